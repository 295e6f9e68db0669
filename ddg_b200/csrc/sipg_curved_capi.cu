// C-ABI of the curved-element SIPG operator (include/ddg_sipg.h,
// ddg_curved_*): host set-up of the per-element fields, the three-pass
// apply, loads, block-Jacobi by coloured probing and the CG graph.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/ddg_sipg.h"
#include "sipg_device.cuh"
#include "sipg_launch.h"
#include "status.h"

using namespace ddg;

#define CK(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return fail(DDG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));             \
  } while (0)

namespace {

struct CvGuard {
  int prev = -1;
  explicit CvGuard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~CvGuard() {
    int cur;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

struct CvGraph {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t exec = nullptr;
};

using CvKey = std::tuple<int, int, double, double>;  // quad, pc, alpha, shift

}  // namespace

struct ddg_curved_op {
  int N = 0, Np = 0, Nfp = 0, K = 0, dev = 0, Ncub = 0, Nfq = 0, ncol = 0;
  double tau_scale = 0.0;
  double *gN = nullptr, *fN = nullptr, *sJ0 = nullptr, *tauF = nullptr;
  double *cG = nullptr, *cQ = nullptr, *cMat = nullptr;
  double *tr = nullptr, *dl = nullptr, *zero = nullptr;
  int ldc = 0;                      // row stride of cG (K rounded up to 128)
  int *tag = nullptr, *slotP = nullptr, *mapP = nullptr, *colour = nullptr;
  unsigned int* status = nullptr;
  CgCtl* ctl = nullptr;
  double *partA = nullptr, *partB = nullptr;
  // block Jacobi
  double *blocks = nullptr, *binv = nullptr;
  bool pc_ready = false;
  int pc_quad = 0;
  double pc_alpha = 0.0;
  // CG work vectors (lazy)
  double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr, *b = nullptr;
  std::map<CvKey, CvGraph> graphs;
  cudaStream_t cap = nullptr;
};

namespace {

CvArgs cv_args(const ddg_curved_op* op, int gate) {
  CvArgs a{};
  a.K = op->K;
  a.Ncub = op->Ncub;
  a.gN = op->gN;
  a.fN = op->fN;
  a.sJ0 = op->sJ0;
  a.tauF = op->tauF;
  a.tag = op->tag;
  a.slotP = op->slotP;
  a.mapP = op->mapP;
  a.cG = op->cG;
  a.cQ = op->cQ;
  a.cMat = op->cMat;
  a.tr = op->tr;
  a.dl = op->dl;
  a.ldc = op->ldc;
  a.ctl = op->ctl;
  a.partA = op->partA;
  a.partB = op->partB;
  a.gate = gate;
  return a;
}

// the three passes of one operator application (mode: CV pass-3 mode)
cudaError_t cv_run(const ddg_curved_op* op, int quad, int mode, double alpha, double shift, const double* u,
                   const double* udir, const double* b, double* y, cudaStream_t s, int gate) {
  const CvArgs a = cv_args(op, gate);
  cudaError_t e = launch_cv_pass(op->N, 1, quad, 0, a, u, nullptr, nullptr, nullptr, 0.0, 0.0, s);
  if (e == cudaSuccess) e = launch_cv_pass(op->N, 2, quad, 0, a, u, udir, nullptr, nullptr, 0.0, 0.0, s);
  if (e == cudaSuccess) e = launch_cv_pass(op->N, 3, quad, mode, a, u, nullptr, b, y, alpha, shift, s);
  return e;
}

int cv_check_quad(const ddg_curved_op* op, int quad, const char* who) {
  if (quad != DDG_QUAD_NODAL && quad != DDG_QUAD_CUBATURE)
    return fail(DDG_ERR_INVALID, std::string(who) + ": quad must be DDG_QUAD_NODAL or DDG_QUAD_CUBATURE");
  if (quad == DDG_QUAD_CUBATURE && op->Ncub == 0)
    return fail(DDG_ERR_INVALID, std::string(who) + ": the handle was created without cubature data");
  return DDG_OK;
}

int cv_status(ddg_curved_op* op) {
  unsigned int st = 0;
  CK(cudaMemcpy(&st, op->status, sizeof(st), cudaMemcpyDeviceToHost));
  if (st != 0u) {
    cudaMemset(op->status, 0, sizeof(unsigned int));
    return fail(DDG_ERR_DEVICE, "curved operator: a kernel reported a singular block (status " +
                                    std::to_string(st) + ")");
  }
  return DDG_OK;
}

void cv_free(ddg_curved_op* op) {
  for (auto& kv : op->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.g) cudaGraphDestroy(kv.second.g);
  }
  op->graphs.clear();
  for (void* ptr : {(void*)op->gN, (void*)op->fN, (void*)op->sJ0, (void*)op->tauF, (void*)op->cG, (void*)op->cQ,
                    (void*)op->cMat, (void*)op->tr, (void*)op->dl, (void*)op->zero, (void*)op->tag,
                    (void*)op->slotP, (void*)op->mapP, (void*)op->colour, (void*)op->status, (void*)op->ctl,
                    (void*)op->partA, (void*)op->partB, (void*)op->blocks, (void*)op->binv, (void*)op->x,
                    (void*)op->r, (void*)op->z, (void*)op->p, (void*)op->Ap, (void*)op->b})
    if (ptr) cudaFree(ptr);
  if (op->cap) cudaStreamDestroy(op->cap);
  delete op;
}

int cv_set_tags(ddg_curved_op* op, const int32_t* bc) {
  const int K = op->K;
  std::vector<int> t((size_t)3 * K);
  for (int k = 0; k < K; ++k)
    for (int f = 0; f < 3; ++f) {
      const int v = bc[(size_t)k * 3 + f];
      if (v < 0 || v > 2) return fail(DDG_ERR_INVALID, "bc_types entries must be 0, 1 or 2");
      t[(size_t)f * K + k] = v;
    }
  CK(cudaMemcpy(op->tag, t.data(), t.size() * sizeof(int), cudaMemcpyHostToDevice));
  op->pc_ready = false;
  return DDG_OK;
}

int cv_ensure_work(ddg_curved_op* op) {
  if (op->x) return DDG_OK;
  const size_t bytes = (size_t)op->K * op->Np * sizeof(double);
  for (double** v : {&op->x, &op->r, &op->z, &op->p, &op->Ap, &op->b}) {
    cudaError_t e = cudaMalloc((void**)v, bytes);
    if (e != cudaSuccess) return fail(DDG_ERR_NOMEM, "curved CG work vectors: " + std::string(cudaGetErrorString(e)));
  }
  return DDG_OK;
}

cudaError_t cv_body(ddg_curved_op* op, const CvKey& key, cudaStream_t s, cudaGraphConditionalHandle h) {
  const int quad = std::get<0>(key), pc = std::get<1>(key);
  const double alpha = std::get<2>(key), shift = std::get<3>(key);
  const int64_t n = (int64_t)op->K * op->Np;
  const double* z = pc ? op->z : op->r;
  cudaError_t e = launch_cv_pupd(n, z, op->p, op->ctl, s);
  if (e == cudaSuccess) e = cv_run(op, quad, 2 /*PDOT*/, alpha, shift, op->p, nullptr, nullptr, op->Ap, s, 1);
  if (e == cudaSuccess) e = launch_cg_xr<double>(op->x, op->p, op->r, op->Ap, n, op->ctl, op->partA, s);
  if (e == cudaSuccess && pc) e = launch_cv_pc(op->N, op->K, op->binv, op->r, op->z, op->ctl, s);
  if (e == cudaSuccess) e = launch_cg_finish<double>(false, op->r, z, n, op->ctl, op->partA, op->status, 1, h, s);
  return e;
}

int cv_graph(ddg_curved_op* op, const CvKey& key, CvGraph** out) {
  auto it = op->graphs.find(key);
  if (it != op->graphs.end()) {
    *out = &it->second;
    return DDG_OK;
  }
  CvGraph cg;
  CK(cudaGraphCreate(&cg.g, 0));
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, cg.g, 1, cudaGraphCondAssignDefault));
  alignas(cudaGraphNodeParams) unsigned char np_buf[sizeof(cudaGraphNodeParams)];
  std::memset(np_buf, 0, sizeof(np_buf));
  cudaGraphNodeParams& np = *reinterpret_cast<cudaGraphNodeParams*>(np_buf);
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, cg.g, nullptr, 0, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  CK(cudaStreamBeginCaptureToGraph(op->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  const cudaError_t e = cv_body(op, key, op->cap, h);
  cudaGraph_t outg = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(op->cap, &outg);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    cudaGraphDestroy(cg.g);
    return fail(DDG_ERR_CUDA, std::string("curved CG body capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  CK(cudaGraphInstantiate(&cg.exec, cg.g, 0));
  op->graphs[key] = cg;
  *out = &op->graphs[key];
  return DDG_OK;
}

}  // namespace

extern "C" int ddg_curved_create(const ddg_curved_desc* d, ddg_curved_op** out) {
  if (!d || !out) return fail(DDG_ERR_INVALID, "ddg_curved_create: null argument");
  *out = nullptr;
  if (d->N < 1 || d->N > DDG_MAX_DEGREE)
    return fail(DDG_ERR_UNSUPPORTED, "polynomial degree " + std::to_string(d->N) + " not built");
  const int N = d->N, Np = (N + 1) * (N + 2) / 2, Nfp = N + 1, Ns = 3 * Nfp, K = d->K;
  if (K < 1 || (int64_t)K * Np >= INT_MAX || (int64_t)Ns * K >= INT_MAX)
    return fail(DDG_ERR_INVALID, "element count out of range");
  if (!d->Dr || !d->Ds || !d->M || !d->m1d || !d->Fmask || !d->rx || !d->sx || !d->ry || !d->sy || !d->J ||
      !d->nx || !d->ny || !d->sJ || !d->Fscale || !d->EToE || !d->EToF || !d->vmapM || !d->vmapP || !d->bc_types)
    return fail(DDG_ERR_INVALID, "ddg_curved_create: null array in descriptor");
  const int Ncub = d->Ncub, Nfq = d->Nfq;
  if (Ncub < 0) return fail(DDG_ERR_INVALID, "Ncub must be >= 0");
  if (Ncub > 0 && (Nfq < 1 || !d->cw || !d->Drq || !d->Dsq || !d->Lq || !d->cJ || !d->crx || !d->csx || !d->cry ||
                   !d->csy || !d->face_w || !d->face_L1d || !d->face_sJ))
    return fail(DDG_ERR_INVALID, "ddg_curved_create: cubature arrays missing");
  if (Ncub > 0 && cv_gather_smem_bytes(N, Ncub) > (size_t)CV_SMEM_LIMIT)
    return fail(DDG_ERR_UNSUPPORTED, "cubature rule too large for the staged kernels (Ncub = " + std::to_string(Ncub) +
                                         ")");
  for (int p = 0; p < Nfp; ++p)
    for (int f = 0; f < 3; ++f)
      if (d->Fmask[p * 3 + f] != fmask_idx(N, f, p))
        return fail(DDG_ERR_INVALID, "Fmask differs from the warp-and-blend row numbering");
  for (int64_t i = 0; i < (int64_t)Ns * K; ++i) {
    const int64_t k = i / Ns, m = i % Ns;
    if (d->vmapM[i] != k * Np + fmask_idx(N, (int)(m / Nfp), (int)(m % Nfp)))
      return fail(DDG_ERR_INVALID, "vmapM inconsistent with Fmask");
    if (d->vmapP[i] < 0 || d->vmapP[i] >= (int64_t)K * Np) return fail(DDG_ERR_INVALID, "vmapP out of range");
  }
  // the neighbour face slot of every face slot (where its vmapP node sits
  // on the neighbour's face EToF)
  std::vector<int> slotP((size_t)Ns * K), mapP((size_t)Ns * K);
  for (int k = 0; k < K; ++k)
    for (int f = 0; f < 3; ++f) {
      const int64_t kp = d->EToE[(size_t)k * 3 + f], fp = d->EToF[(size_t)k * 3 + f];
      if (kp < 0 || kp >= K || fp < 0 || fp > 2) return fail(DDG_ERR_INVALID, "EToE/EToF out of range");
      for (int p = 0; p < Nfp; ++p) {
        const int m = f * Nfp + p;
        const int64_t target = d->vmapP[(size_t)k * Ns + m];
        int found = -1;
        for (int q = 0; q < Nfp && found < 0; ++q)
          if (d->vmapM[(size_t)kp * Ns + fp * Nfp + q] == target) found = (int)fp * Nfp + q;
        if (found < 0) return fail(DDG_ERR_INVALID, "vmapP names no node of the neighbour face EToF");
        slotP[(size_t)m * K + k] = (int)target;
        mapP[(size_t)m * K + k] = found * K + (int)kp;
      }
    }
  // greedy colouring in element order (src/ddg/dg2d/sipg.py:651-668)
  std::vector<int> colour(K, -1);
  int ncol = 0;
  for (int k = 0; k < K; ++k) {
    std::set<int> used;
    for (int f = 0; f < 3; ++f) {
      const int64_t nb = d->EToE[(size_t)k * 3 + f];
      if (nb != k && colour[nb] >= 0) used.insert(colour[nb]);
    }
    int c = 0;
    while (used.count(c)) ++c;
    colour[k] = c;
    ncol = std::max(ncol, c + 1);
  }
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (d->device < 0 || d->device >= ndev) return fail(DDG_ERR_INVALID, "bad device ordinal");
  CvGuard guard(d->device);
  {
    const int urc = ddg_sipg_upload_reference(N, d->Dr, d->Ds, d->M, d->m1d, d->device);
    if (urc != DDG_OK) return urc;
  }
  // host images of the device fields
  const size_t KN = (size_t)Np * K, KS = (size_t)Ns * K;
  std::vector<double> gN(5 * KN), fN(2 * KS), sJ0((size_t)3 * K), tauF((size_t)3 * K);
  std::memcpy(gN.data() + 0 * KN, d->rx, KN * 8);
  std::memcpy(gN.data() + 1 * KN, d->sx, KN * 8);
  std::memcpy(gN.data() + 2 * KN, d->ry, KN * 8);
  std::memcpy(gN.data() + 3 * KN, d->sy, KN * 8);
  std::memcpy(gN.data() + 4 * KN, d->J, KN * 8);
  std::memcpy(fN.data(), d->nx, KS * 8);
  std::memcpy(fN.data() + KS, d->ny, KS * 8);
  const double tscale = d->tau_scale * (N + 1) * (N + 1);
  for (int f = 0; f < 3; ++f)
    for (int k = 0; k < K; ++k) {
      sJ0[(size_t)f * K + k] = d->sJ[(size_t)f * Nfp * K + k];
      tauF[(size_t)f * K + k] = tscale * d->Fscale[(size_t)f * Nfp * K + k];
    }
  std::vector<double> cG, cQ, cMat;
  const int NQ = Nfp * (Nfp + 1) / 2;
  const int ldc = (K + 127) / 128 * 128;
  if (Ncub > 0) {
    cG.assign((size_t)4 * Ncub * ldc, 0.0);
    for (int q = 0; q < Ncub; ++q)
      for (int k = 0; k < K; ++k) {
        const size_t i = (size_t)q * K + k;
        const double wJ = d->cw[q] * d->cJ[i];
        const double rx = d->crx[i], sx = d->csx[i], ry = d->cry[i], sy = d->csy[i];
        cG[(size_t)(0 * Ncub + q) * ldc + k] = wJ * (rx * rx + ry * ry);
        cG[(size_t)(1 * Ncub + q) * ldc + k] = wJ * (rx * sx + ry * sy);
        cG[(size_t)(2 * Ncub + q) * ldc + k] = wJ * (sx * sx + sy * sy);
        cG[(size_t)(3 * Ncub + q) * ldc + k] = wJ;
      }
    cQ.assign((size_t)3 * NQ * K, 0.0);
    for (int f = 0; f < 3; ++f)
      for (int i = 0; i < Nfq; ++i) {
        const double* L = d->face_L1d + ((size_t)f * Nfq + i) * Nfp;
        for (int k = 0; k < K; ++k) {
          const double wq = d->face_w[i] * d->face_sJ[((size_t)f * Nfq + i) * K + k];
          for (int p = 0; p < Nfp; ++p)
            for (int q = p; q < Nfp; ++q) {
              const int idx = p * Nfp - p * (p - 1) / 2 + (q - p);
              cQ[(size_t)(f * NQ + idx) * K + k] += wq * L[p] * L[q];
            }
        }
      }
    cMat.resize((size_t)3 * Ncub * Np);
    std::memcpy(cMat.data(), d->Drq, (size_t)Ncub * Np * 8);
    std::memcpy(cMat.data() + (size_t)Ncub * Np, d->Dsq, (size_t)Ncub * Np * 8);
    std::memcpy(cMat.data() + (size_t)2 * Ncub * Np, d->Lq, (size_t)Ncub * Np * 8);
  }

  ddg_curved_op* op = new ddg_curved_op();
  op->N = N;
  op->Np = Np;
  op->Nfp = Nfp;
  op->K = K;
  op->dev = d->device;
  op->Ncub = Ncub;
  op->Nfq = Nfq;
  op->ncol = ncol;
  op->ldc = ldc;
  op->tau_scale = d->tau_scale;
  const int nparts = std::max((K + 127) / 128, xr_grid((int64_t)K * Np)) + 32;
  cudaError_t e = cudaSuccess;
#define ALLOC(ptr, bytes) \
  if (e == cudaSuccess) e = cudaMalloc((void**)&(ptr), (bytes))
#define UPLOAD(ptr, vec) \
  if (e == cudaSuccess) e = cudaMemcpy((ptr), (vec).data(), (vec).size() * sizeof((vec)[0]), cudaMemcpyHostToDevice)
  ALLOC(op->gN, gN.size() * 8);
  ALLOC(op->fN, fN.size() * 8);
  ALLOC(op->sJ0, sJ0.size() * 8);
  ALLOC(op->tauF, tauF.size() * 8);
  ALLOC(op->tag, (size_t)3 * K * sizeof(int));
  ALLOC(op->slotP, slotP.size() * sizeof(int));
  ALLOC(op->mapP, mapP.size() * sizeof(int));
  ALLOC(op->colour, colour.size() * sizeof(int));
  ALLOC(op->tr, 2 * KS * 8);
  ALLOC(op->dl, 3 * KS * 8);
  ALLOC(op->zero, KN * 8);
  ALLOC(op->status, sizeof(unsigned int));
  ALLOC(op->ctl, sizeof(CgCtl));
  ALLOC(op->partA, (size_t)nparts * 8);
  ALLOC(op->partB, (size_t)nparts * 8);
  if (Ncub > 0) {
    ALLOC(op->cG, cG.size() * 8);
    ALLOC(op->cQ, cQ.size() * 8);
    ALLOC(op->cMat, cMat.size() * 8);
  }
  UPLOAD(op->gN, gN);
  UPLOAD(op->fN, fN);
  UPLOAD(op->sJ0, sJ0);
  UPLOAD(op->tauF, tauF);
  UPLOAD(op->slotP, slotP);
  UPLOAD(op->mapP, mapP);
  UPLOAD(op->colour, colour);
  if (Ncub > 0) {
    UPLOAD(op->cG, cG);
    UPLOAD(op->cQ, cQ);
    UPLOAD(op->cMat, cMat);
  }
#undef ALLOC
#undef UPLOAD
  if (e == cudaSuccess) e = cudaMemset(op->zero, 0, KN * 8);
  if (e == cudaSuccess) e = cudaMemset(op->status, 0, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(op->ctl, 0, sizeof(CgCtl));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&op->cap, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cv_prepare(N);
  if (e != cudaSuccess) {
    cv_free(op);
    return fail(e == cudaErrorMemoryAllocation ? DDG_ERR_NOMEM : DDG_ERR_CUDA,
                std::string("ddg_curved_create: ") + cudaGetErrorString(e));
  }
  const int rc = cv_set_tags(op, d->bc_types);
  if (rc != DDG_OK) {
    cv_free(op);
    return rc;
  }
  *out = op;
  return DDG_OK;
}

extern "C" int ddg_curved_destroy(ddg_curved_op* op) {
  if (!op) return DDG_OK;
  CvGuard guard(op->dev);
  cudaDeviceSynchronize();
  cv_free(op);
  return DDG_OK;
}

extern "C" int ddg_curved_set_bc(ddg_curved_op* op, const int32_t* bc) {
  if (!op || !bc) return fail(DDG_ERR_INVALID, "ddg_curved_set_bc: null argument");
  CvGuard guard(op->dev);
  return cv_set_tags(op, bc);
}

extern "C" int ddg_curved_apply(ddg_curved_op* op, int quad, double alpha, const double* u, double* y, void* stream) {
  if (!op || !u || !y) return fail(DDG_ERR_INVALID, "ddg_curved_apply: null argument");
  if (int rc = cv_check_quad(op, quad, "ddg_curved_apply")) return rc;
  if (u == y) return fail(DDG_ERR_INVALID, "ddg_curved_apply: u and y must not alias");
  CvGuard guard(op->dev);
  const cudaError_t e = cv_run(op, quad, 0, alpha, 0.0, u, nullptr, nullptr, y, (cudaStream_t)stream, 0);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("ddg_curved_apply: ") + cudaGetErrorString(e));
  return DDG_OK;
}

extern "C" int ddg_curved_apply_dir(ddg_curved_op* op, int quad, const double* u, const double* u_dir, double* y,
                                    void* stream) {
  if (!op || !u_dir || !y) return fail(DDG_ERR_INVALID, "ddg_curved_apply_dir: null argument");
  if (int rc = cv_check_quad(op, quad, "ddg_curved_apply_dir")) return rc;
  if (u == y || u_dir == y) return fail(DDG_ERR_INVALID, "ddg_curved_apply_dir: y aliases an input");
  CvGuard guard(op->dev);
  const double* uu = u ? u : op->zero;
  const cudaError_t e = cv_run(op, quad, 0, 0.0, 0.0, uu, u_dir, nullptr, y, (cudaStream_t)stream, 0);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("ddg_curved_apply_dir: ") + cudaGetErrorString(e));
  return DDG_OK;
}

extern "C" int ddg_curved_mass(ddg_curved_op* op, int quad, const double* f, double* y, void* stream) {
  if (!op || !f || !y) return fail(DDG_ERR_INVALID, "ddg_curved_mass: null argument");
  if (int rc = cv_check_quad(op, quad, "ddg_curved_mass")) return rc;
  if (f == y) return fail(DDG_ERR_INVALID, "ddg_curved_mass: f and y must not alias");
  CvGuard guard(op->dev);
  const cudaError_t e = launch_cv_mass(op->N, quad, cv_args(op, 0), f, y, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("ddg_curved_mass: ") + cudaGetErrorString(e));
  return DDG_OK;
}

extern "C" int ddg_curved_rhs(ddg_curved_op* op, int quad, const double* f, const double* u_dir, const double* q_neu,
                              double* rhs, void* stream) {
  if (!op || !rhs) return fail(DDG_ERR_INVALID, "ddg_curved_rhs: null argument");
  if (int rc = cv_check_quad(op, quad, "ddg_curved_rhs")) return rc;
  if (rhs == f || rhs == u_dir || rhs == q_neu) return fail(DDG_ERR_INVALID, "ddg_curved_rhs: rhs aliases an input");
  CvGuard guard(op->dev);
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = f ? launch_cv_mass(op->N, quad, cv_args(op, 0), f, rhs, s)
                    : cudaMemsetAsync(rhs, 0, (size_t)op->K * op->Np * 8, s);
  // - L_D: the nodal operator applied to zero with the Dirichlet ghost u_dir
  if (e == cudaSuccess && u_dir)
    e = cv_run(op, DDG_QUAD_NODAL, 1 /*SUB*/, 0.0, 0.0, op->zero, u_dir, nullptr, rhs, s, 0);
  if (e == cudaSuccess && q_neu) e = launch_cv_neumann(op->N, cv_args(op, 0), q_neu, rhs, s);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("ddg_curved_rhs: ") + cudaGetErrorString(e));
  return DDG_OK;
}

extern "C" int ddg_curved_pc_build(ddg_curved_op* op, int quad, double alpha, void* stream) {
  if (!op) return fail(DDG_ERR_INVALID, "ddg_curved_pc_build: null handle");
  if (int rc = cv_check_quad(op, quad, "ddg_curved_pc_build")) return rc;
  CvGuard guard(op->dev);
  if (int rc = cv_ensure_work(op)) return rc;
  const size_t nb = (size_t)op->K * op->Np * op->Np * sizeof(double);
  if (!op->blocks) CK(cudaMalloc((void**)&op->blocks, nb));
  if (!op->binv) CK(cudaMalloc((void**)&op->binv, nb));
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaSuccess;
  for (int c = 0; c < op->ncol && e == cudaSuccess; ++c)
    for (int j = 0; j < op->Np && e == cudaSuccess; ++j) {
      e = launch_cv_probe(op->K, op->Np, op->colour, c, j, op->p, s);
      if (e == cudaSuccess) e = cv_run(op, quad, 0, alpha, 0.0, op->p, nullptr, nullptr, op->Ap, s, 0);
      if (e == cudaSuccess) e = launch_cv_collect(op->K, op->Np, op->colour, c, j, 0.0, op->Ap, op->blocks, s);
    }
  if (e == cudaSuccess) e = launch_cv_invert(op->N, op->K, op->blocks, op->binv, op->status, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("ddg_curved_pc_build: ") + cudaGetErrorString(e));
  if (int rc = cv_status(op)) return rc;
  op->pc_ready = true;
  op->pc_quad = quad;
  op->pc_alpha = alpha;
  return DDG_OK;
}

extern "C" int ddg_curved_pc_apply(ddg_curved_op* op, const double* r, double* z, void* stream) {
  if (!op || !r || !z) return fail(DDG_ERR_INVALID, "ddg_curved_pc_apply: null argument");
  if (!op->pc_ready) return fail(DDG_ERR_INVALID, "ddg_curved_pc_apply: call ddg_curved_pc_build first");
  if (r == z) return fail(DDG_ERR_INVALID, "ddg_curved_pc_apply: r and z must not alias");
  CvGuard guard(op->dev);
  const cudaError_t e = launch_cv_pc(op->N, op->K, op->binv, r, z, nullptr, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("ddg_curved_pc_apply: ") + cudaGetErrorString(e));
  return DDG_OK;
}

extern "C" int ddg_curved_pc_blocks(ddg_curved_op* op, double* blocks, void* stream) {
  if (!op || !blocks) return fail(DDG_ERR_INVALID, "ddg_curved_pc_blocks: null argument");
  if (!op->pc_ready) return fail(DDG_ERR_INVALID, "ddg_curved_pc_blocks: call ddg_curved_pc_build first");
  CvGuard guard(op->dev);
  CK(cudaMemcpyAsync(blocks, op->blocks, (size_t)op->K * op->Np * op->Np * 8, cudaMemcpyDeviceToDevice,
                     (cudaStream_t)stream));
  return DDG_OK;
}

extern "C" int ddg_curved_cg(ddg_curved_op* op, int quad, const ddg_cg_config* cfg, const double* b, double* x,
                             void* stream, ddg_solve_info* info) {
  if (!op || !cfg || !b || !x) return fail(DDG_ERR_INVALID, "ddg_curved_cg: null argument");
  if (int rc = cv_check_quad(op, quad, "ddg_curved_cg")) return rc;
  if (cfg->maxiter < 0 || !(cfg->tol >= 0) || !(cfg->atol >= 0))
    return fail(DDG_ERR_INVALID, "ddg_curved_cg: tol/atol/maxiter must be non-negative");
  if (cfg->precision != DDG_FP64) return fail(DDG_ERR_UNSUPPORTED, "ddg_curved_cg: float64 only");
  if (cfg->pc != DDG_PC_NONE && cfg->pc != DDG_PC_JACOBI)
    return fail(DDG_ERR_UNSUPPORTED, "ddg_curved_cg: pc must be DDG_PC_NONE or DDG_PC_JACOBI");
  const int pc = cfg->pc == DDG_PC_JACOBI;
  if (pc && !op->pc_ready) return fail(DDG_ERR_INVALID, "ddg_curved_cg: call ddg_curved_pc_build first");
  CvGuard guard(op->dev);
  if (int rc = cv_ensure_work(op)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const CvKey key{quad, pc, cfg->alpha, cfg->shift};
  CvGraph* gr = nullptr;
  if (int rc = cv_graph(op, key, &gr)) return rc;
  const int64_t n = (int64_t)op->K * op->Np;
  const size_t bytes = (size_t)n * 8;
  CgCtl h{};
  h.tol2 = cfg->tol * cfg->tol;
  h.atol_sq = cfg->atol * cfg->atol;
  h.maxiter = cfg->maxiter;
  h.use_pc = pc;
  h.cont = 1;
  h.zcoef = 1.0;
  CK(cudaMemcpyAsync(op->ctl, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(op->b, b, bytes, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(op->x, x, bytes, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemsetAsync(op->p, 0, bytes, s));
  cudaError_t e = cv_run(op, quad, 3 /*RESID*/, cfg->alpha, cfg->shift, op->x, nullptr, op->b, op->r, s, 0);
  if (e == cudaSuccess && pc) e = launch_cv_pc(op->N, op->K, op->binv, op->r, op->z, nullptr, s);
  if (e == cudaSuccess)
    e = launch_cg_finish<double>(true, op->r, pc ? op->z : op->r, n, op->ctl, op->partA, op->status, 0, 0, s);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("ddg_curved_cg init: ") + cudaGetErrorString(e));
  CK(cudaGraphLaunch(gr->exec, s));
  CK(cudaMemcpyAsync(x, op->x, bytes, cudaMemcpyDeviceToDevice, s));
  CgCtl res{};
  CK(cudaMemcpyAsync(&res, op->ctl, sizeof(res), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (int rc = cv_status(op)) return rc;
  if (info) {
    info->status = res.status;
    info->iterations = res.iter;
    info->res_norm2 = res.rr;
    info->b_norm2 = res.bb;
    info->updates = 0;
    info->reserved = 0;
  }
  return DDG_OK;
}
