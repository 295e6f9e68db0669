// C-ABI implementation: handle lifetime, uploads, and the entry points of
// include/ddg_sipg.h.  No exception crosses the boundary; every CUDA error
// becomes a status code plus a thread-local message.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ddg_sipg.h"
#include "sipg_device.cuh"
#include "sipg_launch.h"
#include "status.h"

namespace ddg {
static thread_local std::string g_err;
void set_error(const std::string& m) { g_err = m; }
}  // namespace ddg

using namespace ddg;

#define CK(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return fail(DDG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));             \
  } while (0)

namespace {

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~DevGuard() {
    int cur;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Reference-element matrices already in constant memory, per (device, N).
std::mutex g_ref_mu;
std::map<std::pair<int, int>, std::vector<double>> g_ref_loaded;

struct Work {  // CG vectors of one precision (element-major, K*Np)
  void *x = nullptr, *b = nullptr, *r = nullptr, *z = nullptr, *p0 = nullptr, *p1 = nullptr, *Ap = nullptr;
  size_t bytes = 0;
};

struct GraphKey {
  int prec, pc;
  double alpha, shift;
  bool operator<(const GraphKey& o) const {
    if (prec != o.prec) return prec < o.prec;
    if (pc != o.pc) return pc < o.pc;
    if (alpha != o.alpha) return alpha < o.alpha;
    return shift < o.shift;
  }
};
struct CgGraph {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t exec = nullptr;
};

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

struct ddg_sipg_op {
  int N = 0, Np = 0, Nfp = 0, K = 0, dev = 0, ldg = 0, ldb = 0;
  double tau_scale = 0, tau = 0;
  double* geo64 = nullptr;
  float* geo32 = nullptr;
  uint32_t* nbr = nullptr;
  int* perm = nullptr;
  unsigned int* status = nullptr;   // device status word
  CgCtl* ctl = nullptr;
  double* partA = nullptr;
  double* partB = nullptr;
  unsigned int* ticket = nullptr;   // for the free dot helper
  double* dotbuf = nullptr;
  // block Jacobi
  double* blocks = nullptr;
  double* binv64 = nullptr;
  float* binv32 = nullptr;
  bool pc_ready = false;
  double pc_alpha = 0.0;
  Work w[2];
  std::map<GraphKey, CgGraph> graphs;
  cudaStream_t cap = nullptr;       // private stream for graph capture
  // host copies for set_bc
  std::vector<int64_t> EToE, EToF, vmapP;
  std::vector<int64_t> rot;         // (3, Np)
  std::vector<uint32_t> nbr_host;
};

namespace {

int build_nbr(ddg_sipg_op* op, const int32_t* bc) {
  const int K = op->K, N = op->N, Np = op->Np, Nfp = op->Nfp;
  op->nbr_host.assign((size_t)3 * K, 0u);
  for (int k = 0; k < K; ++k)
    for (int f = 0; f < 3; ++f) {
      const int64_t kp = op->EToE[(size_t)k * 3 + f], fp = op->EToF[(size_t)k * 3 + f];
      const int tag = bc[(size_t)k * 3 + f];
      if (tag < 0 || tag > 2) return fail(DDG_ERR_INVALID, "bc_types entries must be 0, 1 or 2");
      if (kp < 0 || kp >= K || fp < 0 || fp > 2) return fail(DDG_ERR_INVALID, "EToE/EToF out of range");
      const bool self = (kp == k && fp == f);
      bool flip = false, pact = false, mint = false;
      if (!self) {
        const int tagp = bc[(size_t)kp * 3 + fp];
        pact = (tagp == DDG_BC_INTERIOR);
        mint = (tag == DDG_BC_INTERIOR);
        // node order of the partner face (re-labelled so its face is face 0)
        int nsame = 0, nrev = 0;
        for (int p = 0; p < Nfp; ++p) {
          const int64_t j = op->vmapP[((size_t)k * 3 + f) * Nfp + p];
          if (j / Np != kp) return fail(DDG_ERR_INVALID, "vmapP does not point into the EToE neighbour (non-conforming face)");
          const int64_t loc = j % Np;
          int q = -1;
          for (int qq = 0; qq < Nfp; ++qq)
            if (op->rot[(size_t)fp * Np + qq] == loc) q = qq;
          if (q == p) ++nsame;
          if (q == N - p) ++nrev;
        }
        if (nrev == Nfp) flip = true;
        else if (nsame != Nfp) return fail(DDG_ERR_INVALID, "face node matching is neither aligned nor reversed");
      }
      // a self-pointing face tagged interior contributes nothing (its jump
      // vanishes and its two scatters cancel: sipg.py:241-249)
      op->nbr_host[(size_t)f * K + k] = nbr_pack((uint32_t)kp, (uint32_t)fp, flip, (uint32_t)tag, pact, mint);
    }
  return DDG_OK;
}

int ensure_work(ddg_sipg_op* op, int prec) {
  Work& w = op->w[prec];
  const size_t bytes = (size_t)op->K * op->Np * (prec == DDG_FP64 ? 8 : 4);
  if (w.bytes == bytes) return DDG_OK;
  void** ptrs[] = {&w.x, &w.b, &w.r, &w.z, &w.p0, &w.p1, &w.Ap};
  for (void** p : ptrs) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  w.bytes = 0;
  for (void** p : ptrs) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return fail(DDG_ERR_NOMEM, std::string("CG workspace: ") + cudaGetErrorString(e));
  }
  w.bytes = bytes;
  return DDG_OK;
}

template <typename T>
ApplyArgs<T> apply_args(ddg_sipg_op* op) {
  ApplyArgs<T> a{};
  a.geo = (sizeof(T) == 8) ? (const T*)op->geo64 : (const T*)op->geo32;
  a.nbr = op->nbr;
  a.perm = op->perm;
  a.ctl = op->ctl;
  a.partA = op->partA;
  a.partB = op->partB;
  a.ctl_status = op->status;
  a.K = op->K;
  a.ldg = op->ldg;
  a.tau = op->tau;
  return a;
}

int check_status(ddg_sipg_op* op) {
  unsigned int st = 0;
  CK(cudaMemcpy(&st, op->status, sizeof(st), cudaMemcpyDeviceToHost));
  if (st) {
    cudaMemset(op->status, 0, sizeof(unsigned int));
    return fail(DDG_ERR_DEVICE, st & ST_TMA_TIMEOUT ? "a kernel timed out waiting for a bulk copy"
                                                       : "a kernel reported a singular block or bad index");
  }
  return DDG_OK;
}

template <typename T>
int capture_body(ddg_sipg_op* op, const GraphKey& key, cudaGraph_t body, cudaGraphConditionalHandle h) {
  Work& w = op->w[key.prec];
  CK(cudaStreamBeginCaptureToGraph(op->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  ApplyArgs<T> a = apply_args<T>(op);
  a.alpha = key.alpha;
  a.shift = key.shift;
  a.use_tma = 1;
  CgArgs<T> c{};
  c.x = (T*)w.x;
  c.r = (T*)w.r;
  c.Ap = (const T*)w.Ap;
  c.z = key.pc ? (T*)w.z : (T*)w.r;
  c.binv = (sizeof(T) == 8) ? (const T*)op->binv64 : (const T*)op->binv32;
  c.ldb = op->ldb;
  c.ctl = op->ctl;
  c.partA = op->partA;
  c.partB = op->partB;
  c.K = op->K;
  c.dev_status = op->status;
  c.has_cond = 1;
  c.cond = h;
  cudaError_t e = cudaSuccess;
  for (int half = 0; half < 2 && e == cudaSuccess; ++half) {
    void* pin = half == 0 ? w.p0 : w.p1;
    void* pout = half == 0 ? w.p1 : w.p0;
    a.in0 = (const T*)c.z;
    a.in1 = (const T*)pin;
    a.out0 = (T*)w.Ap;
    a.out1 = (T*)pout;
    e = launch_apply<T>(op->N, AM_PFUSE, a, op->cap);
    if (e != cudaSuccess) break;
    c.p = (const T*)pout;
    e = launch_cg_step<T>(op->N, key.pc != 0, false, c, op->cap);
  }
  cudaGraph_t out = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(op->cap, &out);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("CG body capture: ") + cudaGetErrorString(e));
  if (e2 != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("CG body capture end: ") + cudaGetErrorString(e2));
  return DDG_OK;
}

int get_graph(ddg_sipg_op* op, const GraphKey& key, CgGraph** out) {
  auto it = op->graphs.find(key);
  if (it != op->graphs.end()) {
    *out = &it->second;
    return DDG_OK;
  }
  CgGraph cg;
  CK(cudaGraphCreate(&cg.g, 0));
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, cg.g, 1, cudaGraphCondAssignDefault));
  // cudaGraphNodeParams holds a union without a default constructor
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
  int rc = key.prec == DDG_FP64 ? capture_body<double>(op, key, body, h) : capture_body<float>(op, key, body, h);
  if (rc != DDG_OK) {
    cudaGraphDestroy(cg.g);
    return rc;
  }
  CK(cudaGraphInstantiate(&cg.exec, cg.g, 0));
  op->graphs[key] = cg;
  *out = &op->graphs[key];
  return DDG_OK;
}

void free_op(ddg_sipg_op* op) {
  for (auto& kv : op->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.g) cudaGraphDestroy(kv.second.g);
  }
  void* ptrs[] = {op->geo64, op->geo32, op->nbr, op->perm, op->status, op->ctl, op->partA, op->partB,
                  op->ticket, op->dotbuf, op->blocks, op->binv64, op->binv32};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (auto& w : op->w) {
    void* wp[] = {w.x, w.b, w.r, w.z, w.p0, w.p1, w.Ap};
    for (void* p : wp)
      if (p) cudaFree(p);
  }
  if (op->cap) cudaStreamDestroy(op->cap);
  delete op;
}

}  // namespace

// ===================================================================== API
extern "C" const char* ddg_last_error(void) { return g_err.c_str(); }
extern "C" const char* ddg_version(void) { return "ddg_sipg 0.1 (sm_100a)"; }

extern "C" int ddg_sipg_create(const ddg_sipg_mesh_desc* d, ddg_sipg_op** out) {
  if (!d || !out) return fail(DDG_ERR_INVALID, "ddg_sipg_create: null argument");
  *out = nullptr;
  if (d->N < 1 || d->N > DDG_MAX_DEGREE)
    return fail(DDG_ERR_UNSUPPORTED, "polynomial degree " + std::to_string(d->N) + " not built (1.." +
                                         std::to_string(DDG_MAX_DEGREE) + ")");
  if (d->K < 1 || (uint32_t)d->K > NBR_MAX_K) return fail(DDG_ERR_INVALID, "element count out of range");
  if (!d->Dr || !d->Ds || !d->M || !d->m1d || !d->Fmask || !d->rot_perm || !d->geo || !d->EToE || !d->EToF ||
      !d->vmapM || !d->vmapP || !d->bc_types)
    return fail(DDG_ERR_INVALID, "ddg_sipg_create: null array in descriptor");
  const int N = d->N, Np = (N + 1) * (N + 2) / 2, Nfp = N + 1, K = d->K;
  for (int p = 0; p < Nfp; ++p)
    for (int f = 0; f < 3; ++f)
      if (d->Fmask[p * 3 + f] != fmask_idx(N, f, p))
        return fail(DDG_ERR_INVALID, "Fmask differs from the warp-and-blend row numbering");
  for (int64_t i = 0; i < (int64_t)3 * Nfp * K; ++i) {
    const int64_t k = i / (3 * Nfp), f = (i / Nfp) % 3, p = i % Nfp;
    if (d->vmapM[i] != k * Np + fmask_idx(N, (int)f, (int)p)) return fail(DDG_ERR_INVALID, "vmapM inconsistent with Fmask");
    if (d->vmapP[i] < 0 || d->vmapP[i] >= (int64_t)K * Np) return fail(DDG_ERR_INVALID, "vmapP out of range");
  }
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (d->device < 0 || d->device >= ndev) return fail(DDG_ERR_INVALID, "bad device ordinal");
  DevGuard guard(d->device);

  ddg_sipg_op* op = new ddg_sipg_op();
  op->N = N;
  op->Np = Np;
  op->Nfp = Nfp;
  op->K = K;
  op->dev = d->device;
  op->ldg = (K + 31) / 32 * 32;
  op->ldb = op->ldg;
  op->tau_scale = d->tau_scale;
  op->tau = d->tau_scale * (N + 1) * (N + 1);
  op->EToE.assign(d->EToE, d->EToE + (size_t)3 * K);
  op->EToF.assign(d->EToF, d->EToF + (size_t)3 * K);
  op->vmapP.assign(d->vmapP, d->vmapP + (size_t)3 * Nfp * K);
  op->rot.assign(d->rot_perm, d->rot_perm + (size_t)3 * Np);
  for (int f = 0; f < 3; ++f) {
    std::vector<int> seen(Np, 0);
    for (int i = 0; i < Np; ++i) {
      const int64_t v = op->rot[(size_t)f * Np + i];
      if (v < 0 || v >= Np || seen[v]++) {
        free_op(op);
        return fail(DDG_ERR_INVALID, "rot_perm is not a permutation");
      }
    }
  }
  int rc = build_nbr(op, d->bc_types);
  if (rc != DDG_OK) {
    free_op(op);
    return rc;
  }
  // constant memory (once per device and degree)
  {
    std::lock_guard<std::mutex> lk(g_ref_mu);
    std::vector<double> blob;
    blob.insert(blob.end(), d->Dr, d->Dr + Np * Np);
    blob.insert(blob.end(), d->Ds, d->Ds + Np * Np);
    blob.insert(blob.end(), d->M, d->M + Np * Np);
    blob.insert(blob.end(), d->m1d, d->m1d + 3 * Nfp * Nfp);
    auto key = std::make_pair(d->device, N);
    auto it = g_ref_loaded.find(key);
    if (it == g_ref_loaded.end()) {
      cudaError_t e = upload_ref(N, d->Dr, d->Ds, d->M, d->m1d);
      if (e != cudaSuccess) {
        free_op(op);
        return fail(DDG_ERR_CUDA, std::string("constant upload: ") + cudaGetErrorString(e));
      }
      g_ref_loaded[key] = blob;
    } else {
      for (size_t i = 0; i < blob.size(); ++i)
        if (std::fabs(blob[i] - it->second[i]) > 1e-12 * (1.0 + std::fabs(blob[i]))) {
          free_op(op);
          return fail(DDG_ERR_INVALID, "reference matrices differ from the ones already loaded for this degree");
        }
    }
  }
  // geometry (SoA, float64 and float32)
  std::vector<double> g64((size_t)G_COUNT * op->ldg, 0.0);
  std::vector<float> g32((size_t)G_COUNT * op->ldg, 0.0f);
  for (int k = 0; k < K; ++k)
    for (int c = 0; c < G_COUNT; ++c) {
      const double v = d->geo[(size_t)k * G_COUNT + c];
      g64[(size_t)c * op->ldg + k] = v;
      g32[(size_t)c * op->ldg + k] = (float)v;
    }
  std::vector<int> perm(op->rot.begin(), op->rot.end());
  cudaError_t e = cudaSuccess;
#define ALLOC(ptr, bytes) \
  if (e == cudaSuccess) e = cudaMalloc((void**)&(ptr), (bytes))
  ALLOC(op->geo64, g64.size() * 8);
  ALLOC(op->geo32, g32.size() * 4);
  ALLOC(op->nbr, op->nbr_host.size() * 4);
  ALLOC(op->perm, perm.size() * sizeof(int));
  ALLOC(op->status, sizeof(unsigned int));
  ALLOC(op->ctl, sizeof(CgCtl));
  const int np_parts = std::max(apply_grid(K), std::max(cg_grid(K), dot_grid((int64_t)K * Np))) + 32;
  ALLOC(op->partA, np_parts * sizeof(double));
  ALLOC(op->partB, np_parts * sizeof(double));
  ALLOC(op->ticket, sizeof(unsigned int));
  ALLOC(op->dotbuf, sizeof(double));
#undef ALLOC
  if (e == cudaSuccess) e = cudaMemcpy(op->geo64, g64.data(), g64.size() * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(op->geo32, g32.data(), g32.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(op->nbr, op->nbr_host.data(), op->nbr_host.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(op->perm, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(op->status, 0, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(op->ctl, 0, sizeof(CgCtl));
  if (e == cudaSuccess) e = cudaMemset(op->ticket, 0, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&op->cap, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    free_op(op);
    return fail(e == cudaErrorMemoryAllocation ? DDG_ERR_NOMEM : DDG_ERR_CUDA,
                std::string("ddg_sipg_create: ") + cudaGetErrorString(e));
  }
  *out = op;
  return DDG_OK;
}

extern "C" int ddg_sipg_destroy(ddg_sipg_op* op) {
  if (!op) return DDG_OK;
  DevGuard guard(op->dev);
  cudaDeviceSynchronize();
  free_op(op);
  return DDG_OK;
}

extern "C" int ddg_sipg_set_bc(ddg_sipg_op* op, const int32_t* bc) {
  if (!op || !bc) return fail(DDG_ERR_INVALID, "ddg_sipg_set_bc: null argument");
  DevGuard guard(op->dev);
  int rc = build_nbr(op, bc);
  if (rc != DDG_OK) return rc;
  CK(cudaMemcpy(op->nbr, op->nbr_host.data(), op->nbr_host.size() * 4, cudaMemcpyHostToDevice));
  op->pc_ready = false;
  return DDG_OK;
}

extern "C" int ddg_sipg_apply(ddg_sipg_op* op, int prec, double alpha, const void* u, void* y, void* stream) {
  if (!op || !u || !y) return fail(DDG_ERR_INVALID, "ddg_sipg_apply: null argument");
  if (u == y) return fail(DDG_ERR_INVALID, "ddg_sipg_apply: u and y must not alias");
  DevGuard guard(op->dev);
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  if (prec == DDG_FP64) {
    ApplyArgs<double> a = apply_args<double>(op);
    a.in0 = (const double*)u;
    a.out0 = (double*)y;
    a.alpha = alpha;
    a.use_tma = aligned16(u) && aligned16(y);
    e = launch_apply<double>(op->N, AM_APPLY, a, s);
  } else if (prec == DDG_FP32) {
    ApplyArgs<float> a = apply_args<float>(op);
    a.in0 = (const float*)u;
    a.out0 = (float*)y;
    a.alpha = alpha;
    a.use_tma = aligned16(u) && aligned16(y);
    e = launch_apply<float>(op->N, AM_APPLY, a, s);
  } else {
    return fail(DDG_ERR_INVALID, "precision must be DDG_FP64 or DDG_FP32");
  }
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("apply launch: ") + cudaGetErrorString(e));
  return DDG_OK;
}

extern "C" int ddg_sipg_rhs(ddg_sipg_op* op, const double* f, const double* u_dir, const double* q_neu,
                            double* rhs, void* stream) {
  if (!op || !rhs) return fail(DDG_ERR_INVALID, "ddg_sipg_rhs: null argument");
  DevGuard guard(op->dev);
  RhsArgs a{};
  a.geo = op->geo64;
  a.nbr = op->nbr;
  a.f = f;
  a.u_dir = u_dir;
  a.q_neu = q_neu;
  a.rhs = rhs;
  a.K = op->K;
  a.ldg = op->ldg;
  a.tau = op->tau;
  cudaError_t e = launch_rhs(op->N, a, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("rhs launch: ") + cudaGetErrorString(e));
  return DDG_OK;
}

extern "C" int ddg_sipg_pc_build(ddg_sipg_op* op, double alpha, void* stream) {
  if (!op) return fail(DDG_ERR_INVALID, "ddg_sipg_pc_build: null handle");
  DevGuard guard(op->dev);
  const size_t nb = (size_t)op->K * op->Np * op->Np;
  if (!op->blocks) {
    CK(cudaMalloc((void**)&op->blocks, nb * 8));
    CK(cudaMalloc((void**)&op->binv64, (size_t)op->Np * op->Np * op->ldb * 8));
    CK(cudaMalloc((void**)&op->binv32, (size_t)op->Np * op->Np * op->ldb * 4));
  }
  BlockArgs a{};
  a.geo = op->geo64;
  a.nbr = op->nbr;
  a.blocks = op->blocks;
  a.binv64 = op->binv64;
  a.binv32 = op->binv32;
  a.status = op->status;
  a.K = op->K;
  a.ldg = op->ldg;
  a.ldb = op->ldb;
  a.tau = op->tau;
  a.alpha = alpha;
  a.shift = 0.0;
  cudaError_t e = launch_block_jacobi(op->N, a, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("block-Jacobi launch: ") + cudaGetErrorString(e));
  CK(cudaStreamSynchronize((cudaStream_t)stream));
  int rc = check_status(op);
  if (rc != DDG_OK) return rc;
  op->pc_ready = true;
  op->pc_alpha = alpha;
  return DDG_OK;
}

extern "C" int ddg_sipg_pc_apply(ddg_sipg_op* op, int prec, const void* r, void* z, void* stream) {
  if (!op || !r || !z) return fail(DDG_ERR_INVALID, "ddg_sipg_pc_apply: null argument");
  if (!op->pc_ready) return fail(DDG_ERR_INVALID, "ddg_sipg_pc_apply: preconditioner not built");
  DevGuard guard(op->dev);
  cudaError_t e;
  if (prec == DDG_FP64)
    e = launch_pc_apply<double>(op->N, (const double*)r, (double*)z, op->binv64, op->ldb, op->K, (cudaStream_t)stream);
  else
    e = launch_pc_apply<float>(op->N, (const float*)r, (float*)z, op->binv32, op->ldb, op->K, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("pc apply launch: ") + cudaGetErrorString(e));
  return DDG_OK;
}

extern "C" int ddg_sipg_pc_blocks(ddg_sipg_op* op, double* blocks, void* stream) {
  if (!op || !blocks) return fail(DDG_ERR_INVALID, "ddg_sipg_pc_blocks: null argument");
  if (!op->pc_ready) return fail(DDG_ERR_INVALID, "ddg_sipg_pc_blocks: preconditioner not built");
  DevGuard guard(op->dev);
  CK(cudaMemcpyAsync(blocks, op->blocks, (size_t)op->K * op->Np * op->Np * 8, cudaMemcpyDeviceToDevice,
                     (cudaStream_t)stream));
  return DDG_OK;
}

extern "C" int ddg_sipg_cg(ddg_sipg_op* op, const ddg_cg_config* cfg, const void* b, void* x, void* stream,
                           ddg_solve_info* info) {
  if (!op || !cfg || !b || !x) return fail(DDG_ERR_INVALID, "ddg_sipg_cg: null argument");
  if (cfg->precision != DDG_FP64 && cfg->precision != DDG_FP32)
    return fail(DDG_ERR_INVALID, "ddg_sipg_cg: bad precision");
  if (cfg->maxiter < 0 || !(cfg->tol >= 0) || !(cfg->atol >= 0))
    return fail(DDG_ERR_INVALID, "ddg_sipg_cg: tol/atol/maxiter must be non-negative");
  if (cfg->pc != DDG_PC_NONE && cfg->pc != DDG_PC_JACOBI) return fail(DDG_ERR_UNSUPPORTED, "ddg_sipg_cg: pc kind");
  if (cfg->pc == DDG_PC_JACOBI && !op->pc_ready) return fail(DDG_ERR_INVALID, "ddg_sipg_cg: preconditioner not built");
  if (cfg->pc == DDG_PC_JACOBI && op->pc_alpha != cfg->alpha)
    return fail(DDG_ERR_INVALID, "ddg_sipg_cg: preconditioner was built for another alpha");
  DevGuard guard(op->dev);
  const int prec = cfg->precision;
  int rc = ensure_work(op, prec);
  if (rc != DDG_OK) return rc;
  Work& w = op->w[prec];
  cudaStream_t s = (cudaStream_t)stream;
  GraphKey key{prec, cfg->pc, cfg->alpha, cfg->shift};
  CgGraph* gr = nullptr;
  rc = get_graph(op, key, &gr);
  if (rc != DDG_OK) return rc;

  CgCtl h{};
  h.tol2 = cfg->tol * cfg->tol;
  h.atol_sq = cfg->atol * cfg->atol;
  h.maxiter = cfg->maxiter;
  h.use_pc = cfg->pc != DDG_PC_NONE;
  h.cont = 1;
  CK(cudaMemcpyAsync(op->ctl, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(w.b, b, w.bytes, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(w.x, x, w.bytes, cudaMemcpyDeviceToDevice, s));
  cudaError_t e;
  // r = b - (alpha M + A + shift) x0 ; z = B^-1 r ; gamma = r.z ; p_old = 0
  if (prec == DDG_FP64) {
    ApplyArgs<double> a = apply_args<double>(op);
    a.in0 = (const double*)w.x;
    a.in1 = (const double*)w.b;
    a.out0 = (double*)w.r;
    a.alpha = cfg->alpha;
    a.shift = cfg->shift;
    a.use_tma = 1;
    e = launch_apply<double>(op->N, AM_RESID, a, s);
    CgArgs<double> c{};
    c.r = (double*)w.r;
    c.z = cfg->pc ? (double*)w.z : (double*)w.r;
    c.p_zero = (double*)w.p0;
    c.binv = op->binv64;
    c.ldb = op->ldb;
    c.ctl = op->ctl;
    c.partA = op->partA;
    c.partB = op->partB;
    c.K = op->K;
    c.dev_status = op->status;
    if (e == cudaSuccess) e = launch_cg_step<double>(op->N, cfg->pc != 0, true, c, s);
  } else {
    ApplyArgs<float> a = apply_args<float>(op);
    a.in0 = (const float*)w.x;
    a.in1 = (const float*)w.b;
    a.out0 = (float*)w.r;
    a.alpha = cfg->alpha;
    a.shift = cfg->shift;
    a.use_tma = 1;
    e = launch_apply<float>(op->N, AM_RESID, a, s);
    CgArgs<float> c{};
    c.r = (float*)w.r;
    c.z = cfg->pc ? (float*)w.z : (float*)w.r;
    c.p_zero = (float*)w.p0;
    c.binv = op->binv32;
    c.ldb = op->ldb;
    c.ctl = op->ctl;
    c.partA = op->partA;
    c.partB = op->partB;
    c.K = op->K;
    c.dev_status = op->status;
    if (e == cudaSuccess) e = launch_cg_step<float>(op->N, cfg->pc != 0, true, c, s);
  }
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("CG init launch: ") + cudaGetErrorString(e));
  CK(cudaGraphLaunch(gr->exec, s));
  CK(cudaMemcpyAsync(x, w.x, w.bytes, cudaMemcpyDeviceToDevice, s));
  CgCtl res{};
  CK(cudaMemcpyAsync(&res, op->ctl, sizeof(res), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  rc = check_status(op);
  if (rc != DDG_OK) return rc;
  if (info) {
    info->status = res.status;
    info->iterations = res.iter;
    info->res_norm2 = res.use_pc ? res.rr : res.gamma;
    info->b_norm2 = res.bb;
  }
  return DDG_OK;
}

extern "C" int ddg_axpby(int64_t n, double a, const double* x, double b, double* y, void* stream) {
  if (n < 0 || (n > 0 && (!x || !y))) return fail(DDG_ERR_INVALID, "ddg_axpby: bad argument");
  if (n == 0) return DDG_OK;
  cudaError_t e = launch_axpby(n, a, x, b, y, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("axpby: ") + cudaGetErrorString(e));
  return DDG_OK;
}

extern "C" int ddg_cast(int64_t n, int to_prec, const void* src, void* dst, void* stream) {
  if (n < 0 || (n > 0 && (!src || !dst))) return fail(DDG_ERR_INVALID, "ddg_cast: bad argument");
  if (to_prec != DDG_FP64 && to_prec != DDG_FP32) return fail(DDG_ERR_INVALID, "ddg_cast: bad precision");
  if (n == 0) return DDG_OK;
  cudaError_t e = launch_cast(n, to_prec, src, dst, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("cast: ") + cudaGetErrorString(e));
  return DDG_OK;
}

namespace {
std::mutex g_dot_mu;
std::map<int, std::pair<double*, unsigned int*>> g_dot_scratch;  // per device
}  // namespace

extern "C" int ddg_dot(int64_t n, int prec, const void* x, const void* y, double* out, void* stream) {
  if (n < 0 || !out || (n > 0 && (!x || !y))) return fail(DDG_ERR_INVALID, "ddg_dot: bad argument");
  if (prec != DDG_FP64 && prec != DDG_FP32) return fail(DDG_ERR_INVALID, "ddg_dot: bad precision");
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::pair<double*, unsigned int*> sc;
  {
    std::lock_guard<std::mutex> lk(g_dot_mu);
    auto it = g_dot_scratch.find(dev);
    if (it == g_dot_scratch.end()) {
      double* part = nullptr;
      unsigned int* t = nullptr;
      CK(cudaMalloc((void**)&part, (148 * 16 + 32) * sizeof(double)));
      CK(cudaMalloc((void**)&t, sizeof(unsigned int)));
      CK(cudaMemset(t, 0, sizeof(unsigned int)));
      it = g_dot_scratch.emplace(dev, std::make_pair(part, t)).first;
    }
    sc = it->second;
  }
  if (n == 0) {
    CK(cudaMemsetAsync(out, 0, sizeof(double), (cudaStream_t)stream));
    return DDG_OK;
  }
  cudaError_t e = launch_dot(n, prec, x, y, sc.first, sc.second, out, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("dot: ") + cudaGetErrorString(e));
  return DDG_OK;
}
