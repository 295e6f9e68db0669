// C-ABI implementation: handle lifetime, uploads, and the entry points of
// include/ddg_sipg.h.  No exception crosses the boundary; every CUDA error
// becomes a status code plus a thread-local message.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <cstddef>
#include <map>
#include <mutex>
#include <string>
#include <thread>
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
  int engine = 0;  // float32 apply engine captured in the graph
  bool operator<(const GraphKey& o) const {
    if (engine != o.engine) return engine < o.engine;
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

#ifndef DDG_HOST_PLAN
#define DDG_HOST_PLAN 1, 1, 1, 1, 1, 1, 1, 1   // relative chunk sizes of the host-buffer apply pipeline
#endif

// State of the host-buffer apply (ddg_sipg_apply_host), created on first use:
// node-major device copies of u and y, pinned staging for pageable host
// arrays, one stream per direction plus one for the kernels, and per-chunk
// events.  Each chunk's elements are applied in two pieces: the leading
// run whose neighbours all lie in chunks <= c (ready as soon as chunk c has
// arrived) and the rest; need[i] is the last chunk piece i reads through a
// face, so its kernel waits only for the host->device copies up to need[i].  With pinned host arrays the
// whole chunked pipeline (about 8 API calls per chunk) is captured once per
// (u, y, alpha) into a CUDA graph and replayed with one launch.
struct HostIO {
  double* d_u = nullptr;   // node-major input, as copied from the host
  double* d_y = nullptr;   // node-major output, copied to the host
  double* e_u = nullptr;   // element-major input (transposed on the device)
  double* e_y = nullptr;   // element-major output of the apply
  double* h_u = nullptr;   // pinned staging (pageable input)
  double* h_y = nullptr;   // pinned staging (pageable output)
  cudaStream_t s_in = nullptr, s_cmp = nullptr, s_out = nullptr;
  cudaEvent_t e_start = nullptr;
  std::vector<cudaEvent_t> e_in, e_cmp, e_out;
  std::vector<int> need;                 // per piece (2 per chunk), running maximum
  std::vector<int> p_lo, p_hi;           // piece element ranges
  int nch = 0;
  std::vector<int> bounds;               // chunk c covers elements [bounds[c], bounds[c + 1])
  int chunk_of(int k) const { return (int)(std::upper_bound(bounds.begin(), bounds.end(), k) - bounds.begin()) - 1; }
  cudaStream_t s_org = nullptr;       // capture origin of the pipeline graph
  cudaGraphExec_t gexec = nullptr;    // the captured pipeline for (g_u, g_y, g_alpha)
  const double* g_u = nullptr;
  double* g_y = nullptr;
  double g_alpha = 0.0;
  bool g_ok = false;
};

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
  double* partC = nullptr;
  unsigned int* ticket = nullptr;   // for the free dot helper
  double* dotbuf = nullptr;
  // block Jacobi
  double* kappa64 = nullptr;        // per-element diffusivity (extension)
  float* kappa32 = nullptr;
  bool kappa_on = false;
  double* blocks = nullptr;
  double* binv64 = nullptr;
  float* binv32 = nullptr;
  bool pc_ready = false;
  double pc_alpha = 0.0;
  Work w[2];
  std::map<GraphKey, CgGraph> graphs;
  std::map<std::pair<void*, GraphKey>, CgGraph> mg_graphs;   // CG with a multigrid preconditioner
  cudaStream_t cap = nullptr;       // private stream for graph capture
  // host copies for set_bc
  std::vector<int64_t> EToE, EToF, vmapP;
  std::vector<int64_t> rot;         // (3, Np)
  std::vector<uint32_t> nbr_host;
  HostIO* hio = nullptr;            // host-buffer apply state (lazy)
  uint8_t* tc_img = nullptr;        // tensor-core B operands of this degree (device)
  int fp32_engine = DDG_ENGINE_TENSOR_CORES;   // stand-alone float32 applies
  int cg32_engine = DDG_ENGINE_TENSOR_CORES;   // float32 CG iterations (CUDA cores where no tensor-core apply is built)
  double* dm_img = nullptr;         // FP64 tensor-core (DMMA) B operands of this degree (device)
  double* dm_geo = nullptr;         // that kernel's element and face coefficients (device)
  int fp64_engine = DDG_ENGINE_TENSOR_CORES;   // every float64 apply (stand-alone, CG, residuals)
  std::vector<ddg_mg*> mgs;         // multigrid objects whose V-cycle is embedded in this handle's CG graphs
};

// Defined after struct ddg_mg: removes op from mg's list of graph holders.
static void mg_forget_user(ddg_mg* mg, ddg_sipg_op* op);

namespace {

}  // namespace

// Neighbour words of K elements (nbr_pack layout, out[f * out_ld + k]);
// element ids inside the words are shifted by k_offset (pools place a
// request's elements at [k_offset, k_offset + K)).
int ddg::pack_neighbours(int K, int N, const int64_t* EToE, const int64_t* EToF, const int64_t* vmapP,
                         const int64_t* rot, const int32_t* bc, uint32_t k_offset, uint32_t* out, size_t out_ld) {
  const int Np = (N + 1) * (N + 2) / 2, Nfp = N + 1;
  for (int k = 0; k < K; ++k)
    for (int f = 0; f < 3; ++f) {
      const int64_t kp = EToE[(size_t)k * 3 + f], fp = EToF[(size_t)k * 3 + f];
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
          const int64_t j = vmapP[((size_t)k * 3 + f) * Nfp + p];
          if (j / Np != kp) return fail(DDG_ERR_INVALID, "vmapP does not point into the EToE neighbour (non-conforming face)");
          const int64_t loc = j % Np;
          int q = -1;
          for (int qq = 0; qq < Nfp; ++qq)
            if (rot[(size_t)fp * Np + qq] == loc) q = qq;
          if (q == p) ++nsame;
          if (q == N - p) ++nrev;
        }
        if (nrev == Nfp) flip = true;
        else if (nsame != Nfp) return fail(DDG_ERR_INVALID, "face node matching is neither aligned nor reversed");
      }
      // a self-pointing face tagged interior contributes nothing (its jump
      // vanishes and its two scatters cancel: sipg.py:241-249)
      out[(size_t)f * out_ld + k] =
          nbr_pack((uint32_t)(kp + k_offset), (uint32_t)fp, flip, (uint32_t)tag, pact, mint);
    }
  return DDG_OK;
}

namespace {

int build_nbr(ddg_sipg_op* op, const int32_t* bc) {
  op->nbr_host.assign((size_t)3 * op->K, 0u);
  return ddg::pack_neighbours(op->K, op->N, op->EToE.data(), op->EToF.data(), op->vmapP.data(), op->rot.data(), bc, 0u,
                         op->nbr_host.data(), (size_t)op->K);
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
  a.kappa = op->kappa_on ? ((sizeof(T) == 8) ? (const T*)op->kappa64 : (const T*)op->kappa32) : nullptr;
  if (sizeof(T) == 8 && op->fp64_engine == DDG_ENGINE_TENSOR_CORES) {
    a.dm_img = op->dm_img;
    a.dm_geo = op->dm_geo;
  }
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

// Two CG iterations (the p ping-pong) of the loop body on stream st: with
// has_cond the step kernel also sets the graph's loop condition.
template <typename T>
cudaError_t issue_body(ddg_sipg_op* op, const GraphKey& key, cudaStream_t st, int has_cond,
                       cudaGraphConditionalHandle h) {
  Work& w = op->w[key.prec];
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
  c.partC = op->partC;
  c.K = op->K;
  c.dev_status = op->status;
  c.has_cond = has_cond;
  c.bulk = 1;  // workspace vectors come from cudaMalloc (256-byte aligned)
  c.cond = h;
  cudaError_t e = cudaSuccess;
  for (int half = 0; half < 2 && e == cudaSuccess; ++half) {
    void* pin = half == 0 ? w.p0 : w.p1;
    void* pout = half == 0 ? w.p1 : w.p0;
    a.in0 = (const T*)c.z;
    a.in1 = (const T*)pin;
    a.out0 = (T*)w.Ap;
    a.out1 = (T*)pout;
    if constexpr (sizeof(T) == 4) {
      if (key.engine == DDG_ENGINE_TENSOR_CORES) {
        // the direction first (one streaming pass), then the tensor-core
        // apply of the formed direction with the p.Ap reduction: its
        // neighbour gathers read one vector instead of two
        // (programmatic dependent launches: each kernel waits for its
        // predecessor on the device, so launches overlap the previous tail)
        e = launch_pupd((int64_t)op->K * op->Np, (const float*)c.z, (const float*)pin, (float*)pout, op->ctl,
                        st, has_cond);
        if (e == cudaSuccess) {
          a.in0 = (const T*)pout;
          a.in1 = nullptr;
          a.out1 = nullptr;
          a.pdl = has_cond;
          e = launch_apply_tc(op->N, AM_PDOT, a, op->tc_img, st);
          a.pdl = 0;
          c.pdl = has_cond;
        }
      } else {
        e = launch_apply<T>(op->N, AM_PFUSE, a, st);
      }
    } else {
      // float64 on the FP64 tensor cores: programmatic dependent launches
      // as in the float32 body (the CUDA-core kernel keeps plain launches)
      const bool dm = key.engine == DDG_ENGINE_TENSOR_CORES && op->dm_img;
      a.pdl = dm ? has_cond : 0;
      e = launch_apply<T>(op->N, AM_PFUSE, a, st);
      a.pdl = 0;
      c.pdl = dm ? has_cond : 0;
    }
    if (e != cudaSuccess) break;
    c.p = (const T*)pout;
    e = launch_cg_step<T>(op->N, key.pc != 0, false, c, st);
    c.pdl = 0;
  }
  return e;
}

template <typename T>
int capture_body(ddg_sipg_op* op, const GraphKey& key, cudaGraph_t body, cudaGraphConditionalHandle h) {
  CK(cudaStreamBeginCaptureToGraph(op->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  const cudaError_t e = issue_body<T>(op, key, op->cap, 1, h);
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
  for (ddg_mg* mg : op->mgs) mg_forget_user(mg, op);   // the multigrid must not reach this handle again
  op->mgs.clear();
  for (auto& kv : op->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.g) cudaGraphDestroy(kv.second.g);
  }
  for (auto& kv : op->mg_graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.g) cudaGraphDestroy(kv.second.g);
  }
  if (op->tc_img) cudaFree(op->tc_img);
  if (op->dm_img) cudaFree(op->dm_img);
  if (op->dm_geo) cudaFree(op->dm_geo);

  void* ptrs[] = {op->kappa64 /* kappa32 lives in the same block */, op->geo64, op->geo32, op->nbr, op->perm, op->status, op->ctl, op->partA, op->partB, op->partC,
                  op->ticket, op->dotbuf, op->blocks, op->binv64, op->binv32};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (auto& w : op->w) {
    void* wp[] = {w.x, w.b, w.r, w.z, w.p0, w.p1, w.Ap};
    for (void* p : wp)
      if (p) cudaFree(p);
  }
  if (op->cap) cudaStreamDestroy(op->cap);
  if (HostIO* h = op->hio) {
    if (h->d_u) cudaFree(h->d_u);
    if (h->d_y) cudaFree(h->d_y);
    if (h->e_u) cudaFree(h->e_u);
    if (h->e_y) cudaFree(h->e_y);
    if (h->h_u) cudaFreeHost(h->h_u);
    if (h->h_y) cudaFreeHost(h->h_y);
    for (auto* v : {&h->e_in, &h->e_cmp, &h->e_out})
      for (cudaEvent_t ev : *v) cudaEventDestroy(ev);
    if (h->e_start) cudaEventDestroy(h->e_start);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    for (cudaStream_t st : {h->s_in, h->s_cmp, h->s_out, h->s_org})
      if (st) cudaStreamDestroy(st);
    delete h;
  }
  delete op;
}

}  // namespace

// ===================================================================== API
extern "C" const char* ddg_last_error(void) { return g_err.c_str(); }
extern "C" const char* ddg_version(void) { return "ddg_sipg 0.1 (sm_100a)"; }

// Reference-element matrices of degree N into constant memory of `device`
// (once per device and degree; later calls must pass the same matrices).
extern "C" int ddg_sipg_upload_reference(int N, const double* Dr, const double* Ds, const double* M,
                                         const double* m1d, int device) {
  if (N < 1 || N > DDG_MAX_DEGREE || !Dr || !Ds || !M || !m1d)
    return fail(DDG_ERR_INVALID, "reference matrices: bad arguments");
  const int Np = (N + 1) * (N + 2) / 2, Nfp = N + 1;
  std::lock_guard<std::mutex> lk(g_ref_mu);
  std::vector<double> blob;
  blob.insert(blob.end(), Dr, Dr + Np * Np);
  blob.insert(blob.end(), Ds, Ds + Np * Np);
  blob.insert(blob.end(), M, M + Np * Np);
  blob.insert(blob.end(), m1d, m1d + 3 * Nfp * Nfp);
  auto key = std::make_pair(device, N);
  auto it = g_ref_loaded.find(key);
  if (it == g_ref_loaded.end()) {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    cudaError_t e = upload_ref(N, Dr, Ds, M, m1d);
    if (e == cudaSuccess) e = cv_upload_ref(N, Dr, Ds, M, m1d);
    cudaSetDevice(cur);
    if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("constant upload: ") + cudaGetErrorString(e));
    g_ref_loaded[key] = blob;
    return DDG_OK;
  }
  for (size_t i = 0; i < blob.size(); ++i)
    if (std::fabs(blob[i] - it->second[i]) > 1e-12 * (1.0 + std::fabs(blob[i])))
      return fail(DDG_ERR_INVALID, "reference matrices differ from the ones already loaded for this degree");
  return DDG_OK;
}

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
    const int urc = ddg_sipg_upload_reference(N, d->Dr, d->Ds, d->M, d->m1d, d->device);
    if (urc != DDG_OK) {
      free_op(op);
      return urc;
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
  // partials: one per block of the largest grid (the bulk CG step of float64
  // runs 64-element blocks)
  const int np_parts = std::max(std::max(apply_grid(K), (K + 63) / 64), std::max(cg_grid(K), dot_grid((int64_t)K * Np))) + 32;
  ALLOC(op->partA, np_parts * sizeof(double));
  ALLOC(op->partB, np_parts * sizeof(double));
  ALLOC(op->partC, np_parts * sizeof(double));
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
  if (e == cudaSuccess && tc_supported(N)) {
    std::vector<uint8_t> img((size_t)tc_image_bytes(N), 0);
    tc_build_image(N, d->Dr, d->Ds, d->M, img.data());
    e = cudaMalloc((void**)&op->tc_img, img.size());
    if (e == cudaSuccess) e = cudaMemcpy(op->tc_img, img.data(), img.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = tc_prepare(N);
  }
  if (!op->tc_img) op->fp32_engine = op->cg32_engine = DDG_ENGINE_CUDA_CORES;
  if (e == cudaSuccess && dm_supported(N)) {
    std::vector<double> img((size_t)dm_image_doubles(N), 0.0);
    dm_build_image(N, d->Dr, d->Ds, d->M, d->m1d, img.data());
    e = cudaMalloc((void**)&op->dm_img, img.size() * sizeof(double));
    if (e == cudaSuccess)
      e = cudaMemcpy(op->dm_img, img.data(), img.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = dm_prepare(N);
    if (e == cudaSuccess) e = cudaMalloc((void**)&op->dm_geo, (size_t)dm_geo_fields() * op->ldg * sizeof(double));
    if (e == cudaSuccess) e = dm_build_geo(op->geo64, op->nbr, op->dm_geo, op->K, op->ldg, op->tau, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
  }
  if (!op->dm_img || !op->dm_geo) op->fp64_engine = DDG_ENGINE_CUDA_CORES;
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
  if (op->dm_geo) {
    CK(dm_build_geo(op->geo64, op->nbr, op->dm_geo, op->K, op->ldg, op->tau, nullptr));
    CK(cudaDeviceSynchronize());
  }
  op->pc_ready = false;
  if (op->hio) op->hio->need.clear();
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
    if (op->fp32_engine == DDG_ENGINE_TENSOR_CORES && op->tc_img && a.use_tma)
      e = launch_apply_tc(op->N, AM_APPLY, a, op->tc_img, s);
    else
      e = launch_apply<float>(op->N, AM_APPLY, a, s);
  } else {
    return fail(DDG_ERR_INVALID, "precision must be DDG_FP64 or DDG_FP32");
  }
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("apply launch: ") + cudaGetErrorString(e));
  return DDG_OK;
}

namespace {

// Lazily create the host-buffer apply state and (after a BC change) its
// chunk dependency table.
int hio_prepare(ddg_sipg_op* op) {
  const int K = op->K;
  if (!op->hio) {
    HostIO* h = new HostIO();
    op->hio = h;  // released by free_op even when set-up stops halfway
    // chunk plan (relative sizes of consecutive element chunks), measured on
    // B200 for the 16 MB-per-direction workload: 8 equal chunks 0.52 ms per
    // call; 4 equal 0.56; small first and last chunks (1,3,4,4,3,1 /
    // 1,2,2,2,2,2,2,1 / 1,3,3,1) 0.53-0.55; 16 equal 0.62
    std::vector<int> wts = {DDG_HOST_PLAN};
    int tot = 0;
    for (int x : wts) tot += x;
    if (K < 4096 * (int)wts.size()) wts.assign(1, 1), tot = 1;
    h->bounds.assign(1, 0);
    int acc = 0;
    for (size_t c = 0; c < wts.size(); ++c) {
      acc += wts[c];
      int b = c + 1 == wts.size() ? K : (int)((int64_t)K * acc / tot) / 64 * 64;  // 64-element tiles
      if (b > h->bounds.back()) h->bounds.push_back(b);
    }
    if (h->bounds.back() != K) h->bounds.back() = K;
    h->nch = (int)h->bounds.size() - 1;
    const size_t bytes = (size_t)K * op->Np * sizeof(double);
    CK(cudaMalloc((void**)&h->d_u, bytes));
    CK(cudaMalloc((void**)&h->d_y, bytes));
    CK(cudaMalloc((void**)&h->e_u, bytes));
    CK(cudaMalloc((void**)&h->e_y, bytes));
    CK(cudaStreamCreateWithFlags(&h->s_in, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&h->s_cmp, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&h->s_out, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&h->s_org, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&h->e_start, cudaEventDisableTiming));
    h->e_in.assign(h->nch, nullptr);
    h->e_cmp.assign(2 * h->nch, nullptr);
    h->e_out.assign(2 * h->nch, nullptr);
    for (auto* v : {&h->e_in, &h->e_cmp, &h->e_out})
      for (cudaEvent_t& ev : *v) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  }
  HostIO* h = op->hio;
  if (h->need.empty()) {
    // mx[k]: the last chunk element k reads (its own, or a neighbour's through
    // a face whose own-interior or neighbour-side bit is set)
    std::vector<int> mx(K);
    for (int k = 0; k < K; ++k) mx[k] = h->chunk_of(k);
    for (int f = 0; f < 3; ++f)
      for (int k = 0; k < K; ++k) {
        const uint32_t w = op->nbr_host[(size_t)f * K + k];
        if (w & (32u | 64u)) mx[k] = std::max(mx[k], h->chunk_of((int)(w >> 7)));
      }
    std::vector<int> need(2 * h->nch), lo(2 * h->nch), hi(2 * h->nch);
    for (int c = 0; c < h->nch; ++c) {
      const int c0 = h->bounds[c], c1 = h->bounds[c + 1];
      int p = c0;
      while (p < c1 && mx[p] <= c) ++p;
      if (p < c1) p = c0 + (p - c0) / 16 * 16;  // ranges of the tensor-core kernel start on 16-element blocks
      int tail = c;
      for (int k = p; k < c1; ++k) tail = std::max(tail, mx[k]);
      lo[2 * c] = c0, hi[2 * c] = p, need[2 * c] = c;
      lo[2 * c + 1] = p, hi[2 * c + 1] = c1, need[2 * c + 1] = tail;
    }
    for (size_t i = 1; i < need.size(); ++i) need[i] = std::max(need[i], need[i - 1]);
    h->need.swap(need);
    h->p_lo.swap(lo);
    h->p_hi.swap(hi);
    h->g_ok = false;  // the captured pipeline followed the old dependencies
  }
  return DDG_OK;
}

bool host_pinned(const void* p) {
  cudaPointerAttributes at{};
  const cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

}  // namespace

namespace {

// memcpy split over a few host threads (staging of pageable arrays: one
// thread moves far less than the memory bandwidth)
void par_copy(void* dst, const void* src, size_t bytes) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::min<size_t>(std::min(8u, hw), std::max<size_t>(1, bytes >> 21));
  const size_t piece = (bytes + nt - 1) / nt;
  std::vector<std::thread> pool;
  for (size_t t = 1; t < nt; ++t) {
    const size_t o = t * piece;
    if (o >= bytes) break;
    pool.emplace_back([=] { std::memcpy((char*)dst + o, (const char*)src + o, std::min(piece, bytes - o)); });
  }
  std::memcpy(dst, src, std::min(piece, bytes));
  for (auto& th : pool) th.join();
}

// Issue the chunked pipeline for pinned (or staged) host arrays src -> dst
// after the work already queued on `us`, and join it back into `us`.  Per
// element chunk: a pitched copy engine transfer of the chunk's Np row
// segments (few large chunks: copies in both directions then overlap), a
// transpose to the element-major layout in device memory, the element-major
// apply of every chunk whose neighbours have all arrived (the tensor-core
// kernel for float64 where built), the transpose back and the pitched copy
// to the host.  src and dst are pinned host arrays.
int hio_issue(ddg_sipg_op* op, double alpha, const double* src, double* dst, cudaStream_t us) {
  HostIO* h = op->hio;
  const int K = op->K, Np = op->Np;
  const size_t pitch = (size_t)K * sizeof(double);
  CK(cudaEventRecord(h->e_start, us));
  for (cudaStream_t st : {h->s_in, h->s_cmp, h->s_out}) CK(cudaStreamWaitEvent(st, h->e_start, 0));
  ApplyArgs<double> a = apply_args<double>(op);
  a.in0 = h->e_u;
  a.out0 = h->e_y;
  a.alpha = alpha;
  a.use_tma = aligned16(h->e_u) && aligned16(h->e_y);
  int next = 0;
  for (int c = 0; c < h->nch; ++c) {
    const int c0 = h->bounds[c], c1 = h->bounds[c + 1];
    const size_t w = (size_t)(c1 - c0) * sizeof(double);
    CK(cudaMemcpy2DAsync(h->d_u + c0, pitch, src + c0, pitch, w, Np, cudaMemcpyHostToDevice, h->s_in));
    CK(cudaEventRecord(h->e_in[c], h->s_in));
    CK(cudaStreamWaitEvent(h->s_cmp, h->e_in[c], 0));
    cudaError_t e = launch_nm_to_em(h->d_u, h->e_u, K, Np, c0, c1, h->s_cmp);
    if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("transpose launch: ") + cudaGetErrorString(e));
    for (; next < 2 * h->nch && h->need[next] <= c; ++next) {
      const int j0 = h->p_lo[next], j1 = h->p_hi[next];
      if (j1 <= j0) continue;
      a.k_lo = j0;
      a.k_hi = j1;
      e = launch_apply<double>(op->N, AM_APPLY, a, h->s_cmp);
      if (e == cudaSuccess) e = launch_em_to_nm(h->e_y, h->d_y, K, Np, j0, j1, h->s_cmp);
      if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("apply launch: ") + cudaGetErrorString(e));
      CK(cudaEventRecord(h->e_cmp[next], h->s_cmp));
      CK(cudaStreamWaitEvent(h->s_out, h->e_cmp[next], 0));
      CK(cudaMemcpy2DAsync(dst + j0, pitch, h->d_y + j0, pitch, (size_t)(j1 - j0) * sizeof(double), Np,
                           cudaMemcpyDeviceToHost, h->s_out));
      CK(cudaEventRecord(h->e_out[next], h->s_out));
    }
  }
  // join: every stream's last piece covers everything issued on it
  int last = 2 * h->nch - 1;
  while (last > 0 && h->p_hi[last] <= h->p_lo[last]) --last;
  CK(cudaStreamWaitEvent(us, h->e_in[h->nch - 1], 0));
  CK(cudaStreamWaitEvent(us, h->e_cmp[last], 0));
  CK(cudaStreamWaitEvent(us, h->e_out[last], 0));
  return DDG_OK;
}

// Capture the pinned-array pipeline for (u, y, alpha) into h->gexec.
int hio_capture(ddg_sipg_op* op, double alpha, const double* u, double* y) {
  HostIO* h = op->hio;
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  h->gexec = nullptr;
  h->g_ok = false;
  CK(cudaStreamBeginCapture(h->s_org, cudaStreamCaptureModeThreadLocal));
  const int rc = hio_issue(op, alpha, u, y, h->s_org);
  cudaGraph_t g = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(h->s_org, &g);
  if (rc != DDG_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e2 != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("host-buffer graph capture: ") + cudaGetErrorString(e2));
  const cudaError_t e3 = cudaGraphInstantiate(&h->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e3 != cudaSuccess) {
    h->gexec = nullptr;
    return fail(DDG_ERR_CUDA, std::string("host-buffer graph instantiate: ") + cudaGetErrorString(e3));
  }
  h->g_u = u;
  h->g_y = y;
  h->g_alpha = alpha;
  h->g_ok = true;
  return DDG_OK;
}

}  // namespace

extern "C" int ddg_sipg_apply_host(ddg_sipg_op* op, double alpha, const double* u, double* y, void* stream) {
  if (!op || !u || !y) return fail(DDG_ERR_INVALID, "ddg_sipg_apply_host: null argument");
  if ((const void*)u == (const void*)y) return fail(DDG_ERR_INVALID, "ddg_sipg_apply_host: u and y must not alias");
  DevGuard guard(op->dev);
  int rc = hio_prepare(op);
  if (rc != DDG_OK) return rc;
  HostIO* h = op->hio;
  const int K = op->K, Np = op->Np;
  const size_t bytes = (size_t)K * Np * sizeof(double);
  const bool u_pin = host_pinned(u), y_pin = host_pinned(y);
  cudaStream_t us = (cudaStream_t)stream;
  // pageable arrays go through the pinned staging buffers (multi-threaded
  // host copies); the pinned arrays' pipeline is replayed from a graph
  if (!u_pin && !h->h_u) CK(cudaMallocHost((void**)&h->h_u, bytes));
  if (!y_pin && !h->h_y) CK(cudaMallocHost((void**)&h->h_y, bytes));
  const double* src = u_pin ? u : h->h_u;
  double* dst = y_pin ? y : h->h_y;
  if (!u_pin) par_copy(h->h_u, u, bytes);
  if (!(h->g_ok && h->g_u == src && h->g_y == dst && h->g_alpha == alpha)) {
    rc = hio_capture(op, alpha, src, dst);
    if (rc != DDG_OK) return rc;
  }
  CK(cudaGraphLaunch(h->gexec, us));
  CK(cudaStreamSynchronize(us));
  if (!y_pin) par_copy(y, h->h_y, bytes);
  return DDG_OK;
}

extern "C" int ddg_sipg_set_engine(ddg_sipg_op* op, int engine) {
  if (!op) return fail(DDG_ERR_INVALID, "ddg_sipg_set_engine: null handle");
  // The captured host-buffer pipeline baked in the previous engine's kernel.
  if (op->hio) op->hio->g_ok = false;
  if (engine == DDG_ENGINE_CUDA_CORES) {
    op->fp32_engine = op->cg32_engine = op->fp64_engine = engine;
    return DDG_OK;
  }
  if (engine == DDG_ENGINE_TENSOR_CORES) {
    if (!op->tc_img && !op->dm_img)
      return fail(DDG_ERR_UNSUPPORTED, "no tensor-core apply is built for this degree");
    if (op->tc_img) op->fp32_engine = op->cg32_engine = engine;
    if (op->dm_img) op->fp64_engine = engine;
    return DDG_OK;
  }
  return fail(DDG_ERR_INVALID, "engine must be DDG_ENGINE_CUDA_CORES or DDG_ENGINE_TENSOR_CORES");
}

extern "C" int ddg_sipg_rhs(ddg_sipg_op* op, const double* f, const double* u_dir, const double* q_neu,
                            double* rhs, void* stream) {
  if (!op || !rhs) return fail(DDG_ERR_INVALID, "ddg_sipg_rhs: null argument");
  if (op->kappa_on && u_dir)
    return fail(DDG_ERR_UNSUPPORTED, "ddg_sipg_rhs: non-homogeneous Dirichlet data with a diffusivity is not built");
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
    const size_t nsym = (size_t)op->Np * (op->Np + 1) / 2;
    CK(cudaMalloc((void**)&op->binv64, nsym * op->ldb * 8));
    CK(cudaMalloc((void**)&op->binv32, nsym * op->ldb * 4));
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
  a.kappa = op->kappa_on ? op->kappa64 : nullptr;
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
  key.engine = prec == DDG_FP32 ? (op->tc_img ? op->cg32_engine : DDG_ENGINE_CUDA_CORES) : op->fp64_engine;
  // DDG_CG_EAGER=1: launch the iteration kernels directly, checking the loop
  // flag from the host every 16 iterations, instead of the conditional graph
  // (same kernels and results; profilers cannot see into conditional graphs)
  static const bool eager = [] {
    const char* v = std::getenv("DDG_CG_EAGER");
    return v && v[0] == '1';
  }();
  CgGraph* gr = nullptr;
  if (!eager) {
    rc = get_graph(op, key, &gr);
    if (rc != DDG_OK) return rc;
  }

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
    c.partC = op->partC;
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
    c.partC = op->partC;
    c.K = op->K;
    c.dev_status = op->status;
    if (e == cudaSuccess) e = launch_cg_step<float>(op->N, cfg->pc != 0, true, c, s);
  }
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("CG init launch: ") + cudaGetErrorString(e));
  if (eager) {
    // every kernel returns at once when the loop flag is down, and the step
    // lowers it at maxiter, so the loop ends within 16 iterations of that
    for (int it = 0; it < cfg->maxiter + 16; it += 2) {
      e = prec == DDG_FP64 ? issue_body<double>(op, key, s, 0, cudaGraphConditionalHandle{})
                           : issue_body<float>(op, key, s, 0, cudaGraphConditionalHandle{});
      if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("CG iteration launch: ") + cudaGetErrorString(e));
      if (it % 16 == 14) {
        int cont = 0;
        CK(cudaMemcpyAsync(&cont, &op->ctl->cont, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (!cont) break;
      }
    }
  } else {
    CK(cudaGraphLaunch(gr->exec, s));
  }
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

extern "C" int ddg_sipg_cg_mixed(ddg_sipg_op* op, const ddg_cg_config* cfg, double delta, const double* b,
                                 double* x, void* stream, ddg_solve_info* info) {
  if (!op || !cfg || !b || !x) return fail(DDG_ERR_INVALID, "ddg_sipg_cg_mixed: null argument");
  if (cfg->maxiter < 0 || !(cfg->tol >= 0) || !(cfg->atol >= 0) || !(delta > 0.0 && delta < 1.0))
    return fail(DDG_ERR_INVALID, "ddg_sipg_cg_mixed: need tol, atol, maxiter >= 0 and 0 < delta < 1");
  if (cfg->pc != DDG_PC_NONE && cfg->pc != DDG_PC_JACOBI) return fail(DDG_ERR_UNSUPPORTED, "ddg_sipg_cg_mixed: pc kind");
  if (cfg->pc == DDG_PC_JACOBI && (!op->pc_ready || op->pc_alpha != cfg->alpha))
    return fail(DDG_ERR_INVALID, "ddg_sipg_cg_mixed: block-Jacobi preconditioner missing or built for another alpha");
  DevGuard guard(op->dev);
  int rc = ensure_work(op, DDG_FP64);
  if (rc == DDG_OK) rc = ensure_work(op, DDG_FP32);
  if (rc != DDG_OK) return rc;
  Work& w64 = op->w[DDG_FP64];
  Work& w32 = op->w[DDG_FP32];
  GraphKey key{DDG_FP32, cfg->pc, cfg->alpha, cfg->shift};
  key.engine = op->tc_img ? op->cg32_engine : DDG_ENGINE_CUDA_CORES;
  CgGraph* gr = nullptr;
  rc = get_graph(op, key, &gr);
  if (rc != DDG_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t n = (int64_t)op->K * op->Np;
  CK(cudaMemcpyAsync(w64.b, b, w64.bytes, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(w64.x, x, w64.bytes, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemsetAsync(op->ctl, 0, sizeof(CgCtl), s));

  ApplyArgs<double> ra = apply_args<double>(op);
  ra.in0 = (const double*)w64.x;
  ra.in1 = (const double*)w64.b;
  ra.out0 = (double*)w64.r;
  ra.alpha = cfg->alpha;
  ra.shift = cfg->shift;
  ra.use_tma = 1;
  CgArgs<float> ci{};
  ci.r = (float*)w32.r;
  ci.z = cfg->pc ? (float*)w32.z : (float*)w32.r;
  ci.p_zero = (float*)w32.p0;
  ci.binv = op->binv32;
  ci.ldb = op->ldb;
  ci.ctl = op->ctl;
  ci.partA = op->partA;
  ci.partB = op->partB;
  ci.partC = op->partC;
  ci.dev_status = op->status;
  ci.K = op->K;

  double target = -1.0;
  std::vector<double> hist;
  int total = 0, updates = 0, status = DDG_SOLVE_MAXITER;
  double rr_last = 0.0, bb0 = 0.0;
  for (int outer = 0; outer < 100000; ++outer) {
    // float64 true residual r = b - (alpha M + A + shift) x
    cudaError_t e = launch_apply<double>(op->N, AM_RESID, ra, s);
    if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("residual launch: ") + cudaGetErrorString(e));
    CgCtl h{};
    CK(cudaMemcpyAsync(&h, op->ctl, sizeof(h), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (target < 0.0) {
      bb0 = h.bb;
      target = std::fmax(cfg->tol * cfg->tol * h.bb, cfg->atol * cfg->atol);
    }
    rr_last = h.rr;
    hist.push_back(h.rr);
    if (!std::isfinite(h.rr)) {
      status = DDG_SOLVE_BREAKDOWN;
      break;
    }
    if (h.rr <= target) {
      status = DDG_SOLVE_CONVERGED;
      break;
    }
    if (total >= cfg->maxiter) {
      status = DDG_SOLVE_MAXITER;
      break;
    }
    // stagnation: the last three replacements together reduced r.r by less
    // than 10 % (each float32 solve asks for a reduction by delta)
    const size_t m = hist.size();
    if (m >= 4 && hist[m - 1] > 0.9 * hist[m - 4]) {
      status = DDG_SOLVE_STAGNATED;
      break;
    }
    // float32 restart from the float64 residual, keeping the direction
    struct {
      double tol2, atol_sq;
    } tl{delta * delta, 0.0};
    struct {
      int iter, maxiter, status, use_pc, cont;
    } it{0, cfg->maxiter - total, 0, cfg->pc != DDG_PC_NONE, 1};
    CK(cudaMemcpyAsync((char*)op->ctl + offsetof(CgCtl, tol2), &tl, sizeof(tl), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync((char*)op->ctl + offsetof(CgCtl, iter), &it, sizeof(it), cudaMemcpyHostToDevice, s));
    e = launch_cast_norm(n, (const double*)w64.r, (float*)w32.r, (float*)w32.x, op->partA, op->ctl, s);
    ci.keep_p = updates > 0 ? 1 : 0;
    if (e == cudaSuccess) e = launch_cg_step<float>(op->N, cfg->pc != 0, true, ci, s);
    if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("mixed restart launch: ") + cudaGetErrorString(e));
    CK(cudaGraphLaunch(gr->exec, s));
    CgCtl h2{};
    CK(cudaMemcpyAsync(&h2, op->ctl, sizeof(h2), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    total += h2.iter;
    // the ping-pong body leaves the newest direction in p1 after an odd count
    if (h2.iter % 2 == 1) CK(cudaMemcpyAsync(w32.p0, w32.p1, w32.bytes, cudaMemcpyDeviceToDevice, s));
    e = launch_axpy_mixed(n, (const float*)w32.x, (double*)w64.x, s);
    if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("mixed update launch: ") + cudaGetErrorString(e));
    ++updates;
    if (h2.status == 2 || h2.status == 3) {
      status = h2.status == 3 ? DDG_SOLVE_DEVICE_ERR : DDG_SOLVE_BREAKDOWN;
      break;
    }
    if (h2.iter == 0) {
      status = DDG_SOLVE_STAGNATED;
      break;
    }
  }
  CK(cudaMemcpyAsync(x, w64.x, w64.bytes, cudaMemcpyDeviceToDevice, s));
  CK(cudaStreamSynchronize(s));
  rc = check_status(op);
  if (rc != DDG_OK) return rc;
  if (info) {
    info->status = status;
    info->iterations = total;
    info->res_norm2 = rr_last;
    info->b_norm2 = bb0;
    info->updates = updates;
  }
  return DDG_OK;
}

// =========================================================== multigrid
struct ddg_mg {
  int L = 0, prec = 1, nu = 2, dev = 0;
  double omega = 0.7, alpha = 0.0;
  std::vector<ddg_sipg_op*> ops;
  struct Lv {
    int n = 0, Kc = 0, prow = 0, pcol = 0;   // Kc: K of the next coarser level
    void *x = nullptr, *t = nullptr, *b = nullptr, *r = nullptr;
    void *P = nullptr, *R = nullptr;          // prolongation / restriction (MG precision)
  };

  std::vector<Lv> lv;
  void* Ainv = nullptr;
  int nc = 0;
  CgCtl* sctl = nullptr;                     // scratch control block for residual kernels
  double *spa = nullptr, *spb = nullptr;
  std::vector<ddg_sipg_op*> users;           // handles holding CG graphs that embed this V-cycle
};

static void mg_forget_user(ddg_mg* mg, ddg_sipg_op* op) {
  mg->users.erase(std::remove(mg->users.begin(), mg->users.end(), op), mg->users.end());
}

namespace {

template <typename T>
int mg_alloc(ddg_mg* mg, const ddg_mg_desc* d) {
  const size_t ts = sizeof(T);
  int maxK = 0;
  for (int l = 0; l < mg->L; ++l) maxK = std::max(maxK, mg->ops[l]->K);
  cudaError_t e = cudaSuccess;
  for (int l = 0; l < mg->L; ++l) {
    auto& v = mg->lv[l];
    v.n = mg->ops[l]->K * mg->ops[l]->Np;
    void** bufs[] = {&v.x, &v.t, &v.b, &v.r};
    for (void** p : bufs)
      if (e == cudaSuccess) e = cudaMalloc(p, (size_t)v.n * ts);
    if (l + 1 < mg->L) {
      const int rows = d->prolong_rows[l], cols = d->prolong_cols[l];
      std::vector<T> P((size_t)rows * cols), R((size_t)rows * cols);
      for (int i = 0; i < rows; ++i)
        for (int j = 0; j < cols; ++j) {
          P[(size_t)i * cols + j] = (T)d->prolong[l][(size_t)i * cols + j];
          R[(size_t)j * rows + i] = (T)d->prolong[l][(size_t)i * cols + j];
        }
      v.prow = rows;
      v.pcol = cols;
      v.Kc = mg->ops[l + 1]->K;
      if (e == cudaSuccess) e = cudaMalloc(&v.P, P.size() * ts);
      if (e == cudaSuccess) e = cudaMalloc(&v.R, R.size() * ts);
      if (e == cudaSuccess) e = cudaMemcpy(v.P, P.data(), P.size() * ts, cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = cudaMemcpy(v.R, R.data(), R.size() * ts, cudaMemcpyHostToDevice);
    }
  }
  const int nc = mg->lv[mg->L - 1].n;
  mg->nc = nc;
  std::vector<T> A((size_t)nc * nc);
  for (size_t i = 0; i < A.size(); ++i) A[i] = (T)d->coarse_inv[i];
  if (e == cudaSuccess) e = cudaMalloc(&mg->Ainv, A.size() * ts);
  if (e == cudaSuccess) e = cudaMemcpy(mg->Ainv, A.data(), A.size() * ts, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc((void**)&mg->sctl, sizeof(CgCtl));
  if (e == cudaSuccess) e = cudaMemset(mg->sctl, 0, sizeof(CgCtl));
  const int np = apply_grid(maxK) + 32;
  if (e == cudaSuccess) e = cudaMalloc((void**)&mg->spa, np * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&mg->spb, np * sizeof(double));
  if (e != cudaSuccess)
    return fail(e == cudaErrorMemoryAllocation ? DDG_ERR_NOMEM : DDG_ERR_CUDA,
                std::string("ddg_mg_create: ") + cudaGetErrorString(e));
  return DDG_OK;
}

void mg_free(ddg_mg* mg) {
  for (auto& v : mg->lv) {
    void* p[] = {v.x, v.t, v.b, v.r, v.P, v.R};
    for (void* q : p)
      if (q) cudaFree(q);
  }
  void* p[] = {mg->Ainv, mg->sctl, mg->spa, mg->spb};
  for (void* q : p)
    if (q) cudaFree(q);
  delete mg;
}

template <typename T>
ApplyArgs<T> mg_args(ddg_mg* mg, int l) {
  ApplyArgs<T> a = apply_args<T>(mg->ops[l]);
  a.ctl = mg->sctl;
  a.partA = mg->spa;
  a.partB = mg->spb;
  a.alpha = mg->alpha;
  a.use_tma = 1;
  a.binv = (sizeof(T) == 8) ? (const T*)mg->ops[l]->binv64 : (const T*)mg->ops[l]->binv32;
  a.ldb = mg->ops[l]->ldb;
  a.omega = mg->omega;
  return a;
}

// One V-cycle on level l: approximately solves A_l x = b_l (b_l in lv[l].b).
// Returns the buffer that holds x_l.  Only kernel launches: capturable.
template <typename T>
cudaError_t mg_vcycle(ddg_mg* mg, int l, cudaStream_t s, T** result) {
  auto& v = mg->lv[l];
  ddg_sipg_op* op = mg->ops[l];
  cudaError_t e;
  if (l == mg->L - 1) {   // coarse: x = A_c^-1 b (multigrid.py:227-228)
    e = launch_dense_gemv<T>(mg->nc, (const T*)mg->Ainv, (const T*)v.b, (T*)v.x, s);
    *result = (T*)v.x;
    return e;
  }
  T* A = (T*)v.x;
  T* B = (T*)v.t;
  const T* binv = (sizeof(T) == 8) ? (const T*)op->binv64 : (const T*)op->binv32;
  ApplyArgs<T> a = mg_args<T>(mg, l);
  // pre-smoothing from x = 0: the first sweep is x = omega B^-1 b
  if (mg->nu > 0) {
    e = launch_bj_scaled<T>(op->N, (const T*)v.b, A, binv, op->ldb, op->K, (T)mg->omega, s);
    if (e != cudaSuccess) return e;
  } else {
    e = cudaMemsetAsync(A, 0, (size_t)v.n * sizeof(T), s);
    if (e != cudaSuccess) return e;
  }
  for (int it = 1; it < mg->nu; ++it) {
    a.in0 = A; a.in1 = (const T*)v.b; a.out0 = B;
    if ((e = launch_apply<T>(op->N, AM_SMOOTH, a, s)) != cudaSuccess) return e;
    std::swap(A, B);
  }
  // coarse-grid correction
  a.in0 = A; a.in1 = (const T*)v.b; a.out0 = (T*)v.r;
  if ((e = launch_apply<T>(op->N, AM_RESID, a, s)) != cudaSuccess) return e;
  auto& c = mg->lv[l + 1];
  if ((e = launch_elem_matvec<T>(v.Kc, v.pcol, v.prow, (const T*)v.R, (const T*)v.r, (T*)c.b, 0, s)) != cudaSuccess)
    return e;
  T* xc = nullptr;
  if ((e = mg_vcycle<T>(mg, l + 1, s, &xc)) != cudaSuccess) return e;
  if ((e = launch_elem_matvec<T>(v.Kc, v.prow, v.pcol, (const T*)v.P, xc, A, 1, s)) != cudaSuccess) return e;
  for (int it = 0; it < mg->nu; ++it) {
    a.in0 = A; a.in1 = (const T*)v.b; a.out0 = B;
    if ((e = launch_apply<T>(op->N, AM_SMOOTH, a, s)) != cudaSuccess) return e;
    std::swap(A, B);
  }
  *result = A;
  return cudaSuccess;
}

// every smoothed level must still carry the smoother built for mg->alpha
int mg_check(ddg_mg* mg) {
  for (int l = 0; l + 1 < mg->L; ++l)
    if (!mg->ops[l]->pc_ready || mg->ops[l]->pc_alpha != mg->alpha)
      return fail(DDG_ERR_INVALID, "multigrid level " + std::to_string(l) +
                                       ": its block-Jacobi smoother was rebuilt for another alpha");
  return DDG_OK;
}

// z = V(r) with float64 r, z (casts around a float32 hierarchy)
cudaError_t mg_apply64(ddg_mg* mg, const double* r, double* z, cudaStream_t s) {
  const int64_t n = mg->lv[0].n;
  cudaError_t e;
  if (mg->prec == DDG_FP32) {
    if ((e = launch_cast(n, DDG_FP32, r, mg->lv[0].b, s)) != cudaSuccess) return e;
    float* res = nullptr;
    if ((e = mg_vcycle<float>(mg, 0, s, &res)) != cudaSuccess) return e;
    return launch_cast(n, DDG_FP64, res, z, s);
  }
  if ((e = cudaMemcpyAsync(mg->lv[0].b, r, n * 8, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
  double* res = nullptr;
  if ((e = mg_vcycle<double>(mg, 0, s, &res)) != cudaSuccess) return e;
  return cudaMemcpyAsync(z, res, n * 8, cudaMemcpyDeviceToDevice, s);
}

int get_mg_graph(ddg_sipg_op* op, ddg_mg* mg, const GraphKey& key, CgGraph** out) {
  auto k2 = std::make_pair((void*)mg, key);
  auto it = op->mg_graphs.find(k2);
  if (it != op->mg_graphs.end()) {
    *out = &it->second;
    return DDG_OK;
  }
  Work& w = op->w[DDG_FP64];
  const int64_t n = (int64_t)op->K * op->Np;
  CgGraph cg;
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
  ApplyArgs<double> a = apply_args<double>(op);
  a.alpha = key.alpha;
  a.shift = key.shift;
  a.use_tma = 1;
  cudaError_t e = cudaSuccess;
  for (int half = 0; half < 2 && e == cudaSuccess; ++half) {
    void* pin = half == 0 ? w.p0 : w.p1;
    void* pout = half == 0 ? w.p1 : w.p0;
    a.in0 = (const double*)w.z;
    a.in1 = (const double*)pin;
    a.out0 = (double*)w.Ap;
    a.out1 = (double*)pout;
    e = launch_apply<double>(op->N, AM_PFUSE, a, op->cap);
    if (e == cudaSuccess)
      e = launch_cg_xr<double>((double*)w.x, (const double*)pout, (double*)w.r, (const double*)w.Ap, n, op->ctl,
                               op->partA, op->cap);
    if (e == cudaSuccess) e = mg_apply64(mg, (const double*)w.r, (double*)w.z, op->cap);
    if (e == cudaSuccess)
      e = launch_cg_finish<double>(false, (const double*)w.r, (const double*)w.z, n, op->ctl, op->partA,
                                   op->status, 1, h, op->cap);
  }
  cudaGraph_t outg = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(op->cap, &outg);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    cudaGraphDestroy(cg.g);
    return fail(DDG_ERR_CUDA, std::string("MG-CG body capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  CK(cudaGraphInstantiate(&cg.exec, cg.g, 0));
  op->mg_graphs[k2] = cg;
  *out = &op->mg_graphs[k2];
  if (std::find(mg->users.begin(), mg->users.end(), op) == mg->users.end()) mg->users.push_back(op);
  if (std::find(op->mgs.begin(), op->mgs.end(), mg) == op->mgs.end()) op->mgs.push_back(mg);
  return DDG_OK;
}

}  // namespace

extern "C" int ddg_mg_create(const ddg_mg_desc* d, ddg_mg** out) {
  if (!d || !out || d->nlevels < 1 || !d->ops || !d->coarse_inv)
    return fail(DDG_ERR_INVALID, "ddg_mg_create: bad descriptor");
  if (d->precision != DDG_FP32 && d->precision != DDG_FP64) return fail(DDG_ERR_INVALID, "ddg_mg_create: precision");
  if (d->nu < 0 || !(d->omega > 0.0)) return fail(DDG_ERR_INVALID, "ddg_mg_create: nu >= 0, omega > 0");
  *out = nullptr;
  for (int l = 0; l < d->nlevels; ++l) {
    ddg_sipg_op* op = d->ops[l];
    if (!op) return fail(DDG_ERR_INVALID, "ddg_mg_create: null level handle");
    if (l + 1 < d->nlevels && (!op->pc_ready || op->pc_alpha != d->alpha))
      return fail(DDG_ERR_INVALID, "ddg_mg_create: level " + std::to_string(l) +
                                       " needs ddg_sipg_pc_build(alpha) for its smoother");
    if (op->dev != d->ops[0]->dev) return fail(DDG_ERR_INVALID, "ddg_mg_create: levels on different devices");
  }
  for (int l = 0; l + 1 < d->nlevels; ++l) {
    ddg_sipg_op *f = d->ops[l], *c = d->ops[l + 1];
    const int rows = d->prolong_rows[l], cols = d->prolong_cols[l];
    const bool pt = (f->K == c->K) && rows == f->Np && cols == c->Np;
    const bool ht = (f->K == 4 * c->K) && f->Np == c->Np && rows == 4 * f->Np && cols == c->Np;
    if (!pt && !ht || !d->prolong[l])
      return fail(DDG_ERR_INVALID, "ddg_mg_create: transfer " + std::to_string(l) +
                                       " is neither a p-transfer (same K) nor an h-transfer (K = 4 Kc)");
  }
  const int Lc = d->nlevels - 1;
  const int64_t nc = (int64_t)d->ops[Lc]->K * d->ops[Lc]->Np;
  if (nc > 20000) return fail(DDG_ERR_INVALID, "ddg_mg_create: coarsest level too large for a dense solve");
  DevGuard guard(d->ops[0]->dev);
  ddg_mg* mg = new ddg_mg();
  mg->L = d->nlevels;
  mg->prec = d->precision;
  mg->nu = d->nu;
  mg->omega = d->omega;
  mg->alpha = d->alpha;
  mg->dev = d->ops[0]->dev;
  mg->ops.assign(d->ops, d->ops + d->nlevels);
  mg->lv.resize(d->nlevels);
  const int rc = d->precision == DDG_FP32 ? mg_alloc<float>(mg, d) : mg_alloc<double>(mg, d);
  if (rc != DDG_OK) {
    mg_free(mg);
    return rc;
  }
  *out = mg;
  return DDG_OK;
}

extern "C" int ddg_mg_destroy(ddg_mg* mg) {
  if (!mg) return DDG_OK;
  DevGuard guard(mg->dev);
  cudaDeviceSynchronize();
  for (ddg_sipg_op* op : mg->users) {     // drop CG graphs that embed this V-cycle
    for (auto it = op->mg_graphs.begin(); it != op->mg_graphs.end();) {
      if (it->first.first == (void*)mg) {
        if (it->second.exec) cudaGraphExecDestroy(it->second.exec);
        if (it->second.g) cudaGraphDestroy(it->second.g);
        it = op->mg_graphs.erase(it);
      } else {
        ++it;
      }
    }
    op->mgs.erase(std::remove(op->mgs.begin(), op->mgs.end(), mg), op->mgs.end());
  }
  mg->users.clear();
  mg_free(mg);
  return DDG_OK;
}

extern "C" int ddg_mg_apply(ddg_mg* mg, const double* r, double* z, void* stream) {
  if (!mg || !r || !z) return fail(DDG_ERR_INVALID, "ddg_mg_apply: null argument");
  if (int rc = mg_check(mg)) return rc;
  DevGuard guard(mg->dev);
  cudaError_t e = mg_apply64(mg, r, z, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("ddg_mg_apply: ") + cudaGetErrorString(e));
  return DDG_OK;
}

extern "C" int ddg_sipg_cg_mg(ddg_sipg_op* op, const ddg_cg_config* cfg, ddg_mg* mg, const double* b, double* x,
                              void* stream, ddg_solve_info* info) {
  if (!op || !cfg || !mg || !b || !x) return fail(DDG_ERR_INVALID, "ddg_sipg_cg_mg: null argument");
  if (cfg->maxiter < 0 || !(cfg->tol >= 0) || !(cfg->atol >= 0))
    return fail(DDG_ERR_INVALID, "ddg_sipg_cg_mg: tol/atol/maxiter must be non-negative");
  if (mg->lv[0].n != op->K * op->Np || mg->ops[0]->N != op->N)
    return fail(DDG_ERR_INVALID, "ddg_sipg_cg_mg: finest multigrid level does not match the operator");
  if (mg->dev != op->dev) return fail(DDG_ERR_INVALID, "ddg_sipg_cg_mg: different devices");
  if (int rc0 = mg_check(mg)) return rc0;
  DevGuard guard(op->dev);
  int rc = ensure_work(op, DDG_FP64);
  if (rc != DDG_OK) return rc;
  Work& w = op->w[DDG_FP64];
  cudaStream_t s = (cudaStream_t)stream;
  GraphKey key{DDG_FP64, 99, cfg->alpha, cfg->shift};
  key.engine = op->fp64_engine;
  CgGraph* gr = nullptr;
  rc = get_mg_graph(op, mg, key, &gr);
  if (rc != DDG_OK) return rc;
  const int64_t n = (int64_t)op->K * op->Np;
  CgCtl h{};
  h.tol2 = cfg->tol * cfg->tol;
  h.atol_sq = cfg->atol * cfg->atol;
  h.maxiter = cfg->maxiter;
  h.use_pc = 1;
  h.cont = 1;
  h.zcoef = 1.0;
  CK(cudaMemcpyAsync(op->ctl, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(w.b, b, w.bytes, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(w.x, x, w.bytes, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemsetAsync(w.p0, 0, w.bytes, s));
  ApplyArgs<double> a = apply_args<double>(op);
  a.in0 = (const double*)w.x;
  a.in1 = (const double*)w.b;
  a.out0 = (double*)w.r;
  a.alpha = cfg->alpha;
  a.shift = cfg->shift;
  a.use_tma = 1;
  cudaError_t e = launch_apply<double>(op->N, AM_RESID, a, s);
  if (e == cudaSuccess) e = mg_apply64(mg, (const double*)w.r, (double*)w.z, s);
  if (e == cudaSuccess)
    e = launch_cg_finish<double>(true, (const double*)w.r, (const double*)w.z, n, op->ctl, op->partA, op->status, 0,
                                 0, s);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("MG-CG init: ") + cudaGetErrorString(e));
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
    info->res_norm2 = res.rr;
    info->b_norm2 = res.bb;
    info->updates = 0;
  }
  return DDG_OK;
}

namespace {
void drop_graphs(ddg_sipg_op* op) {
  for (auto& kv : op->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.g) cudaGraphDestroy(kv.second.g);
  }
  op->graphs.clear();
  for (auto& kv : op->mg_graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.g) cudaGraphDestroy(kv.second.g);
  }
  op->mg_graphs.clear();
  if (op->hio) op->hio->g_ok = false;
}
}  // namespace

extern "C" int ddg_sipg_set_kappa(ddg_sipg_op* op, const double* kappa) {
  if (!op) return fail(DDG_ERR_INVALID, "ddg_sipg_set_kappa: null handle");
  DevGuard guard(op->dev);
  const bool on = kappa != nullptr;
  if (on) {
    for (int k = 0; k < op->K; ++k)
      if (!(kappa[k] > 0.0) || !std::isfinite(kappa[k]))
        return fail(DDG_ERR_INVALID, "ddg_sipg_set_kappa: diffusivity must be positive and finite");
    if (!op->kappa64 || !op->kappa32) {       // one block: both copies or neither
      if (op->kappa64) cudaFree(op->kappa64);
      op->kappa64 = nullptr;
      op->kappa32 = nullptr;
      void* blk = nullptr;
      CK(cudaMalloc(&blk, (size_t)op->K * 8 + (size_t)op->K * 4 + 16));
      op->kappa64 = (double*)blk;
      op->kappa32 = (float*)((char*)blk + (((size_t)op->K * 8 + 15) & ~(size_t)15));
    }
    std::vector<float> k32(kappa, kappa + op->K);
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(op->kappa64, kappa, (size_t)op->K * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(op->kappa32, k32.data(), (size_t)op->K * 4, cudaMemcpyHostToDevice));
  }
  if (on != op->kappa_on) {
    CK(cudaDeviceSynchronize());
    drop_graphs(op);          // captured launches bake the diffusivity pointer in
  }
  op->kappa_on = on;
  op->pc_ready = false;       // the diagonal blocks depend on the diffusivity
  return DDG_OK;
}

extern "C" int ddg_sipg_grad_kappa(ddg_sipg_op* op, const double* u, const double* lam, double* g, void* stream) {
  if (!op || !u || !lam || !g) return fail(DDG_ERR_INVALID, "ddg_sipg_grad_kappa: null argument");
  DevGuard guard(op->dev);
  GradArgs a{};
  a.geo = op->geo64;
  a.nbr = op->nbr;
  a.perm = op->perm;
  a.u = u;
  a.lam = lam;
  a.kappa = op->kappa_on ? op->kappa64 : nullptr;
  a.g = g;
  a.K = op->K;
  a.ldg = op->ldg;
  a.tau = op->tau;
  cudaError_t e = launch_grad_kappa(op->N, a, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("ddg_sipg_grad_kappa: ") + cudaGetErrorString(e));
  return DDG_OK;
}
