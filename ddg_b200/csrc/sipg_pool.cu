// Continuous-batching solve pool (host side): many independent SIPG
// Helmholtz/Poisson solves of one polynomial degree share one packed element
// array.  Requests are admitted into free element ranges while others are
// iterating; a batched CG advances every active request in the same kernel
// launches (captured as a CUDA graph), and finished requests are retired
// between launches, freeing their range for the next arrivals.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <array>
#include <map>
#include <string>
#include <vector>

#include "../../include/ddg_sipg.h"
#include "sipg_device.cuh"
#include "sipg_launch.h"
#include "status.h"

using namespace ddg;

#define PCK(call)                                                                                \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return fail(DDG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));             \
  } while (0)

struct ddg_pool {
  int N = 0, Np = 0, cap = 0, max_req = 0, dev = 0, hw = 0, max_req_K = 0;
  double tau = 0.0;
  // device
  double* geo = nullptr;
  uint32_t* nbr = nullptr;
  int* seg = nullptr;
  double* alpha_e = nullptr;
  double* binv = nullptr;
  int prec = DDG_FP64;          // iteration vectors: DDG_FP64 or DDG_FP32
  double *x = nullptr, *b = nullptr, *r = nullptr, *z = nullptr, *Ap = nullptr;   // float64 pools
  float *x32 = nullptr, *r32 = nullptr, *z32 = nullptr, *Ap32 = nullptr;          // float32 pools
  void *p0 = nullptr, *p1 = nullptr;      // CG directions (the pool's precision)
  float *geo32 = nullptr, *binv32 = nullptr;  // float32 copies (float32 pools)
  double* fsrc = nullptr;       // admission scratch: the request's source (max request size)
  double *epA = nullptr, *epB = nullptr;
  BatchReq* req = nullptr;
  int* perm = nullptr;
  double* blocks = nullptr;     // block-Jacobi build scratch (max request size)
  unsigned int* status = nullptr;
  BatchReq* req_host = nullptr; // pinned mirror for polling
  // host
  std::vector<std::pair<int, int>> free_ranges;   // (start, length), sorted by start
  std::vector<int> slot_k0, slot_K;               // -1 when the slot is free
  int threads = 128, persistent = 0;              // element-kernel tile (ddg_pool_set_tile)
  // captured iteration graphs by (hw, pairs, threads, persistent)
  std::map<std::array<int, 4>, std::pair<cudaGraph_t, cudaGraphExec_t>> graphs;
  cudaStream_t cap_stream = nullptr;
};

extern "C" int ddg_sipg_upload_reference(int N, const double* Dr, const double* Ds, const double* M,
                                         const double* m1d, int device);

namespace {

BatchArgs pool_args(ddg_pool* p) {
  BatchArgs a{};
  a.threads = p->threads;
  a.persistent = p->persistent;
  a.cap = p->cap;
  a.hw = p->hw;
  a.geo = p->geo;
  a.nbr = p->nbr;
  a.seg = p->seg;
  a.alpha_e = p->alpha_e;
  a.binv = p->binv;
  a.x = p->x;
  a.b = p->b;
  a.r = p->r;
  a.z = p->z;
  a.Ap = p->Ap;
  a.prec = p->prec == DDG_FP32 ? 1 : 0;
  a.geo32 = p->geo32;
  a.binv32 = p->binv32;
  a.x32 = p->x32;
  a.r32 = p->r32;
  a.z32 = p->z32;
  a.Ap32 = p->Ap32;
  a.epA = p->epA;
  a.epB = p->epB;
  a.req = p->req;
  a.perm = p->perm;
  a.tau = p->tau;
  a.max_req = p->max_req;
  return a;
}

void pool_free(ddg_pool* p) {
  for (auto& kv : p->graphs) {
    cudaGraphExecDestroy(kv.second.second);
    cudaGraphDestroy(kv.second.first);
  }
  void* d[] = {p->geo, p->nbr, p->seg, p->alpha_e, p->binv, p->x, p->b, p->r, p->z, p->p0, p->p1, p->Ap,
               p->epA, p->epB, p->req, p->perm, p->blocks, p->status, p->x32, p->r32, p->z32, p->Ap32,
               p->geo32, p->binv32, p->fsrc};
  for (void* q : d)
    if (q) cudaFree(q);
  if (p->req_host) cudaFreeHost(p->req_host);
  if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
  delete p;
}

int take_range(ddg_pool* p, int K) {
  for (size_t i = 0; i < p->free_ranges.size(); ++i) {   // first fit
    auto& fr = p->free_ranges[i];
    if (fr.second >= K) {
      const int k0 = fr.first;
      fr.first += K;
      fr.second -= K;
      if (fr.second == 0) p->free_ranges.erase(p->free_ranges.begin() + i);
      return k0;
    }
  }
  return -1;
}

void give_range(ddg_pool* p, int k0, int K) {
  auto& v = p->free_ranges;
  v.push_back({k0, K});
  std::sort(v.begin(), v.end());
  std::vector<std::pair<int, int>> m;
  for (auto& fr : v) {
    if (!m.empty() && m.back().first + m.back().second == fr.first) m.back().second += fr.second;
    else m.push_back(fr);
  }
  v.swap(m);
}

int pool_graph(ddg_pool* p, int pairs, cudaGraphExec_t* out) {
  const std::array<int, 4> key{p->hw, pairs, p->threads, p->persistent};
  auto it = p->graphs.find(key);
  if (it != p->graphs.end()) {
    *out = it->second.second;
    return DDG_OK;
  }
  BatchArgs a = pool_args(p);
  PCK(cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  for (int it2 = 0; it2 < 2 * pairs && e == cudaSuccess; ++it2) {
    void* pin = (it2 % 2 == 0) ? p->p0 : p->p1;
    void* pout = (it2 % 2 == 0) ? p->p1 : p->p0;
    e = launch_batch_pfuse(p->N, a, pin, pout, p->cap_stream);
    if (e == cudaSuccess) e = launch_batch_seg(0, a, 0, p->max_req, p->cap_stream);
    if (e == cudaSuccess) e = launch_batch_step(p->N, a, pout, p->cap_stream);
    if (e == cudaSuccess) e = launch_batch_seg(1, a, 0, p->max_req, p->cap_stream);
  }
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(p->cap_stream, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(DDG_ERR_CUDA, std::string("pool graph capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  cudaGraphExec_t ex = nullptr;
  PCK(cudaGraphInstantiate(&ex, g, 0));
  p->graphs[key] = {g, ex};
  *out = ex;
  return DDG_OK;
}

}  // namespace

extern "C" int ddg_pool_create(int N, int capacity, int max_requests, int max_request_K, double tau_scale,
                               int device, ddg_pool** out) {
  return ddg_pool_create_ex(N, capacity, max_requests, max_request_K, tau_scale, DDG_FP64, device, out);
}

extern "C" int ddg_pool_create_ex(int N, int capacity, int max_requests, int max_request_K, double tau_scale,
                                  int precision, int device, ddg_pool** out) {
  if (!out || N < 1 || N > DDG_MAX_DEGREE || capacity < 1 || (uint32_t)capacity > NBR_MAX_K ||
      max_requests < 1 || max_request_K < 1 || max_request_K > capacity ||
      (precision != DDG_FP64 && precision != DDG_FP32))
    return fail(DDG_ERR_INVALID, "ddg_pool_create: bad arguments");
  *out = nullptr;
  int cur = 0;
  cudaGetDevice(&cur);
  PCK(cudaSetDevice(device));
  ddg_pool* p = new ddg_pool();
  p->N = N;
  p->Np = (N + 1) * (N + 2) / 2;
  p->cap = (capacity + 31) / 32 * 32;
  p->max_req = max_requests;
  p->max_req_K = max_request_K;
  p->dev = device;
  p->tau = tau_scale * (N + 1) * (N + 1);
  const size_t nE = (size_t)p->cap, nV = nE * p->Np, nS = (size_t)p->Np * (p->Np + 1) / 2;
  cudaError_t e = cudaSuccess;
#define PA(ptr, bytes) \
  if (e == cudaSuccess) e = cudaMalloc((void**)&(ptr), (bytes))
  PA(p->geo, G_COUNT * nE * 8);
  PA(p->nbr, 3 * nE * 4);
  PA(p->seg, nE * 4);
  PA(p->alpha_e, nE * 8);
  PA(p->binv, nS * nE * 8);
  PA(p->b, nV * 8);
  PA(p->fsrc, (size_t)max_request_K * p->Np * 8);
  p->prec = precision;
  if (precision == DDG_FP64) {
    PA(p->x, nV * 8);
    PA(p->r, nV * 8);
    PA(p->z, nV * 8);
    PA(p->p0, nV * 8);
    PA(p->p1, nV * 8);
    PA(p->Ap, nV * 8);
  } else {
    PA(p->x32, nV * 4);
    PA(p->r32, nV * 4);
    PA(p->z32, nV * 4);
    PA(p->p0, nV * 4);
    PA(p->p1, nV * 4);
    PA(p->Ap32, nV * 4);
    PA(p->geo32, G_COUNT * nE * 4);
    PA(p->binv32, nS * nE * 4);
  }
  PA(p->epA, nE * 8);
  PA(p->epB, nE * 8);
  PA(p->req, max_requests * sizeof(BatchReq));
  PA(p->perm, 3 * p->Np * sizeof(int));
  PA(p->blocks, (size_t)max_request_K * p->Np * p->Np * 8);
  PA(p->status, sizeof(unsigned int));
#undef PA
  if (e == cudaSuccess) e = cudaMallocHost((void**)&p->req_host, max_requests * sizeof(BatchReq));
  if (e == cudaSuccess) e = cudaMemset(p->seg, 0xff, nE * 4);   // -1: free
  if (e == cudaSuccess) e = cudaMemset(p->req, 0, max_requests * sizeof(BatchReq));
  if (e == cudaSuccess) e = cudaMemset(p->status, 0, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking);
  cudaSetDevice(cur);
  if (e != cudaSuccess) {
    pool_free(p);
    return fail(e == cudaErrorMemoryAllocation ? DDG_ERR_NOMEM : DDG_ERR_CUDA,
                std::string("ddg_pool_create: ") + cudaGetErrorString(e));
  }
  p->free_ranges.push_back({0, capacity});
  p->slot_k0.assign(max_requests, -1);
  p->slot_K.assign(max_requests, 0);
  *out = p;
  return DDG_OK;
}

extern "C" int ddg_pool_destroy(ddg_pool* p) {
  if (!p) return DDG_OK;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(p->dev);
  cudaDeviceSynchronize();
  pool_free(p);
  cudaSetDevice(cur);
  return DDG_OK;
}

// Admit one request: mesh (its own element numbering), Helmholtz alpha,
// tolerances, nodal source f (K x Np element-major, host).  Returns the slot
// in *slot, or DDG_ERR_NOMEM when no slot or element range is free now.
extern "C" int ddg_pool_admit(ddg_pool* p, const ddg_sipg_mesh_desc* d, double alpha, double tol, double atol,
                              int maxiter, const double* f, void* stream, int* slot) {
  if (!p || !d || !f || !slot) return fail(DDG_ERR_INVALID, "ddg_pool_admit: null argument");
  if (d->N != p->N) return fail(DDG_ERR_INVALID, "ddg_pool_admit: degree differs from the pool's");
  if (d->K < 1 || d->K > p->max_req_K) return fail(DDG_ERR_INVALID, "ddg_pool_admit: request larger than the pool's limit");
  if (!(tol >= 0.0) || !(atol >= 0.0) || maxiter < 0) return fail(DDG_ERR_INVALID, "ddg_pool_admit: tolerances");
  int s = -1;
  for (int i = 0; i < p->max_req; ++i)
    if (p->slot_k0[i] < 0) {
      s = i;
      break;
    }
  if (s < 0) return fail(DDG_ERR_NOMEM, "ddg_pool_admit: no free request slot");
  const int K = d->K, Np = p->Np;
  const int k0 = take_range(p, K);
  if (k0 < 0) return fail(DDG_ERR_NOMEM, "ddg_pool_admit: no free element range");
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(p->dev);
  struct Restore {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{cur};
  auto undo = [&](int code, const std::string& m) {
    give_range(p, k0, K);
    return fail(code, m);
  };
  int rc = ddg_sipg_upload_reference(p->N, d->Dr, d->Ds, d->M, d->m1d, p->dev);
  if (rc != DDG_OK) return undo(rc, "ddg_pool_admit: reference matrices");
  // neighbour words with the element offset, geometry, segment ids, alpha
  std::vector<uint32_t> nb((size_t)3 * K);
  rc = pack_neighbours(K, p->N, d->EToE, d->EToF, d->vmapP, d->rot_perm, d->bc_types, (uint32_t)k0, nb.data(),
                       (size_t)K);
  if (rc != DDG_OK) return undo(rc, std::string("ddg_pool_admit: ") + ddg_last_error());
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<double> geo((size_t)G_COUNT * K);
  for (int k = 0; k < K; ++k)
    for (int c = 0; c < G_COUNT; ++c) geo[(size_t)c * K + k] = d->geo[(size_t)k * G_COUNT + c];
  std::vector<int> perm(d->rot_perm, d->rot_perm + 3 * Np);
  std::vector<int> segv(K, s);
  std::vector<double> alv(K, alpha);
  cudaError_t e = cudaMemcpy2DAsync(p->geo + k0, (size_t)p->cap * 8, geo.data(), (size_t)K * 8, (size_t)K * 8,
                                    G_COUNT, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(p->nbr + k0, (size_t)p->cap * 4, nb.data(), (size_t)K * 4, (size_t)K * 4, 3,
                          cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p->perm, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p->alpha_e + k0, alv.data(), (size_t)K * 8, cudaMemcpyHostToDevice, st);
  // source into the scratch, b = J M f
  if (e == cudaSuccess) e = cudaMemcpyAsync(p->fsrc, f, (size_t)K * Np * 8, cudaMemcpyHostToDevice, st);
  // block-Jacobi blocks of the range
  BlockArgs ba{};
  ba.geo = p->geo;
  ba.nbr = p->nbr;
  ba.blocks = p->blocks;
  ba.binv64 = p->binv;
  ba.binv32 = nullptr;
  ba.status = p->status;
  ba.K = K;
  ba.ldg = p->cap;
  ba.ldb = p->cap;
  ba.tau = p->tau;
  ba.alpha = alpha;
  ba.k0 = k0;
  ba.nbr_ld = p->cap;
  if (e == cudaSuccess) e = launch_block_jacobi(p->N, ba, st);
  BatchArgs a = pool_args(p);
  if (e == cudaSuccess && p->prec == DDG_FP32) {   // float32 copies of the range's geometry and inverses
    e = launch_rows_to_f32(p->geo, p->geo32, G_COUNT, p->cap, k0, K, st);
    if (e == cudaSuccess) e = launch_rows_to_f32(p->binv, p->binv32, Np * (Np + 1) / 2, p->cap, k0, K, st);
  }
  if (e == cudaSuccess) e = launch_batch_rhs(p->N, a, p->fsrc, k0, K, st);
  if (e == cudaSuccess) e = launch_batch_init(p->N, a, p->p0, k0, K, st);
  BatchReq q{};
  q.k0 = k0;
  q.K = K;
  q.maxiter = maxiter;
  q.tol2 = tol * tol;
  q.atol_sq = atol * atol;
  if (e == cudaSuccess) e = cudaMemcpyAsync(p->req + s, &q, sizeof(q), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = launch_batch_seg(2, a, s, 1, st);
  // the element range joins the iteration only now (segment ids last)
  if (e == cudaSuccess) e = cudaMemcpyAsync(p->seg + k0, segv.data(), (size_t)K * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // host staging buffers go out of scope
  if (e != cudaSuccess) return undo(DDG_ERR_CUDA, std::string("ddg_pool_admit: ") + cudaGetErrorString(e));
  p->slot_k0[s] = k0;
  p->slot_K[s] = K;
  p->hw = std::max(p->hw, (k0 + K + 16383) / 16384 * 16384);
  p->hw = std::min(p->hw, p->cap);
  *slot = s;
  return DDG_OK;
}

// Advance every active request by 2*pairs CG iterations (one graph launch).
extern "C" int ddg_pool_iterate(ddg_pool* p, int pairs, void* stream) {
  if (!p || pairs < 1) return fail(DDG_ERR_INVALID, "ddg_pool_iterate: bad arguments");
  if (p->hw == 0) return DDG_OK;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(p->dev);
  cudaGraphExec_t ex = nullptr;
  int rc = pool_graph(p, pairs, &ex);
  if (rc == DDG_OK) {
    cudaError_t e = cudaGraphLaunch(ex, (cudaStream_t)stream);
    if (e != cudaSuccess) rc = fail(DDG_ERR_CUDA, std::string("ddg_pool_iterate: ") + cudaGetErrorString(e));
  }
  cudaSetDevice(cur);
  return rc;
}

// Tile shape of the element kernels of later ddg_pool_iterate calls:
// threads per block (64, 128 or 256) and persistent (0: one thread per
// element; 1: at most 2048 / threads blocks per SM looping over the
// elements).  Results do not depend on it.
extern "C" int ddg_pool_set_tile(ddg_pool* p, int threads, int persistent) {
  if (!p || !(threads == 64 || threads == 128 || threads == 256) || (persistent != 0 && persistent != 1))
    return fail(DDG_ERR_INVALID, "ddg_pool_set_tile: threads must be 64, 128 or 256 and persistent 0 or 1");
  p->threads = threads;
  p->persistent = persistent;
  return DDG_OK;
}

// Copy the per-request state to the host and report, per slot, 1 when the
// request is still iterating, 0 when it has finished (or the slot is empty).
extern "C" int ddg_pool_poll(ddg_pool* p, int32_t* active, int32_t* iterations, void* stream) {
  if (!p || !active) return fail(DDG_ERR_INVALID, "ddg_pool_poll: null argument");
  cudaStream_t st = (cudaStream_t)stream;
  PCK(cudaMemcpyAsync(p->req_host, p->req, p->max_req * sizeof(BatchReq), cudaMemcpyDeviceToHost, st));
  PCK(cudaStreamSynchronize(st));
  for (int i = 0; i < p->max_req; ++i) {
    active[i] = (p->slot_k0[i] >= 0 && p->req_host[i].active) ? 1 : 0;
    if (iterations) iterations[i] = p->slot_k0[i] >= 0 ? p->req_host[i].iter : 0;
  }
  return DDG_OK;
}

// Copy a finished request's solution (K x Np element-major) to host memory x
// and free its slot and element range.
extern "C" int ddg_pool_retire(ddg_pool* p, int slot, double* x, void* stream, ddg_solve_info* info) {
  if (!p || !x || slot < 0 || slot >= p->max_req || p->slot_k0[slot] < 0)
    return fail(DDG_ERR_INVALID, "ddg_pool_retire: bad slot");
  const int k0 = p->slot_k0[slot], K = p->slot_K[slot];
  cudaStream_t st = (cudaStream_t)stream;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(p->dev);
  BatchReq q{};
  cudaError_t e = cudaMemcpyAsync(&q, p->req + slot, sizeof(q), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && q.active) {
    cudaSetDevice(cur);
    return fail(DDG_ERR_INVALID, "ddg_pool_retire: request still iterating");
  }
  std::vector<float> x32;
  if (e == cudaSuccess) {
    if (p->prec == DDG_FP64) {
      e = cudaMemcpyAsync(x, p->x + (size_t)k0 * p->Np, (size_t)K * p->Np * 8, cudaMemcpyDeviceToHost, st);
    } else {
      x32.resize((size_t)K * p->Np);
      e = cudaMemcpyAsync(x32.data(), p->x32 + (size_t)k0 * p->Np, x32.size() * 4, cudaMemcpyDeviceToHost, st);
    }
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(p->seg + k0, 0xff, (size_t)K * 4, st);
  BatchReq zero{};
  if (e == cudaSuccess) e = cudaMemcpyAsync(p->req + slot, &zero, sizeof(zero), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaSetDevice(cur);
  if (e != cudaSuccess) return fail(DDG_ERR_CUDA, std::string("ddg_pool_retire: ") + cudaGetErrorString(e));
  for (size_t i = 0; i < x32.size(); ++i) x[i] = (double)x32[i];
  p->slot_k0[slot] = -1;
  p->slot_K[slot] = 0;
  give_range(p, k0, K);
  if (info) {
    info->status = q.status;
    info->iterations = q.iter;
    info->res_norm2 = q.rr;
    info->b_norm2 = q.bb;
    info->updates = 0;
  }
  return DDG_OK;
}
