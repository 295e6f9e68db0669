// Multigrid and external-preconditioner CG kernels.
//
// Transfers (ddg src/ddg/dg2d/multigrid.py:106-184) are all per-element
// small matrix products out[k] (+)= M in[k]:
//   p-prolong   x_hi[k] += I x_lo[k]                 M = I       (Np_hi x Np_lo)
//   p-restrict  b_lo[k]  = I^T r_hi[k]               M = I^T     (Np_lo x Np_hi)
//   h-prolong   x_f[4k..4k+3] += [I_0;..;I_3] x_c[k] M (4 Np x Np)
//   h-restrict  b_c[k] = [I_0^T .. I_3^T] r_f[4k..4k+3]  M (Np x 4 Np)
// (fine element 4k+c is child c of coarse element k, so a coarse element's
// four children are contiguous in the element-major fine vector).
#include <cuda_runtime.h>
#include <stdint.h>

#include "sipg_device.cuh"
#include "sipg_launch.h"

namespace ddg {

// out[k*rows + i] = (add ? out : 0) + sum_j M[i*cols + j] in[k*cols + j]
template <typename T>
__global__ void k_elem_matvec(int Kout, int rows, int cols, const T* __restrict__ M, const T* __restrict__ in,
                              T* __restrict__ out, int add) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sM = reinterpret_cast<T*>(smraw);
  for (int i = threadIdx.x; i < rows * cols; i += blockDim.x) sM[i] = M[i];
  __syncthreads();
  const int64_t total = (int64_t)Kout * rows;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = t / rows;
    const int i = (int)(t - k * rows);
    const T* v = in + k * cols;
    const T* m = sM + i * cols;
    T acc = add ? out[t] : T(0);
    for (int j = 0; j < cols; ++j) acc = fma(m[j], v[j], acc);
    out[t] = acc;
  }
}

// x = A_inv b (dense n x n, row-major): one warp per row.
template <typename T>
__global__ void k_dense_gemv(int n, const T* __restrict__ A, const T* __restrict__ b, T* __restrict__ x) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  const T* row = A + (size_t)warp * n;
  double acc = 0.0;
  for (int j = lane; j < n; j += 32) acc += (double)row[j] * (double)b[j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) x[warp] = (T)acc;
}

// x = scale * B^-1 b, one element per thread (packed inverses: each entry
// loaded once, coalesced across the warp's elements, used for (i,j), (j,i)).
template <int N, typename T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_bj_scaled(const T* __restrict__ b, T* __restrict__ x,
                                                     const T* __restrict__ binv, int ldb, int K, T scale) {
  constexpr int Np = Dim<N>::Np;
  __shared__ __align__(16) T s[BLOCK * Np];
  const int tid = threadIdx.x, k0 = blockIdx.x * BLOCK, nk = min(BLOCK, K - k0);
  const size_t off = (size_t)k0 * Np;
  for (int i = tid; i < nk * Np; i += BLOCK) s[i] = b[off + i];
  __syncthreads();
  if (tid < nk) {
    T rv[Np], zv[Np];
#pragma unroll
    for (int j = 0; j < Np; ++j) {
      rv[j] = s[tid * Np + j];
      zv[j] = T(0);
    }
    const T* bk = binv + k0 + tid;
#pragma unroll
    for (int i = 0; i < Np; ++i)
#pragma unroll
      for (int j = i; j < Np; ++j) {
        const T c = __ldg(bk + (size_t)sym_idx(Np, i, j) * ldb);
        zv[i] = fma(c, rv[j], zv[i]);
        if (j != i) zv[j] = fma(c, rv[i], zv[j]);
      }
#pragma unroll
    for (int i = 0; i < Np; ++i) s[tid * Np + i] = scale * zv[i];
  }
  __syncthreads();
  for (int i = tid; i < nk * Np; i += BLOCK) x[off + i] = s[i];
}

// CG with an external preconditioner, part 1: x += alpha p, r -= alpha Ap,
// r.r -> ctl->rr.  (The preconditioner kernels then compute z from r.)
template <typename T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_cg_xr(T* __restrict__ x, const T* __restrict__ p, T* __restrict__ r,
                                                 const T* __restrict__ Ap, int64_t n, CgCtl* ctl, double* part) {
  __shared__ double s_red[64];
  if (ctl->cont == 0) return;
  const T al = T(ctl->alpha);
  double rr = 0.0, d = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * BLOCK) {
    x[i] = fma(al, p[i], x[i]);
    const T rn = fma(-al, Ap[i], r[i]);
    r[i] = rn;
    rr += (double)rn * (double)rn;
  }
  block_sum2<BLOCK>(rr, d, s_red);
  if (threadIdx.x == 0) part[blockIdx.x] = rr;
  if (!is_last_block(&ctl->ticket)) return;
  double t, u;
  reduce_partials2<BLOCK>(part, nullptr, gridDim.x, t, u, s_red);
  if (threadIdx.x == 0) {
    ctl->rr = t;
    ctl->ticket = 0u;
  }
}

// Part 2: gamma = r.z, beta, iteration count, loop condition (as k_cg_step).
template <typename T, bool INIT, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_cg_finish(const T* __restrict__ r, const T* __restrict__ z, int64_t n,
                                                     CgCtl* ctl, double* part, const unsigned int* dev_status,
                                                     int has_cond, cudaGraphConditionalHandle cond) {
  __shared__ double s_red[64];
  if (!INIT && ctl->cont == 0) {
    if (has_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0u);
    return;
  }
  double rz = 0.0, d = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * BLOCK)
    rz += (double)r[i] * (double)z[i];
  block_sum2<BLOCK>(rz, d, s_red);
  if (threadIdx.x == 0) part[blockIdx.x] = rz;
  if (!is_last_block(&ctl->ticket)) return;
  double g, u;
  reduce_partials2<BLOCK>(part, nullptr, gridDim.x, g, u, s_red);
  if (threadIdx.x == 0) {
    CgCtl* c = ctl;
    if (INIT) {
      c->atol2 = fmax(c->tol2 * c->bb, c->atol_sq);
      c->beta = 0.0;
      c->iter = 0;
      c->status = 0;
    } else {
      c->gamma_prev = c->gamma;
      c->beta = g / c->gamma;
      c->iter += 1;
    }
    c->zcoef = 1.0;
    c->gamma = g;
    const double rs = c->rr;
    int cont = (rs > c->atol2) && (c->iter < c->maxiter) && (c->status == 0);
    if (!isfinite(g) || !isfinite(rs) || (!INIT && !isfinite(c->beta))) {
      c->status = 2;
      cont = 0;
    }
    if (dev_status && *(volatile const unsigned int*)dev_status != 0u) {
      c->status = 3;
      cont = 0;
    }
    if (cont == 0 && c->status == 0 && rs > c->atol2) c->status = 1;
    c->cont = cont;
    c->ticket = 0u;
    if (has_cond) cudaGraphSetConditional(cond, (unsigned)cont);
  }
}

// ------------------------------------------------------------- launchers
static int grid_for(int64_t n, int block, int cap) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  return (int)(g < cap ? g : cap);
}

template <typename T>
cudaError_t launch_elem_matvec(int Kout, int rows, int cols, const T* M, const T* in, T* out, int add,
                               cudaStream_t s) {
  const size_t smem = (size_t)rows * cols * sizeof(T);
  const int64_t total = (int64_t)Kout * rows;
  k_elem_matvec<T><<<grid_for(total, 256, 148 * 16), 256, smem, s>>>(Kout, rows, cols, M, in, out, add);
  return cudaGetLastError();
}
template cudaError_t launch_elem_matvec<double>(int, int, int, const double*, const double*, double*, int,
                                                cudaStream_t);
template cudaError_t launch_elem_matvec<float>(int, int, int, const float*, const float*, float*, int, cudaStream_t);

template <typename T>
cudaError_t launch_dense_gemv(int n, const T* A, const T* b, T* x, cudaStream_t s) {
  const int warps_per_block = 8;
  k_dense_gemv<T><<<(n + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, s>>>(n, A, b, x);
  return cudaGetLastError();
}
template cudaError_t launch_dense_gemv<double>(int, const double*, const double*, double*, cudaStream_t);
template cudaError_t launch_dense_gemv<float>(int, const float*, const float*, float*, cudaStream_t);

template <int N, typename T>
static cudaError_t launch_bj_n(const T* b, T* x, const T* binv, int ldb, int K, T scale, cudaStream_t s) {
  constexpr int B = 128;
  k_bj_scaled<N, T, B><<<(K + B - 1) / B, B, 0, s>>>(b, x, binv, ldb, K, scale);
  return cudaGetLastError();
}
template <typename T>
cudaError_t launch_bj_scaled(int N, const T* b, T* x, const T* binv, int ldb, int K, T scale, cudaStream_t s) {
  switch (N) {
    case 1: return launch_bj_n<1, T>(b, x, binv, ldb, K, scale, s);
    case 2: return launch_bj_n<2, T>(b, x, binv, ldb, K, scale, s);
    case 3: return launch_bj_n<3, T>(b, x, binv, ldb, K, scale, s);
    case 4: return launch_bj_n<4, T>(b, x, binv, ldb, K, scale, s);
    case 5: return launch_bj_n<5, T>(b, x, binv, ldb, K, scale, s);
  }
  return cudaErrorInvalidValue;
}
template cudaError_t launch_bj_scaled<double>(int, const double*, double*, const double*, int, int, double,
                                              cudaStream_t);
template cudaError_t launch_bj_scaled<float>(int, const float*, float*, const float*, int, int, float, cudaStream_t);

int xr_grid(int64_t n) { return grid_for(n, 256, 148 * 8); }

template <typename T>
cudaError_t launch_cg_xr(T* x, const T* p, T* r, const T* Ap, int64_t n, CgCtl* ctl, double* part, cudaStream_t s) {
  k_cg_xr<T, 256><<<xr_grid(n), 256, 0, s>>>(x, p, r, Ap, n, ctl, part);
  return cudaGetLastError();
}
template cudaError_t launch_cg_xr<double>(double*, const double*, double*, const double*, int64_t, CgCtl*, double*,
                                          cudaStream_t);

template <typename T>
cudaError_t launch_cg_finish(bool init, const T* r, const T* z, int64_t n, CgCtl* ctl, double* part,
                             const unsigned int* dev_status, int has_cond, cudaGraphConditionalHandle cond,
                             cudaStream_t s) {
  if (init)
    k_cg_finish<T, true, 256><<<xr_grid(n), 256, 0, s>>>(r, z, n, ctl, part, dev_status, has_cond, cond);
  else
    k_cg_finish<T, false, 256><<<xr_grid(n), 256, 0, s>>>(r, z, n, ctl, part, dev_status, has_cond, cond);
  return cudaGetLastError();
}
template cudaError_t launch_cg_finish<double>(bool, const double*, const double*, int64_t, CgCtl*, double*,
                                              const unsigned int*, int, cudaGraphConditionalHandle, cudaStream_t);

}  // namespace ddg
