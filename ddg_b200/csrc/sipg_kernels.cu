// Kernels of the SIPG operator, its CG loop, the block-Jacobi
// preconditioner and the right-hand-side loads, plus their host launchers.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "sipg_device.cuh"
#include "sipg_launch.h"

namespace ddg {

#define DDG_DEFINE_CONST(NN)                       \
  __constant__ RefMats<NN, double> c_ref64_##NN; \
  __constant__ RefMats<NN, float> c_ref32_##NN;  \
  __constant__ RefPairs<NN> c_pair32_##NN;
DDG_DEFINE_CONST(1)
DDG_DEFINE_CONST(2)
DDG_DEFINE_CONST(3)
DDG_DEFINE_CONST(4)
DDG_DEFINE_CONST(5)

#define DDG_CREF(NN)                                                                    \
  template <> struct CRef<NN, double> {                                                \
    static __device__ __forceinline__ const RefMats<NN, double>& get() { return c_ref64_##NN; } \
  };                                                                                   \
  template <> struct CRef<NN, float> {                                                 \
    static __device__ __forceinline__ const RefMats<NN, float>& get() { return c_ref32_##NN; } \
  };
DDG_CREF(1)
DDG_CREF(2)
DDG_CREF(3)
DDG_CREF(4)
DDG_CREF(5)

#define DDG_CPAIRS(NN)                                                                   \
  template <> struct CPairs<NN> {                                                      \
    static __device__ __forceinline__ const RefPairs<NN>& get() { return c_pair32_##NN; } \
  };
DDG_CPAIRS(1)
DDG_CPAIRS(2)
DDG_CPAIRS(3)
DDG_CPAIRS(4)
DDG_CPAIRS(5)

// ================================================================ apply
// MODE: AM_APPLY  out0 = A in0 + alpha J M in0 + shift in0
//       AM_PFUSE  u = in0 + beta in1 (CG direction, beta from ctl);
//                 out1 = u; out0 = A u (+...); partial u.out0 -> ctl->pAp,
//                 ctl->alpha = gamma / pAp  (last block)
//       AM_RESID  out0 = in1 - (A in0 + ...); partials in1.in1, out0.out0
//                 -> ctl->bb, ctl->rr (last block)
//       AM_SMOOTH out0 = in0 + omega B^-1 (in1 - (A in0 + ...)): one weighted
//                 block-Jacobi sweep (multigrid.py:238-243); out0 != in0
template <int N, typename T, int MODE, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_apply(ApplyArgs<T> a) {
  constexpr int Np = Dim<N>::Np;
  constexpr int NT = (MODE == AM_APPLY) ? 1 : 2;
  constexpr bool HASB = (MODE == AM_RESID || MODE == AM_SMOOTH);
  __shared__ __align__(128) T s_tile[NT][BLOCK * Np];
  __shared__ int s_perm[3 * Np];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ double s_red[64];

  if (MODE == AM_PFUSE && a.ctl->cont == 0) return;  // uniform across the grid
  const int tid = threadIdx.x;
  const int k_hi = (MODE == AM_APPLY && a.k_hi > 0) ? a.k_hi : a.K;
  const int k0 = (MODE == AM_APPLY ? a.k_lo : 0) + blockIdx.x * BLOCK;
  const int nk = min(BLOCK, k_hi - k0);
  const size_t off = (size_t)k0 * Np;
  const uint32_t bytes = (uint32_t)(nk * Np * sizeof(T));
  const bool tma = a.use_tma && (bytes % 16u == 0u);

  for (int i = tid; i < 3 * Np; i += BLOCK) s_perm[i] = a.perm[i];
  if (tma && tid == 0) {
    mbar_init(&s_bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tma) {
    __shared__ int s_ok;
    if (tid == 0) {
      mbar_expect_tx(&s_bar, bytes * NT);
      bulk_load(s_tile[0], a.in0 + off, bytes, &s_bar);
      if (NT > 1) bulk_load(s_tile[NT - 1], a.in1 + off, bytes, &s_bar);
      s_ok = mbar_wait_bounded(&s_bar, 0, &a.ctl_status[0]) ? 1 : 0;
    }
    __syncthreads();           // one waiter; the whole block sees its outcome
    if (!s_ok) return;         // uniform exit: no thread is left at a barrier
  } else {
    for (int i = tid; i < nk * Np; i += BLOCK) {
      s_tile[0][i] = a.in0[off + i];
      if (NT > 1) s_tile[NT - 1][i] = a.in1[off + i];
    }
    __syncthreads();
  }

  const T beta = (MODE == AM_PFUSE) ? T(a.ctl->beta) : T(0);
  const T zc = (MODE == AM_PFUSE) ? T(a.ctl->zcoef) : T(1);
  const int k = k0 + tid;
  const bool active = tid < nk;
  T u[Np], y[Np], b2[Np];
  double dA = 0.0, dB = 0.0;
  if (active) {
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      if (MODE == AM_PFUSE) {
        u[i] = zc * s_tile[0][tid * Np + i] + beta * s_tile[1][tid * Np + i];
      } else {
        u[i] = s_tile[0][tid * Np + i];
      }
      if (HASB) b2[i] = s_tile[1][tid * Np + i];
    }
    uint32_t w[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) w[f] = __ldg(a.nbr + (size_t)f * a.K + k);
    const Geo<T> g = load_geo(a.geo, a.ldg, k);
    if (MODE == AM_PFUSE) {
      NbrPfuse<T, Np> src{a.in0, a.in1, zc, beta, s_perm};
      elem_apply<N, T, true>(u, y, g, w, a.geo, a.ldg, T(a.tau), T(a.alpha), src, a.kappa, k);
    } else {
      NbrPlain<T, Np> src{a.in0, s_perm};
      elem_apply<N, T, true>(u, y, g, w, a.geo, a.ldg, T(a.tau), T(a.alpha), src, a.kappa, k);
    }
    if (a.shift != 0.0) {
#pragma unroll
      for (int i = 0; i < Np; ++i) y[i] += T(a.shift) * u[i];
    }
    if (HASB) {
#pragma unroll
      for (int i = 0; i < Np; ++i) {
        y[i] = b2[i] - y[i];
        dA += (double)b2[i] * (double)b2[i];
        dB += (double)y[i] * (double)y[i];
      }
    }
    if (MODE == AM_PFUSE) {
#pragma unroll
      for (int i = 0; i < Np; ++i) dA += (double)u[i] * (double)y[i];
    }
  }
  __syncthreads();  // every tile read done before the tiles are overwritten
  if (MODE == AM_SMOOTH) {
    // x += omega B^-1 r for this thread's element: the residual is already in
    // registers; each packed-symmetric entry of the inverse is loaded once
    // (coalesced across the warp's elements) and used for (i, j) and (j, i)
    if (active) {
      T zv[Np];
#pragma unroll
      for (int i = 0; i < Np; ++i) zv[i] = T(0);
      const T* bk = a.binv + k0 + tid;
#pragma unroll
      for (int i = 0; i < Np; ++i)
#pragma unroll
        for (int j = i; j < Np; ++j) {
          const T b = __ldg(bk + (size_t)sym_idx(Np, i, j) * a.ldb);
          zv[i] = fma(b, y[j], zv[i]);
          if (j != i) zv[j] = fma(b, y[i], zv[j]);
        }
      const T om = T(a.omega);
#pragma unroll
      for (int i = 0; i < Np; ++i) s_tile[0][tid * Np + i] += om * zv[i];
    }
  } else if (active) {
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      s_tile[0][tid * Np + i] = y[i];
      if (MODE == AM_PFUSE) s_tile[1][tid * Np + i] = u[i];
    }
  }
  if (tma) fence_proxy_async_smem();
  __syncthreads();
  if (tma) {
    if (tid == 0) {
      bulk_store(a.out0 + off, s_tile[0], bytes);
      if (MODE == AM_PFUSE) bulk_store(a.out1 + off, s_tile[1], bytes);
      bulk_commit();
      bulk_wait_read_all();
    }
  } else {
    for (int i = tid; i < nk * Np; i += BLOCK) {
      a.out0[off + i] = s_tile[0][i];
      if (MODE == AM_PFUSE) a.out1[off + i] = s_tile[1][i];
    }
  }
  if (MODE == AM_APPLY || MODE == AM_SMOOTH) return;

  // reductions: block partials -> last block -> control block
  block_sum2<BLOCK>(dA, dB, s_red);
  if (tid == 0) {
    a.partA[blockIdx.x] = dA;
    a.partB[blockIdx.x] = dB;
  }
  if (!is_last_block(&a.ctl->ticket)) return;
  double sA, sB;
  reduce_partials2<BLOCK>(a.partA, a.partB, gridDim.x, sA, sB, s_red);
  if (tid == 0) {
    CgCtl* c = a.ctl;
    if (MODE == AM_PFUSE) {
      c->pAp = sA;
      const double al = c->gamma / sA;
      if (!(sA > 0.0) || !isfinite(al)) {
        c->status = 2;  // breakdown
        c->alpha = 0.0;
      } else {
        c->alpha = al;
      }
    } else {
      c->bb = sA;
      c->rr = sB;
    }
    c->ticket = 0u;
  }
}

// ====================================================== node-major apply
// y = A u + alpha J M u for the elements [k_begin, k_end) of fields stored
// node-major, (Np, ld) row-major with ld = K: the reference's own (Np, K)
// field layout (src/ddg/dg2d/sipg.py:304-337 takes and returns (Np, K)).
// Thread k reads u[i * ld + k], so each warp load is one coalesced 256-byte
// (float64) row segment and no shared-memory staging is needed.  Used by the
// host-buffer entry point, which copies (Np, K) fields chunk by chunk and
// launches this kernel per element chunk as soon as the chunk's neighbours
// have arrived.
template <typename T, int Np>
struct NbrNodeMajor {
  const T* __restrict__ u;
  int ld;
  const int* perm;  // shared memory, 3*Np
  __device__ __forceinline__ void operator()(int kp, int fp, T (&ut)[Np]) const {
#pragma unroll
    for (int i = 0; i < Np; ++i) ut[i] = __ldg(u + (size_t)perm[fp * Np + i] * ld + kp);
  }
};

template <int N, typename T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_apply_nm(ApplyArgs<T> a, int k_begin, int k_end) {
  constexpr int Np = Dim<N>::Np;
  __shared__ int s_perm[3 * Np];
  for (int i = threadIdx.x; i < 3 * Np; i += BLOCK) s_perm[i] = a.perm[i];
  __syncthreads();
  const int k = k_begin + blockIdx.x * BLOCK + threadIdx.x;
  if (k >= k_end) return;
  const int ld = a.K;
  T u[Np], y[Np];
#pragma unroll
  for (int i = 0; i < Np; ++i) u[i] = __ldg(a.in0 + (size_t)i * ld + k);
  uint32_t w[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) w[f] = __ldg(a.nbr + (size_t)f * a.K + k);
  const Geo<T> g = load_geo(a.geo, a.ldg, k);
  NbrNodeMajor<T, Np> src{a.in0, ld, s_perm};
  elem_apply<N, T, true>(u, y, g, w, a.geo, a.ldg, T(a.tau), T(a.alpha), src, a.kappa, k);
  if (a.shift != 0.0) {
#pragma unroll
    for (int i = 0; i < Np; ++i) y[i] += T(a.shift) * u[i];
  }
#pragma unroll
  for (int i = 0; i < Np; ++i) a.out0[(size_t)i * ld + k] = y[i];
}

// ================================================================= CG
// One CG step after the apply: x += alpha p; r -= alpha Ap; z = B^-1 r;
// partials r.z, r.r -> last block: gamma, beta, iter, loop condition.
// INIT: r given (from AM_RESID), no x/p update; zeroes p_old, sets
// gamma0 = r.z, beta = 0, iter = 0.
template <int N, typename T, bool PC, bool INIT, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_cg_step(CgArgs<T> a) {
  constexpr int Np = Dim<N>::Np;
  __shared__ __align__(16) T s_r[BLOCK * Np];  // r tile, then z tile (PC)
  __shared__ double s_red[64];
  if (!INIT && a.ctl->cont == 0) {
    // the loop already stopped: make sure the while node sees 0
    if (a.has_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.cond, 0u);
    return;
  }
  const int tid = threadIdx.x;
  const T al = INIT ? T(0) : T(a.ctl->alpha);
  double rr = 0.0, rz = 0.0, rp = 0.0;
  // persistent over element tiles: one partial per block, so the last
  // block's reduction (the serial tail of the step) stays short
  const int ntiles = (a.K + BLOCK - 1) / BLOCK;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
  const int k0 = tile * BLOCK;
  const int nk = min(BLOCK, a.K - k0);
  const size_t off = (size_t)k0 * Np;
  if (!INIT && nk == BLOCK) {
    // full tile: x += alpha p, r -= alpha Ap with the vectors marked
    // non-aliasing and the loads of five tile rows issued together (the
    // plain-pointer loop serialised every load behind the previous store)
    T* __restrict__ x = a.x + off;
    const T* __restrict__ p = a.p + off;
    T* __restrict__ r = a.r + off;
    const T* __restrict__ Ap = a.Ap + off;
    constexpr int STEP = (Np % 5 == 0) ? 5 : ((Np % 3 == 0) ? 3 : 1);  // rows per batch, divides Np
#pragma unroll
    for (int c = 0; c < Np; c += STEP) {
      T xv[STEP], pv[STEP], rv0[STEP], av[STEP];
#pragma unroll
      for (int u = 0; u < STEP; ++u) {
        const int i = tid + (c + u) * BLOCK;
        xv[u] = x[i];
        pv[u] = __ldg(p + i);
        rv0[u] = r[i];
        av[u] = __ldg(Ap + i);
      }
#pragma unroll
      for (int u = 0; u < STEP; ++u) {
        const int i = tid + (c + u) * BLOCK;
        x[i] = fma(al, pv[u], xv[u]);
        const T rn = fma(-al, av[u], rv0[u]);
        r[i] = rn;
        rr += (double)rn * (double)rn;
        if (PC) s_r[i] = rn;
      }
    }
  } else {
    for (int i = tid; i < nk * Np; i += BLOCK) {
      T rn;
      if (INIT) {
        rn = a.r[off + i];
        if (!a.keep_p) a.p_zero[off + i] = T(0);
        else rp += (double)rn * (double)a.p_zero[off + i];
      } else {
        a.x[off + i] += al * a.p[off + i];
        rn = a.r[off + i] - al * a.Ap[off + i];
        a.r[off + i] = rn;
      }
      rr += (double)rn * (double)rn;
      if (PC) s_r[i] = rn;
    }
  }
  if (PC) {
    // z = B^-1 r, one element per thread with the packed-symmetric indices
    // known at compile time: each load of the inverse is one coalesced row
    // segment across the warp's elements and each entry is loaded once
    __syncthreads();
    if (tid < nk) {
      T rv[Np], zv[Np];
#pragma unroll
      for (int j = 0; j < Np; ++j) {
        rv[j] = s_r[tid * Np + j];
        zv[j] = T(0);
      }
      const T* bk = a.binv + k0 + tid;
#pragma unroll
      for (int i = 0; i < Np; ++i)
#pragma unroll
        for (int j = i; j < Np; ++j) {
          const T b = __ldg(bk + (size_t)sym_idx(Np, i, j) * a.ldb);
          zv[i] = fma(b, rv[j], zv[i]);
          if (j != i) zv[j] = fma(b, rv[i], zv[j]);
        }
#pragma unroll
      for (int i = 0; i < Np; ++i) {
        s_r[tid * Np + i] = zv[i];  // own slots only: rv was read above
        rz += (double)rv[i] * (double)zv[i];
      }
    }
    __syncthreads();
    for (int i = tid; i < nk * Np; i += BLOCK) a.z[off + i] = s_r[i];
    __syncthreads();  // the next tile refills s_r
  }
  }  // tiles
  if (!PC) rz = rr;
  block_sum2<BLOCK>(rz, rr, s_red);
  if (INIT) {
    double d0 = 0.0;
    block_sum2<BLOCK>(rp, d0, s_red);
  }
  if (tid == 0) {
    a.partA[blockIdx.x] = rz;
    a.partB[blockIdx.x] = rr;
    if (INIT) a.partC[blockIdx.x] = rp;
  }
  if (!is_last_block(&a.ctl->ticket)) return;
  double g, r2, gp = 0.0, d1;
  reduce_partials2<BLOCK>(a.partA, a.partB, gridDim.x, g, r2, s_red);
  if (INIT && a.keep_p) reduce_partials2<BLOCK>(a.partC, nullptr, gridDim.x, gp, d1, s_red);
  if (tid == 0) {
    CgCtl* c = a.ctl;
    if (INIT) {
      c->atol2 = fmax(c->tol2 * c->bb, c->atol_sq);
      // a reliable-update restart keeps the search direction: beta from the
      // previous gamma; a fresh start has p_old = 0 and beta = 0
      c->beta = (a.keep_p && c->gamma_prev != 0.0) ? g / c->gamma_prev : 0.0;
      // restore r.p = 0 after the residual replacement:
      // p_old <- p_old - (r.p_old / r.z) z, folded into the next direction
      c->zcoef = (a.keep_p && g != 0.0) ? 1.0 - c->beta * (gp / g) : 1.0;
      c->iter = 0;
      c->status = 0;
    } else {
      c->gamma_prev = c->gamma;
      c->beta = g / c->gamma;
      c->zcoef = 1.0;
      c->iter += 1;
    }
    c->gamma = g;
    c->rr = r2;
    const double rs = c->use_pc ? r2 : g;
    int cont = (rs > c->atol2) && (c->iter < c->maxiter) && (c->status == 0);
    if (!isfinite(g) || !isfinite(r2)) {
      c->status = 2;
      cont = 0;
    }
    if (!INIT && !isfinite(c->beta)) {
      c->status = 2;
      cont = 0;
    }
    if (a.dev_status && *(volatile const unsigned int*)a.dev_status != 0u) {
      c->status = 3;  // a kernel reported a device-side error: stop now
      cont = 0;
    }
    if (cont == 0 && c->status == 0 && rs > c->atol2) c->status = 1;  // maxiter
    c->cont = cont;
    c->ticket = 0u;
    if (a.has_cond) cudaGraphSetConditional(a.cond, (unsigned)cont);
  }
}

// CG step with the element tiles staged by bulk copies (the regular
// iteration, all vectors 16-byte aligned): thread 0 copies the x, p, r and
// Ap tiles into shared memory at once, each thread updates its own element
// (x += alpha p, r -= alpha Ap, z = B^-1 r with the packed-symmetric inverse
// loaded once per entry), and the x, r, z tiles go back by bulk stores.
// Same scalars, partials and loop control as k_cg_step.
template <int N, typename T, bool PC, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_cg_step_bulk(CgArgs<T> a) {
  constexpr int Np = Dim<N>::Np;
  __shared__ __align__(128) T s_x[BLOCK * Np];
  __shared__ __align__(128) T s_p[BLOCK * Np];   // p, then z
  __shared__ __align__(128) T s_r[BLOCK * Np];
  __shared__ __align__(128) T s_a[BLOCK * Np];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ double s_red[64];
  __shared__ int s_ok;
  grid_dep_wait();
  if (a.ctl->cont == 0) {
    if (a.has_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(a.cond, 0u);
    return;
  }
  const int tid = threadIdx.x;
  const int k0 = blockIdx.x * BLOCK, nk = min(BLOCK, a.K - k0);
  const size_t off = (size_t)k0 * Np;
  const uint32_t bytes = (uint32_t)(nk * Np * sizeof(T));
  const bool bulk = (bytes % 16u) == 0u;  // the launcher checked the base alignment
  const T al = T(a.ctl->alpha);
  double rr = 0.0, rz = 0.0;
  if (bulk) {
    if (tid == 0) {
      mbar_init(&s_bar, 1);
      fence_mbar_init();
      mbar_expect_tx(&s_bar, 4u * bytes);
      bulk_load(s_x, a.x + off, bytes, &s_bar);
      bulk_load(s_p, a.p + off, bytes, &s_bar);
      bulk_load(s_r, a.r + off, bytes, &s_bar);
      bulk_load(s_a, a.Ap + off, bytes, &s_bar);
      s_ok = mbar_wait_bounded(&s_bar, 0, const_cast<unsigned int*>(a.dev_status)) ? 1 : 0;
    }
    __syncthreads();
  } else {
    for (int i = tid; i < nk * Np; i += BLOCK) {
      s_x[i] = a.x[off + i];
      s_p[i] = a.p[off + i];
      s_r[i] = a.r[off + i];
      s_a[i] = a.Ap[off + i];
    }
    if (tid == 0) s_ok = 1;
    __syncthreads();
  }
  if (s_ok && tid < nk) {
    T rv[Np];
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      const int j = tid * Np + i;
      s_x[j] = fma(al, s_p[j], s_x[j]);
      rv[i] = fma(-al, s_a[j], s_r[j]);
      s_r[j] = rv[i];
      rr += (double)rv[i] * (double)rv[i];
    }
    if (PC) {
      T zv[Np];
      sym_block_apply<Np, T>(a.binv + k0 + tid, (size_t)a.ldb, rv, zv);
#pragma unroll
      for (int i = 0; i < Np; ++i) {
        s_p[tid * Np + i] = zv[i];  // own slots: p was read above
        rz += (double)rv[i] * (double)zv[i];
      }
    } else {
      rz = rr;
    }
  }
  if (s_ok) {
    if (bulk) {
      fence_proxy_async_smem();
      __syncthreads();
      if (tid == 0) {
        bulk_store(a.x + off, s_x, bytes);
        bulk_store(a.r + off, s_r, bytes);
        if (PC) bulk_store(a.z + off, s_p, bytes);
        bulk_commit();
        bulk_wait_read_all();
      }
    } else {
      __syncthreads();
      for (int i = tid; i < nk * Np; i += BLOCK) {
        a.x[off + i] = s_x[i];
        a.r[off + i] = s_r[i];
        if (PC) a.z[off + i] = s_p[i];
      }
    }
  }
  block_sum2<BLOCK>(rz, rr, s_red);
  if (tid == 0) {
    a.partA[blockIdx.x] = rz;
    a.partB[blockIdx.x] = rr;
  }
  if (!is_last_block(&a.ctl->ticket)) return;
  double g, r2, d1;
  reduce_partials2<BLOCK>(a.partA, a.partB, gridDim.x, g, r2, s_red);
  (void)d1;
  if (tid == 0) {
    CgCtl* c = a.ctl;
    c->gamma_prev = c->gamma;
    c->beta = g / c->gamma;
    c->zcoef = 1.0;
    c->iter += 1;
    c->gamma = g;
    c->rr = r2;
    const double rs = c->use_pc ? r2 : g;
    int cont = (rs > c->atol2) && (c->iter < c->maxiter) && (c->status == 0);
    if (!isfinite(g) || !isfinite(r2) || !isfinite(c->beta)) {
      c->status = 2;
      cont = 0;
    }
    if (a.dev_status && *(volatile const unsigned int*)a.dev_status != 0u) {
      c->status = 3;  // a kernel reported a device-side error: stop now
      cont = 0;
    }
    if (cont == 0 && c->status == 0 && rs > c->atol2) c->status = 1;  // maxiter
    c->cont = cont;
    c->ticket = 0u;
    if (a.has_cond) cudaGraphSetConditional(a.cond, (unsigned)cont);
  }
}

// ========================================================= block Jacobi
// Self block column j of element k = (local operator with zero neighbour
// values) applied to e_j: the coloured probe of sipg.py:671-704 without
// the colouring.  Output blocks[k][i][j] (row-major per element, float64).
template <int N, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_self_blocks(BlockArgs a) {
  constexpr int Np = Dim<N>::Np;
  const int kl = blockIdx.x * BLOCK + threadIdx.x;
  if (kl >= a.K) return;
  const int k = a.k0 + kl;
  const size_t ld = a.nbr_ld ? (size_t)a.nbr_ld : (size_t)a.K;
  uint32_t w[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) w[f] = __ldg(a.nbr + (size_t)f * ld + k);
  const Geo<double> g = load_geo(a.geo, a.ldg, k);
  const double al = a.alpha_e ? a.alpha_e[k] : a.alpha;
  NbrZero<double, Np> src;
  for (int j = 0; j < Np; ++j) {
    double u[Np], y[Np];
#pragma unroll
    for (int i = 0; i < Np; ++i) u[i] = (i == j) ? 1.0 : 0.0;
    elem_apply<N, double, false>(u, y, g, w, a.geo, a.ldg, a.tau, al, src, a.kappa, k);
#pragma unroll
    for (int i = 0; i < Np; ++i) a.blocks[(size_t)kl * Np * Np + i * Np + j] = y[i] + (i == j ? a.shift : 0.0);
  }
}

// Gauss-Jordan inverse with partial pivoting per element; writes the
// inverse, symmetrised and packed (upper triangle), structure-of-arrays
// binv[sym_idx(i, j) ldb + k] in float64 and float32.
template <int N, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_invert_blocks(BlockArgs a) {
  constexpr int Np = Dim<N>::Np;
  const int kl = blockIdx.x * BLOCK + threadIdx.x;
  if (kl >= a.K) return;
  const int k = a.k0 + kl;
  double m[Np][2 * Np];
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) {
      m[i][j] = a.blocks[(size_t)kl * Np * Np + i * Np + j];
      m[i][Np + j] = (i == j) ? 1.0 : 0.0;
    }
  bool ok = true;
  for (int c = 0; c < Np; ++c) {
    int piv = c;
    double best = fabs(m[c][c]);
    for (int i = c + 1; i < Np; ++i)
      if (fabs(m[i][c]) > best) {
        best = fabs(m[i][c]);
        piv = i;
      }
    if (!(best > 0.0)) {
      ok = false;
      break;
    }
    if (piv != c)
      for (int j = 0; j < 2 * Np; ++j) {
        const double t = m[c][j];
        m[c][j] = m[piv][j];
        m[piv][j] = t;
      }
    const double inv = 1.0 / m[c][c];
    for (int j = 0; j < 2 * Np; ++j) m[c][j] *= inv;
    for (int i = 0; i < Np; ++i) {
      if (i == c) continue;
      const double fct = m[i][c];
      if (fct != 0.0)
        for (int j = 0; j < 2 * Np; ++j) m[i][j] -= fct * m[c][j];
    }
  }
  if (!ok) atomicOr(a.status, ST_BAD_INDEX);
  for (int i = 0; i < Np; ++i)
    for (int j = i; j < Np; ++j) {
      const double v = ok ? 0.5 * (m[i][Np + j] + m[j][Np + i]) : NAN;
      a.binv64[(size_t)sym_idx(Np, i, j) * a.ldb + k] = v;
      if (a.binv32) a.binv32[(size_t)sym_idx(Np, i, j) * a.ldb + k] = (float)v;
    }
}

// z = B^-1 r for every element (the standalone preconditioner callable).
template <int N, typename T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_pc_apply(const T* __restrict__ r, T* __restrict__ z,
                                                      const T* __restrict__ binv, int ldb, int K) {
  constexpr int Np = Dim<N>::Np;
  __shared__ __align__(16) T s[BLOCK * Np];
  const int tid = threadIdx.x, k0 = blockIdx.x * BLOCK, nk = min(BLOCK, K - k0);
  const size_t off = (size_t)k0 * Np;
  for (int i = tid; i < nk * Np; i += BLOCK) s[i] = r[off + i];
  __syncthreads();
  if (tid < nk) {
    const int k = k0 + tid;
    T rv[Np], zv[Np];
#pragma unroll
    for (int j = 0; j < Np; ++j) {
      rv[j] = s[tid * Np + j];
      zv[j] = T(0);
    }
    // each packed-symmetric entry loaded once, used for (i, j) and (j, i)
#pragma unroll
    for (int i = 0; i < Np; ++i)
#pragma unroll
      for (int j = i; j < Np; ++j) {
        const T b = __ldg(binv + (size_t)sym_idx(Np, i, j) * ldb + k);
        zv[i] = fma(b, rv[j], zv[i]);
        if (j != i) zv[j] = fma(b, rv[i], zv[j]);
      }
#pragma unroll
    for (int i = 0; i < Np; ++i) s[tid * Np + i] = zv[i];
  }
  __syncthreads();
  for (int i = tid; i < nk * Np; i += BLOCK) z[off + i] = s[i];
}

// ================================================================ RHS
// rhs = J M f - L_D(u_dir) + L_N(q_neu)   (sipg.py:852-864, 398-453)
template <int N, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_rhs(RhsArgs a) {
  constexpr int Np = Dim<N>::Np, Nfp = Dim<N>::Nfp;
  const int k = blockIdx.x * BLOCK + threadIdx.x;
  if (k >= a.K) return;
  const RefMats<N, double>& R = CRef<N, double>::get();
  const Geo<double> g = load_geo(a.geo, a.ldg, k);
  double y[Np];
#pragma unroll
  for (int i = 0; i < Np; ++i) y[i] = 0.0;
  if (a.f) {
    double fv[Np];
#pragma unroll
    for (int j = 0; j < Np; ++j) fv[j] = a.f[(size_t)k * Np + j];
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < Np; ++j) s = fma(R.M[i * Np + j], fv[j], s);
      y[i] = g.J * s;
    }
  }
  uint32_t w[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) w[f] = __ldg(a.nbr + (size_t)f * a.K + k);
  if (a.u_dir) {
    // Dirichlet load with u = 0: only Dirichlet-tagged faces contribute.
    double yd[Np], ex[Np], ey[Np];
#pragma unroll
    for (int i = 0; i < Np; ++i) yd[i] = ex[i] = ey[i] = 0.0;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      if (((w[f] >> 3) & 3) != 1) continue;
      const double sJ = g.sJ[f], tauM = a.tau * sJ / g.J;
      double ud[Nfp];
#pragma unroll
      for (int p = 0; p < Nfp; ++p) ud[p] = a.u_dir[(size_t)k * Np + fmask_idx(N, f, p)];
#pragma unroll
      for (int q = 0; q < Nfp; ++q) {
        double s1 = 0.0, s2 = 0.0;
#pragma unroll
        for (int p = 0; p < Nfp; ++p) {
          const double m = R.m1d[(f * Nfp + p) * Nfp + q];
          s1 = fma(m, -tauM * ud[p], s1);
          s2 = fma(m, -ud[p], s2);
        }
        const int n = fmask_idx(N, f, q);
        yd[n] += sJ * s1;
        ex[n] -= sJ * g.nx[f] * s2;
        ey[n] -= sJ * g.ny[f] * s2;
      }
    }
    double tr[Np], ts[Np];
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      tr[i] = g.rx * ex[i] + g.ry * ey[i];
      ts[i] = g.sx * ex[i] + g.sy * ey[i];
    }
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      double s = yd[i];
#pragma unroll
      for (int j = 0; j < Np; ++j) {
        s = fma(R.Dr[j * Np + i], tr[j], s);
        s = fma(R.Ds[j * Np + i], ts[j], s);
      }
      y[i] -= s;
    }
  }
  if (a.q_neu) {
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      if (((w[f] >> 3) & 3) != 2) continue;
      double q[Nfp];
#pragma unroll
      for (int p = 0; p < Nfp; ++p) q[p] = a.q_neu[(size_t)k * 3 * Nfp + f * Nfp + p];
#pragma unroll
      for (int p = 0; p < Nfp; ++p) {
        double s = 0.0;
#pragma unroll
        for (int qq = 0; qq < Nfp; ++qq) s = fma(R.m1d[(f * Nfp + p) * Nfp + qq], q[qq], s);
        y[fmask_idx(N, f, p)] += g.sJ[f] * s;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < Np; ++i) a.rhs[(size_t)k * Np + i] = y[i];
}

// ================================================= mixed precision helpers
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_cast_norm(int64_t n, const double* __restrict__ r64,
                                                      float* __restrict__ r32, float* __restrict__ x32,
                                                      double* part, CgCtl* ctl) {
  __shared__ double s_red[64];
  double s = 0.0, d = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * BLOCK) {
    const float v = (float)r64[i];
    r32[i] = v;
    x32[i] = 0.0f;
    s += (double)v * (double)v;
  }
  block_sum2<BLOCK>(s, d, s_red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
  if (!is_last_block(&ctl->ticket)) return;
  double t, u;
  reduce_partials2<BLOCK>(part, nullptr, gridDim.x, t, u, s_red);
  if (threadIdx.x == 0) {
    ctl->bb = t;
    ctl->ticket = 0u;
  }
}

__global__ void k_axpy_mixed(int64_t n, const float* __restrict__ x32, double* __restrict__ x64) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x64[i] += (double)x32[i];
}

// ================================================= kappa gradient (adjoint)
// g_k = d a(u, lam; kappa) / d kappa_k: the volume term of element k plus,
// per face, the derivative of the kappa-weighted average and penalty terms
// (own side and, through the neighbour's half of an interior face, the
// neighbour side).  Only the neighbours' traces are needed.
template <int N, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_grad_kappa(GradArgs a) {
  constexpr int Np = Dim<N>::Np, Nfp = Dim<N>::Nfp;
  __shared__ int s_perm[3 * Np];
  for (int i = threadIdx.x; i < 3 * Np; i += BLOCK) s_perm[i] = a.perm[i];
  __syncthreads();
  const int k = blockIdx.x * BLOCK + threadIdx.x;
  if (k >= a.K) return;
  const RefMats<N, double>& R = CRef<N, double>::get();
  const Geo<double> g = load_geo(a.geo, a.ldg, k);
  double u[Np], l[Np], ux[Np], uy[Np], lx[Np], ly[Np];
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    u[i] = a.u[(size_t)k * Np + i];
    l[i] = a.lam[(size_t)k * Np + i];
  }
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    double ur = 0, us = 0, lr = 0, ls = 0;
#pragma unroll
    for (int j = 0; j < Np; ++j) {
      ur = fma(R.Dr[i * Np + j], u[j], ur);
      us = fma(R.Ds[i * Np + j], u[j], us);
      lr = fma(R.Dr[i * Np + j], l[j], lr);
      ls = fma(R.Ds[i * Np + j], l[j], ls);
    }
    ux[i] = g.rx * ur + g.sx * us;
    uy[i] = g.ry * ur + g.sy * us;
    lx[i] = g.rx * lr + g.sx * ls;
    ly[i] = g.ry * lr + g.sy * ls;
  }
  double acc = 0.0;   // volume: J ux.(M lx) + uy.(M ly)   (sipg.py:189 with v = lam)
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    double mx = 0, my = 0;
#pragma unroll
    for (int j = 0; j < Np; ++j) {
      mx = fma(R.M[i * Np + j], lx[j], mx);
      my = fma(R.M[i * Np + j], ly[j], my);
    }
    acc += ux[i] * mx + uy[i] * my;
  }
  acc *= g.J;
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    const uint32_t wf = __ldg(a.nbr + (size_t)f * a.K + k);
    const int bc = (wf >> 3) & 3;
    const bool pact = (wf >> 5) & 1, mint = (wf >> 6) & 1, mdir = (bc == 1);
    if (!(pact || mint || mdir)) continue;
    const double sJ = g.sJ[f], nx = g.nx[f], ny = g.ny[f];
    const double tauM = a.tau * sJ / g.J;
    double uM[Nfp], lM[Nfp], dU[Nfp], dL[Nfp], uP[Nfp], lP[Nfp];
#pragma unroll
    for (int p = 0; p < Nfp; ++p) {
      const int n = fmask_idx(N, f, p);
      uM[p] = u[n];
      lM[p] = l[n];
      dU[p] = nx * ux[n] + ny * uy[n];
      dL[p] = nx * lx[n] + ny * ly[n];
      uP[p] = lP[p] = 0.0;
    }
    double tauP = tauM;
    if (pact || mint) {
      const int kp = (int)(wf >> 7), fp = (int)(wf & 3);
      const bool flip = (wf >> 2) & 1;
      tauP = a.tau * sJ / __ldg(a.geo + G_J * a.ldg + kp);
      double ut[Nfp], lt[Nfp];
#pragma unroll
      for (int q = 0; q < Nfp; ++q) {
        const size_t o = (size_t)kp * Np + s_perm[fp * Np + q];
        ut[q] = __ldg(a.u + o);
        lt[q] = __ldg(a.lam + o);
      }
#pragma unroll
      for (int p = 0; p < Nfp; ++p) {
        uP[p] = flip ? ut[N - p] : ut[p];
        lP[p] = flip ? lt[N - p] : lt[p];
      }
    }
    // weights: Dirichlet own side 1 (jumps against zero), interior halves 1/4
    const double cA = mdir ? 1.0 : (mint ? 0.25 : 0.0) + (pact ? 0.25 : 0.0);
    const double cT = mdir ? tauM : (mint ? 0.25 * tauM : 0.0) + (pact ? 0.25 * tauP : 0.0);
    const double* m1 = R.m1d + f * Nfp * Nfp;
    double face = 0.0;
#pragma unroll
    for (int p = 0; p < Nfp; ++p) {
      const double jU = mdir ? uM[p] : uM[p] - uP[p];
#pragma unroll
      for (int q = 0; q < Nfp; ++q) {
        const double jL = mdir ? lM[q] : lM[q] - lP[q];
        face += m1[p * Nfp + q] * (-cA * (dU[p] * jL + jU * dL[q]) + cT * jU * jL);
      }
    }
    if (mdir && pact) {   // neighbour's interior half across a Dirichlet-tagged face
#pragma unroll
      for (int p = 0; p < Nfp; ++p)
#pragma unroll
        for (int q = 0; q < Nfp; ++q) {
          const double jU = uM[p] - uP[p], jL = lM[q] - lP[q];
          face += m1[p * Nfp + q] * (-0.25 * (dU[p] * jL + jU * dL[q]) + 0.25 * tauP * jU * jL);
        }
    }
    acc += sJ * face;
  }
  a.g[k] = acc;
}

template <int N>
static cudaError_t launch_grad_n(const GradArgs& a, cudaStream_t s) {
  constexpr int B = 128;
  k_grad_kappa<N, B><<<(a.K + B - 1) / B, B, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_grad_kappa(int N, const GradArgs& a, cudaStream_t s) {
  switch (N) {
    case 1: return launch_grad_n<1>(a, s);
    case 2: return launch_grad_n<2>(a, s);
    case 3: return launch_grad_n<3>(a, s);
    case 4: return launch_grad_n<4>(a, s);
    case 5: return launch_grad_n<5>(a, s);
  }
  return cudaErrorInvalidValue;
}

// ============================================================ vectors
__global__ void k_axpby(int64_t n, double al, const double* __restrict__ x, double be, double* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = al * x[i] + be * y[i];
}
template <typename S, typename D>
__global__ void k_cast(int64_t n, const S* __restrict__ s, D* __restrict__ d) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = (D)s[i];
}
template <typename T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_dot(int64_t n, const T* __restrict__ x, const T* __restrict__ y,
                                                double* part, unsigned int* ticket, double* out) {
  __shared__ double s_red[64];
  double s = 0.0, d = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * BLOCK)
    s += (double)x[i] * (double)y[i];
  block_sum2<BLOCK>(s, d, s_red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
  if (!is_last_block(ticket)) return;
  double t, u;
  reduce_partials2<BLOCK>(part, nullptr, gridDim.x, t, u, s_red);
  if (threadIdx.x == 0) {
    *out = t;
    *ticket = 0u;
  }
}

// ============================================================ launchers
template <int N, typename T> struct CRefSym;
#define DDG_SYM(NN)                                                                        \
  template <> struct CRefSym<NN, double> { static const void* sym() { return &c_ref64_##NN; } }; \
  template <> struct CRefSym<NN, float> { static const void* sym() { return &c_ref32_##NN; } };
DDG_SYM(1)
DDG_SYM(2)
DDG_SYM(3)
DDG_SYM(4)
DDG_SYM(5)
template <int N> struct CPairSym;
#define DDG_PSYM(NN) \
  template <> struct CPairSym<NN> { static const void* sym() { return &c_pair32_##NN; } };
DDG_PSYM(1)
DDG_PSYM(2)
DDG_PSYM(3)
DDG_PSYM(4)
DDG_PSYM(5)

namespace {
template <int N, typename T>
cudaError_t upload_one(const double* Dr, const double* Ds, const double* M, const double* m1d) {
  constexpr int Np = Dim<N>::Np, Nfp = Dim<N>::Nfp;
  RefMats<N, T> h;
  for (int i = 0; i < Np * Np; ++i) {
    h.Dr[i] = (T)Dr[i];
    h.Ds[i] = (T)Ds[i];
    h.M[i] = (T)M[i];
  }
  for (int i = 0; i < 3 * Nfp * Nfp; ++i) h.m1d[i] = (T)m1d[i];
  cudaError_t e = cudaMemcpyToSymbol(CRefSym<N, T>::sym(), &h, sizeof(h));
  if (e != cudaSuccess || sizeof(T) != 4) return e;
  RefPairs<N> pr{};
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) {
      pr.DrDs[i * Np + j] = make_float2((float)Dr[i * Np + j], (float)Ds[i * Np + j]);
      pr.DrDsT[i * Np + j] = make_float2((float)Dr[j * Np + i], (float)Ds[j * Np + i]);
    }
  for (int r = 0; r < Np / 2; ++r)
    for (int j = 0; j < Np; ++j)
      pr.MP[r * Np + j] = make_float2((float)M[2 * r * Np + j], (float)M[(2 * r + 1) * Np + j]);
  return cudaMemcpyToSymbol(CPairSym<N>::sym(), &pr, sizeof(pr));
}
}  // namespace



template <int N>
static cudaError_t upload_n(const double* Dr, const double* Ds, const double* M, const double* m1d) {
  cudaError_t e = upload_one<N, double>(Dr, Ds, M, m1d);
  if (e != cudaSuccess) return e;
  return upload_one<N, float>(Dr, Ds, M, m1d);
}

cudaError_t upload_ref(int N, const double* Dr, const double* Ds, const double* M, const double* m1d) {
  switch (N) {
    case 1: return upload_n<1>(Dr, Ds, M, m1d);
    case 2: return upload_n<2>(Dr, Ds, M, m1d);
    case 3: return upload_n<3>(Dr, Ds, M, m1d);
    case 4: return upload_n<4>(Dr, Ds, M, m1d);
    case 5: return upload_n<5>(Dr, Ds, M, m1d);
  }
  return cudaErrorInvalidValue;
}

template <typename T> constexpr int apply_block() { return sizeof(T) == 8 ? 128 : 128; }

template <int N, typename T>
static cudaError_t launch_apply_n(int mode, const ApplyArgs<T>& a, cudaStream_t s) {
  if constexpr (sizeof(T) == 8) {
    if (dm_handles(mode, a)) return launch_apply_dm(N, mode, a, s);
  }
  constexpr int B = apply_block<T>();
  const int span = (mode == AM_APPLY && a.k_hi > 0) ? a.k_hi - a.k_lo : a.K;
  if (span <= 0) return cudaSuccess;
  const int grid = (span + B - 1) / B;
  switch (mode) {
    case AM_APPLY: k_apply<N, T, AM_APPLY, B><<<grid, B, 0, s>>>(a); break;
    case AM_PFUSE: k_apply<N, T, AM_PFUSE, B><<<grid, B, 0, s>>>(a); break;
    case AM_RESID: k_apply<N, T, AM_RESID, B><<<grid, B, 0, s>>>(a); break;
    case AM_SMOOTH: k_apply<N, T, AM_SMOOTH, B><<<grid, B, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_apply(int N, int mode, const ApplyArgs<T>& a, cudaStream_t s) {
  switch (N) {
    case 1: return launch_apply_n<1, T>(mode, a, s);
    case 2: return launch_apply_n<2, T>(mode, a, s);
    case 3: return launch_apply_n<3, T>(mode, a, s);
    case 4: return launch_apply_n<4, T>(mode, a, s);
    case 5: return launch_apply_n<5, T>(mode, a, s);
  }
  return cudaErrorInvalidValue;
}
template cudaError_t launch_apply<double>(int, int, const ApplyArgs<double>&, cudaStream_t);
template cudaError_t launch_apply<float>(int, int, const ApplyArgs<float>&, cudaStream_t);

template <int N, typename T>
static cudaError_t launch_apply_nm_n(const ApplyArgs<T>& a, int k_begin, int k_end, cudaStream_t s) {
  constexpr int B = 128;
  const int n = k_end - k_begin;
  if (n <= 0) return cudaSuccess;
  k_apply_nm<N, T, B><<<(n + B - 1) / B, B, 0, s>>>(a, k_begin, k_end);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_apply_nm(int N, const ApplyArgs<T>& a, int k_begin, int k_end, cudaStream_t s) {
  switch (N) {
    case 1: return launch_apply_nm_n<1, T>(a, k_begin, k_end, s);
    case 2: return launch_apply_nm_n<2, T>(a, k_begin, k_end, s);
    case 3: return launch_apply_nm_n<3, T>(a, k_begin, k_end, s);
    case 4: return launch_apply_nm_n<4, T>(a, k_begin, k_end, s);
    case 5: return launch_apply_nm_n<5, T>(a, k_begin, k_end, s);
  }
  return cudaErrorInvalidValue;
}
template cudaError_t launch_apply_nm<double>(int, const ApplyArgs<double>&, int, int, cudaStream_t);

// Node-major (rows, ld) <-> element-major (ld, rows) transposes of elements
// [k0, k1) for the host-buffer apply (its host arrays are the reference's
// (Np, K) layout).  Tiles of 64 elements: the node-major side is read or
// written one row segment (64 consecutive doubles) at a time, the
// element-major side as one contiguous 64 x rows block; both coalesced.
template <bool TO_EM>
__global__ void __launch_bounds__(256) k_transpose_nm(const double* __restrict__ src, double* __restrict__ dst,
                                                      int ld, int rows, int k0, int k1) {
  extern __shared__ double s_t[];  // [rows][65]
  const int kb = k0 + blockIdx.x * 64, nk = min(64, k1 - kb);
  if (nk <= 0) return;
  if (TO_EM) {
    for (int i = threadIdx.x; i < rows * 64; i += 256) {
      const int r = i / 64, c = i % 64;
      if (c < nk) s_t[r * 65 + c] = src[(size_t)r * ld + kb + c];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nk * rows; i += 256) {
      const int e = i / rows, r = i % rows;
      dst[(size_t)(kb + e) * rows + r] = s_t[r * 65 + e];
    }
  } else {
    for (int i = threadIdx.x; i < nk * rows; i += 256) {
      const int e = i / rows, r = i % rows;
      s_t[r * 65 + e] = src[(size_t)(kb + e) * rows + r];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < rows * 64; i += 256) {
      const int r = i / 64, c = i % 64;
      if (c < nk) dst[(size_t)r * ld + kb + c] = s_t[r * 65 + c];
    }
  }
}

cudaError_t launch_nm_to_em(const double* nm, double* em, int ld, int rows, int k0, int k1, cudaStream_t s) {
  if (k1 <= k0 || rows <= 0) return cudaSuccess;
  k_transpose_nm<true><<<(k1 - k0 + 63) / 64, 256, (size_t)rows * 65 * sizeof(double), s>>>(nm, em, ld, rows, k0, k1);
  return cudaGetLastError();
}

cudaError_t launch_em_to_nm(const double* em, double* nm, int ld, int rows, int k0, int k1, cudaStream_t s) {
  if (k1 <= k0 || rows <= 0) return cudaSuccess;
  k_transpose_nm<false><<<(k1 - k0 + 63) / 64, 256, (size_t)rows * 65 * sizeof(double), s>>>(em, nm, ld, rows, k0, k1);
  return cudaGetLastError();
}


int apply_grid(int K) { return (K + 127) / 128; }
int cg_grid(int K) { return (K + 127) / 128; }

static int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  }
  return n;
}

// Blocks of `kernel` that fill every SM once (occupancy API; cached per
// kernel instantiation by the caller's static).
template <typename Kern>
static int full_wave(Kern kernel, int block) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  return per_sm * sm_count();
}

template <int N, typename T, bool PC, bool INIT>
static void launch_cg_one(const CgArgs<T>& a, cudaStream_t s) {
  if (!INIT && a.bulk) {
    // regular iteration with aligned vectors: tiles staged by bulk copies
    constexpr int BB = sizeof(T) == 8 ? 64 : 128;  // four tiles within the 48 KB of static shared memory
    PdlLaunch l(dim3((a.K + BB - 1) / BB), dim3(BB), 0, s, a.pdl);
    cudaLaunchKernelEx(&l.cfg, k_cg_step_bulk<N, T, PC, BB>, a);
    return;
  }
  constexpr int B = 128;
  static const int wave = full_wave(k_cg_step<N, T, PC, INIT, B>, B);
  const int ntiles = (a.K + B - 1) / B;
  // one resident wave at most: each block loops over tiles and publishes a
  // single partial, so the serial last-block reduction stays short
  k_cg_step<N, T, PC, INIT, B><<<ntiles < wave ? ntiles : wave, B, 0, s>>>(a);
}

template <int N, typename T>
static cudaError_t launch_cg_n(bool pc, bool init, const CgArgs<T>& a, cudaStream_t s) {
  if (pc) {
    if (init) launch_cg_one<N, T, true, true>(a, s);
    else launch_cg_one<N, T, true, false>(a, s);
  } else {
    if (init) launch_cg_one<N, T, false, true>(a, s);
    else launch_cg_one<N, T, false, false>(a, s);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_cg_step(int N, bool pc, bool init, const CgArgs<T>& a, cudaStream_t s) {
  switch (N) {
    case 1: return launch_cg_n<1, T>(pc, init, a, s);
    case 2: return launch_cg_n<2, T>(pc, init, a, s);
    case 3: return launch_cg_n<3, T>(pc, init, a, s);
    case 4: return launch_cg_n<4, T>(pc, init, a, s);
    case 5: return launch_cg_n<5, T>(pc, init, a, s);
  }
  return cudaErrorInvalidValue;
}
template cudaError_t launch_cg_step<double>(int, bool, bool, const CgArgs<double>&, cudaStream_t);
template cudaError_t launch_cg_step<float>(int, bool, bool, const CgArgs<float>&, cudaStream_t);

template <int N>
static cudaError_t launch_blocks_n(const BlockArgs& a, cudaStream_t s) {
  constexpr int B = 64;
  const int grid = (a.K + B - 1) / B;
  k_self_blocks<N, B><<<grid, B, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_invert_blocks<N, B><<<grid, B, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_block_jacobi(int N, const BlockArgs& a, cudaStream_t s) {
  switch (N) {
    case 1: return launch_blocks_n<1>(a, s);
    case 2: return launch_blocks_n<2>(a, s);
    case 3: return launch_blocks_n<3>(a, s);
    case 4: return launch_blocks_n<4>(a, s);
    case 5: return launch_blocks_n<5>(a, s);
  }
  return cudaErrorInvalidValue;
}

template <int N, typename T>
static cudaError_t launch_pc_n(const T* r, T* z, const T* binv, int ldb, int K, cudaStream_t s) {
  constexpr int B = 128;
  k_pc_apply<N, T, B><<<(K + B - 1) / B, B, 0, s>>>(r, z, binv, ldb, K);
  return cudaGetLastError();
}
template <typename T>
cudaError_t launch_pc_apply(int N, const T* r, T* z, const T* binv, int ldb, int K, cudaStream_t s) {
  switch (N) {
    case 1: return launch_pc_n<1, T>(r, z, binv, ldb, K, s);
    case 2: return launch_pc_n<2, T>(r, z, binv, ldb, K, s);
    case 3: return launch_pc_n<3, T>(r, z, binv, ldb, K, s);
    case 4: return launch_pc_n<4, T>(r, z, binv, ldb, K, s);
    case 5: return launch_pc_n<5, T>(r, z, binv, ldb, K, s);
  }
  return cudaErrorInvalidValue;
}
template cudaError_t launch_pc_apply<double>(int, const double*, double*, const double*, int, int, cudaStream_t);
template cudaError_t launch_pc_apply<float>(int, const float*, float*, const float*, int, int, cudaStream_t);

template <int N>
static cudaError_t launch_rhs_n(const RhsArgs& a, cudaStream_t s) {
  constexpr int B = 128;
  k_rhs<N, B><<<(a.K + B - 1) / B, B, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_rhs(int N, const RhsArgs& a, cudaStream_t s) {
  switch (N) {
    case 1: return launch_rhs_n<1>(a, s);
    case 2: return launch_rhs_n<2>(a, s);
    case 3: return launch_rhs_n<3>(a, s);
    case 4: return launch_rhs_n<4>(a, s);
    case 5: return launch_rhs_n<5>(a, s);
  }
  return cudaErrorInvalidValue;
}

static int vec_grid(int64_t n) {
  int64_t g = (n + 255) / 256;
  return (int)(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}
cudaError_t launch_axpby(int64_t n, double al, const double* x, double be, double* y, cudaStream_t s) {
  k_axpby<<<vec_grid(n), 256, 0, s>>>(n, al, x, be, y);
  return cudaGetLastError();
}
// p = zc z + beta p_old for the CG direction (zc, beta from the control
// block; nothing once the loop has stopped), float32, four values per thread
// step; the same rounding as the fused direction update of the applies
__global__ void k_pupd(int64_t n, const float* __restrict__ z, const float* __restrict__ p_old,
                       float* __restrict__ p, const CgCtl* ctl) {
  grid_dep_wait();
  if (ctl->cont == 0) return;
  const float zc = (float)ctl->zcoef, be = (float)ctl->beta;
  const int64_t n4 = n / 4;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    const float4 a = reinterpret_cast<const float4*>(z)[i];
    const float4 b = reinterpret_cast<const float4*>(p_old)[i];
    float4 c;
    c.x = fmaf(zc, a.x, be * b.x);
    c.y = fmaf(zc, a.y, be * b.y);
    c.z = fmaf(zc, a.z, be * b.z);
    c.w = fmaf(zc, a.w, be * b.w);
    reinterpret_cast<float4*>(p)[i] = c;
  }
  for (int64_t i = 4 * n4 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    p[i] = fmaf(zc, z[i], be * p_old[i]);
}
cudaError_t launch_pupd(int64_t n, const float* z, const float* p_old, float* p, const CgCtl* ctl, cudaStream_t s,
                        int pdl) {
  PdlLaunch l(dim3(vec_grid((n + 3) / 4)), dim3(256), 0, s, pdl);
  return cudaLaunchKernelEx(&l.cfg, k_pupd, n, z, p_old, p, ctl);
}

cudaError_t launch_cast(int64_t n, int to_prec, const void* src, void* dst, cudaStream_t s) {
  if (to_prec == 1) k_cast<double, float><<<vec_grid(n), 256, 0, s>>>(n, (const double*)src, (float*)dst);
  else k_cast<float, double><<<vec_grid(n), 256, 0, s>>>(n, (const float*)src, (double*)dst);
  return cudaGetLastError();
}
int dot_grid(int64_t n) { return vec_grid(n); }
cudaError_t launch_cast_norm(int64_t n, const double* r64, float* r32, float* x32, double* part, CgCtl* ctl,
                             cudaStream_t s) {
  k_cast_norm<256><<<vec_grid(n), 256, 0, s>>>(n, r64, r32, x32, part, ctl);
  return cudaGetLastError();
}
cudaError_t launch_axpy_mixed(int64_t n, const float* x32, double* x64, cudaStream_t s) {
  k_axpy_mixed<<<vec_grid(n), 256, 0, s>>>(n, x32, x64);
  return cudaGetLastError();
}
cudaError_t launch_dot(int64_t n, int prec, const void* x, const void* y, double* part, unsigned int* ticket,
                       double* out, cudaStream_t s) {
  const int g = vec_grid(n);
  if (prec == 0) k_dot<double, 256><<<g, 256, 0, s>>>(n, (const double*)x, (const double*)y, part, ticket, out);
  else k_dot<float, 256><<<g, 256, 0, s>>>(n, (const float*)x, (const float*)y, part, ticket, out);
  return cudaGetLastError();
}

}  // namespace ddg

#include "sipg_batch_kernels.cuh"
#include "sipg_tc.cuh"
#include "sipg_dm.cuh"
