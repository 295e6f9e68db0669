// Device code of the matrix-free SIPG operator (sm_100a).
//
// One thread owns one element.  The reference-element matrices (Dr, Ds, M,
// the three face masses) live in __constant__ memory per degree and
// precision; every thread of a warp reads the same entry at the same time,
// so each multiply-add takes its matrix operand straight from the constant
// bank.  Element tiles of the element-major vectors are staged into shared
// memory with TMA bulk copies (cp.async.bulk) and written back the same way.
//
// The operator is the gradient of ddg's SIPG bilinear form
// (src/ddg/dg2d/sipg.py:142-337) written "gather-only": every element
// computes all contributions to its own nodes, including the ones the
// reference scatters from the neighbouring element's side of a shared face,
// so no atomics are needed.  For an interior face (own side M, neighbour P,
// w = 1/2 from each side, sipg.py:135-138):
//   y[Fmask_f]  += sJ * m1d_f^T ( -c_a * avg + c_j * jmp )
//   g_x[Fmask_f] -= sJ * nx * m1d_f^T ( c_g * jmp )      (g_y likewise)
//   y           += Dr^T (rx gx + ry gy) + Ds^T (sx gx + sy gy),
//   gx = M^T (J ux) + face part,
// with avg = (Dn_M + Dn_P)/2, jmp = u_M - u_P and the coefficients
//   own side:  interior c_a=1/2, c_j=tau_M/2, c_g=1/4;
//              Dirichlet c_a=1, c_j=tau_M, c_g=1 (avg=Dn_M, jmp=u_M);
//   neighbour side (its tag interior): c_a+=1/2, c_j+=tau_P/2, c_g+=1/4,
// tau = tau_scale (N+1)^2 sJ / J on each side (sipg.py:263).
//
// The neighbour's normal derivative at the shared face needs face rows of
// Dr/Ds for the neighbour's face f'.  To keep the constant-bank operands
// uniform across a warp (f' differs between neighbouring threads), the
// neighbour's nodal values are gathered through a rotation permutation that
// relabels its vertices so that f' becomes face 0; the chain-rule
// coefficients are rotated to match.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ddg {

template <int N>
struct Dim {
  static constexpr int Np = (N + 1) * (N + 2) / 2;
  static constexpr int Nfp = N + 1;
};

// Face-node indices of the row-by-row warp-and-blend numbering.
__host__ __device__ constexpr int fmask_idx(int N, int f, int p) {
  return f == 0 ? p : (f == 1 ? p * (N + 1) - p * (p - 1) / 2 + (N - p) : p * (N + 1) - p * (p - 1) / 2);
}

template <int N, typename T>
struct RefMats {
  T Dr[Dim<N>::Np * Dim<N>::Np];
  T Ds[Dim<N>::Np * Dim<N>::Np];
  T M[Dim<N>::Np * Dim<N>::Np];
  T m1d[3 * Dim<N>::Nfp * Dim<N>::Nfp];
};

// Constant-memory matrices are defined in sipg_kernels.cu, which also
// specialises CRef for every built degree.
template <int N, typename T> struct CRef;

// float32 operator: the reference matrices paired for the packed FP32 FMA
// of sm_100 (__ffma2_rn, two independent accumulations per instruction):
//   DrDs[i Np + j]  = (Dr[i][j], Ds[i][j])   gradient rows
//   DrDsT[i Np + j] = (Dr[j][i], Ds[j][i])   lift (transposed) rows
//   MP[r Np + j]    = (M[2r][j], M[2r+1][j]) mass rows in pairs
template <int N>
struct RefPairs {
  float2 DrDs[Dim<N>::Np * Dim<N>::Np];
  float2 DrDsT[Dim<N>::Np * Dim<N>::Np];
  float2 MP[(Dim<N>::Np / 2) * Dim<N>::Np + 1];
};
template <int N> struct CPairs;

// Symmetric packed index of (i, j), upper triangle (block-Jacobi inverses
// are stored as Np (Np + 1) / 2 entries per element).
__host__ __device__ constexpr int sym_idx(int Np, int i, int j) {
  return i <= j ? i * Np - i * (i - 1) / 2 + (j - i) : j * Np - j * (j - 1) / 2 + (i - j);
}

// z = B^-1 r for one element from its packed symmetric inverse, stored
// structure-of-arrays with stride ld (bk points at entry 0 of the element):
// every entry is loaded once and used for (i, j) and (j, i).
template <int Np, typename T>
__device__ __forceinline__ void sym_block_apply(const T* __restrict__ bk, size_t ld, const T (&rv)[Np],
                                                T (&zv)[Np]) {
#pragma unroll
  for (int i = 0; i < Np; ++i) zv[i] = T(0);
#pragma unroll
  for (int i = 0; i < Np; ++i)
#pragma unroll
    for (int j = i; j < Np; ++j) {
      const T b = __ldg(bk + (size_t)sym_idx(Np, i, j) * ld);
      zv[i] = fma(b, rv[j], zv[i]);
      if (j != i) zv[j] = fma(b, rv[i], zv[j]);
    }
}

// ---------------------------------------------------------------- layout
// Geometry: structure-of-arrays geo[c * ldg + k].
enum GeoField { G_RX = 0, G_SX, G_RY, G_SY, G_J, G_F0 = 5, G_COUNT = 14 };
// Neighbour word per (face f, element k), nbr[f * K + k]:
//   bits 0-1 neighbour face f' | bit 2 flip | bits 3-4 BC tag of (k,f)
//   bit 5 neighbour side contributes (its tag interior, real neighbour)
//   bit 6 own side interior active (tag interior, real neighbour)
//   bits 7-31 neighbour element k'
__host__ __device__ constexpr uint32_t nbr_pack(uint32_t kp, uint32_t fp, bool flip, uint32_t bc,
                                                bool pact, bool mint) {
  return fp | (flip ? 4u : 0u) | (bc << 3) | (pact ? 32u : 0u) | (mint ? 64u : 0u) | (kp << 7);
}
constexpr uint32_t NBR_MAX_K = (1u << 25) - 1u;

// Device status word bits (written by kernels, read by the host).
enum DevStatus : unsigned int { ST_TMA_TIMEOUT = 1u, ST_BAD_INDEX = 2u };

// ------------------------------------------------------- PTX helpers (TMA)
// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may start while the previous kernel's last CTAs drain; it
// waits here, before touching anything that kernel wrote (returns at once
// for an ordinary launch).
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_load(void* sdst, const void* gsrc, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(sdst)),
      "l"(gsrc), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_addr(ssrc)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Bounded wait on a bulk-copy barrier; on timeout records ST_TMA_TIMEOUT and
// returns false (the caller then skips the tile; nothing spins forever).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, unsigned int* status) {
  for (int it = 0; it < (1 << 22); ++it)
    if (mbar_try_wait(bar, phase)) return true;
  atomicOr(status, ST_TMA_TIMEOUT);
  return false;
}

// ------------------------------------------------------------ reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block sum of two doubles; the result is valid in thread 0.
template <int BLOCK>
__device__ __forceinline__ void block_sum2(double& a, double& b, double* s_red) {
  a = warp_sum(a);
  b = warp_sum(b);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) {
    s_red[warp] = a;
    s_red[32 + warp] = b;
  }
  __syncthreads();
  if (warp == 0) {
    a = lane < BLOCK / 32 ? s_red[lane] : 0.0;
    b = lane < BLOCK / 32 ? s_red[32 + lane] : 0.0;
    a = warp_sum(a);
    b = warp_sum(b);
  }
}

// "Last block done" detection (threadfence reduction).  Every block has
// written its partials before calling; returns true in exactly one block.
__device__ __forceinline__ bool is_last_block(unsigned int* ticket) {
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  return s_last;
}

// Deterministic sum of n partials (fixed order) by one block; valid in thread 0.
template <int BLOCK>
__device__ __forceinline__ void reduce_partials2(const double* pa, const double* pb, int n, double& a, double& b,
                                                 double* s_red) {
  a = 0.0;
  b = 0.0;
  for (int i = threadIdx.x; i < n; i += BLOCK) {
    a += __ldcg(pa + i);
    if (pb) b += __ldcg(pb + i);
  }
  block_sum2<BLOCK>(a, b, s_red);
}

// --------------------------------------------------- CG control block
struct CgCtl {
  double gamma;   // r.z
  double gamma_prev;  // r.z one iteration earlier (reliable-update restarts)
  double pAp;
  double alpha;
  double beta;
  double rr;      // r.r
  double bb;      // b.b
  double atol2;   // max(tol^2 b.b, atol^2)
  double tol2, atol_sq;
  double zcoef;   // next direction p = zcoef z + beta p (1 except right after a restart)
  int iter, maxiter, status, use_pc;
  int cont;       // loop condition mirror (1 = keep iterating)
  unsigned int ticket;
  unsigned int dev_status;
  int pad;
};

// ---------------------------------------------------- element operator
template <typename T>
struct Geo {
  T rx, sx, ry, sy, J;
  T nx[3], ny[3], sJ[3];
};

template <typename T>
__device__ __forceinline__ Geo<T> load_geo(const T* __restrict__ geo, int ldg, int k) {
  Geo<T> g;
  g.rx = __ldg(geo + G_RX * ldg + k);
  g.sx = __ldg(geo + G_SX * ldg + k);
  g.ry = __ldg(geo + G_RY * ldg + k);
  g.sy = __ldg(geo + G_SY * ldg + k);
  g.J = __ldg(geo + G_J * ldg + k);
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    g.nx[f] = __ldg(geo + (G_F0 + 3 * f) * ldg + k);
    g.ny[f] = __ldg(geo + (G_F0 + 3 * f + 1) * ldg + k);
    g.sJ[f] = __ldg(geo + (G_F0 + 3 * f + 2) * ldg + k);
  }
  return g;
}

// Neighbour-value sources (the rotated neighbour vector u~ of face f').
template <typename T, int Np>
struct NbrPlain {  // u~[i] = u[k' Np + perm[f'][i]]
  const T* __restrict__ u;
  const int* perm;  // shared memory, 3*Np
  __device__ __forceinline__ void operator()(int kp, int fp, T (&ut)[Np]) const {
    const T* base = u + (size_t)kp * Np;
#pragma unroll
    for (int i = 0; i < Np; ++i) ut[i] = __ldg(base + perm[fp * Np + i]);
  }
};
template <typename T, int Np>
struct NbrPfuse {  // u~ = zc z~ + beta p_old~  (the CG direction update, fused)
  const T* __restrict__ z;
  const T* __restrict__ p;
  T zc, beta;
  const int* perm;
  __device__ __forceinline__ void operator()(int kp, int fp, T (&ut)[Np]) const {
    const size_t o = (size_t)kp * Np;
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      const int j = perm[fp * Np + i];
      ut[i] = zc * __ldg(z + o + j) + beta * __ldg(p + o + j);
    }
  }
};
template <typename T, int Np>
struct NbrZero {  // self-block extraction: the neighbour carries no value
  __device__ __forceinline__ void operator()(int, int, T (&ut)[Np]) const {
#pragma unroll
    for (int i = 0; i < Np; ++i) ut[i] = T(0);
  }
};

template <int N, bool USE_NBR, class NbrSrc>
__device__ __forceinline__ void elem_apply_f2(const float (&u)[Dim<N>::Np], float (&y)[Dim<N>::Np],
                                              const Geo<float>& g, const uint32_t (&w)[3],
                                              const float* __restrict__ geo, int ldg, float tau, float alpha,
                                              const NbrSrc& nbr, const float* __restrict__ kappa, int k);

// y = A u + alpha J M u  for element k (u, y in registers).
// USE_NBR=false skips the neighbour value gather (self-block mode: the
// neighbour's value is zero, its geometry still sets tau_P).
// kappa (per-element diffusivity, may be null = 1; no reference counterpart):
// volume kappa_k grad u.grad v, face averages (kappa_M Dn_M + kappa_P Dn_P)/2,
// penalty weighted by kappa_F = (kappa_M + kappa_P)/2 (kappa_M on Dirichlet
// faces).  With kappa null every product by kappa is skipped, so the
// reference operator is reproduced bit for bit.
template <int N, typename T, bool USE_NBR, class NbrSrc>
__device__ __forceinline__ void elem_apply(const T (&u)[Dim<N>::Np], T (&y)[Dim<N>::Np], const Geo<T>& g,
                                           const uint32_t (&w)[3], const T* __restrict__ geo, int ldg, T tau,
                                           T alpha, const NbrSrc& nbr, const T* __restrict__ kappa = nullptr,
                                           int k = 0) {
  if constexpr (sizeof(T) == 4) {
    elem_apply_f2<N, USE_NBR>(u, y, g, w, geo, ldg, tau, alpha, nbr, kappa, k);
    return;
  }
  constexpr int Np = Dim<N>::Np, Nfp = Dim<N>::Nfp;
  const RefMats<N, T>& R = CRef<N, T>::get();
  const T kM = kappa ? __ldg(kappa + k) : T(1);

  // physical gradient at the nodes
  T ux[Np], uy[Np];
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    T ar = T(0), as = T(0);
#pragma unroll
    for (int j = 0; j < Np; ++j) {
      ar = fma(R.Dr[i * Np + j], u[j], ar);
      as = fma(R.Ds[i * Np + j], u[j], as);
    }
    ux[i] = g.rx * ar + g.sx * as;
    uy[i] = g.ry * ar + g.sy * as;
  }
  // own normal derivative at face nodes
  T dnm[3][Nfp];
#pragma unroll
  for (int f = 0; f < 3; ++f)
#pragma unroll
    for (int p = 0; p < Nfp; ++p) {
      const int n = fmask_idx(N, f, p);
      dnm[f][p] = g.nx[f] * ux[n] + g.ny[f] * uy[n];
    }
  // volume part of the lifted gradient: ex = M^T (J ux), ey = M^T (J uy)
  T ex[Np], ey[Np];
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    T a = T(0), b = T(0);
#pragma unroll
    for (int j = 0; j < Np; ++j) {
      a = fma(R.M[j * Np + i], ux[j], a);
      b = fma(R.M[j * Np + i], uy[j], b);
    }
    ex[i] = kM * g.J * a;
    ey[i] = kM * g.J * b;
  }
  // mass term (Helmholtz): alpha J (M u)
#pragma unroll
  for (int i = 0; i < Np; ++i) y[i] = T(0);
  if (alpha != T(0)) {
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      T a = T(0);
#pragma unroll
      for (int j = 0; j < Np; ++j) a = fma(R.M[i * Np + j], u[j], a);
      y[i] = alpha * g.J * a;
    }
  }
  // faces
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    const uint32_t wf = w[f];
    const int bc = (wf >> 3) & 3;
    const bool pact = (wf >> 5) & 1;
    const bool mint = (wf >> 6) & 1;
    const bool mdir = (bc == 1);
    if (!(pact || mint || mdir)) continue;
    const T sJ = g.sJ[f], nx = g.nx[f], ny = g.ny[f];
    const T tauM = tau * sJ / g.J;
    T uP[Nfp], dnP[Nfp];
    T tauP = tauM;
    T kP = kM;
    if (pact || mint) {
      const int kp = (int)(wf >> 7), fp = (int)(wf & 3);
      const bool flip = (wf >> 2) & 1;
      if (kappa) kP = __ldg(kappa + kp);
      const T rxn = __ldg(geo + G_RX * ldg + kp), sxn = __ldg(geo + G_SX * ldg + kp);
      const T ryn = __ldg(geo + G_RY * ldg + kp), syn = __ldg(geo + G_SY * ldg + kp);
      const T Jn = __ldg(geo + G_J * ldg + kp);
      tauP = tau * sJ / Jn;
      if (USE_NBR) {
        T ut[Np];
        nbr(kp, fp, ut);
        const T ar = nx * rxn + ny * ryn, as = nx * sxn + ny * syn;
        // derivative along the re-labelled reference axes (r~, s~)
        const T cr = fp == 0 ? ar : (fp == 1 ? as : -ar - as);
        const T cs = fp == 0 ? as : (fp == 1 ? -ar - as : ar);
        T dq[Nfp];
#pragma unroll
        for (int q = 0; q < Nfp; ++q) {
          T a = T(0), b = T(0);
#pragma unroll
          for (int j = 0; j < Np; ++j) {
            a = fma(R.Dr[q * Np + j], ut[j], a);  // face-0 rows: fmask_idx(N,0,q) == q
            b = fma(R.Ds[q * Np + j], ut[j], b);
          }
          dq[q] = cr * a + cs * b;
        }
#pragma unroll
        for (int p = 0; p < Nfp; ++p) {
          uP[p] = flip ? ut[N - p] : ut[p];
          dnP[p] = flip ? dq[N - p] : dq[p];
        }
      } else {
#pragma unroll
        for (int p = 0; p < Nfp; ++p) {
          uP[p] = T(0);
          dnP[p] = T(0);
        }
      }
    } else {
#pragma unroll
      for (int p = 0; p < Nfp; ++p) {
        uP[p] = T(0);
        dnP[p] = T(0);
      }
    }
    // coefficients (kappa_F: penalty weight of an interior face)
    const T kF = kappa ? T(0.5) * (kM + kP) : T(1);
    const T caM = mdir ? T(1) : (mint ? T(0.5) : T(0));
    const T cjM = mdir ? (kappa ? tauM * kM : tauM) : (mint ? (kappa ? T(0.5) * tauM * kF : T(0.5) * tauM) : T(0));
    const T cgM = (mdir ? T(1) : (mint ? T(0.25) : T(0))) * kM;
    const T caP = pact ? T(0.5) : T(0);
    const T cjP = pact ? (kappa ? T(0.5) * tauP * kF : T(0.5) * tauP) : T(0);
    const T cgP = (pact ? T(0.25) : T(0)) * kM;
    T v1[Nfp], v2[Nfp];
#pragma unroll
    for (int p = 0; p < Nfp; ++p) {
      const T uM = u[fmask_idx(N, f, p)];
      const T avgI = kappa ? T(0.5) * (kM * dnm[f][p] + kP * dnP[p]) : T(0.5) * (dnm[f][p] + dnP[p]);
      const T jmpI = uM - uP[p];
      const T avgM = mdir ? (kappa ? kM * dnm[f][p] : dnm[f][p]) : avgI;
      const T jmpM = mdir ? uM : jmpI;
      v1[p] = -caM * avgM + cjM * jmpM - caP * avgI + cjP * jmpI;
      v2[p] = cgM * jmpM + cgP * jmpI;
    }
#pragma unroll
    for (int q = 0; q < Nfp; ++q) {
      T a = T(0), b = T(0);
#pragma unroll
      for (int p = 0; p < Nfp; ++p) {
        a = fma(R.m1d[(f * Nfp + p) * Nfp + q], v1[p], a);
        b = fma(R.m1d[(f * Nfp + p) * Nfp + q], v2[p], b);
      }
      const int n = fmask_idx(N, f, q);
      y[n] += sJ * a;
      ex[n] -= sJ * nx * b;
      ey[n] -= sJ * ny * b;
    }
  }
  // lift: y += Dr^T (rx ex + ry ey) + Ds^T (sx ex + sy ey)
  T tr[Np], ts[Np];
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    tr[i] = g.rx * ex[i] + g.ry * ey[i];
    ts[i] = g.sx * ex[i] + g.sy * ey[i];
  }
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    T a = y[i];
#pragma unroll
    for (int j = 0; j < Np; ++j) {
      a = fma(R.Dr[j * Np + i], tr[j], a);
      a = fma(R.Ds[j * Np + i], ts[j], a);
    }
    y[i] = a;
  }
}


// float32 version of elem_apply with paired accumulations (same terms and
// coefficients; every component follows the scalar FMA sequence except the
// lift, which sums its Dr and Ds parts in two accumulators).
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

template <int N, bool USE_NBR, class NbrSrc>
__device__ __forceinline__ void elem_apply_f2(const float (&u)[Dim<N>::Np], float (&y)[Dim<N>::Np],
                                              const Geo<float>& g, const uint32_t (&w)[3],
                                              const float* __restrict__ geo, int ldg, float tau, float alpha,
                                              const NbrSrc& nbr, const float* __restrict__ kappa, int k) {
  constexpr int Np = Dim<N>::Np, Nfp = Dim<N>::Nfp;
  const RefMats<N, float>& R = CRef<N, float>::get();
  const RefPairs<N>& P = CPairs<N>::get();
  const float kM = kappa ? __ldg(kappa + k) : 1.0f;

  // Every derivative product acts on values centred on c = u[0]: Dr and Ds
  // annihilate constants, so Dr (u - c) = Dr u exactly, while the float32
  // rounding error now scales with the element's variation |u - c| ~ h |grad u|
  // instead of |u|.  On smooth vectors (the slow modes of an iterative solve)
  // this removes a cancellation error of order eps / (k h)^2 relative to A u.
  const float c0 = u[0];
  float uc[Np];
#pragma unroll
  for (int j = 0; j < Np; ++j) uc[j] = u[j] - c0;
  // physical gradient at the nodes: (ux, uy)
  float2 uxy[Np];
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    float2 a = f2(0.f, 0.f);  // (Dr u, Ds u)_i
#pragma unroll
    for (int j = 0; j < Np; ++j) a = __ffma2_rn(P.DrDs[i * Np + j], f2(uc[j], uc[j]), a);
    uxy[i] = f2(g.rx * a.x + g.sx * a.y, g.ry * a.x + g.sy * a.y);
  }
  float dnm[3][Nfp];
#pragma unroll
  for (int f = 0; f < 3; ++f)
#pragma unroll
    for (int p = 0; p < Nfp; ++p) {
      const int n = fmask_idx(N, f, p);
      dnm[f][p] = g.nx[f] * uxy[n].x + g.ny[f] * uxy[n].y;
    }
  // (ex, ey) = M^T (J ux, J uy)
  float2 exy[Np];
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    float2 a = f2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < Np; ++j) {
      const float m = R.M[j * Np + i];
      a = __ffma2_rn(f2(m, m), uxy[j], a);
    }
    exy[i] = f2(kM * g.J * a.x, kM * g.J * a.y);
  }
  // mass term (Helmholtz): alpha J (M u), rows in pairs
#pragma unroll
  for (int i = 0; i < Np; ++i) y[i] = 0.f;
  if (alpha != 0.f) {
#pragma unroll
    for (int r = 0; r < Np / 2; ++r) {
      float2 a = f2(0.f, 0.f);
#pragma unroll
      for (int j = 0; j < Np; ++j) a = __ffma2_rn(P.MP[r * Np + j], f2(u[j], u[j]), a);
      y[2 * r] = alpha * g.J * a.x;
      y[2 * r + 1] = alpha * g.J * a.y;
    }
    if (Np % 2) {
      float a = 0.f;
#pragma unroll
      for (int j = 0; j < Np; ++j) a = fmaf(R.M[(Np - 1) * Np + j], u[j], a);
      y[Np - 1] = alpha * g.J * a;
    }
  }
  // faces
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    const uint32_t wf = w[f];
    const int bc = (wf >> 3) & 3;
    const bool pact = (wf >> 5) & 1;
    const bool mint = (wf >> 6) & 1;
    const bool mdir = (bc == 1);
    if (!(pact || mint || mdir)) continue;
    const float sJ = g.sJ[f], nx = g.nx[f], ny = g.ny[f];
    const float tauM = tau * sJ / g.J;
    float uP[Nfp], dnP[Nfp];
    float tauP = tauM;
    float kP = kM;
#pragma unroll
    for (int p = 0; p < Nfp; ++p) {
      uP[p] = 0.f;
      dnP[p] = 0.f;
    }
    if (pact || mint) {
      const int kp = (int)(wf >> 7), fp = (int)(wf & 3);
      const bool flip = (wf >> 2) & 1;
      if (kappa) kP = __ldg(kappa + kp);
      const float rxn = __ldg(geo + G_RX * ldg + kp), sxn = __ldg(geo + G_SX * ldg + kp);
      const float ryn = __ldg(geo + G_RY * ldg + kp), syn = __ldg(geo + G_SY * ldg + kp);
      const float Jn = __ldg(geo + G_J * ldg + kp);
      tauP = tau * sJ / Jn;
      if (USE_NBR) {
        float ut[Np];
        nbr(kp, fp, ut);
        const float ar = nx * rxn + ny * ryn, as = nx * sxn + ny * syn;
        const float cr = fp == 0 ? ar : (fp == 1 ? as : -ar - as);
        const float cs = fp == 0 ? as : (fp == 1 ? -ar - as : ar);
        float dq[Nfp], utc[Np];
#pragma unroll
        for (int j = 0; j < Np; ++j) utc[j] = ut[j] - c0;  // centred as the own values
#pragma unroll
        for (int q = 0; q < Nfp; ++q) {
          float2 a = f2(0.f, 0.f);  // face-0 rows: fmask_idx(N,0,q) == q
#pragma unroll
          for (int j = 0; j < Np; ++j) a = __ffma2_rn(P.DrDs[q * Np + j], f2(utc[j], utc[j]), a);
          dq[q] = cr * a.x + cs * a.y;
        }
#pragma unroll
        for (int p = 0; p < Nfp; ++p) {
          uP[p] = flip ? ut[N - p] : ut[p];
          dnP[p] = flip ? dq[N - p] : dq[p];
        }
      }
    }
    const float kF = kappa ? 0.5f * (kM + kP) : 1.0f;
    const float caM = mdir ? 1.f : (mint ? 0.5f : 0.f);
    const float cjM = mdir ? (kappa ? tauM * kM : tauM) : (mint ? (kappa ? 0.5f * tauM * kF : 0.5f * tauM) : 0.f);
    const float cgM = (mdir ? 1.f : (mint ? 0.25f : 0.f)) * kM;
    const float caP = pact ? 0.5f : 0.f;
    const float cjP = pact ? (kappa ? 0.5f * tauP * kF : 0.5f * tauP) : 0.f;
    const float cgP = (pact ? 0.25f : 0.f) * kM;
    float2 v12[Nfp];
#pragma unroll
    for (int p = 0; p < Nfp; ++p) {
      const float uM = u[fmask_idx(N, f, p)];
      const float avgI = kappa ? 0.5f * (kM * dnm[f][p] + kP * dnP[p]) : 0.5f * (dnm[f][p] + dnP[p]);
      const float jmpI = uM - uP[p];
      const float avgM = mdir ? (kappa ? kM * dnm[f][p] : dnm[f][p]) : avgI;
      const float jmpM = mdir ? uM : jmpI;
      v12[p] = f2(-caM * avgM + cjM * jmpM - caP * avgI + cjP * jmpI, cgM * jmpM + cgP * jmpI);
    }
#pragma unroll
    for (int q = 0; q < Nfp; ++q) {
      float2 a = f2(0.f, 0.f);
#pragma unroll
      for (int p = 0; p < Nfp; ++p) {
        const float m = R.m1d[(f * Nfp + p) * Nfp + q];
        a = __ffma2_rn(f2(m, m), v12[p], a);
      }
      const int n = fmask_idx(N, f, q);
      y[n] += sJ * a.x;
      exy[n].x -= sJ * nx * a.y;
      exy[n].y -= sJ * ny * a.y;
    }
  }
  // lift: y += Dr^T (rx ex + ry ey) + Ds^T (sx ex + sy ey)
  float2 trs[Np];
#pragma unroll
  for (int i = 0; i < Np; ++i) trs[i] = f2(g.rx * exy[i].x + g.ry * exy[i].y, g.sx * exy[i].x + g.sy * exy[i].y);
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    float2 a = f2(y[i], 0.f);
#pragma unroll
    for (int j = 0; j < Np; ++j) a = __ffma2_rn(P.DrDsT[i * Np + j], trs[j], a);
    y[i] = a.x + a.y;
  }
}

}  // namespace ddg
