// Curved-element SIPG operator (sm_100a, float64).
//
// The reference's bilinear form (src/ddg/dg2d/sipg.py:142-301) on a Mesh2D
// whose geometric factors vary node by node (curved boundary elements,
// src/ddg/dg2d/curved.py:93-236), with either quadrature the reference
// offers:
//   nodal     (cub=None)  volume  sum_i J_i (ux_i (M vx)_i + uy_i (M vy)_i),
//                         faces   w sJ_f0 X^T m1d_f Y          (sipg.py:188-189, 265-280)
//   cubature  (cub=...)   volume  sum_q w_q J_q grad u . grad v at the points,
//                         faces   interpolated to the 1D face points and
//                         weighted by face_w sJ_q               (sipg.py:190-201, 281-299)
// Both face rules are one symmetric Nfp x Nfp matrix Q per (element, face):
// Q = sJ_f0 m1d_f (nodal) or L1d_f^T diag(face_w sJ_q) L1d_f (cubature), so
// one kernel family serves both.
//
// Gather-only in three passes, one thread per element (elements are
// independent inside a pass; passes meet only through global memory):
//   1. trace   gradient (gx, gy) of u at every face slot, with the nodal
//              metrics of the element                        -> tr[2][3Nfp][K]
//   2. dual    per side (k, f): jmp = u_M - u_P, avg = n.(g_M + g_P)/2 (one-
//              sided on boundary faces, sipg.py:235-249), then
//                a = w Q (tau jmp - avg)     (coefficient of jmp_v)
//                b = -w Q jmp / 2            (coefficient of Dn_v)
//              stored as (a, b nx, b ny) per face slot      -> dl[3][3Nfp][K]
//   3. gather  y = volume + sum over own sides (a at the face node,
//              Grad^T (b n) with b doubled on Dirichlet sides, sipg.py:241-245)
//              + sum over the neighbours' sides facing this element
//              (-a and Grad^T (b n) at the node the neighbour's vmapP names)
// where Grad^T h = Dr^T (rx hx + ry hy) + Ds^T (sx hx + sy hy) with nodal
// metrics.  Every field is structure-of-arrays [field][row][K] so a warp's
// 32 elements read 32 consecutive doubles.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>

#include "../../include/ddg_sipg.h"
#include "sipg_device.cuh"
#include "sipg_launch.h"

namespace ddg {

// this translation unit's copy of the reference-element matrices (filled by
// cv_upload_ref together with the other kernels' copy)
#define CV_DEFINE_CONST(NN) __constant__ RefMats<NN, double> c_cv_ref_##NN;
CV_DEFINE_CONST(1)
CV_DEFINE_CONST(2)
CV_DEFINE_CONST(3)
CV_DEFINE_CONST(4)
CV_DEFINE_CONST(5)
#undef CV_DEFINE_CONST

template <int N> struct CvRef;
#define CV_REF(NN)                                                                              \
  template <> struct CvRef<NN> {                                                                \
    static __device__ __forceinline__ const RefMats<NN, double>& get() { return c_cv_ref_##NN; } \
    static const void* sym() { return &c_cv_ref_##NN; }                                         \
  };
CV_REF(1)
CV_REF(2)
CV_REF(3)
CV_REF(4)
CV_REF(5)
#undef CV_REF

namespace cv {

constexpr int CV_BLOCK = 128;
constexpr int CV_GQ = 4;    // cubature points per staged chunk of the G table

__host__ __device__ constexpr int cv_even(int n) { return (n + 1) & ~1; }

// asynchronous 16-byte global -> shared copies (no registers held in flight)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// every group but the most recent one has completed
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int N>
struct CvDim {
  static constexpr int Np = (N + 1) * (N + 2) / 2;
  static constexpr int Nfp = N + 1;
  static constexpr int Ns = 3 * (N + 1);            // face slots per element
  static constexpr int NQ = (N + 1) * (N + 2) / 2;  // packed symmetric Nfp x Nfp
};

__device__ __forceinline__ int qidx(int Nfp, int p, int q) {
  return p <= q ? p * Nfp - p * (p - 1) / 2 + (q - p) : q * Nfp - q * (q - 1) / 2 + (p - q);
}

// stage elements [k0, k0 + nk) of an element-major vector into shared memory
template <int Np>
__device__ __forceinline__ void stage_tile(const double* __restrict__ v, int k0, int nk, double* s) {
  const size_t off = (size_t)k0 * Np;
  for (int i = threadIdx.x; i < nk * Np; i += blockDim.x) s[i] = v[off + i];
}

// ---------------------------------------------------------------- pass 1
template <int N>
__global__ void __launch_bounds__(CV_BLOCK) k_cv_trace(CvArgs a, const double* __restrict__ u) {
  constexpr int Np = CvDim<N>::Np, Nfp = CvDim<N>::Nfp, Ns = CvDim<N>::Ns;
  if (a.ctl && a.gate && a.ctl->cont == 0) return;
  __shared__ double s_u[CV_BLOCK * Np];
  const int k0 = blockIdx.x * CV_BLOCK, nk = min(CV_BLOCK, a.K - k0);
  stage_tile<Np>(u, k0, nk, s_u);
  __syncthreads();
  if ((int)threadIdx.x >= nk) return;
  const int k = k0 + threadIdx.x;
  const size_t K = (size_t)a.K;
  const RefMats<N, double>& R = CvRef<N>::get();
  double uv[Np];
#pragma unroll
  for (int j = 0; j < Np; ++j) uv[j] = s_u[threadIdx.x * Np + j];
#pragma unroll
  for (int f = 0; f < 3; ++f)
#pragma unroll
    for (int p = 0; p < Nfp; ++p) {
      const int n = fmask_idx(N, f, p), m = f * Nfp + p;
      double ur = 0.0, us = 0.0;
#pragma unroll
      for (int j = 0; j < Np; ++j) {
        ur = fma(R.Dr[n * Np + j], uv[j], ur);
        us = fma(R.Ds[n * Np + j], uv[j], us);
      }
      const double rx = a.gN[(0 * Np + n) * K + k], sx = a.gN[(1 * Np + n) * K + k];
      const double ry = a.gN[(2 * Np + n) * K + k], sy = a.gN[(3 * Np + n) * K + k];
      a.tr[(size_t)(0 * Ns + m) * K + k] = rx * ur + sx * us;
      a.tr[(size_t)(1 * Ns + m) * K + k] = ry * ur + sy * us;
    }
}

// ---------------------------------------------------------------- pass 2
template <int N, bool CUB>
__global__ void __launch_bounds__(CV_BLOCK, 8) k_cv_dual(CvArgs a, const double* __restrict__ u,
                                                      const double* __restrict__ udir) {
  constexpr int Np = CvDim<N>::Np, Nfp = CvDim<N>::Nfp, Ns = CvDim<N>::Ns, NQ = CvDim<N>::NQ;
  if (a.ctl && a.gate && a.ctl->cont == 0) return;
  const int k = blockIdx.x * CV_BLOCK + threadIdx.x;
  if (k >= a.K) return;
  const size_t K = (size_t)a.K;
  const RefMats<N, double>& R = CvRef<N>::get();
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    const int t = a.tag[f * K + k];
    double jm[Nfp], av[Nfp], nxv[Nfp], nyv[Nfp];
    const double w = t == DDG_BC_DIRICHLET ? 1.0 : (t == DDG_BC_NEUMANN ? 0.0 : 0.5);
#pragma unroll
    for (int p = 0; p < Nfp; ++p) {
      const int n = fmask_idx(N, f, p), m = f * Nfp + p;
      const double nx = a.fN[(size_t)(0 * Ns + m) * K + k], ny = a.fN[(size_t)(1 * Ns + m) * K + k];
      nxv[p] = nx;
      nyv[p] = ny;
      const double uM = u[(size_t)k * Np + n];
      const double DnM = nx * a.tr[(size_t)(0 * Ns + m) * K + k] + ny * a.tr[(size_t)(1 * Ns + m) * K + k];
      if (t == DDG_BC_DIRICHLET) {
        jm[p] = uM - (udir ? udir[(size_t)k * Np + n] : 0.0);
        av[p] = DnM;
      } else if (t == DDG_BC_NEUMANN) {
        jm[p] = 0.0;
        av[p] = 0.0;
      } else {
        const int sp = a.slotP[(size_t)m * K + k];
        const size_t mp = (size_t)a.mapP[(size_t)m * K + k];
        const double DnP = nx * a.tr[mp] + ny * a.tr[(size_t)Ns * K + mp];
        jm[p] = uM - u[sp];
        av[p] = 0.5 * (DnM + DnP);
      }
    }
    const double tau = a.tauF[f * K + k];
    const double sj = CUB ? 1.0 : a.sJ0[f * K + k];
#pragma unroll
    for (int p = 0; p < Nfp; ++p) {
      double sa = 0.0, sb = 0.0;
#pragma unroll
      for (int q = 0; q < Nfp; ++q) {
        const double Q = CUB ? a.cQ[(size_t)(f * NQ + qidx(Nfp, p, q)) * K + k] : R.m1d[(f * Nfp + p) * Nfp + q];
        sa = fma(Q, fma(tau, jm[q], -av[q]), sa);
        sb = fma(Q, jm[q], sb);
      }
      const double ca = w * sj * sa, cb = -0.5 * w * sj * sb;
      const int m = f * Nfp + p;
      a.dl[(size_t)(0 * Ns + m) * K + k] = ca;
      a.dl[(size_t)(1 * Ns + m) * K + k] = cb * nxv[p];
      a.dl[(size_t)(2 * Ns + m) * K + k] = cb * nyv[p];
    }
  }
}

// ---------------------------------------------------------------- pass 3
enum CvMode { CV_APPLY = 0, CV_SUB = 1, CV_PDOT = 2, CV_RESID = 3 };

// dynamic shared memory: the element tile (CV_BLOCK Np doubles), then (CUB)
// Drq, Dsq, Lq (3 Ncub Np) and two buffers of the block's G table for
// CV_GQ cubature points (2 x 4 x CV_GQ x CV_BLOCK), filled by cp.async while
// the previous points (or the face terms) are computed.
// Register budget: only the output row and, for the nodal volume, J grad u
// are held per thread.  The gradient part of every face slot is applied as a
// rank-one update Dr^T e_n (rx bx + ry by) + Ds^T e_n (sx bx + sy by), the
// nodal volume node by node, and the element's u stays in the shared tile.
template <int N, bool CUB, int MODE>
__global__ void __launch_bounds__(CV_BLOCK, CUB ? (N >= 5 ? 2 : 3) : 4) k_cv_gather(CvArgs a, const double* __restrict__ u,
                                                                    const double* __restrict__ b,
                                                                    double* __restrict__ y, double alpha,
                                                                    double shift) {
  constexpr int Np = CvDim<N>::Np, Nfp = CvDim<N>::Nfp, Ns = CvDim<N>::Ns;
  if (a.ctl && a.gate && a.ctl->cont == 0) return;
  extern __shared__ __align__(16) double s_dyn[];
  __shared__ double s_red[64];
  double* s_u = s_dyn;
  double* s_m = s_dyn + CV_BLOCK * Np;
  const int k0 = blockIdx.x * CV_BLOCK, nk = min(CV_BLOCK, a.K - k0);
  stage_tile<Np>(u, k0, nk, s_u);
  double* s_g = s_m + (CUB ? cv_even(3 * a.Ncub * Np) : 0);   // 16-byte aligned for cp.async
  const int nch = CUB ? (a.Ncub + CV_GQ - 1) / CV_GQ : 0;
  // the block's G rows of points [ch CV_GQ, (ch + 1) CV_GQ): 128 consecutive
  // doubles per (field, point), 16-byte pieces (a.ldc and k0 are multiples
  // of CV_BLOCK, so every piece is aligned and inside the padded table)
  auto issue = [&](int ch) {
    double* dst = s_g + (size_t)(ch & 1) * 4 * CV_GQ * CV_BLOCK;
    for (int idx = threadIdx.x; idx < 4 * CV_GQ * (CV_BLOCK / 2); idx += CV_BLOCK) {
      const int row = idx / (CV_BLOCK / 2), piece = idx - row * (CV_BLOCK / 2);
      const int c = row / CV_GQ, q = ch * CV_GQ + (row - c * CV_GQ);
      if (q < a.Ncub)
        cp_async16(dst + (size_t)row * CV_BLOCK + 2 * piece,
                   a.cG + (size_t)(c * a.Ncub + q) * a.ldc + k0 + 2 * piece);
    }
    cp_async_commit();
  };
  if (CUB) {
    // (Drq, Dsq) interleaved as 16-byte pairs, then Lq: one 128-bit and one
    // 64-bit shared load per basis function and cubature point
    const int nq = a.Ncub * Np;
    for (int i = threadIdx.x; i < nq; i += CV_BLOCK) {
      s_m[2 * i] = a.cMat[i];
      s_m[2 * i + 1] = a.cMat[nq + i];
      s_m[2 * nq + i] = a.cMat[2 * nq + i];
    }
    issue(0);
  }
  __syncthreads();
  const bool active = (int)threadIdx.x < nk;
  const int k = k0 + threadIdx.x;
  const size_t K = (size_t)a.K;
  const RefMats<N, double>& R = CvRef<N>::get();
  const double* ue = s_u + threadIdx.x * Np;
  double out[Np];
  double dA = 0.0, dB = 0.0;
  if (active) {
#pragma unroll
    for (int i = 0; i < Np; ++i) out[i] = 0.0;
    // faces: own sides, then the neighbours' sides facing this element
    // (one slot per iteration: the node index is warp-uniform, so the
    // constant-bank rows stay broadcasts and the scalar part is a
    // predicated add into the statically indexed output)
#pragma unroll 1
    for (int m = 0; m < Ns; ++m) {
      const int f = m / Nfp, n = fmask_idx(N, f, m - f * Nfp);
      const int t = a.tag[f * K + k];
      const double c = t == DDG_BC_DIRICHLET ? 2.0 : 1.0;
      double av = 0.0, bx = 0.0, by = 0.0;
      if (t != DDG_BC_NEUMANN) {
        av = a.dl[(size_t)(0 * Ns + m) * K + k];
        bx = c * a.dl[(size_t)(1 * Ns + m) * K + k];
        by = c * a.dl[(size_t)(2 * Ns + m) * K + k];
      }
      const int mp = a.mapP[(size_t)m * K + k];
      const int k2 = mp % a.K, f2 = (mp / a.K) / Nfp;
      if (a.tag[f2 * K + k2] == DDG_BC_INTERIOR) {
        av -= a.dl[(size_t)mp];
        bx += a.dl[(size_t)Ns * K + mp];
        by += a.dl[(size_t)2 * Ns * K + mp];
      }
      const double rx = a.gN[(0 * Np + n) * K + k], sx = a.gN[(1 * Np + n) * K + k];
      const double ry = a.gN[(2 * Np + n) * K + k], sy = a.gN[(3 * Np + n) * K + k];
      const double tr = fma(rx, bx, ry * by), ts = fma(sx, bx, sy * by);
#pragma unroll
      for (int i = 0; i < Np; ++i) {
        out[i] = fma(R.Dr[n * Np + i], tr, fma(R.Ds[n * Np + i], ts, out[i]));
        if (i == n) out[i] += av;
      }
    }
    if (!CUB) {
      // nodal volume: Grad^T M^T (J grad u), node by node
      double jx[Np], jy[Np];
#pragma unroll
      for (int i = 0; i < Np; ++i) {
        double ur = 0.0, us = 0.0;
#pragma unroll
        for (int j = 0; j < Np; ++j) {
          ur = fma(R.Dr[i * Np + j], ue[j], ur);
          us = fma(R.Ds[i * Np + j], ue[j], us);
        }
        const double J = a.gN[(4 * Np + i) * K + k];
        jx[i] = J * fma(a.gN[(0 * Np + i) * K + k], ur, a.gN[(1 * Np + i) * K + k] * us);
        jy[i] = J * fma(a.gN[(2 * Np + i) * K + k], ur, a.gN[(3 * Np + i) * K + k] * us);
      }
#pragma unroll 1
      for (int n = 0; n < Np; ++n) {
        double hx = 0.0, hy = 0.0;
#pragma unroll
        for (int j = 0; j < Np; ++j) {
          hx = fma(R.M[j * Np + n], jx[j], hx);
          hy = fma(R.M[j * Np + n], jy[j], hy);
        }
        const double rx = a.gN[(0 * Np + n) * K + k], sx = a.gN[(1 * Np + n) * K + k];
        const double ry = a.gN[(2 * Np + n) * K + k], sy = a.gN[(3 * Np + n) * K + k];
        const double tr = fma(rx, hx, ry * hy), ts = fma(sx, hx, sy * hy);
#pragma unroll
        for (int i = 0; i < Np; ++i) out[i] = fma(R.Dr[n * Np + i], tr, fma(R.Ds[n * Np + i], ts, out[i]));
      }
      if (alpha != 0.0) {
#pragma unroll
        for (int i = 0; i < Np; ++i) {
          double s = 0.0;
#pragma unroll
          for (int j = 0; j < Np; ++j) s = fma(R.M[i * Np + j], ue[j], s);
          out[i] = fma(alpha * a.gN[(4 * Np + i) * K + k], s, out[i]);
        }
      }
    }
  }
  if (CUB) {
    // cubature volume and mass, CV_GQ points at a time from the staged G
    const double2* DD = reinterpret_cast<const double2*>(s_m);
    const double* Lq = s_m + 2 * a.Ncub * Np;
    double uv[Np];
#pragma unroll
    for (int j = 0; j < Np; ++j) uv[j] = active ? ue[j] : 0.0;
    for (int ch = 0; ch < nch; ++ch) {
      if (ch + 1 < nch) issue(ch + 1);
      else cp_async_commit();                      // an empty group keeps the count uniform
      cp_async_wait_1();                           // chunk ch has landed (this thread's pieces)
      __syncthreads();                             // ... and every thread's
      const double* g = s_g + (size_t)(ch & 1) * 4 * CV_GQ * CV_BLOCK + threadIdx.x;
      if (active) {
#pragma unroll 1
        for (int qq = 0; qq < CV_GQ; ++qq) {
          const int q = ch * CV_GQ + qq;
          if (q >= a.Ncub) break;
          double ur = 0.0, us = 0.0, uq = 0.0;
#pragma unroll
          for (int j = 0; j < Np; ++j) {
            const double2 d = DD[q * Np + j];
            ur = fma(d.x, uv[j], ur);
            us = fma(d.y, uv[j], us);
            uq = fma(Lq[q * Np + j], uv[j], uq);
          }
          const double Grr = g[(0 * CV_GQ + qq) * CV_BLOCK], Grs = g[(1 * CV_GQ + qq) * CV_BLOCK];
          const double Gss = g[(2 * CV_GQ + qq) * CV_BLOCK], wJ = g[(3 * CV_GQ + qq) * CV_BLOCK];
          const double vr = fma(Grr, ur, Grs * us), vs = fma(Grs, ur, Gss * us), vm = alpha * wJ * uq;
#pragma unroll
          for (int i = 0; i < Np; ++i) {
            const double2 d = DD[q * Np + i];
            out[i] = fma(d.x, vr, fma(d.y, vs, fma(Lq[q * Np + i], vm, out[i])));
          }
        }
      }
      __syncthreads();                             // the buffer is refilled two chunks later
    }
  }
  if (active) {
    if (shift != 0.0) {
#pragma unroll
      for (int i = 0; i < Np; ++i) out[i] = fma(shift, ue[i], out[i]);
    }
    if (MODE == CV_PDOT) {
#pragma unroll
      for (int i = 0; i < Np; ++i) dA = fma(ue[i], out[i], dA);
    } else if (MODE == CV_RESID) {
#pragma unroll
      for (int i = 0; i < Np; ++i) {
        const double bi = b[(size_t)k * Np + i];
        out[i] = bi - out[i];
        dA = fma(bi, bi, dA);
        dB = fma(out[i], out[i], dB);
      }
    } else if (MODE == CV_SUB) {
#pragma unroll
      for (int i = 0; i < Np; ++i) out[i] = y[(size_t)k * Np + i] - out[i];
    }
  }
  __syncthreads();
  if (active) {
#pragma unroll
    for (int i = 0; i < Np; ++i) s_u[threadIdx.x * Np + i] = out[i];
  }
  __syncthreads();
  {
    const size_t off = (size_t)k0 * Np;
    for (int i = threadIdx.x; i < nk * Np; i += CV_BLOCK) y[off + i] = s_u[i];
  }
  if (MODE != CV_PDOT && MODE != CV_RESID) return;
  block_sum2<CV_BLOCK>(dA, dB, s_red);
  if (threadIdx.x == 0) {
    a.partA[blockIdx.x] = dA;
    a.partB[blockIdx.x] = dB;
  }
  if (!is_last_block(&a.ctl->ticket)) return;
  double sA, sB;
  reduce_partials2<CV_BLOCK>(a.partA, a.partB, gridDim.x, sA, sB, s_red);
  if (threadIdx.x == 0) {
    CgCtl* c = a.ctl;
    if (MODE == CV_PDOT) {
      c->pAp = sA;
      const double al = c->gamma / sA;
      if (!(sA > 0.0) || !isfinite(al)) {
        c->status = 2;
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

// ------------------------------------------------------------- mass, loads
// y = M_quad f: J (M f) at the nodes (nodal) or Lq^T (w J (Lq f)) (cubature,
// src/ddg/dg2d/cubature.py:243-254)
template <int N, bool CUB>
__global__ void __launch_bounds__(CV_BLOCK) k_cv_mass(CvArgs a, const double* __restrict__ f,
                                                      double* __restrict__ y) {
  constexpr int Np = CvDim<N>::Np;
  extern __shared__ __align__(16) double s_dyn[];
  double* s_u = s_dyn;
  double* s_m = s_dyn + CV_BLOCK * Np;
  const int k0 = blockIdx.x * CV_BLOCK, nk = min(CV_BLOCK, a.K - k0);
  stage_tile<Np>(f, k0, nk, s_u);
  if (CUB)
    for (int i = threadIdx.x; i < a.Ncub * Np; i += CV_BLOCK) s_m[i] = a.cMat[2 * a.Ncub * Np + i];
  __syncthreads();
  const bool active = (int)threadIdx.x < nk;
  const int k = k0 + threadIdx.x;
  const size_t K = (size_t)a.K;
  double out[Np];
  if (active) {
    double fv[Np];
#pragma unroll
    for (int j = 0; j < Np; ++j) {
      fv[j] = s_u[threadIdx.x * Np + j];
      out[j] = 0.0;
    }
    if (CUB) {
      for (int q = 0; q < a.Ncub; ++q) {
        double fq = 0.0;
#pragma unroll
        for (int j = 0; j < Np; ++j) fq = fma(s_m[q * Np + j], fv[j], fq);
        fq *= a.cG[(size_t)(3 * a.Ncub + q) * a.ldc + k];
#pragma unroll
        for (int i = 0; i < Np; ++i) out[i] = fma(s_m[q * Np + i], fq, out[i]);
      }
    } else {
      const RefMats<N, double>& R = CvRef<N>::get();
#pragma unroll
      for (int i = 0; i < Np; ++i) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < Np; ++j) s = fma(R.M[i * Np + j], fv[j], s);
        out[i] = a.gN[(4 * Np + i) * K + k] * s;
      }
    }
  }
  __syncthreads();
  if (active) {
#pragma unroll
    for (int i = 0; i < Np; ++i) s_u[threadIdx.x * Np + i] = out[i];
  }
  __syncthreads();
  const size_t off = (size_t)k0 * Np;
  for (int i = threadIdx.x; i < nk * Np; i += CV_BLOCK) y[off + i] = s_u[i];
}

// y += sJ_f0 m1d_f q on Neumann faces (src/ddg/dg2d/sipg.py:420-453);
// q is a face vector, index k 3 Nfp + f Nfp + p
template <int N>
__global__ void __launch_bounds__(CV_BLOCK) k_cv_neumann(CvArgs a, const double* __restrict__ q,
                                                         double* __restrict__ y) {
  constexpr int Np = CvDim<N>::Np, Nfp = CvDim<N>::Nfp;
  const int k = blockIdx.x * CV_BLOCK + threadIdx.x;
  if (k >= a.K) return;
  const size_t K = (size_t)a.K;
  const RefMats<N, double>& R = CvRef<N>::get();
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    if (a.tag[f * K + k] != DDG_BC_NEUMANN) continue;
    const double sj = a.sJ0[f * K + k];
    double qv[Nfp];
#pragma unroll
    for (int p = 0; p < Nfp; ++p) qv[p] = q[(size_t)k * 3 * Nfp + f * Nfp + p];
#pragma unroll
    for (int p = 0; p < Nfp; ++p) {
      double s = 0.0;
#pragma unroll
      for (int qq = 0; qq < Nfp; ++qq) s = fma(R.m1d[(f * Nfp + p) * Nfp + qq], qv[qq], s);
      y[(size_t)k * Np + fmask_idx(N, f, p)] += sj * s;
    }
  }
}

// ------------------------------------------------------- block Jacobi
// coloured probe: P = e_j on every element of colour c (src/ddg/dg2d/sipg.py:671-704)
__global__ void k_cv_probe(int K, int Np, const int* __restrict__ colour, int c, int j, double* __restrict__ P) {
  const int64_t n = (int64_t)K * Np;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(i / Np), r = (int)(i % Np);
    P[i] = (r == j && colour[k] == c) ? 1.0 : 0.0;
  }
}

// column j of the diagonal block of every element of colour c
__global__ void k_cv_collect(int K, int Np, const int* __restrict__ colour, int c, int j, double shift,
                             const double* __restrict__ Y, double* __restrict__ blocks) {
  const int64_t n = (int64_t)K * Np;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(i / Np), r = (int)(i % Np);
    if (colour[k] == c) blocks[(size_t)k * Np * Np + (size_t)r * Np + j] = Y[i] + (r == j ? shift : 0.0);
  }
}

// explicit inverse of each block (Gauss-Jordan, partial pivoting), stored
// SoA binv[(i Np + j) K + k]; the blocks of the nodal curved operator are
// not symmetric, so the full inverse is kept (src/ddg/dg2d/sipg.py:707-715)
template <int N>
__global__ void __launch_bounds__(64) k_cv_invert(int K, const double* __restrict__ blocks, double* __restrict__ binv,
                                                   unsigned int* status) {
  constexpr int Np = CvDim<N>::Np;
  const int k = blockIdx.x * 64 + threadIdx.x;
  if (k >= K) return;
  double m[Np][2 * Np];
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) {
      m[i][j] = blocks[(size_t)k * Np * Np + i * Np + j];
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
  if (!ok) atomicOr(status, ST_BAD_INDEX);
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) binv[(size_t)(i * Np + j) * K + k] = ok ? m[i][Np + j] : NAN;
}

// z = B^-1 r per element
template <int N>
__global__ void __launch_bounds__(CV_BLOCK) k_cv_pc(int K, const double* __restrict__ binv,
                                                    const double* __restrict__ r, double* __restrict__ z,
                                                    const CgCtl* ctl) {
  constexpr int Np = CvDim<N>::Np;
  if (ctl && ctl->cont == 0) return;
  __shared__ double s[CV_BLOCK * Np];
  const int k0 = blockIdx.x * CV_BLOCK, nk = min(CV_BLOCK, K - k0);
  stage_tile<Np>(r, k0, nk, s);
  __syncthreads();
  double zv[Np];
  const bool active = (int)threadIdx.x < nk;
  if (active) {
    const int k = k0 + threadIdx.x;
    double rv[Np];
#pragma unroll
    for (int j = 0; j < Np; ++j) rv[j] = s[threadIdx.x * Np + j];
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < Np; ++j) acc = fma(binv[(size_t)(i * Np + j) * K + k], rv[j], acc);
      zv[i] = acc;
    }
  }
  __syncthreads();
  if (active) {
#pragma unroll
    for (int i = 0; i < Np; ++i) s[threadIdx.x * Np + i] = zv[i];
  }
  __syncthreads();
  const size_t off = (size_t)k0 * Np;
  for (int i = threadIdx.x; i < nk * Np; i += CV_BLOCK) z[off + i] = s[i];
}

// CG direction p = zcoef z + beta p (float64, in place)
__global__ void k_cv_pupd(int64_t n, const double* __restrict__ z, double* __restrict__ p, const CgCtl* ctl) {
  if (ctl->cont == 0) return;
  const double zc = ctl->zcoef, be = ctl->beta;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = fma(zc, z[i], be * p[i]);
}

// ------------------------------------------------------------- launchers
template <int N, bool CUB, int MODE>
cudaError_t gather_n(const CvArgs& a, const double* u, const double* b, double* y, double alpha, double shift,
                     cudaStream_t s) {
  constexpr int Np = CvDim<N>::Np;
  const size_t smem =
      (size_t)(CV_BLOCK * Np + (CUB ? cv_even(3 * a.Ncub * Np) + 2 * 4 * CV_GQ * CV_BLOCK : 0)) * sizeof(double);
  k_cv_gather<N, CUB, MODE><<<(a.K + CV_BLOCK - 1) / CV_BLOCK, CV_BLOCK, smem, s>>>(a, u, b, y, alpha, shift);
  return cudaGetLastError();
}

template <int N>
cudaError_t cv_apply_n(int pass, int quad, int mode, const CvArgs& a, const double* u, const double* udir,
                       const double* b, double* y, double alpha, double shift, cudaStream_t s) {
  const int grid = (a.K + CV_BLOCK - 1) / CV_BLOCK;
  if (pass == 1) {
    k_cv_trace<N><<<grid, CV_BLOCK, 0, s>>>(a, u);
    return cudaGetLastError();
  }
  if (pass == 2) {
    if (quad) k_cv_dual<N, true><<<grid, CV_BLOCK, 0, s>>>(a, u, udir);
    else k_cv_dual<N, false><<<grid, CV_BLOCK, 0, s>>>(a, u, udir);
    return cudaGetLastError();
  }
#define CV_G(Q, M) return gather_n<N, Q, M>(a, u, b, y, alpha, shift, s)
  if (quad) {
    switch (mode) {
      case CV_APPLY: CV_G(true, CV_APPLY);
      case CV_SUB: CV_G(true, CV_SUB);
      case CV_PDOT: CV_G(true, CV_PDOT);
      case CV_RESID: CV_G(true, CV_RESID);
    }
  } else {
    switch (mode) {
      case CV_APPLY: CV_G(false, CV_APPLY);
      case CV_SUB: CV_G(false, CV_SUB);
      case CV_PDOT: CV_G(false, CV_PDOT);
      case CV_RESID: CV_G(false, CV_RESID);
    }
  }
#undef CV_G
  return cudaErrorInvalidValue;
}

template <int N>
cudaError_t cv_mass_n(int quad, const CvArgs& a, const double* f, double* y, cudaStream_t s) {
  constexpr int Np = CvDim<N>::Np;
  const size_t smem = (size_t)(CV_BLOCK * Np + (quad ? a.Ncub * Np : 0)) * sizeof(double);
  const int grid = (a.K + CV_BLOCK - 1) / CV_BLOCK;
  if (quad) k_cv_mass<N, true><<<grid, CV_BLOCK, smem, s>>>(a, f, y);
  else k_cv_mass<N, false><<<grid, CV_BLOCK, smem, s>>>(a, f, y);
  return cudaGetLastError();
}

// dynamic shared memory limits of the kernels that stage matrices (once per
// degree, before any launch or graph capture)
template <int N>
cudaError_t cv_prepare_n() {
  constexpr int lim = CV_SMEM_LIMIT;
  cudaError_t e = cudaSuccess;
#define CV_A(fn) \
  if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, lim)
  CV_A((k_cv_gather<N, true, CV_APPLY>));
  CV_A((k_cv_gather<N, true, CV_SUB>));
  CV_A((k_cv_gather<N, true, CV_PDOT>));
  CV_A((k_cv_gather<N, true, CV_RESID>));
  CV_A((k_cv_gather<N, false, CV_APPLY>));
  CV_A((k_cv_gather<N, false, CV_SUB>));
  CV_A((k_cv_gather<N, false, CV_PDOT>));
  CV_A((k_cv_gather<N, false, CV_RESID>));
  CV_A((k_cv_mass<N, true>));
  CV_A((k_cv_mass<N, false>));
#undef CV_A
  return e;
}

}  // namespace cv

#define CV_DISPATCH(N_, CALL)   \
  switch (N_) {                 \
    case 1: return CALL(1);     \
    case 2: return CALL(2);     \
    case 3: return CALL(3);     \
    case 4: return CALL(4);     \
    case 5: return CALL(5);     \
  }                             \
  return cudaErrorInvalidValue

cudaError_t launch_cv_pass(int N, int pass, int quad, int mode, const CvArgs& a, const double* u, const double* udir,
                           const double* b, double* y, double alpha, double shift, cudaStream_t s) {
#define C_(n) cv::cv_apply_n<n>(pass, quad, mode, a, u, udir, b, y, alpha, shift, s)
  CV_DISPATCH(N, C_);
#undef C_
}

namespace {
template <int N>
cudaError_t cv_upload_n(const double* Dr, const double* Ds, const double* M, const double* m1d) {
  constexpr int Np = (N + 1) * (N + 2) / 2, Nfp = N + 1;
  RefMats<N, double> h;
  for (int i = 0; i < Np * Np; ++i) {
    h.Dr[i] = Dr[i];
    h.Ds[i] = Ds[i];
    h.M[i] = M[i];
  }
  for (int i = 0; i < 3 * Nfp * Nfp; ++i) h.m1d[i] = m1d[i];
  return cudaMemcpyToSymbol(CvRef<N>::sym(), &h, sizeof(h));
}
}  // namespace

cudaError_t cv_upload_ref(int N, const double* Dr, const double* Ds, const double* M, const double* m1d) {
#define C_(n) cv_upload_n<n>(Dr, Ds, M, m1d)
  CV_DISPATCH(N, C_);
#undef C_
}

size_t cv_gather_smem_bytes(int N, int Ncub) {
  const int Np = (N + 1) * (N + 2) / 2;
  return (size_t)(cv::CV_BLOCK * Np + cv::cv_even(3 * Ncub * Np) + 2 * 4 * cv::CV_GQ * cv::CV_BLOCK) * sizeof(double);
}

cudaError_t cv_prepare(int N) {
#define C_(n) cv::cv_prepare_n<n>()
  CV_DISPATCH(N, C_);
#undef C_
}

cudaError_t launch_cv_mass(int N, int quad, const CvArgs& a, const double* f, double* y, cudaStream_t s) {
#define C_(n) cv::cv_mass_n<n>(quad, a, f, y, s)
  CV_DISPATCH(N, C_);
#undef C_
}

cudaError_t launch_cv_neumann(int N, const CvArgs& a, const double* q, double* y, cudaStream_t s) {
  const int grid = (a.K + cv::CV_BLOCK - 1) / cv::CV_BLOCK;
#define C_(n) (cv::k_cv_neumann<n><<<grid, cv::CV_BLOCK, 0, s>>>(a, q, y), cudaGetLastError())
  CV_DISPATCH(N, C_);
#undef C_
}

cudaError_t launch_cv_probe(int K, int Np, const int* colour, int c, int j, double* P, cudaStream_t s) {
  const int64_t n = (int64_t)K * Np;
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  cv::k_cv_probe<<<grid, 256, 0, s>>>(K, Np, colour, c, j, P);
  return cudaGetLastError();
}

cudaError_t launch_cv_collect(int K, int Np, const int* colour, int c, int j, double shift, const double* Y,
                              double* blocks, cudaStream_t s) {
  const int64_t n = (int64_t)K * Np;
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  cv::k_cv_collect<<<grid, 256, 0, s>>>(K, Np, colour, c, j, shift, Y, blocks);
  return cudaGetLastError();
}

cudaError_t launch_cv_invert(int N, int K, const double* blocks, double* binv, unsigned int* status, cudaStream_t s) {
  const int grid = (K + 63) / 64;
#define C_(n) (cv::k_cv_invert<n><<<grid, 64, 0, s>>>(K, blocks, binv, status), cudaGetLastError())
  CV_DISPATCH(N, C_);
#undef C_
}

cudaError_t launch_cv_pc(int N, int K, const double* binv, const double* r, double* z, const CgCtl* ctl,
                         cudaStream_t s) {
  const int grid = (K + cv::CV_BLOCK - 1) / cv::CV_BLOCK;
#define C_(n) (cv::k_cv_pc<n><<<grid, cv::CV_BLOCK, 0, s>>>(K, binv, r, z, ctl), cudaGetLastError())
  CV_DISPATCH(N, C_);
#undef C_
}

cudaError_t launch_cv_pupd(int64_t n, const double* z, double* p, const CgCtl* ctl, cudaStream_t s) {
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  cv::k_cv_pupd<<<grid, 256, 0, s>>>(n, z, p, ctl);
  return cudaGetLastError();
}
#undef CV_DISPATCH

}  // namespace ddg
