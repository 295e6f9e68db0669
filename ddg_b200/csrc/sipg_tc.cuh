// float32 SIPG apply on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Included at the end of sipg_kernels.cu (it reads that file's
// __constant__ reference matrices).
//
// One CTA of 128 threads owns a tile of 128 elements; thread e, TMEM lane e
// and MMA row e are element k0 + e.  The CTA is persistent (it loops over
// tiles) and holds 256 TMEM columns for its lifetime.  Per tile:
//
//   stage 1 (tensor cores):  D1 = u . [Srr; Srs; Sss; M; Dr; Ds]^T
//       A = u (this element's nodal values, K = Kp >= Np) written by each
//       thread into its TMEM lane; B = the six stacked reference matrices,
//       K-major in shared memory.  Srr = Dr^T M^T Dr, Srs = Dr^T M^T Ds +
//       Ds^T M^T Dr, Sss = Ds^T M^T Ds are the reference stiffness blocks, so
//       the affine volume term is kappa J (c_rr Srr + c_rs Srs + c_ss Sss) u
//       with c_rr = rx^2 + ry^2, c_rs = rx sx + ry sy, c_ss = sx^2 + sy^2, and
//       the mass term is alpha J M u (src/ddg/dg2d/sipg.py:175-189, 597-601).
//   CUDA cores (overlapping stage 1): the neighbour's normal derivative at
//       each shared face (face-0 rows of Dr/Ds on the neighbour's re-labelled
//       values), then, from D1, the own normal derivative, the SIPG
//       jump/average flux through the 1D face mass (sipg.py:246-279) into y
//       at the face nodes, and the gradient-test weights gr, gs.
//   stage 2 (tensor cores):  D2 = [gr | gs] . [Dr[F,:]; Ds[F,:]]^T
//       the face part of the lift Dr^T(rx ex + ry ey) + Ds^T(sx ex + sy ey),
//       which only touches the face rows F of Dr and Ds.
//
// Precision: every product is split 3xTF32 (x = x_hi + x_lo with x_hi the
// TF32 rounding; a.b ~ a_hi.b_hi + a_lo.b_hi + a_hi.b_lo, float32
// accumulation), which keeps the apply at float32 accuracy (single-pass TF32
// would lose three decimal digits and stall iterative refinement at SIPG
// condition numbers).  The B matrices are split on the host from their
// float64 values.
//
// Layouts: A in TMEM, row = lane, one 32-bit column per K index.  B in shared
// memory in the canonical K-major no-swizzle layout: core matrices of 8 rows
// x 16 bytes, element (n, k) at byte ((n/8)(Kc/4) + k/4) 128 + (n%8) 16 +
// (k%4) 4, so the leading-dimension offset (next 4 K values) is 128 bytes and
// the stride-dimension offset (next 8 rows) is (Kc/4) 128 bytes.
//
// Every wait (bulk copy or MMA completion) is bounded; on time-out the CTA
// records ST_TMA_TIMEOUT, stops issuing work, waits (bounded) for what it
// already issued and frees its TMEM before returning.
#pragma once

namespace ddg {
namespace tc {

template <int N>
struct TcDim {
  static constexpr int Np = Dim<N>::Np, Nfp = Dim<N>::Nfp;
  static constexpr int Kp = (Np + 7) / 8 * 8;             // K of stage 1
  static constexpr int K2 = (6 * Nfp + 7) / 8 * 8;        // K of stage 2: [gr | gs]
  static constexpr int N1 = 6 * Kp;                        // stage-1 output columns
  static constexpr int N2 = (Np + 15) / 16 * 16;           // stage-2 output columns
  static constexpr int KpS = (Kp + 15) / 16 * 16;          // TMEM column offset hi -> lo (stage 1)
  static constexpr int K2S = (K2 + 15) / 16 * 16;          // TMEM column offset hi -> lo (stage 2)
  // TMEM columns of this CTA's 128 (four CTAs per SM share the 512).  Stage
  // operands and results reuse columns once consumed: A2 is written over D1
  // after every thread has read its D1 lane, and D2 lands on the u operand
  // after stage 1 has completed.
  static constexpr int COL_AU = 0;                         // u_hi | u_lo      (stage 1 A)
  static constexpr int COL_D1 = 32;                        // stage 1 D
  static constexpr int COL_A2 = 32;                        // A2_hi | A2_lo    (stage 2 A)
  static constexpr int COL_D2 = 0;                         // stage 2 D
  static constexpr int TMEM_COLS = 128;
  static constexpr int CTAS_PER_SM = 4;
  // B image in shared memory (bytes): B1hi | B1lo | B2hi | B2lo
  static constexpr int B1_BYTES = N1 * Kp * 4;
  static constexpr int B2_BYTES = N2 * K2 * 4;
  static constexpr int IMG_BYTES = 2 * B1_BYTES + 2 * B2_BYTES;
  static_assert(2 * KpS <= COL_D1 - COL_AU, "u operand does not fit its TMEM columns");
  static_assert(COL_D1 + N1 <= TMEM_COLS, "stage-1 accumulator does not fit");
  static_assert(COL_A2 + 2 * K2S <= TMEM_COLS, "face operand does not fit its TMEM columns");
  static_assert(COL_D2 + N2 <= COL_A2, "stage-2 accumulator overlaps its operand");
  static_assert(N1 % 16 == 0 && N1 <= 256 && N2 % 16 == 0, "MMA N must be a multiple of 16 (M = 128)");
};

// ---------------------------------------------------------------- PTX
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D (TMEM) (+)= A (TMEM, 128 x 8 tf32) . B (shared memory descriptor)^T
__device__ __forceinline__ void mma_tf32(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
      "r"(a), "l"(bdesc), "r"(idesc), "r"(acc)
      : "memory");
}
// arrive once on `bar` when every MMA issued so far by this thread is done
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

// 16 consecutive 32-bit columns of this thread's lane (warp w owns lanes 32w..)
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16};" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
// load 16 columns and wait for them in one statement (the values are only
// defined after the wait)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&f)[16]) {
  uint32_t v[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n\ttcgen05.wait::ld.sync.aligned;"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) f[i] = __uint_as_float(v[i]);
}
__device__ __forceinline__ uint32_t tf32_bits(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
// x = hi + lo, both TF32: hi is x rounded to TF32 (nearest, ties away from
// zero: add half a unit of the 10-bit mantissa to the magnitude bits and
// clear the 13 low bits -- a carry into the exponent is the correct
// rounding; finite inputs only), lo the TF32 rounding of the exact float32
// remainder x - hi.
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = (__float_as_uint(x) + 0x1000u) & 0xffffe000u;
  lo = tf32_bits(x - __uint_as_float(hi));
}


// shared-memory matrix descriptor, K-major, no swizzle
__device__ __forceinline__ uint64_t smem_desc(const void* p, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((smem_addr(p) & 0x3FFFFu) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, relative LBO, layout type 0 (no swizzle)
}
// instruction descriptor: kind::tf32, float32 accumulate, A and B K-major
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int Nn) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(Nn >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait_all(uint64_t* bar, uint32_t phase) {
  for (int it = 0; it < (1 << 22); ++it)
    if (mbar_try_wait(bar, phase)) return true;
  return false;
}

struct TcArgs {
  const float* u;           // APPLY: u | PFUSE: z
  const float* p_old;       // PFUSE: previous direction
  float* y;                 // A u  (PFUSE: A p)
  float* p_new;             // PFUSE: p = zc z + beta p_old
  const float* geo;
  const uint32_t* nbr;
  const int* perm;
  const uint8_t* img;       // B image (IMG_BYTES, 16-byte aligned)
  const float* kappa;
  unsigned int* status;
  CgCtl* ctl;               // PFUSE: CG scalars (beta, zcoef in; pAp, alpha out)
  double* part;             // PFUSE: one partial of p.Ap per CTA
  int K, ldg;
  float tau, alpha, shift;
};

// Stage-1 MMAs: D1 = A_hi.B_hi + A_lo.B_hi + A_hi.B_lo over Kc (multiple of 8).
template <int NN, int Kc>
__device__ __forceinline__ void issue_3xtf32(uint32_t d, uint32_t a_hi, uint32_t a_lo, const uint8_t* b_hi,
                                             const uint8_t* b_lo) {
  constexpr uint32_t idesc = idesc_tf32(128, NN);
  constexpr uint32_t sbo = (Kc / 4) * 128;
#pragma unroll
  for (int s = 0; s < Kc / 8; ++s) mma_tf32(d, a_hi + 8 * s, smem_desc(b_hi + 256 * s, 128, sbo), idesc, s > 0);
#pragma unroll
  for (int s = 0; s < Kc / 8; ++s) mma_tf32(d, a_lo + 8 * s, smem_desc(b_hi + 256 * s, 128, sbo), idesc, 1u);
#pragma unroll
  for (int s = 0; s < Kc / 8; ++s) mma_tf32(d, a_hi + 8 * s, smem_desc(b_lo + 256 * s, 128, sbo), idesc, 1u);
}

// write Kc split values (zero padded) into this lane's TMEM: hi parts at
// columns [col, col + KS), lo parts at [col + KS, col + 2 KS), KS = Kc
// rounded up to 16 (the 16-column store width)
template <int Kc>
__device__ __forceinline__ void store_split(uint32_t taddr_lane, int col, const float* v, int nv) {
  constexpr int KS = (Kc + 15) / 16 * 16;
#pragma unroll
  for (int c = 0; c < KS / 16; ++c) {
    uint32_t h[16], l[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const int k = 16 * c + i;
      if (k < nv) {
        split_tf32(v[k], h[i], l[i]);
      } else {
        h[i] = 0u;
        l[i] = 0u;
      }
    }
    tmem_st16(taddr_lane + col + 16 * c, h);
    tmem_st16(taddr_lane + col + KS + 16 * c, l);
  }
}

// MODE AM_APPLY: y = A u + alpha J M u (+ shift u).
// MODE AM_PFUSE (one CG step's operator half, as k_apply's PFUSE mode):
//   p = zc z + beta p_old (beta, zc from the control block), p_new = p,
//   y = A p, and the last CTA to finish turns the per-CTA partials of p.Ap
//   into ctl->pAp and ctl->alpha = gamma / pAp (breakdown flagged).
// MODE AM_PDOT: the same with p already formed (u = p): one input tile and
//   plain neighbour gathers.
template <int N, int MODE>
__global__ void __launch_bounds__(128, TcDim<N>::CTAS_PER_SM) k_apply_tc(TcArgs a) {
  using D = TcDim<N>;
  constexpr int Np = D::Np, Nfp = D::Nfp, Kp = D::Kp, K2 = D::K2;
  constexpr int NT = (MODE == AM_PFUSE) ? 2 : 1;  // input tiles per element tile
  constexpr bool DOT = (MODE == AM_PFUSE || MODE == AM_PDOT);  // p.Ap and alpha
  constexpr int TILE = 128 * Np;                   // floats per tile
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* s_img = smem;                                          // IMG_BYTES
  float* s_t = reinterpret_cast<float*>(smem + D::IMG_BYTES);     // [2 buffers][NT][TILE]
  int* s_perm = reinterpret_cast<int*>(s_t + 2 * NT * TILE);      // 3 Np
  __shared__ __align__(8) uint64_t bar_img, bar_u[2], bar_mma;
  __shared__ float s_msum[Np];                                    // row sums of M (centring)
  __shared__ uint32_t s_taddr;
  __shared__ double s_red[64];

  grid_dep_wait();
  if (DOT && a.ctl->cont == 0) return;  // the loop has stopped (uniform)
  const RefMats<N, float>& R = CRef<N, float>::get();
  const RefPairs<N>& P = CPairs<N>::get();
  const int tid = threadIdx.x, warp = tid >> 5;
  const int ntiles = (a.K + 127) / 128;
  const float beta = (MODE == AM_PFUSE) ? (float)a.ctl->beta : 0.0f;
  const float zc = (MODE == AM_PFUSE) ? (float)a.ctl->zcoef : 1.0f;

  if (warp == 0) {
    tmem_alloc(&s_taddr, D::TMEM_COLS);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bar_img, 1);
    mbar_init(&bar_u[0], 1);
    mbar_init(&bar_u[1], 1);
    mbar_init(&bar_mma, 1);
    fence_mbar_init();
  }
  for (int i = tid; i < 3 * Np; i += 128) s_perm[i] = a.perm[i];
  if (tid < Np) {
    float m = 0.0f;
    for (int j = 0; j < Np; ++j) m += R.M[tid * Np + j];
    s_msum[tid] = m;
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tbase = s_taddr;
  const uint32_t tlane = tbase + ((uint32_t)(warp * 32) << 16);  // this warp's lane quarter

  auto tile_bytes = [&](int t) { return (uint32_t)(min(128, a.K - t * 128) * Np * 4); };
  // every tile goes through bulk copies when all byte counts are multiples of
  // 16 (the launcher guarantees 16-byte aligned vectors)
  const bool bulk_ok = (tile_bytes(ntiles - 1) % 16u) == 0u;
  auto issue_tile = [&](int t, int buf) {
    const uint32_t bytes = tile_bytes(t);
    mbar_expect_tx(&bar_u[buf], bytes * NT);
    bulk_load(s_t + (buf * NT) * TILE, a.u + (size_t)t * TILE, bytes, &bar_u[buf]);
    if (NT > 1) bulk_load(s_t + (buf * NT + 1) * TILE, a.p_old + (size_t)t * TILE, bytes, &bar_u[buf]);
  };
  if (tid == 0) {
    mbar_expect_tx(&bar_img, (uint32_t)D::IMG_BYTES);
    bulk_load(s_img, a.img, (uint32_t)D::IMG_BYTES, &bar_img);
    if (bulk_ok && blockIdx.x < ntiles) issue_tile(blockIdx.x, 0);
  }
  bool ok = mbar_wait_all(&bar_img, 0);
  bool failed = false;  // block-uniform: some wait of this CTA timed out
  uint32_t mma_phase = 0;
  double dA = 0.0;      // PFUSE: this thread's share of p.Ap
  int it = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
    if (__syncthreads_or(!ok)) {  // uniform stop after any time-out
      failed = true;
      break;
    }
    const int buf = it & 1;
    const int k0 = t * 128, nk = min(128, a.K - k0);
    const int k = k0 + tid;
    const bool active = tid < nk;
    float* s0 = s_t + (buf * NT) * TILE;
    float* s1 = s_t + (buf * NT + NT - 1) * TILE;
    if (bulk_ok) {
      if (tid == 0 && t + (int)gridDim.x < ntiles) {
        bulk_wait_read_all();  // the other buffer's output stores have left it
        issue_tile(t + gridDim.x, buf ^ 1);
      }
      ok = mbar_wait_all(&bar_u[buf], (uint32_t)((it >> 1) & 1));
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
    } else {
      for (int i = tid; i < nk * Np; i += 128) {
        s0[i] = a.u[(size_t)k0 * Np + i];
        if (NT > 1) s1[i] = a.p_old[(size_t)k0 * Np + i];
      }
      __syncthreads();
    }

    // ---- this element's values, geometry and neighbour words
    float u[Np];
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      float v = active ? s0[tid * Np + i] : 0.0f;
      if (MODE == AM_PFUSE) v = active ? fmaf(zc, v, beta * s1[tid * Np + i]) : 0.0f;
      u[i] = v;
    }
    uint32_t w[3] = {0u, 0u, 0u};
    Geo<float> g{};
    float kM = 1.0f;
    if (active) {
#pragma unroll
      for (int f = 0; f < 3; ++f) w[f] = __ldg(a.nbr + (size_t)f * a.K + k);
      g = load_geo(a.geo, a.ldg, k);
      if (a.kappa) kM = __ldg(a.kappa + k);
    }

    // ---- stage 1: A = u - c (3xTF32) into TMEM, MMA into D1.  The
    // stiffness and derivative blocks annihilate constants, so centring on
    // c = u[0] leaves them unchanged while their float32 rounding error
    // scales with the element's variation instead of |u| (the mass block
    // gets c M 1 back in the epilogue); on smooth vectors, the slow modes of
    // an iterative solve, this removes a cancellation error of order
    // eps / (k h)^2.
    const float c0 = u[0];
    {
      float uc[Np];
#pragma unroll
      for (int i = 0; i < Np; ++i) uc[i] = u[i] - c0;
      store_split<Kp>(tlane, D::COL_AU, uc, Np);
    }
    tmem_wait_st();
    fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
      issue_3xtf32<D::N1, Kp>(tbase + D::COL_D1, tbase + D::COL_AU, tbase + D::COL_AU + D::KpS, s_img,
                              s_img + D::B1_BYTES);
      mma_commit(&bar_mma);
    }

    // ---- CUDA cores meanwhile: neighbour values, normal derivatives, tau
    float uP[3][Nfp], dnP[3][Nfp], tauP[3], kP[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const uint32_t wf = w[f];
      tauP[f] = 0.0f;
      kP[f] = kM;
#pragma unroll
      for (int p = 0; p < Nfp; ++p) uP[f][p] = dnP[f][p] = 0.0f;
      if (active && ((wf >> 5) & 3u)) {
        const int kp = (int)(wf >> 7), fp = (int)(wf & 3);
        const bool flip = (wf >> 2) & 1;
        const float sJ = g.sJ[f], nx = g.nx[f], ny = g.ny[f];
        const float rxn = __ldg(a.geo + G_RX * a.ldg + kp), sxn = __ldg(a.geo + G_SX * a.ldg + kp);
        const float ryn = __ldg(a.geo + G_RY * a.ldg + kp), syn = __ldg(a.geo + G_SY * a.ldg + kp);
        const float Jn = __ldg(a.geo + G_J * a.ldg + kp);
        if (a.kappa) kP[f] = __ldg(a.kappa + kp);
        tauP[f] = a.tau * sJ / Jn;
        float ut[Np];
        const size_t nb = (size_t)kp * Np;
#pragma unroll
        for (int i = 0; i < Np; ++i) {
          const int j = s_perm[fp * Np + i];
          ut[i] = (MODE == AM_PFUSE) ? fmaf(zc, __ldg(a.u + nb + j), beta * __ldg(a.p_old + nb + j))
                                     : __ldg(a.u + nb + j);
        }
        const float ar = nx * rxn + ny * ryn, as = nx * sxn + ny * syn;
        const float cr = fp == 0 ? ar : (fp == 1 ? as : -ar - as);
        const float cs = fp == 0 ? as : (fp == 1 ? -ar - as : ar);
        float dq[Nfp];
#pragma unroll
        for (int q = 0; q < Nfp; ++q) {
          float2 s = make_float2(0.0f, 0.0f);  // (Dr_F0 u~, Ds_F0 u~), packed FP32 FMA
#pragma unroll
          for (int j = 0; j < Np; ++j) {
            const float v = ut[j] - c0;  // centred as the own values
            s = __ffma2_rn(P.DrDs[q * Np + j], make_float2(v, v), s);
          }
          dq[q] = cr * s.x + cs * s.y;
        }
#pragma unroll
        for (int p = 0; p < Nfp; ++p) {
          uP[f][p] = flip ? ut[N - p] : ut[p];
          dnP[f][p] = flip ? dq[N - p] : dq[p];
        }
      }
    }

    // ---- stage-1 results
    ok = mbar_wait_all(&bar_mma, mma_phase);
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    mma_phase ^= 1u;
    fence_after_sync();
    float y[Np], dr[Np], ds[Np];
    {
      const float kJ = kM * g.J;
      const float crr = kJ * (g.rx * g.rx + g.ry * g.ry), crs = kJ * (g.rx * g.sx + g.ry * g.sy);
      const float css = kJ * (g.sx * g.sx + g.sy * g.sy), cm = a.alpha * g.J;
      float v[16];
#pragma unroll
      for (int i = 0; i < Np; ++i) y[i] = 0.0f;
#pragma unroll
      for (int blk = 0; blk < 6; ++blk) {
#pragma unroll
        for (int c = 0; c < Kp; c += 16) {
          tmem_ld16(tlane + D::COL_D1 + blk * Kp + c, v);
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int n = c + i;
            if (n < Np) {
              if (blk == 0) y[n] = fmaf(crr, v[i], y[n]);
              else if (blk == 1) y[n] = fmaf(crs, v[i], y[n]);
              else if (blk == 2) y[n] = fmaf(css, v[i], y[n]);
              else if (blk == 3) y[n] = fmaf(cm, v[i] + c0 * s_msum[n], y[n]);
              else if (blk == 4) dr[n] = v[i];
              else ds[n] = v[i];
            }
          }
        }
      }
    }

    // ---- faces: SIPG flux into y, gradient-test weights into A2
    float a2[6 * Nfp];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const uint32_t wf = w[f];
      const int bc = (wf >> 3) & 3;
      const bool pact = (wf >> 5) & 1, mint = (wf >> 6) & 1, mdir = (bc == 1);
#pragma unroll
      for (int q = 0; q < Nfp; ++q) a2[f * Nfp + q] = a2[3 * Nfp + f * Nfp + q] = 0.0f;
      if (!active || !(pact || mint || mdir)) continue;
      const float sJ = g.sJ[f], nx = g.nx[f], ny = g.ny[f];
      const float tauM = a.tau * sJ / g.J;
      const float arM = nx * g.rx + ny * g.ry, asM = nx * g.sx + ny * g.sy;
      const float tP = (pact || mint) ? tauP[f] : tauM;
      const float kPf = (pact || mint) ? kP[f] : kM;
      const bool kap = a.kappa != nullptr;
      const float kF = kap ? 0.5f * (kM + kPf) : 1.0f;
      const float caM = mdir ? 1.0f : (mint ? 0.5f : 0.0f);
      const float cjM = mdir ? (kap ? tauM * kM : tauM) : (mint ? (kap ? 0.5f * tauM * kF : 0.5f * tauM) : 0.0f);
      const float cgM = (mdir ? 1.0f : (mint ? 0.25f : 0.0f)) * kM;
      const float caP = pact ? 0.5f : 0.0f;
      const float cjP = pact ? (kap ? 0.5f * tP * kF : 0.5f * tP) : 0.0f;
      const float cgP = (pact ? 0.25f : 0.0f) * kM;
      float v1[Nfp], v2[Nfp];
#pragma unroll
      for (int p = 0; p < Nfp; ++p) {
        const int n = fmask_idx(N, f, p);
        const float dnm = arM * dr[n] + asM * ds[n];
        const float uM = u[n];
        const float avgI = kap ? 0.5f * (kM * dnm + kPf * dnP[f][p]) : 0.5f * (dnm + dnP[f][p]);
        const float jmpI = uM - uP[f][p];
        const float avgM = mdir ? (kap ? kM * dnm : dnm) : avgI;
        const float jmpM = mdir ? uM : jmpI;
        v1[p] = -caM * avgM + cjM * jmpM - caP * avgI + cjP * jmpI;
        v2[p] = cgM * jmpM + cgP * jmpI;
      }
#pragma unroll
      for (int q = 0; q < Nfp; ++q) {
        float2 s = make_float2(0.0f, 0.0f);  // the face mass on both flux vectors, packed FP32 FMA
#pragma unroll
        for (int p = 0; p < Nfp; ++p) {
          const float m = R.m1d[(f * Nfp + p) * Nfp + q];
          s = __ffma2_rn(make_float2(m, m), make_float2(v1[p], v2[p]), s);
        }
        const float s1f = s.x, s2f = s.y;
        y[fmask_idx(N, f, q)] += sJ * s1f;
        a2[f * Nfp + q] = -sJ * arM * s2f;
        a2[3 * Nfp + f * Nfp + q] = -sJ * asM * s2f;
      }
    }

    // ---- stage 2: face lift on the tensor cores
    store_split<K2>(tlane, D::COL_A2, a2, 6 * Nfp);
    tmem_wait_st();
    fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
      issue_3xtf32<D::N2, K2>(tbase + D::COL_D2, tbase + D::COL_A2, tbase + D::COL_A2 + D::K2S,
                              s_img + 2 * D::B1_BYTES, s_img + 2 * D::B1_BYTES + D::B2_BYTES);
      mma_commit(&bar_mma);
    }
    ok = mbar_wait_all(&bar_mma, mma_phase);
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    mma_phase ^= 1u;
    fence_after_sync();
    {
      float v[16];
#pragma unroll
      for (int c = 0; c < D::N2; c += 16) {
        tmem_ld16(tlane + D::COL_D2 + c, v);
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (c + i < Np) y[c + i] += v[i];
      }
    }
    if (a.shift != 0.0f) {
#pragma unroll
      for (int i = 0; i < Np; ++i) y[i] = fmaf(a.shift, u[i], y[i]);
    }
    if (DOT && active) {
#pragma unroll
      for (int i = 0; i < Np; ++i) dA += (double)u[i] * (double)y[i];
    }

    // ---- outputs into the consumed input tiles, then back to global memory
    // (every thread read its tile slots right after the tile arrived, and the
    // CTA has passed barriers since)
    if (active) {
#pragma unroll
      for (int i = 0; i < Np; ++i) {
        if (MODE == AM_PFUSE) s0[tid * Np + i] = u[i];
        s1[tid * Np + i] = y[i];
      }
    }
    if (bulk_ok) {
      fence_proxy_async_smem();
      __syncthreads();
      if (tid == 0) {
        bulk_store(a.y + (size_t)k0 * Np, s1, tile_bytes(t));
        if (MODE == AM_PFUSE) bulk_store(a.p_new + (size_t)k0 * Np, s0, tile_bytes(t));
        bulk_commit();
      }
    } else {
      __syncthreads();
      for (int i = tid; i < nk * Np; i += 128) {
        a.y[(size_t)k0 * Np + i] = s1[i];
        if (MODE == AM_PFUSE) a.p_new[(size_t)k0 * Np + i] = s0[i];
      }
      __syncthreads();  // the next tile overwrites these buffers
    }
  }
  if (failed && tid == 0) {
    atomicOr(a.status, ST_TMA_TIMEOUT);
    // let an MMA group this CTA issued finish (bounded) before its TMEM goes
    (void)mbar_wait_all(&bar_mma, mma_phase);
  }
  if (bulk_ok && tid == 0) bulk_wait_read_all();
  fence_before_sync();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tbase, D::TMEM_COLS);
  if (!DOT) return;

  // ---- p.Ap: CTA partial -> last CTA -> control block (every CTA takes part,
  // also after a time-out, so the ticket always completes)
  double d0 = 0.0;
  block_sum2<128>(dA, d0, s_red);
  if (tid == 0) a.part[blockIdx.x] = dA;
  if (!is_last_block(&a.ctl->ticket)) return;
  double sA, sB;
  reduce_partials2<128>(a.part, nullptr, gridDim.x, sA, sB, s_red);
  if (tid == 0) {
    CgCtl* c = a.ctl;
    c->pAp = sA;
    const double al = c->gamma / sA;
    if (!(sA > 0.0) || !isfinite(al)) {
      c->status = 2;  // breakdown
      c->alpha = 0.0;
    } else {
      c->alpha = al;
    }
    c->ticket = 0u;
  }
}

// ------------------------------------------------------------- host side
// Byte image of the B operands for degree N (host, from the float64
// reference matrices): B1 = [Srr; Srs; Sss; M; Dr; Ds] (N1 x Kp),
// B2[i][k] = Dr[F(k)][i] (k < 3 Nfp), Ds[F(k - 3 Nfp)][i] (3 Nfp <= k < 6 Nfp);
// each split into TF32 hi and lo parts, canonical K-major layout.
template <int N>
int build_image(const double* Dr, const double* Ds, const double* M, uint8_t* out) {
  using D = TcDim<N>;
  constexpr int Np = D::Np, Nfp = D::Nfp, Kp = D::Kp, K2 = D::K2;
  auto at = [](const double* A, int i, int j) { return A[i * Np + j]; };
  std::vector<double> B1((size_t)D::N1 * Kp, 0.0), B2((size_t)D::N2 * K2, 0.0);
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) {
      double rr = 0.0, rs = 0.0, ss = 0.0;
      for (int p = 0; p < Np; ++p)
        for (int q = 0; q < Np; ++q) {
          const double m = at(M, q, p);  // (M^T)[p][q]
          rr += at(Dr, p, i) * m * at(Dr, q, j);
          rs += at(Dr, p, i) * m * at(Ds, q, j) + at(Ds, p, i) * m * at(Dr, q, j);
          ss += at(Ds, p, i) * m * at(Ds, q, j);
        }
      B1[(size_t)(0 * Kp + i) * Kp + j] = rr;
      B1[(size_t)(1 * Kp + i) * Kp + j] = rs;
      B1[(size_t)(2 * Kp + i) * Kp + j] = ss;
      B1[(size_t)(3 * Kp + i) * Kp + j] = at(M, i, j);
      B1[(size_t)(4 * Kp + i) * Kp + j] = at(Dr, i, j);
      B1[(size_t)(5 * Kp + i) * Kp + j] = at(Ds, i, j);
    }
  for (int i = 0; i < Np; ++i)
    for (int f = 0; f < 3; ++f)
      for (int q = 0; q < Nfp; ++q) {
        const int n = fmask_idx(N, f, q);
        B2[(size_t)i * K2 + f * Nfp + q] = at(Dr, n, i);
        B2[(size_t)i * K2 + 3 * Nfp + f * Nfp + q] = at(Ds, n, i);
      }
  // TF32 = float32 with the low 13 mantissa bits cleared, round to nearest
  // (ties away from zero), as cvt.rna.tf32.f32 does on the device
  auto tf32 = [](double x) {
    float f = (float)x;
    uint32_t b;
    std::memcpy(&b, &f, 4);
    if ((b & 0x7f800000u) != 0x7f800000u) {
      b += 0x1000u;
      b &= 0xffffe000u;
    }
    float r;
    std::memcpy(&r, &b, 4);
    return r;
  };
  auto put = [&](const std::vector<double>& B, int rows, int Kc, uint8_t* hi, uint8_t* lo) {
    for (int n = 0; n < rows; ++n)
      for (int kk = 0; kk < Kc; ++kk) {
        const double x = B[(size_t)n * Kc + kk];
        const float h = tf32(x);
        const float l = tf32(x - (double)h);
        const size_t off = ((size_t)(n / 8) * (Kc / 4) + kk / 4) * 128 + (n % 8) * 16 + (kk % 4) * 4;
        std::memcpy(hi + off, &h, 4);
        std::memcpy(lo + off, &l, 4);
      }
  };
  put(B1, D::N1, Kp, out, out + D::B1_BYTES);
  put(B2, D::N2, K2, out + 2 * D::B1_BYTES, out + 2 * D::B1_BYTES + D::B2_BYTES);
  return D::IMG_BYTES;
}

}  // namespace tc

// Degrees with a tensor-core float32 apply.
bool tc_supported(int N) { return N >= 1 && N <= 4; }


int tc_image_bytes(int N) {
  switch (N) {
    case 1: return tc::TcDim<1>::IMG_BYTES;
    case 2: return tc::TcDim<2>::IMG_BYTES;
    case 3: return tc::TcDim<3>::IMG_BYTES;
    case 4: return tc::TcDim<4>::IMG_BYTES;
  }
  return 0;
}

int tc_build_image(int N, const double* Dr, const double* Ds, const double* M, uint8_t* out) {
  switch (N) {
    case 1: return tc::build_image<1>(Dr, Ds, M, out);
    case 2: return tc::build_image<2>(Dr, Ds, M, out);
    case 3: return tc::build_image<3>(Dr, Ds, M, out);
    case 4: return tc::build_image<4>(Dr, Ds, M, out);
  }
  return 0;
}

template <int N, int MODE>
static int tc_smem_request() {
  using D = tc::TcDim<N>;
  constexpr int NT = (MODE == AM_PFUSE) ? 2 : 1;
  const int smem = D::IMG_BYTES + (2 * NT * 128 * D::Np + 3 * D::Np) * 4 + 64;
  // at most CTAS_PER_SM CTAs per SM (their TMEM columns add up to the SM's
  // 512): ask for enough shared memory that one more cannot be resident
  const int cap = (228 * 1024) / (D::CTAS_PER_SM + 1) + 1024;
  return smem < cap ? cap : smem;
}

template <int N, int MODE>
static cudaError_t tc_prepare_n() {
  return cudaFuncSetAttribute(tc::k_apply_tc<N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              tc_smem_request<N, MODE>());
}

// Kernel attributes of the tensor-core apply (current device); call before
// any launch or stream capture of it.
cudaError_t tc_prepare(int N) {
  cudaError_t e = cudaErrorInvalidValue;
  switch (N) {
    case 1: e = tc_prepare_n<1, AM_APPLY>(); if (e == cudaSuccess) e = tc_prepare_n<1, AM_PFUSE>(); break;
    case 2: e = tc_prepare_n<2, AM_APPLY>(); if (e == cudaSuccess) e = tc_prepare_n<2, AM_PFUSE>(); break;
    case 3: e = tc_prepare_n<3, AM_APPLY>(); if (e == cudaSuccess) e = tc_prepare_n<3, AM_PFUSE>(); break;
    case 4: e = tc_prepare_n<4, AM_APPLY>(); if (e == cudaSuccess) e = tc_prepare_n<4, AM_PFUSE>(); break;
  }
  if (e != cudaSuccess) return e;
  switch (N) {
    case 1: e = tc_prepare_n<1, AM_PDOT>(); break;
    case 2: e = tc_prepare_n<2, AM_PDOT>(); break;
    case 3: e = tc_prepare_n<3, AM_PDOT>(); break;
    case 4: e = tc_prepare_n<4, AM_PDOT>(); break;
  }
  return e;
}

template <int N, int MODE>
static cudaError_t launch_tc_n(const ApplyArgs<float>& a, const uint8_t* img, cudaStream_t s) {
  using D = tc::TcDim<N>;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = (a.K + 127) / 128;
  const int grid = ntiles < D::CTAS_PER_SM * nsm ? ntiles : D::CTAS_PER_SM * nsm;
  tc::TcArgs t{};
  t.u = a.in0;
  t.p_old = a.in1;
  t.y = a.out0;
  t.p_new = a.out1;
  t.geo = a.geo;
  t.nbr = a.nbr;
  t.perm = a.perm;
  t.img = img;
  t.kappa = a.kappa;
  t.status = a.ctl_status;
  t.ctl = a.ctl;
  t.part = a.partA;
  t.K = a.K;
  t.ldg = a.ldg;
  t.tau = (float)a.tau;
  t.alpha = (float)a.alpha;
  t.shift = (float)a.shift;
  PdlLaunch l(dim3(grid), dim3(128), tc_smem_request<N, MODE>(), s, a.pdl);
  return cudaLaunchKernelEx(&l.cfg, tc::k_apply_tc<N, MODE>, t);
}

template <int MODE>
static cudaError_t launch_tc_mode(int N, const ApplyArgs<float>& a, const uint8_t* img, cudaStream_t s) {
  switch (N) {
    case 1: return launch_tc_n<1, MODE>(a, img, s);
    case 2: return launch_tc_n<2, MODE>(a, img, s);
    case 3: return launch_tc_n<3, MODE>(a, img, s);
    case 4: return launch_tc_n<4, MODE>(a, img, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_apply_tc(int N, int mode, const ApplyArgs<float>& a, const uint8_t* img, cudaStream_t s) {
  if (mode == AM_APPLY) return launch_tc_mode<AM_APPLY>(N, a, img, s);
  if (mode == AM_PFUSE) return launch_tc_mode<AM_PFUSE>(N, a, img, s);
  if (mode == AM_PDOT) return launch_tc_mode<AM_PDOT>(N, a, img, s);
  return cudaErrorInvalidValue;
}

}  // namespace ddg
