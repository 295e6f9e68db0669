// float64 SIPG apply on the FP64 tensor cores (mma.sync m16n8k8 .f64, DMMA).
//
// tcgen05 has no float64 kind; the FP64 tensor path of sm_100a is the
// warp-level mma.sync f64 family, whose m16n8k8 shape runs at the full
// float64 rate (64 multiply-adds per clock per SM) with one instruction per
// 1,024 multiply-adds.  The CUDA-core float64 apply issues one DFMA per 32
// multiply-adds and is bound by instruction issue and gather latency, not by
// the float64 pipe; here the element contractions become a few dozen MMAs
// per 16 elements.
//
// Work unit: a row block of 16 consecutive elements (the MMA's M), owned by
// one warp; warps loop over row blocks (persistent grid) and never wait on
// each other.  Per row block, with u the (16 x Np) element tile:
//   stage 1   [Srr u | Srs u | Sss u | M u | Dr_F u | Ds_F u]   (K = Np)
//             Srr = Dr^T M^T Dr, Srs = Dr^T M^T Ds + Ds^T M^T Dr,
//             Sss = Ds^T M^T Ds are the reference stiffness blocks, so the
//             affine volume term is J (c_rr Srr + c_rs Srs + c_ss Sss) u
//             with c_rr = rx^2 + ry^2, c_rs = rx sx + ry sy,
//             c_ss = sx^2 + sy^2, and the mass term alpha J M u; Dr_F, Ds_F
//             (the face-node rows) give the own normal derivative;
//   stage 2   per face, the neighbour's gradient at the shared face: its
//             nodal values gathered through the rotation relabelling that
//             makes the shared face its face 0, times [Dr_F0 | Ds_F0]; the
//             MMA's result fragments go straight into the SIPG flux of each
//             (element, face node): v1 = -c_a avg + c_j jmp (penalty and
//             consistency) and v2 = c_g jmp (symmetry), as in elem_apply;
//   stage 3   y += [c_r v2 | c_s v2 | sJ v1] . B3 (K = 3 * 3 (N+1)), where
//             B3 holds m1d_f Dr[Fmask_f, :], m1d_f Ds[Fmask_f, :] and m1d_f
//             injected at the face nodes: the 1D face mass, the lift of the
//             gradient-test terms (c_r = -sJ n.(rx, ry), c_s = -sJ n.(sx, sy))
//             and the face-node flux all in one MMA.
// The B operands (all reference-element matrices, float64) are laid out on
// the host in per-lane fragment order and staged once per CTA in shared
// memory; every fragment load is one conflict-free 16-byte load per lane.
#pragma once

namespace ddg {
namespace dm {

constexpr int WARPS = 8;
constexpr int BLOCK = 32 * WARPS;
constexpr int RB = 16;  // elements per row block

__host__ __device__ constexpr int rup8(int x) { return (x + 7) / 8 * 8; }

struct ShapeRT {
  int Np, Nfp, NF, KP, KS, NTV, NTF, NT1, K3, KS3, GS, NTN, TN, T3, TILES, IMG, WSZ, OFF_DN, OFF_UP, OFF_G;
  size_t smem;
};
__host__ __device__ constexpr ShapeRT shape_of(int N) {
  const int Np = (N + 1) * (N + 2) / 2, Nfp = N + 1, NF = 3 * Nfp;
  const int KP = rup8(Np), KS = KP / 8, NTV = KP / 8, NTF = rup8(NF) / 8, NT1 = 4 * NTV + 2 * NTF;
  const int K3 = rup8(3 * NF), KS3 = K3 / 8, NTN = 2 * (rup8(Nfp) / 8);
  // row stride of the stage-3 operand: 4 (mod 16) doubles keeps its fragment loads conflict-free
  const int GS = K3 + ((4 - K3 % 16) + 16) % 16;
  const int TN = KS * NT1, T3 = TN + KS * NTN, TILES = T3 + KS3 * NTV, IMG = TILES * 64;
  const int OFF_DN = RB * Np, OFF_UP = OFF_DN + RB * NF, OFF_G = OFF_UP + RB * Nfp, WSZ = OFF_G + RB * GS;
  const int tab_ints = 3 * Np;
  const size_t smem = (size_t)(IMG + WARPS * WSZ) * 8 + (size_t)((tab_ints + 3) / 4 * 4) * 4;
  return ShapeRT{Np, Nfp, NF, KP, KS, NTV, NTF, NT1, K3, KS3, GS, NTN, TN, T3, TILES, IMG, WSZ, OFF_DN, OFF_UP,
                 OFF_G, smem};
}

// D += A B for one 16 x 8 x 8 float64 tile (fragments in the PTX layout:
// a = A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4]; b = B[t][g], B[t+4][g];
// d = D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1]; g = lane/4, t = lane%4)
__device__ __forceinline__ void dmma(double (&d)[4], const double (&a)[4], const double2 b) {
  asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b.x), "d"(b.y));
}

__device__ __forceinline__ double sel3(const double (&v)[3], int f) { return f == 0 ? v[0] : (f == 1 ? v[1] : v[2]); }

// Per-element coefficients of this kernel, structure-of-arrays dg[c * ldg + k],
// computed once per operator and boundary-tag set (k_dm_geo):
//   D_CRR, D_CRS, D_CSS   J (rx^2 + ry^2), J (rx sx + ry sy), J (sx^2 + sy^2)
//   D_J                   J (the mass term is alpha J M u)
//   D_DR + f, D_DS + f    n_f . (rx, ry), n_f . (sx, sy): own normal derivative
//   D_T + 9 f + c         face f's flux coefficients: with v1, v2 of elem_apply,
//                         sJ v1 = T0 dnM + T1 (Dr_F0 u~) + T2 (Ds_F0 u~) + T3 uM + T4 uP,
//                         c_r v2 = T5 uM + T6 uP, c_s v2 = T7 uM + T8 uP
//                         (u~ the rotated neighbour values; zero on inactive faces)
enum DmField { D_CRR = 0, D_CRS, D_CSS, D_J, D_DR, D_DS = D_DR + 3, D_T = D_DS + 3, D_COUNT = D_T + 27 };

__global__ void k_dm_geo(const double* __restrict__ geo, const uint32_t* __restrict__ nbr, double* __restrict__ dg,
                         int K, int ldg, double tau) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  const double rx = geo[G_RX * ldg + k], sx = geo[G_SX * ldg + k];
  const double ry = geo[G_RY * ldg + k], sy = geo[G_SY * ldg + k];
  const double J = geo[G_J * ldg + k];
  dg[D_CRR * ldg + k] = J * (rx * rx + ry * ry);
  dg[D_CRS * ldg + k] = J * (rx * sx + ry * sy);
  dg[D_CSS * ldg + k] = J * (sx * sx + sy * sy);
  dg[D_J * ldg + k] = J;
  for (int f = 0; f < 3; ++f) {
    const double nx = geo[(G_F0 + 3 * f) * ldg + k], ny = geo[(G_F0 + 3 * f + 1) * ldg + k];
    const double sJ = geo[(G_F0 + 3 * f + 2) * ldg + k];
    const double dr = nx * rx + ny * ry, ds = nx * sx + ny * sy;
    dg[(D_DR + f) * ldg + k] = dr;
    dg[(D_DS + f) * ldg + k] = ds;
    // coefficients as in elem_apply (kappa = 1)
    const uint32_t wf = nbr[(size_t)f * K + k];
    const int bc = (wf >> 3) & 3;
    const bool pact = (wf >> 5) & 1, mint = (wf >> 6) & 1, mdir = (bc == 1);
    const double tauM = tau * sJ / J;
    double tauP = tauM, crn = 0.0, csn = 0.0;
    if (pact || mint) {
      const int kp = (int)(wf >> 7), fp = (int)(wf & 3u);
      const double rxn = geo[G_RX * ldg + kp], sxn = geo[G_SX * ldg + kp];
      const double ryn = geo[G_RY * ldg + kp], syn = geo[G_SY * ldg + kp];
      tauP = tau * sJ / geo[G_J * ldg + kp];
      const double ar = nx * rxn + ny * ryn, as = nx * sxn + ny * syn;
      crn = fp == 0 ? ar : (fp == 1 ? as : -ar - as);
      csn = fp == 0 ? as : (fp == 1 ? -ar - as : ar);
    }
    const double caM = mdir ? 1.0 : (mint ? 0.5 : 0.0);
    const double cjM = mdir ? tauM : (mint ? 0.5 * tauM : 0.0);
    const double cgM = mdir ? 1.0 : (mint ? 0.25 : 0.0);
    const double caP = pact ? 0.5 : 0.0;
    const double cjP = pact ? 0.5 * tauP : 0.0;
    const double cgP = pact ? 0.25 : 0.0;
    // v1 = cA0 dnM + cA1 dnP + cA2 uM + cA3 uP, v2 = cG0 uM + cG1 uP, dnP = crn (Dr_F0 u~) + csn (Ds_F0 u~);
    // avgI = (dnM + dnP) / 2, jmpI = uM - uP; a Dirichlet face has avgM = dnM, jmpM = uM
    const double cA0 = -((mdir ? caM : 0.5 * caM) + 0.5 * caP);
    const double cA1 = -(mdir ? 0.0 : 0.5 * caM) - 0.5 * caP;
    const double cA2 = cjM + cjP;
    const double cA3 = -(mdir ? 0.0 : cjM) - cjP;
    const double cG0 = cgM + cgP;
    const double cG1 = -(mdir ? 0.0 : cgM) - cgP;
    const double cR = -sJ * dr, cS = -sJ * ds;
    const double T[9] = {sJ * cA0, sJ * cA1 * crn, sJ * cA1 * csn, sJ * cA2, sJ * cA3,
                         cR * cG0, cR * cG1,       cS * cG0,        cS * cG1};
    for (int c = 0; c < 9; ++c) dg[(D_T + 9 * f + c) * ldg + k] = T[c];
  }
}

// MODE: AM_APPLY, AM_PFUSE or AM_RESID with the meaning of k_apply (no kappa).
template <int N, int MODE>
__global__ void __launch_bounds__(BLOCK, (N <= 4 ? 2 : 1)) k_apply_dm(ApplyArgs<double> a) {
  constexpr ShapeRT S = shape_of(N);
  constexpr int Np = S.Np, Nfp = S.Nfp, NF = S.NF, GS = S.GS;
  static_assert(Nfp <= 8, "neighbour operand holds one n-tile per derivative");
  constexpr bool TWO = (MODE == AM_PFUSE);
  extern __shared__ __align__(128) double dsm[];
  double* s_img = dsm;
  double* s_w = dsm + S.IMG;
  int* s_perm = reinterpret_cast<int*>(s_w + WARPS * S.WSZ);
  __shared__ __align__(8) uint64_t s_bar[WARPS + 1];
  __shared__ double s_red[64];
  __shared__ int s_ok;

  grid_dep_wait();
  if (MODE == AM_PFUSE && a.ctl->cont == 0) return;  // uniform across the grid
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  if (tid == 0) {
    for (int i = 0; i <= WARPS; ++i) mbar_init(&s_bar[i], 1);
    fence_mbar_init();
  }
  for (int i = tid; i < 3 * Np; i += BLOCK) s_perm[i] = a.perm[i];
  __syncthreads();
  if (tid == 0) {
    mbar_expect_tx(&s_bar[WARPS], (uint32_t)(S.IMG * 8));
    bulk_load(s_img, a.dm_img, (uint32_t)(S.IMG * 8), &s_bar[WARPS]);
    s_ok = mbar_wait_bounded(&s_bar[WARPS], 0, a.ctl_status) ? 1 : 0;
  }
  __syncthreads();

  double* sU = s_w + warp * S.WSZ;  // own tile (u, or the CG direction p)
  double* sDN = sU + S.OFF_DN;      // own normal derivative at the face nodes
  double* sUP = sU + S.OFF_UP;      // neighbour's face values (rotated order) of the current face
  double* sG = sU + S.OFF_G;        // second input tile, then the stage-3 operand, then the output tile
  const double beta = (MODE == AM_PFUSE) ? a.ctl->beta : 0.0;
  const double zc = (MODE == AM_PFUSE) ? a.ctl->zcoef : 1.0;
  const double alpha = a.alpha, shift = a.shift;
  const int K = a.K, ldg = a.ldg;
  const double* __restrict__ dgeo = a.dm_geo;
  const uint32_t* __restrict__ nbr = a.nbr;
  const double* __restrict__ in0 = a.in0;
  const double* __restrict__ in1 = a.in1;
  auto tile = [&](int i) { return *reinterpret_cast<const double2*>(s_img + i * 64 + lane * 2); };
  // the gathered neighbour value (the CG direction is formed on the fly)
  auto src = [&](size_t idx) {
    if (MODE == AM_PFUSE) return zc * __ldg(in0 + idx) + beta * __ldg(in1 + idx);
    return __ldg(in0 + idx);
  };

  double dA = 0.0, dB = 0.0;
  uint32_t phase = 0;
  bool dead = (s_ok == 0);
  bool pending = false;  // a bulk store of this warp may still read its tiles
  // AM_APPLY may cover the element range [k_lo, k_hi) only (k_lo a multiple of RB)
  const int k_hi = (MODE == AM_APPLY && a.k_hi > 0) ? a.k_hi : K;
  const int rb_lo = (MODE == AM_APPLY) ? a.k_lo / RB : 0;
  const int nrb = (k_hi + RB - 1) / RB;
  for (int rb = rb_lo + blockIdx.x * WARPS + warp; rb < nrb && !dead; rb += gridDim.x * WARPS) {
    const int k0 = rb * RB;
    const int nw = min(RB, k_hi - k0);
    const size_t off = (size_t)k0 * Np;
    const uint32_t bytes = (uint32_t)(nw * Np * 8);
    const bool tma = a.use_tma && (bytes % 16u == 0u);
    // this thread's two rows of the MMA fragments: g and g + 8
    bool rv[2];
    int kr[2];
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
      rv[rr] = g + 8 * rr < nw;
      kr[rr] = k0 + min(g + 8 * rr, nw - 1);
    }
    uint32_t wr[3][2];  // neighbour words of the two rows
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
      for (int rr = 0; rr < 2; ++rr) wr[f][rr] = rv[rr] ? __ldg(nbr + (size_t)f * K + kr[rr]) : 0u;

    // ---------------------------------------------------------- own tile(s)
    // the previous row block's bulk stores have read the tiles, and every
    // generic access to them is ordered before the next bulk load
    if (lane == 0 && pending) bulk_wait_read_all();
    pending = false;
    fence_proxy_async_smem();
    __syncwarp();
    if (tma) {
      if (lane == 0) {
        mbar_expect_tx(&s_bar[warp], bytes * (TWO ? 2u : 1u));
        bulk_load(sU, in0 + off, bytes, &s_bar[warp]);
        if (TWO) bulk_load(sG, in1 + off, bytes, &s_bar[warp]);
      }
    }
    // element coefficients of the two rows (overlap the bulk copy)
    double crr[2], crs[2], css[2], cm[2], dr[2][3], ds[2][3];
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
      const double* gk = dgeo + kr[rr];
      crr[rr] = __ldg(gk + D_CRR * ldg);
      crs[rr] = __ldg(gk + D_CRS * ldg);
      css[rr] = __ldg(gk + D_CSS * ldg);
      cm[rr] = alpha * __ldg(gk + D_J * ldg);
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        dr[rr][f] = __ldg(gk + (D_DR + f) * ldg);
        ds[rr][f] = __ldg(gk + (D_DS + f) * ldg);
      }
    }
    if (tma) {
      const bool ok = mbar_wait_bounded(&s_bar[warp], phase, a.ctl_status);
      if (!__all_sync(0xffffffffu, ok)) {
        dead = true;
        break;
      }
      phase ^= 1u;
    } else {
      for (int i = lane; i < nw * Np; i += 32) {
        sU[i] = in0[off + i];
        if (TWO) sG[i] = in1[off + i];
      }
    }
    __syncwarp();
    if (MODE == AM_PFUSE) {
      for (int i = lane; i < nw * Np; i += 32) sU[i] = zc * sU[i] + beta * sG[i];
      __syncwarp();
    }

    // ------------------------------------------- stage 1: volume and own gradient
    double yv[S.NTV][4];
    {
      double af[S.KS][4];
#pragma unroll
      for (int ks = 0; ks < S.KS; ++ks)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int row = g + (i & 1) * 8, col = ks * 8 + t + (i >> 1) * 4;
          af[ks][i] = (row < nw && col < Np) ? sU[row * Np + col] : 0.0;
        }
      const int npr = (alpha != 0.0) ? 4 : 3;  // no mass product for Poisson
#pragma unroll
      for (int j = 0; j < S.NTV; ++j) {
        double acc[4][4] = {};
#pragma unroll
        for (int ks = 0; ks < S.KS; ++ks)
#pragma unroll
          for (int pr = 0; pr < 4; ++pr)
            if (pr < npr) dmma(acc[pr], af[ks], tile(ks * S.NT1 + pr * S.NTV + j));
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int rr = i >> 1;
          yv[j][i] = crr[rr] * acc[0][i] + crs[rr] * acc[1][i] + css[rr] * acc[2][i] + cm[rr] * acc[3][i];
        }
      }
#pragma unroll
      for (int j = 0; j < S.NTF; ++j) {
        double p4[4] = {}, p5[4] = {};
#pragma unroll
        for (int ks = 0; ks < S.KS; ++ks) {
          dmma(p4, af[ks], tile(ks * S.NT1 + 4 * S.NTV + j));
          dmma(p5, af[ks], tile(ks * S.NT1 + 4 * S.NTV + S.NTF + j));
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int rr = i >> 1, row = g + 8 * rr, c = j * 8 + 2 * t + (i & 1);
          if (row < nw && c < NF) {
            const int f = c / Nfp;
            sDN[row * NF + c] = sel3(dr[rr], f) * p4[i] + sel3(ds[rr], f) * p5[i];
          }
        }
      }
    }
    // zero the stage-3 operand's padding columns (K3 > 3 NF)
    for (int i = lane; i < RB * (S.K3 - 3 * NF); i += 32) {
      const int row = i / (S.K3 - 3 * NF), c = 3 * NF + i % (S.K3 - 3 * NF);
      sG[row * GS + c] = 0.0;
    }
    __syncwarp();

    // -------------- stage 2: neighbours' gradients at the shared faces, and the flux
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      bool use[2];
#pragma unroll
      for (int rr = 0; rr < 2; ++rr) use[rr] = ((wr[f][rr] >> 5) & 1u) || ((wr[f][rr] >> 6) & 1u);
      double an[S.KS][4];
#pragma unroll
      for (int ks = 0; ks < S.KS; ++ks)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int rr = i & 1, col = ks * 8 + t + (i >> 1) * 4;
          const int kp = (int)(wr[f][rr] >> 7), fp = (int)(wr[f][rr] & 3u);
          an[ks][i] = (use[rr] && col < Np) ? src((size_t)kp * Np + s_perm[fp * Np + col]) : 0.0;
        }
      // the neighbour's face-0 values (rotated order) for the jumps
#pragma unroll
      for (int ks = 0; ks < S.KS; ++ks)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int row = g + (i & 1) * 8, col = ks * 8 + t + (i >> 1) * 4;
          if (col < Nfp) sUP[row * Nfp + col] = an[ks][i];
        }
      double cd[4] = {}, cs[4] = {};
#pragma unroll
      for (int ks = 0; ks < S.KS; ++ks) {
        dmma(cd, an[ks], tile(S.TN + ks * S.NTN));
        dmma(cs, an[ks], tile(S.TN + ks * S.NTN + S.NTN / 2));
      }
      // the face's flux coefficients of the two rows
      double T[2][9];
#pragma unroll
      for (int rr = 0; rr < 2; ++rr)
#pragma unroll
        for (int c = 0; c < 9; ++c) T[rr][c] = __ldg(dgeo + (D_T + 9 * f + c) * ldg + kr[rr]);
      __syncwarp();  // sUP written
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int rr = i >> 1, row = g + 8 * rr, q = 2 * t + (i & 1);
        if (rv[rr] && q < Nfp) {
          const int p = ((wr[f][rr] >> 2) & 1u) ? N - q : q;
          const double uP = sUP[row * Nfp + q];
          const double uM = sU[row * Np + fmask_idx(N, f, p)];
          const double dnM = sDN[row * NF + f * Nfp + p];
          sG[row * GS + f * Nfp + p] = T[rr][5] * uM + T[rr][6] * uP;
          sG[row * GS + NF + f * Nfp + p] = T[rr][7] * uM + T[rr][8] * uP;
          sG[row * GS + 2 * NF + f * Nfp + p] =
              T[rr][0] * dnM + T[rr][1] * cd[i] + T[rr][2] * cs[i] + T[rr][3] * uM + T[rr][4] * uP;
        }
      }
      __syncwarp();  // sUP read before the next face overwrites it
    }

    // ----------------------------------------------------------- stage 3: lift
    double cl[S.NTV][4] = {};
#pragma unroll
    for (int ks = 0; ks < S.KS3; ++ks) {
      double al[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int row = g + (i & 1) * 8, col = ks * 8 + t + (i >> 1) * 4;
        al[i] = sG[row * GS + col];
      }
#pragma unroll
      for (int j = 0; j < S.NTV; ++j) dmma(cl[j], al, tile(S.T3 + ks * S.NTV + j));
    }
    __syncwarp();  // every lane's stage-3 operand is read before the output tile overwrites it

    // ------------------------------------------------------------- epilogue
    double* sY = sG;
#pragma unroll
    for (int j = 0; j < S.NTV; ++j)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int rr = i >> 1, row = g + 8 * rr, c = j * 8 + 2 * t + (i & 1);
        if (rv[rr] && c < Np) {
          double y = yv[j][i] + cl[j][i];
          const double uv = sU[row * Np + c];
          if (shift != 0.0) y += shift * uv;
          if (MODE == AM_RESID) {
            const double bv = __ldg(in1 + off + row * Np + c);
            y = bv - y;
            dA += bv * bv;
            dB += y * y;
          }
          if (MODE == AM_PFUSE) dA += uv * y;
          sY[row * Np + c] = y;
        }
      }
    if (tma) fence_proxy_async_smem();
    __syncwarp();
    if (tma) {
      if (lane == 0) {
        bulk_store(a.out0 + off, sY, bytes);
        if (MODE == AM_PFUSE) bulk_store(a.out1 + off, sU, bytes);
        bulk_commit();
      }
      pending = true;
    } else {
      for (int i = lane; i < nw * Np; i += 32) {
        a.out0[off + i] = sY[i];
        if (MODE == AM_PFUSE) a.out1[off + i] = sU[i];
      }
    }
  }
  if (lane == 0 && pending) bulk_wait_read_all();
  if (MODE == AM_APPLY) return;

  // reductions: block partials -> last block -> control block (as k_apply)
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

// ------------------------------------------------------------------ host
// B operands in fragment order: tile i holds, for lane l (g = l/4, t = l%4),
// B[8 ks + t][8 nt + g] and B[8 ks + t + 4][8 nt + g] at doubles 64 i + 2 l.
inline void put_tile(double* img, int tile, const std::vector<double>& B, int ncols, int ks, int nt) {
  for (int l = 0; l < 32; ++l) {
    const int g = l >> 2, t = l & 3, n = nt * 8 + g;
    img[tile * 64 + 2 * l] = B[(size_t)(ks * 8 + t) * ncols + n];
    img[tile * 64 + 2 * l + 1] = B[(size_t)(ks * 8 + t + 4) * ncols + n];
  }
}

}  // namespace dm

bool dm_supported(int N) { return N >= 1 && N <= 5; }
int dm_image_doubles(int N) { return dm_supported(N) ? dm::shape_of(N).IMG : 0; }

int dm_build_image(int N, const double* Dr, const double* Ds, const double* M, const double* m1d, double* out) {
  if (!dm_supported(N)) return -1;
  const dm::ShapeRT S = dm::shape_of(N);
  const int Np = S.Np, Nfp = S.Nfp, NF = S.NF;
  auto at = [Np](const double* A, int i, int j) { return A[(size_t)i * Np + j]; };
  // stiffness blocks: T_a = M^T D_a, S_ab = D_a^T T_b
  std::vector<double> Tr((size_t)Np * Np), Ts((size_t)Np * Np);
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) {
      double r = 0.0, s = 0.0;
      for (int b = 0; b < Np; ++b) {
        r += at(M, b, i) * at(Dr, b, j);
        s += at(M, b, i) * at(Ds, b, j);
      }
      Tr[(size_t)i * Np + j] = r;
      Ts[(size_t)i * Np + j] = s;
    }
  auto Sab = [&](const double* Da, const std::vector<double>& Tb, int n, int j) {
    double v = 0.0;
    for (int i = 0; i < Np; ++i) v += at(Da, i, n) * Tb[(size_t)i * Np + j];
    return v;
  };
  // stage 1: B1[j][col] (KP x NT1*8)
  const int c1 = S.NT1 * 8;
  std::vector<double> B1((size_t)S.KP * c1, 0.0);
  for (int j = 0; j < Np; ++j)
    for (int n = 0; n < Np; ++n) {
      B1[(size_t)j * c1 + 0 * S.NTV * 8 + n] = Sab(Dr, Tr, n, j);
      B1[(size_t)j * c1 + 1 * S.NTV * 8 + n] = Sab(Dr, Ts, n, j) + Sab(Ds, Tr, n, j);
      B1[(size_t)j * c1 + 2 * S.NTV * 8 + n] = Sab(Ds, Ts, n, j);
      B1[(size_t)j * c1 + 3 * S.NTV * 8 + n] = at(M, n, j);
    }
  for (int j = 0; j < Np; ++j)
    for (int f = 0; f < 3; ++f)
      for (int p = 0; p < Nfp; ++p) {
        const int c = f * Nfp + p, fn = fmask_idx(N, f, p);
        B1[(size_t)j * c1 + 4 * S.NTV * 8 + c] = at(Dr, fn, j);
        B1[(size_t)j * c1 + (4 * S.NTV + S.NTF) * 8 + c] = at(Ds, fn, j);
      }
  for (int ks = 0; ks < S.KS; ++ks)
    for (int nt = 0; nt < S.NT1; ++nt) dm::put_tile(out, ks * S.NT1 + nt, B1, c1, ks, nt);
  // stage 2: BN[j][q] = Dr[q][j] | Ds[q][j] (face-0 rows are nodes 0..N)
  const int cn = S.NTN * 8;
  std::vector<double> BN((size_t)S.KP * cn, 0.0);
  for (int j = 0; j < Np; ++j)
    for (int q = 0; q < Nfp; ++q) {
      BN[(size_t)j * cn + q] = at(Dr, q, j);
      BN[(size_t)j * cn + (S.NTN / 2) * 8 + q] = at(Ds, q, j);
    }
  for (int ks = 0; ks < S.KS; ++ks)
    for (int nt = 0; nt < S.NTN; ++nt) dm::put_tile(out, S.TN + ks * S.NTN + nt, BN, cn, ks, nt);
  // stage 3, row (f, p) of each block, m_f[p][q] = m1d[(f Nfp + p) Nfp + q]:
  //   B3[f Nfp + p][n]        = sum_q m_f[p][q] Dr[Fmask(f, q)][n]
  //   B3[NF + f Nfp + p][n]   = sum_q m_f[p][q] Ds[Fmask(f, q)][n]
  //   B3[2 NF + f Nfp + p][n] = sum_q m_f[p][q] [Fmask(f, q) == n]
  const int c3 = S.NTV * 8;
  std::vector<double> B3((size_t)S.K3 * c3, 0.0);
  for (int f = 0; f < 3; ++f)
    for (int p = 0; p < Nfp; ++p) {
      const int k = f * Nfp + p;
      for (int q = 0; q < Nfp; ++q) {
        const double mq = m1d[(size_t)(f * Nfp + p) * Nfp + q];
        const int fn = fmask_idx(N, f, q);
        for (int n = 0; n < Np; ++n) {
          B3[(size_t)k * c3 + n] += mq * at(Dr, fn, n);
          B3[(size_t)(NF + k) * c3 + n] += mq * at(Ds, fn, n);
        }
        B3[(size_t)(2 * NF + k) * c3 + fn] += mq;
      }
    }
  for (int ks = 0; ks < S.KS3; ++ks)
    for (int nt = 0; nt < S.NTV; ++nt) dm::put_tile(out, S.T3 + ks * S.NTV + nt, B3, c3, ks, nt);
  return 0;
}

namespace dm {
struct Occ {
  int blocks[6][4] = {};
};
inline Occ& occ() {
  static Occ o;
  return o;
}
template <int N, int MODE>
cudaError_t prepare_one() {
  const size_t smem = shape_of(N).smem;
  cudaError_t e = cudaFuncSetAttribute(k_apply_dm<N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int nb = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_apply_dm<N, MODE>, BLOCK, smem);
  if (e != cudaSuccess) return e;
  occ().blocks[N][MODE] = nb > 0 ? nb : 1;
  return cudaSuccess;
}
template <int N>
cudaError_t prepare_n() {
  cudaError_t e = prepare_one<N, AM_APPLY>();
  if (e == cudaSuccess) e = prepare_one<N, AM_PFUSE>();
  if (e == cudaSuccess) e = prepare_one<N, AM_RESID>();
  return e;
}
template <int N, int MODE>
cudaError_t launch_one(const ApplyArgs<double>& a, cudaStream_t s) {
  const int nb = occ().blocks[N][MODE];
  if (nb <= 0) return cudaErrorInitializationError;  // dm_prepare not called for this degree
  const bool ranged = MODE == AM_APPLY && a.k_hi > 0;
  if (ranged && (a.k_lo % RB != 0 || a.k_hi > a.K || a.k_lo < 0)) return cudaErrorInvalidValue;
  const int nrb = ranged ? (a.k_hi + RB - 1) / RB - a.k_lo / RB : (a.K + RB - 1) / RB;
  if (nrb <= 0) return cudaSuccess;
  const int grid = std::max(1, std::min((nrb + WARPS - 1) / WARPS, nb * sm_count()));
  PdlLaunch l(dim3(grid), dim3(BLOCK), shape_of(N).smem, s, a.pdl);
  return cudaLaunchKernelEx(&l.cfg, k_apply_dm<N, MODE>, a);
}
template <int N>
cudaError_t launch_n(int mode, const ApplyArgs<double>& a, cudaStream_t s) {
  switch (mode) {
    case AM_APPLY: return launch_one<N, AM_APPLY>(a, s);
    case AM_PFUSE: return launch_one<N, AM_PFUSE>(a, s);
    case AM_RESID: return launch_one<N, AM_RESID>(a, s);
  }
  return cudaErrorInvalidValue;
}
}  // namespace dm

cudaError_t dm_prepare(int N) {
  switch (N) {
    case 1: return dm::prepare_n<1>();
    case 2: return dm::prepare_n<2>();
    case 3: return dm::prepare_n<3>();
    case 4: return dm::prepare_n<4>();
    case 5: return dm::prepare_n<5>();
  }
  return cudaErrorInvalidValue;
}

bool dm_handles(int mode, const ApplyArgs<double>& a) {
  return a.dm_img != nullptr && a.dm_geo != nullptr && a.kappa == nullptr &&
         (mode == AM_APPLY || mode == AM_PFUSE || mode == AM_RESID);
}

int dm_geo_fields() { return dm::D_COUNT; }

cudaError_t dm_build_geo(const double* geo, const uint32_t* nbr, double* dg, int K, int ldg, double tau,
                         cudaStream_t s) {
  if (K <= 0) return cudaSuccess;
  dm::k_dm_geo<<<(K + 127) / 128, 128, 0, s>>>(geo, nbr, dg, K, ldg, tau);
  return cudaGetLastError();
}

cudaError_t launch_apply_dm(int N, int mode, const ApplyArgs<double>& a, cudaStream_t s) {
  switch (N) {
    case 1: return dm::launch_n<1>(mode, a, s);
    case 2: return dm::launch_n<2>(mode, a, s);
    case 3: return dm::launch_n<3>(mode, a, s);
    case 4: return dm::launch_n<4>(mode, a, s);
    case 5: return dm::launch_n<5>(mode, a, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace ddg
