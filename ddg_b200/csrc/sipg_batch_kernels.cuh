// Continuous-batching kernels: many independent SIPG solves packed into one
// element array ("mesh of meshes").  Request r owns elements
// [req[r].k0, req[r].k0 + req[r].K); its neighbour words point inside its
// own range, so requests never couple.  Every CG scalar is per request
// (segmented reductions over the element partials), so a request's iterates
// do not depend on which other requests share the launch.
// Included by sipg_kernels.cu (it needs the constant-memory matrices).
#pragma once

namespace ddg {

template <int N, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_pfuse(BatchArgs a, const double* __restrict__ pin,
                                                       double* __restrict__ pout) {
  constexpr int Np = Dim<N>::Np;
  __shared__ int s_perm[3 * Np];
  for (int i = threadIdx.x; i < 3 * Np; i += BLOCK) s_perm[i] = a.perm[i];
  __syncthreads();
  const int k = blockIdx.x * BLOCK + threadIdx.x;
  if (k >= a.hw) return;
  const int s = a.seg[k];
  if (s < 0 || !a.req[s].active) return;
  const double beta = a.req[s].beta;
  double u[Np], y[Np];
  const size_t o = (size_t)k * Np;
#pragma unroll
  for (int i = 0; i < Np; ++i) u[i] = a.z[o + i] + beta * pin[o + i];
  uint32_t w[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) w[f] = __ldg(a.nbr + (size_t)f * a.cap + k);
  const Geo<double> g = load_geo(a.geo, a.cap, k);
  NbrPfuse<double, Np> src{a.z, pin, 1.0, beta, s_perm};
  elem_apply<N, double, true>(u, y, g, w, a.geo, a.cap, a.tau, a.alpha_e[k], src);
  double d = 0.0;
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    pout[o + i] = u[i];
    a.Ap[o + i] = y[i];
    d += u[i] * y[i];
  }
  a.epA[k] = d;
}

template <int N, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_step(BatchArgs a, const double* __restrict__ p) {
  constexpr int Np = Dim<N>::Np;
  const int k = blockIdx.x * BLOCK + threadIdx.x;
  if (k >= a.hw) return;
  const int s = a.seg[k];
  if (s < 0 || !a.req[s].active) return;
  const double al = a.req[s].alpha;
  const size_t o = (size_t)k * Np;
  double rv[Np];
  double rr = 0.0, rz = 0.0;
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    a.x[o + i] = fma(al, p[o + i], a.x[o + i]);
    rv[i] = fma(-al, a.Ap[o + i], a.r[o + i]);
    a.r[o + i] = rv[i];
    rr += rv[i] * rv[i];
  }
  {
    double zv[Np];
    sym_block_apply<Np, double>(a.binv + k, (size_t)a.cap, rv, zv);
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      a.z[o + i] = zv[i];
      rz += rv[i] * zv[i];
    }
  }
  a.epA[k] = rz;
  a.epB[k] = rr;
}

// Segmented reduction, one block per request.
//   mode 0 (after the apply): pAp -> alpha (breakdown stops the request)
//   mode 1 (after the step):  gamma, r.r -> beta, iteration count, stop test
//   mode 2 (admission):       gamma0 = r.z, b.b = r.r (r = b), tolerance
template <int MODE, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_seg(BatchArgs a, int first) {
  __shared__ double s_red[64];
  BatchReq& q = a.req[first + blockIdx.x];
  if (MODE != 2 && !q.active) return;
  double sA = 0.0, sB = 0.0;
  for (int k = q.k0 + threadIdx.x; k < q.k0 + q.K; k += BLOCK) {
    sA += a.epA[k];
    if (MODE != 0) sB += a.epB[k];
  }
  block_sum2<BLOCK>(sA, sB, s_red);
  if (threadIdx.x != 0) return;
  if (MODE == 0) {
    q.pAp = sA;
    const double al = q.gamma / sA;
    if (!(sA > 0.0) || !isfinite(al)) {
      q.alpha = 0.0;
      q.status = 2;
      q.active = 0;
    } else {
      q.alpha = al;
    }
  } else if (MODE == 1) {
    q.gamma_prev = q.gamma;
    q.beta = sA / q.gamma;
    q.gamma = sA;
    q.rr = sB;
    q.iter += 1;
    if (!isfinite(sA) || !isfinite(sB) || !isfinite(q.beta)) {
      q.status = 2;
      q.active = 0;
    } else if (!(sB > q.atol2)) {
      q.status = 0;
      q.active = 0;
    } else if (q.iter >= q.maxiter) {
      q.status = 1;
      q.active = 0;
    }
  } else {
    q.gamma = sA;
    q.rr = sB;
    q.bb = sB;
    q.atol2 = fmax(q.tol2 * sB, q.atol_sq);
    q.beta = 0.0;
    q.iter = 0;
    q.status = 0;
    q.active = (sB > q.atol2 && q.maxiter > 0) ? 1 : 0;
  }
}

// Admission of one request: r = b, x = 0, p = 0, z = B^-1 r, partials.
template <int N, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_init(BatchArgs a, double* __restrict__ p0, int k0, int K) {
  constexpr int Np = Dim<N>::Np;
  const int kl = blockIdx.x * BLOCK + threadIdx.x;
  if (kl >= K) return;
  const int k = k0 + kl;
  const size_t o = (size_t)k * Np;
  double rv[Np];
  double rr = 0.0, rz = 0.0;
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    rv[i] = a.b[o + i];
    a.r[o + i] = rv[i];
    a.x[o + i] = 0.0;
    p0[o + i] = 0.0;
    rr += rv[i] * rv[i];
  }
  {
    double zv[Np];
    sym_block_apply<Np, double>(a.binv + k, (size_t)a.cap, rv, zv);
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      a.z[o + i] = zv[i];
      rz += rv[i] * zv[i];
    }
  }
  a.epA[k] = rz;
  a.epB[k] = rr;
}

// b = J (M_ref f) for one request's elements (homogeneous Dirichlet data).
template <int N, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_rhs(BatchArgs a, const double* __restrict__ f, int k0, int K) {
  constexpr int Np = Dim<N>::Np;
  const int kl = blockIdx.x * BLOCK + threadIdx.x;
  if (kl >= K) return;
  const int k = k0 + kl;
  const RefMats<N, double>& R = CRef<N, double>::get();
  const double J = a.geo[G_J * (size_t)a.cap + k];
  double fv[Np];
#pragma unroll
  for (int j = 0; j < Np; ++j) fv[j] = f[(size_t)kl * Np + j];
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < Np; ++j) s = fma(R.M[i * Np + j], fv[j], s);
    a.b[(size_t)k * Np + i] = J * s;
  }
}

// ---------------------------------------------------------------- launchers
template <int N>
static cudaError_t batch_pfuse_n(const BatchArgs& a, const double* pin, double* pout, cudaStream_t s) {
  constexpr int B = 128;
  k_batch_pfuse<N, B><<<(a.hw + B - 1) / B, B, 0, s>>>(a, pin, pout);
  return cudaGetLastError();
}
template <int N>
static cudaError_t batch_step_n(const BatchArgs& a, const double* p, cudaStream_t s) {
  constexpr int B = 128;
  k_batch_step<N, B><<<(a.hw + B - 1) / B, B, 0, s>>>(a, p);
  return cudaGetLastError();
}
template <int N>
static cudaError_t batch_init_n(const BatchArgs& a, double* p0, int k0, int K, cudaStream_t s) {
  constexpr int B = 128;
  k_batch_init<N, B><<<(K + B - 1) / B, B, 0, s>>>(a, p0, k0, K);
  return cudaGetLastError();
}
template <int N>
static cudaError_t batch_rhs_n(const BatchArgs& a, const double* f, int k0, int K, cudaStream_t s) {
  constexpr int B = 128;
  k_batch_rhs<N, B><<<(K + B - 1) / B, B, 0, s>>>(a, f, k0, K);
  return cudaGetLastError();
}

#define DDG_BATCH_DISPATCH(CALL)          \
  switch (N) {                            \
    case 1: return CALL(1);               \
    case 2: return CALL(2);               \
    case 3: return CALL(3);               \
    case 4: return CALL(4);               \
    case 5: return CALL(5);               \
  }                                       \
  return cudaErrorInvalidValue;

cudaError_t launch_batch_pfuse(int N, const BatchArgs& a, const double* pin, double* pout, cudaStream_t s) {
#define C_(NN) batch_pfuse_n<NN>(a, pin, pout, s)
  DDG_BATCH_DISPATCH(C_)
#undef C_
}
cudaError_t launch_batch_step(int N, const BatchArgs& a, const double* p, cudaStream_t s) {
#define C_(NN) batch_step_n<NN>(a, p, s)
  DDG_BATCH_DISPATCH(C_)
#undef C_
}
cudaError_t launch_batch_init(int N, const BatchArgs& a, double* p0, int k0, int K, cudaStream_t s) {
#define C_(NN) batch_init_n<NN>(a, p0, k0, K, s)
  DDG_BATCH_DISPATCH(C_)
#undef C_
}
cudaError_t launch_batch_rhs(int N, const BatchArgs& a, const double* f, int k0, int K, cudaStream_t s) {
#define C_(NN) batch_rhs_n<NN>(a, f, k0, K, s)
  DDG_BATCH_DISPATCH(C_)
#undef C_
}
cudaError_t launch_batch_seg(int mode, const BatchArgs& a, int first_req, int nreq, cudaStream_t s) {
  if (nreq <= 0) return cudaSuccess;
  switch (mode) {
    case 0: k_batch_seg<0, 256><<<nreq, 256, 0, s>>>(a, first_req); break;
    case 1: k_batch_seg<1, 256><<<nreq, 256, 0, s>>>(a, first_req); break;
    case 2: k_batch_seg<2, 256><<<nreq, 256, 0, s>>>(a, first_req); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace ddg
