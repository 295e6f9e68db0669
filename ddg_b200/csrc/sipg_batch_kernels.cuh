// Continuous-batching kernels: many independent SIPG solves packed into one
// element array ("mesh of meshes").  Request r owns elements
// [req[r].k0, req[r].k0 + req[r].K); its neighbour words point inside its
// own range, so requests never couple.  Every CG scalar is per request
// (segmented reductions over the element partials), so a request's iterates
// do not depend on which other requests share the launch.
// Included by sipg_kernels.cu (it needs the constant-memory matrices).
#pragma once

namespace ddg {

// The element kernels loop over the elements with a grid stride, so the
// same code runs with one thread per element (grid = ceil(hw / BLOCK)) or as
// a persistent grid of a few blocks per SM; the tile shape (BLOCK, grid
// mode) is chosen per pool by the serving autotuner and never changes the
// arithmetic of an element.
// Vectors, geometry and inverses of the element kernels: float64, or the
// float32 copies of a float32 pool (CG scalars and partial sums stay float64).
template <typename T>
struct BatchVec {
  const T *geo, *binv;
  T *x, *r, *z, *Ap;
  __device__ __forceinline__ explicit BatchVec(const BatchArgs& a) {
    if constexpr (sizeof(T) == 8) {
      geo = a.geo; binv = a.binv; x = a.x; r = a.r; z = a.z; Ap = a.Ap;
    } else {
      geo = a.geo32; binv = a.binv32; x = a.x32; r = a.r32; z = a.z32; Ap = a.Ap32;
    }
  }
};

template <int N, typename T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_pfuse(BatchArgs a, const T* __restrict__ pin,
                                                       T* __restrict__ pout) {
  constexpr int Np = Dim<N>::Np;
  __shared__ int s_perm[3 * Np];
  for (int i = threadIdx.x; i < 3 * Np; i += BLOCK) s_perm[i] = a.perm[i];
  __syncthreads();
  const BatchVec<T> v(a);
  for (int k = blockIdx.x * BLOCK + threadIdx.x; k < a.hw; k += gridDim.x * BLOCK) {
  const int s = a.seg[k];
  if (s < 0 || !a.req[s].active) continue;
  const T beta = (T)a.req[s].beta;
  T u[Np], y[Np];
  const size_t o = (size_t)k * Np;
#pragma unroll
  for (int i = 0; i < Np; ++i) u[i] = v.z[o + i] + beta * pin[o + i];
  uint32_t w[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) w[f] = __ldg(a.nbr + (size_t)f * a.cap + k);
  const Geo<T> g = load_geo(v.geo, a.cap, k);
  NbrPfuse<T, Np> src{v.z, pin, T(1), beta, s_perm};
  elem_apply<N, T, true>(u, y, g, w, v.geo, a.cap, (T)a.tau, (T)a.alpha_e[k], src);
  double d = 0.0;
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    pout[o + i] = u[i];
    v.Ap[o + i] = y[i];
    d += (double)u[i] * (double)y[i];
  }
  a.epA[k] = d;
  }
}

template <int N, typename T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_step(BatchArgs a, const T* __restrict__ p) {
  constexpr int Np = Dim<N>::Np;
  const BatchVec<T> v(a);
  for (int k = blockIdx.x * BLOCK + threadIdx.x; k < a.hw; k += gridDim.x * BLOCK) {
  const int s = a.seg[k];
  if (s < 0 || !a.req[s].active) continue;
  const T al = (T)a.req[s].alpha;
  const size_t o = (size_t)k * Np;
  T rv[Np];
  double rr = 0.0, rz = 0.0;
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    v.x[o + i] = fma(al, p[o + i], v.x[o + i]);
    rv[i] = fma(-al, v.Ap[o + i], v.r[o + i]);
    v.r[o + i] = rv[i];
    rr += (double)rv[i] * (double)rv[i];
  }
  {
    T zv[Np];
    sym_block_apply<Np, T>(v.binv + k, (size_t)a.cap, rv, zv);
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      v.z[o + i] = zv[i];
      rz += (double)rv[i] * (double)zv[i];
    }
  }
  a.epA[k] = rz;
  a.epB[k] = rr;
  }
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
template <int N, typename T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_init(BatchArgs a, T* __restrict__ p0, int k0, int K) {
  constexpr int Np = Dim<N>::Np;
  const int kl = blockIdx.x * BLOCK + threadIdx.x;
  if (kl >= K) return;
  const BatchVec<T> v(a);
  const int k = k0 + kl;
  const size_t o = (size_t)k * Np;
  T rv[Np];
  double rr = 0.0, rz = 0.0;
#pragma unroll
  for (int i = 0; i < Np; ++i) {
    rv[i] = (T)a.b[o + i];
    v.r[o + i] = rv[i];
    v.x[o + i] = T(0);
    p0[o + i] = T(0);
    rr += (double)rv[i] * (double)rv[i];
  }
  {
    T zv[Np];
    sym_block_apply<Np, T>(v.binv + k, (size_t)a.cap, rv, zv);
#pragma unroll
    for (int i = 0; i < Np; ++i) {
      v.z[o + i] = zv[i];
      rz += (double)rv[i] * (double)zv[i];
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
// grid of an element kernel: one thread per element, or (persistent) at
// most `per_sm` blocks per SM looping over the elements
static int batch_grid(int hw, int B, int persistent) {
  const int full = (hw + B - 1) / B;
  if (!persistent) return full < 1 ? 1 : full;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int cap = nsm * (2048 / B);
  return full < cap ? (full < 1 ? 1 : full) : cap;
}
template <int N, typename T, int B>
static cudaError_t batch_pfuse_b(const BatchArgs& a, const void* pin, void* pout, cudaStream_t s) {
  k_batch_pfuse<N, T, B><<<batch_grid(a.hw, B, a.persistent), B, 0, s>>>(a, (const T*)pin, (T*)pout);
  return cudaGetLastError();
}
template <int N, typename T, int B>
static cudaError_t batch_step_b(const BatchArgs& a, const void* p, cudaStream_t s) {
  k_batch_step<N, T, B><<<batch_grid(a.hw, B, a.persistent), B, 0, s>>>(a, (const T*)p);
  return cudaGetLastError();
}
template <int N, typename T>
static cudaError_t batch_pfuse_t(const BatchArgs& a, const void* pin, void* pout, cudaStream_t s) {
  if (a.threads == 64) return batch_pfuse_b<N, T, 64>(a, pin, pout, s);
  if (a.threads == 256) return batch_pfuse_b<N, T, 256>(a, pin, pout, s);
  return batch_pfuse_b<N, T, 128>(a, pin, pout, s);
}
template <int N, typename T>
static cudaError_t batch_step_t(const BatchArgs& a, const void* p, cudaStream_t s) {
  if (a.threads == 64) return batch_step_b<N, T, 64>(a, p, s);
  if (a.threads == 256) return batch_step_b<N, T, 256>(a, p, s);
  return batch_step_b<N, T, 128>(a, p, s);
}
template <int N>
static cudaError_t batch_pfuse_n(const BatchArgs& a, const void* pin, void* pout, cudaStream_t s) {
  return a.prec ? batch_pfuse_t<N, float>(a, pin, pout, s) : batch_pfuse_t<N, double>(a, pin, pout, s);
}
template <int N>
static cudaError_t batch_step_n(const BatchArgs& a, const void* p, cudaStream_t s) {
  return a.prec ? batch_step_t<N, float>(a, p, s) : batch_step_t<N, double>(a, p, s);
}
template <int N>
static cudaError_t batch_init_n(const BatchArgs& a, void* p0, int k0, int K, cudaStream_t s) {
  constexpr int B = 128;
  if (a.prec)
    k_batch_init<N, float, B><<<(K + B - 1) / B, B, 0, s>>>(a, (float*)p0, k0, K);
  else
    k_batch_init<N, double, B><<<(K + B - 1) / B, B, 0, s>>>(a, (double*)p0, k0, K);
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

cudaError_t launch_batch_pfuse(int N, const BatchArgs& a, const void* pin, void* pout, cudaStream_t s) {
#define C_(NN) batch_pfuse_n<NN>(a, pin, pout, s)
  DDG_BATCH_DISPATCH(C_)
#undef C_
}
cudaError_t launch_batch_step(int N, const BatchArgs& a, const void* p, cudaStream_t s) {
#define C_(NN) batch_step_n<NN>(a, p, s)
  DDG_BATCH_DISPATCH(C_)
#undef C_
}
cudaError_t launch_batch_init(int N, const BatchArgs& a, void* p0, int k0, int K, cudaStream_t s) {
#define C_(NN) batch_init_n<NN>(a, p0, k0, K, s)
  DDG_BATCH_DISPATCH(C_)
#undef C_
}
cudaError_t launch_batch_rhs(int N, const BatchArgs& a, const double* f, int k0, int K, cudaStream_t s) {
#define C_(NN) batch_rhs_n<NN>(a, f, k0, K, s)
  DDG_BATCH_DISPATCH(C_)
#undef C_
}
__global__ void k_rows_to_f32(const double* __restrict__ src, float* __restrict__ dst, int rows, int ld, int k0,
                              int K) {
  const int64_t n = (int64_t)rows * K;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const size_t o = (size_t)(i / K) * ld + k0 + (i % K);
    dst[o] = (float)src[o];
  }
}
cudaError_t launch_rows_to_f32(const double* src, float* dst, int rows, int ld, int k0, int K, cudaStream_t s) {
  const int64_t n = (int64_t)rows * K;
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  k_rows_to_f32<<<grid < 1 ? 1 : grid, 256, 0, s>>>(src, dst, rows, ld, k0, K);
  return cudaGetLastError();
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
