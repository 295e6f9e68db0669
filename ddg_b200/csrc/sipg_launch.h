// Kernel argument blocks and host launchers (shared by the kernels and the
// C-ABI implementation).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ddg {

struct CgCtl;

enum ApplyMode { AM_APPLY = 0, AM_PFUSE = 1, AM_RESID = 2 };

template <typename T>
struct ApplyArgs {
  const T* in0;             // APPLY: u | PFUSE: z | RESID: x
  const T* in1;             // PFUSE: p_old | RESID: b
  T* out0;                  // y (A u, A p, or b - A x)
  T* out1;                  // PFUSE: p_new
  const T* geo;             // SoA geometry [14][ldg]
  const uint32_t* nbr;      // [3][K] neighbour words
  const int* perm;          // [3][Np] rotation permutations
  CgCtl* ctl;               // PFUSE / RESID
  double* partA;            // per-block partials
  double* partB;
  unsigned int* ctl_status; // device status word
  int K, ldg;
  double tau;               // tau_scale (N+1)^2
  double alpha;             // mass coefficient
  double shift;             // + shift * u
  int use_tma;              // all vector pointers 16-byte aligned
};

template <typename T>
struct CgArgs {
  T* x;
  const T* p;      // current direction (written by the PFUSE apply)
  T* r;
  const T* Ap;
  T* z;            // == r when no preconditioner
  T* p_zero;       // INIT: buffer zeroed (first p_old)
  const T* binv;   // SoA [Np*Np][ldb]
  int ldb;
  CgCtl* ctl;
  double* partA;
  double* partB;
  const unsigned int* dev_status;  // non-zero: a kernel reported an error
  int K;
  int has_cond;
  cudaGraphConditionalHandle cond;
};

struct BlockArgs {
  const double* geo;
  const uint32_t* nbr;
  double* blocks;     // (K, Np, Np)
  double* binv64;     // SoA
  float* binv32;
  unsigned int* status;
  int K, ldg, ldb;
  double tau, alpha, shift;
};

struct RhsArgs {
  const double* geo;
  const uint32_t* nbr;
  const double* f;
  const double* u_dir;
  const double* q_neu;
  double* rhs;
  int K, ldg;
  double tau;
};

cudaError_t upload_ref(int N, const double* Dr, const double* Ds, const double* M, const double* m1d);
template <typename T>
cudaError_t launch_apply(int N, int mode, const ApplyArgs<T>& a, cudaStream_t s);
template <typename T>
cudaError_t launch_cg_step(int N, bool pc, bool init, const CgArgs<T>& a, cudaStream_t s);
cudaError_t launch_block_jacobi(int N, const BlockArgs& a, cudaStream_t s);
template <typename T>
cudaError_t launch_pc_apply(int N, const T* r, T* z, const T* binv, int ldb, int K, cudaStream_t s);
cudaError_t launch_rhs(int N, const RhsArgs& a, cudaStream_t s);
cudaError_t launch_axpby(int64_t n, double al, const double* x, double be, double* y, cudaStream_t s);
cudaError_t launch_cast(int64_t n, int to_prec, const void* src, void* dst, cudaStream_t s);
cudaError_t launch_dot(int64_t n, int prec, const void* x, const void* y, double* part, unsigned int* ticket,
                       double* out, cudaStream_t s);
int apply_grid(int K);
int cg_grid(int K);
int dot_grid(int64_t n);

}  // namespace ddg
