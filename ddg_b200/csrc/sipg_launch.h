// Kernel argument blocks and host launchers (shared by the kernels and the
// C-ABI implementation).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ddg {

struct CgCtl;

// AM_PDOT (tensor-core float32 apply only): y = A p for an already formed
// direction p, with the p.Ap reduction and alpha of AM_PFUSE.
enum ApplyMode { AM_APPLY = 0, AM_PFUSE = 1, AM_RESID = 2, AM_SMOOTH = 3, AM_PDOT = 4 };

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
  const T* binv;            // SMOOTH: packed block-Jacobi inverses (SoA)
  int ldb;
  double omega;             // SMOOTH: damping
  const T* kappa;           // per-element diffusivity (null: 1)
  const double* dm_img;     // float64: FP64 tensor-core operand image (null: CUDA cores)
  const double* dm_geo;     // float64: that kernel's element and face coefficients ([D_COUNT][ldg])
  int k_lo, k_hi;           // AM_APPLY: elements [k_lo, k_hi) only (k_hi = 0: all; k_lo a multiple of 16)
  int pdl;                  // launch with programmatic stream serialization (CG graph bodies)
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
  double* partC;   // INIT with keep_p: r.p_old partials
  const unsigned int* dev_status;  // non-zero: a kernel reported an error
  int keep_p;      // INIT: continue with the existing direction (reliable update)
  int K;
  int has_cond;
  cudaGraphConditionalHandle cond;
  int bulk;        // x, p, r, Ap, z 16-byte aligned: stage tiles by bulk copies
  int pdl;         // launch with programmatic stream serialization (CG graph bodies)
};

struct BlockArgs {
  const double* geo;
  const uint32_t* nbr;
  double* blocks;     // (K, Np, Np) for elements k0 .. k0+K-1
  double* binv64;     // SoA, indexed by the global element id
  float* binv32;      // (may be null)
  unsigned int* status;
  int K, ldg, ldb;
  double tau, alpha, shift;
  int k0;             // first element
  int nbr_ld;         // element stride of the neighbour words (0: K)
  const double* alpha_e;  // per-element alpha (overrides alpha when set)
  const double* kappa;    // per-element diffusivity (null: 1)
};

struct GradArgs {
  const double* geo;
  const uint32_t* nbr;
  const int* perm;
  const double* u;
  const double* lam;
  const double* kappa;    // unused by the contraction (a is linear in kappa)
  double* g;              // out: d a(u, lam) / d kappa_k
  int K, ldg;
  double tau;
};

// Continuous-batching pool: per-request CG state on the device.
struct BatchReq {
  int k0, K, active, iter, maxiter, status, pad0, pad1;
  double gamma, gamma_prev, pAp, alpha, beta, rr, bb, tol2, atol_sq, atol2;
};

struct BatchArgs {
  int cap, hw;             // element capacity (SoA stride) and launch range
  const double* geo;       // SoA [14][cap]
  const uint32_t* nbr;     // [3][cap]
  const int* seg;          // [cap] request slot of each element, -1 when free
  const double* alpha_e;   // [cap] Helmholtz coefficient of each element
  const double* binv;      // packed block-Jacobi inverses, SoA [Np(Np+1)/2][cap]
  double *x, *b, *r, *z, *Ap;
  double *epA, *epB;       // per-element partial sums
  BatchReq* req;
  const int* perm;
  double tau;
  int max_req;
  int threads;             // element-kernel tile: threads per block (64, 128 or 256)
  int persistent;          // 1: a persistent grid of a few blocks per SM
  int prec;                // iteration vectors: 0 float64 (x, r, z, Ap above), 1 float32 (below)
  const float* geo32;      // float32 copies of geo and binv (float32 pools)
  const float* binv32;
  float *x32, *r32, *z32, *Ap32;
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

// Curved-element operator (per-node geometric factors, nodal or cubature
// quadrature): every per-element field is [field][row][K].
struct CvArgs {
  int K;               // elements (the SoA stride of every field)
  int Ncub;            // volume cubature points (cubature quadrature)
  const double* gN;    // [5][Np][K] rx sx ry sy J at the nodes
  const double* fN;    // [2][3Nfp][K] nx ny at the face nodes
  const double* sJ0;   // [3][K] sJ at each face's first node
  const double* tauF;  // [3][K] tau_scale (N+1)^2 Fscale at each face's first node
  const int* tag;      // [3][K] BC tag of (k, f)
  const int* slotP;    // [3Nfp][K] vmapP: element-major index of the outside trace node
  const int* mapP;     // [3Nfp][K] the matching face slot of the neighbour, m' K + k'
  const double* cG;    // [4][Ncub][ldc] wJ(rx^2+ry^2), wJ(rx sx+ry sy), wJ(sx^2+sy^2), wJ
  int ldc;             // row stride of cG: K rounded up to a multiple of 128 (zero padded)
  const double* cQ;    // [3][Nfp(Nfp+1)/2][K] packed face rule L1d^T diag(face_w sJ) L1d
  const double* cMat;  // [3][Ncub][Np] Drq, Dsq, Lq
  double* tr;          // [2][3Nfp][K] gradient traces (pass 1)
  double* dl;          // [3][3Nfp][K] face duals (pass 2)
  CgCtl* ctl;          // CG control block (PDOT, RESID; gating inside CG graphs)
  double* partA;       // per-block partials
  double* partB;
  int gate;            // skip the launch once ctl->cont == 0 (CG graph bodies)
};
// dynamic shared memory ceiling of the curved kernels (bytes)
#define CV_SMEM_LIMIT (200 * 1024)
// pass 1 (traces of u), 2 (face duals, udir = Dirichlet data or null),
// 3 (gather: mode 0 y = A u + alpha M u + shift u, 1 y -= that, 2 with the
// p.Ap reduction, 3 y = b - that with b.b and r.r); quad 1 = cubature
cudaError_t launch_cv_pass(int N, int pass, int quad, int mode, const CvArgs& a, const double* u, const double* udir,
                           const double* b, double* y, double alpha, double shift, cudaStream_t s);
cudaError_t cv_prepare(int N);
// dynamic shared memory of the cubature gather pass for degree N, Ncub points
size_t cv_gather_smem_bytes(int N, int Ncub);
// the curved kernels' copy of the reference-element matrices
cudaError_t cv_upload_ref(int N, const double* Dr, const double* Ds, const double* M, const double* m1d);
cudaError_t launch_cv_mass(int N, int quad, const CvArgs& a, const double* f, double* y, cudaStream_t s);
cudaError_t launch_cv_neumann(int N, const CvArgs& a, const double* q, double* y, cudaStream_t s);
cudaError_t launch_cv_probe(int K, int Np, const int* colour, int c, int j, double* P, cudaStream_t s);
cudaError_t launch_cv_collect(int K, int Np, const int* colour, int c, int j, double shift, const double* Y,
                              double* blocks, cudaStream_t s);
cudaError_t launch_cv_invert(int N, int K, const double* blocks, double* binv, unsigned int* status, cudaStream_t s);
cudaError_t launch_cv_pc(int N, int K, const double* binv, const double* r, double* z, const CgCtl* ctl,
                         cudaStream_t s);
cudaError_t launch_cv_pupd(int64_t n, const double* z, double* p, const CgCtl* ctl, cudaStream_t s);

cudaError_t upload_ref(int N, const double* Dr, const double* Ds, const double* M, const double* m1d);
template <typename T>
cudaError_t launch_apply(int N, int mode, const ApplyArgs<T>& a, cudaStream_t s);
// float32 apply on the tensor cores (tcgen05, 3xTF32); `img` is the device
// copy of the degree's B-operand image (tc_build_image)
bool tc_supported(int N);
int tc_image_bytes(int N);
int tc_build_image(int N, const double* Dr, const double* Ds, const double* M, uint8_t* out);
// modes AM_APPLY and AM_PFUSE; tc_prepare sets the kernels' attributes
cudaError_t tc_prepare(int N);
cudaError_t launch_apply_tc(int N, int mode, const ApplyArgs<float>& a, const uint8_t* img, cudaStream_t s);
// float64 apply on the FP64 tensor cores (mma.sync f64, degrees 1..5):
// modes AM_APPLY, AM_PFUSE, AM_RESID without kappa; launch_apply<double>
// dispatches to it whenever ApplyArgs::dm_img is set.  dm_prepare sets the
// kernels' shared-memory attribute and occupancy (once per degree).
bool dm_supported(int N);
int dm_image_doubles(int N);
int dm_build_image(int N, const double* Dr, const double* Ds, const double* M, const double* m1d, double* out);
cudaError_t dm_prepare(int N);
bool dm_handles(int mode, const ApplyArgs<double>& a);
int dm_geo_fields();
// element and face coefficients of the FP64 tensor-core kernel from the
// geometry and the neighbour words (again after every boundary-tag change)
cudaError_t dm_build_geo(const double* geo, const uint32_t* nbr, double* dg, int K, int ldg, double tau,
                         cudaStream_t s);
cudaError_t launch_apply_dm(int N, int mode, const ApplyArgs<double>& a, cudaStream_t s);
// node-major (Np, K) fields, elements [k_begin, k_end) only (in0 -> out0)
template <typename T>
cudaError_t launch_apply_nm(int N, const ApplyArgs<T>& a, int k_begin, int k_end, cudaStream_t s);
// node-major (rows, ld) <-> element-major (ld, rows) float64 for elements
// [k0, k1), through shared-memory tiles
cudaError_t launch_nm_to_em(const double* nm, double* em, int ld, int rows, int k0, int k1, cudaStream_t s);
cudaError_t launch_em_to_nm(const double* em, double* nm, int ld, int rows, int k0, int k1, cudaStream_t s);
template <typename T>
cudaError_t launch_cg_step(int N, bool pc, bool init, const CgArgs<T>& a, cudaStream_t s);
cudaError_t launch_block_jacobi(int N, const BlockArgs& a, cudaStream_t s);
template <typename T>
cudaError_t launch_pc_apply(int N, const T* r, T* z, const T* binv, int ldb, int K, cudaStream_t s);
cudaError_t launch_rhs(int N, const RhsArgs& a, cudaStream_t s);
cudaError_t launch_grad_kappa(int N, const GradArgs& a, cudaStream_t s);
cudaError_t launch_axpby(int64_t n, double al, const double* x, double be, double* y, cudaStream_t s);
cudaError_t launch_cast(int64_t n, int to_prec, const void* src, void* dst, cudaStream_t s);
// float32 CG direction p = zc z + beta p_old (16-byte aligned vectors)
cudaError_t launch_pupd(int64_t n, const float* z, const float* p_old, float* p, const CgCtl* ctl, cudaStream_t s,
                        int pdl = 0);
// launch configuration with programmatic stream serialization when pdl != 0
struct PdlLaunch {
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute attr[1];
  PdlLaunch(dim3 grid, dim3 block, size_t smem, cudaStream_t s, int pdl) {
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
  }
};
// r32 = float(r64), x32 = 0, ctl->bb = r32.r32 (reliable-update restart)
cudaError_t launch_cast_norm(int64_t n, const double* r64, float* r32, float* x32, double* part, CgCtl* ctl,
                             cudaStream_t s);
// x64 += double(x32)
cudaError_t launch_axpy_mixed(int64_t n, const float* x32, double* x64, cudaStream_t s);
cudaError_t launch_dot(int64_t n, int prec, const void* x, const void* y, double* part, unsigned int* ticket,
                       double* out, cudaStream_t s);
template <typename T>
cudaError_t launch_elem_matvec(int Kout, int rows, int cols, const T* M, const T* in, T* out, int add,
                               cudaStream_t s);
template <typename T>
cudaError_t launch_dense_gemv(int n, const T* A, const T* b, T* x, cudaStream_t s);
template <typename T>
cudaError_t launch_bj_scaled(int N, const T* b, T* x, const T* binv, int ldb, int K, T scale, cudaStream_t s);
template <typename T>
cudaError_t launch_cg_xr(T* x, const T* p, T* r, const T* Ap, int64_t n, CgCtl* ctl, double* part, cudaStream_t s);
template <typename T>
cudaError_t launch_cg_finish(bool init, const T* r, const T* z, int64_t n, CgCtl* ctl, double* part,
                             const unsigned int* dev_status, int has_cond, cudaGraphConditionalHandle cond,
                             cudaStream_t s);
int xr_grid(int64_t n);
// pin / pout / p / p0: float64 or float32 vectors as a.prec says
cudaError_t launch_batch_pfuse(int N, const BatchArgs& a, const void* pin, void* pout, cudaStream_t s);
cudaError_t launch_batch_step(int N, const BatchArgs& a, const void* p, cudaStream_t s);
cudaError_t launch_batch_seg(int mode, const BatchArgs& a, int first_req, int nreq, cudaStream_t s);
cudaError_t launch_batch_init(int N, const BatchArgs& a, void* p0, int k0, int K, cudaStream_t s);
// float32 copy of `rows` SoA rows of elements [k0, k0 + K) (row stride ld)
cudaError_t launch_rows_to_f32(const double* src, float* dst, int rows, int ld, int k0, int K, cudaStream_t s);
cudaError_t launch_batch_rhs(int N, const BatchArgs& a, const double* f, int k0, int K, cudaStream_t s);
// host: neighbour words of a mesh, element ids shifted by k_offset
int pack_neighbours(int K, int N, const int64_t* EToE, const int64_t* EToF, const int64_t* vmapP,
                    const int64_t* rot, const int32_t* bc, uint32_t k_offset, uint32_t* out, size_t out_ld);
int apply_grid(int K);
int cg_grid(int K);
int dot_grid(int64_t n);

}  // namespace ddg
