/*
 * ddg_sipg.h -- C ABI of the B200 (sm_100a) matrix-free SIPG
 * Poisson/Helmholtz solver.
 *
 * Plain C: pointers, sizes and int status codes.  No C++ or torch types
 * cross this boundary and no exception escapes it.  Every entry point
 * returns DDG_OK (0) on success; ddg_last_error() gives the message of the
 * last failure on the calling thread.
 *
 * Layouts follow ddg (reference project CorbinFoucart/ddg):
 *   volume vectors  element-major flat, index k*Np + n (u.T.reshape(-1) of
 *                   an (Np, K) field)        -- src/ddg/dg2d/sipg.py:204
 *   face vectors    index k*3*Nfp + f*Nfp + p (order='F' of (3 Nfp, K))
 *                                            -- src/ddg/dg2d/sipg.py:442
 *   bc_types        (K, 3) int32, 0 interior / 1 Dirichlet / 2 Neumann
 *                                            -- src/ddg/dg2d/sipg.py:53-56
 * Device vectors are caller-owned device memory on the handle's device.
 * One handle is used by one stream at a time.
 */
#ifndef DDG_SIPG_H
#define DDG_SIPG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define DDG_OK               0
#define DDG_ERR_INVALID      1   /* bad argument / inconsistent mesh        */
#define DDG_ERR_CUDA         2   /* a CUDA runtime call failed              */
#define DDG_ERR_UNSUPPORTED  3   /* degree or option not built              */
#define DDG_ERR_NOMEM        4   /* device allocation failed / over budget  */
#define DDG_ERR_DEVICE       5   /* a kernel reported an error (timeout,    */
                                 /* bad index) through its status word      */

/* ---- BC codes (src/ddg/dg2d/sipg.py:53-56) ---------------------------- */
#define DDG_BC_INTERIOR  0
#define DDG_BC_DIRICHLET 1
#define DDG_BC_NEUMANN   2

/* ---- precisions of the operator apply -------------------------------- */
#define DDG_FP64 0
#define DDG_FP32 1

/* ---- solver status (jax's cg discards its info; we return one) -------- */
#define DDG_SOLVE_CONVERGED  0
#define DDG_SOLVE_MAXITER    1
#define DDG_SOLVE_BREAKDOWN  2   /* p.Ap <= 0 or non-finite scalar */
#define DDG_SOLVE_DEVICE_ERR 3   /* a kernel reported an error; loop stopped */

/* Highest polynomial degree with built kernels. */
#define DDG_MAX_DEGREE 5

typedef struct ddg_sipg_op ddg_sipg_op;      /* opaque, library-owned */

/*
 * Mesh + operator description for ddg_sipg_create.  All pointers are HOST
 * memory and are only read during the call.
 *
 * Replaces the Mesh2D fields the reference's sipg_bilinear_form reads
 * (src/ddg/dg2d/mesh.py:50-101, src/ddg/dg2d/sipg.py:168-263): the
 * reference-element matrices, per-element affine geometry, connectivity,
 * node maps and BC tags.  Geometry is per element (straight-sided
 * triangles: rx..J are constant per element), taken at each element's first
 * node / each face's first node exactly as sipg.py:261-263 takes sJ, Fscale.
 */
typedef struct {
    int32_t N;             /* polynomial degree, 1..DDG_MAX_DEGREE          */
    int32_t K;             /* number of elements                            */
    int32_t device;        /* CUDA device ordinal                           */
    int32_t reserved;
    double  tau_scale;     /* penalty tau = tau_scale (N+1)^2 sJ/J          */
    const double *Dr, *Ds; /* (Np, Np) row-major                            */
    const double *M;       /* (Np, Np) reference mass inv(V V^T)            */
    const double *m1d;     /* (3, Nfp, Nfp) face masses (sipg.py:98-110)    */
    const int64_t *Fmask;  /* (Nfp, 3)                                      */
    const int64_t *rot_perm; /* (3, Np): node of the element re-labelled so
                                that its face f is face 0                    */
    const double *geo;     /* (K, 14): rx sx ry sy J, then for f=0..2:
                              nx_f ny_f sJ_f                                */
    const int64_t *EToE, *EToF;   /* (K, 3)                                 */
    const int64_t *vmapM, *vmapP; /* (3 Nfp K)                              */
    const int32_t *bc_types;      /* (K, 3)                                 */
} ddg_sipg_mesh_desc;

/* Build the device-resident operator.  Replaces the per-call setup of
 * src/ddg/dg2d/sipg.py:849-850 (_local_mass / _face_1d_mass_matrices) and
 * the mesh fields above.  Allocates device memory owned by the handle. */
int ddg_sipg_create(const ddg_sipg_mesh_desc *desc, ddg_sipg_op **out);
int ddg_sipg_destroy(ddg_sipg_op *op);

/* Change the BC tags of an existing handle (same mesh). */
int ddg_sipg_set_bc(ddg_sipg_op *op, const int32_t *bc_types);

/* y = A u + alpha * J (M_ref u).
 * Replaces sipg_apply_2d(mesh, u, bc_types=..., u_dir=None) of
 * src/ddg/dg2d/sipg.py:304-337 (alpha = 0) and the Helmholtz matvec
 * src/ddg/dg2d/sipg.py:589-601 / multigrid.py:53-74 (alpha > 0).
 * u, y: device, K*Np elements of double (DDG_FP64) or float (DDG_FP32). */
int ddg_sipg_apply(ddg_sipg_op *op, int precision, double alpha,
                   const void *u, void *y, void *stream);

/* Engine of the operator applies.  DDG_ENGINE_TENSOR_CORES: float32
 * element contractions run on the tcgen05 tensor cores with 3xTF32
 * splitting (float32-level accuracy, degrees 1..4), float64 ones on the
 * FP64 tensor cores (mma.sync f64, float64 arithmetic, degrees 1..5; not
 * with a per-element diffusivity); DDG_ENGINE_CUDA_CORES: plain FMA on the
 * CUDA cores.  Defaults: every float64 apply (ddg_sipg_apply with DDG_FP64,
 * float64 CG and residuals) and stand-alone float32 applies use the tensor
 * cores, and so do float32 CG iterations (ddg_sipg_cg with DDG_FP32,
 * ddg_sipg_cg_mixed).  Both float32 engines centre each element's values on
 * its first nodal value before the derivative products, so their rounding
 * error on smooth vectors scales with the element's variation (the mixed
 * solver then needs as many iterations as with float64 arithmetic).
 * Calling this sets all three where the degree has the engine
 * (DDG_ERR_UNSUPPORTED if it has none).  The host-buffer
 * apply recaptures its pipeline with the new engine on its next call.  No
 * reference counterpart (the reference's operator is jax.grad of its
 * bilinear form, sipg.py:304-337). */
#define DDG_ENGINE_CUDA_CORES   0
#define DDG_ENGINE_TENSOR_CORES 1
int ddg_sipg_set_engine(ddg_sipg_op *op, int engine);

/* y = A u + alpha * J (M_ref u) for float64 HOST fields in the reference's
 * own (Np, K) row-major layout: sipg_apply_2d(mesh, u, bc_types=...) of
 * src/ddg/dg2d/sipg.py:304-337 as called with numpy arrays, which take and
 * return (Np, K).  The call copies u to the device in element chunks on one
 * stream, runs the apply of each chunk as soon as the chunks holding its
 * face neighbours have arrived, and copies y back on a second stream, so the
 * two transfer directions and the kernels overlap.  Pinned (page-locked)
 * u / y are read / written directly by the copy engines; pageable ones are
 * staged through the handle's pinned buffers (allocated on first use).
 * Returns after y is complete; `stream`'s earlier work is ordered before
 * the copies. */
int ddg_sipg_apply_host(ddg_sipg_op *op, double alpha, const double *u, double *y,
                        void *stream);

/* rhs = J (M_ref f) - L_D(u_dir) + L_N(q_neu), all float64 device vectors.
 * Replaces the RHS assembly of src/ddg/dg2d/sipg.py:852-864 with
 * sipg_dirichlet_load_2d (:398-417) and sipg_neumann_load_2d (:420-453).
 * f may be NULL (zero source), u_dir NULL (no Dirichlet load), q_neu NULL. */
int ddg_sipg_rhs(ddg_sipg_op *op, const double *f, const double *u_dir,
                 const double *q_neu, double *rhs, void *stream);

/* Block-Jacobi preconditioner of alpha M + A: per-element (Np, Np) diagonal
 * blocks, inverted on the device.  Replaces extract_block_diag_matfree +
 * _block_jacobi_apply (src/ddg/dg2d/sipg.py:671-715) and the two builders
 * make_sipg/helmholtz_block_jacobi_preconditioner (:718-805). */
int ddg_sipg_pc_build(ddg_sipg_op *op, double alpha, void *stream);
/* z = B^-1 r on device vectors (the M^-1(v_flat) callable, sipg.py:711-713). */
int ddg_sipg_pc_apply(ddg_sipg_op *op, int precision, const void *r, void *z,
                      void *stream);
/* Copy the (K, Np, Np) float64 diagonal blocks (not inverted) to device
 * memory `blocks` (for tests; the inverse is kept internally). */
int ddg_sipg_pc_blocks(ddg_sipg_op *op, double *blocks, void *stream);

/* ---- Krylov solve ----------------------------------------------------- */
#define DDG_PC_NONE   0
#define DDG_PC_JACOBI 1   /* block-Jacobi from ddg_sipg_pc_build           */
#define DDG_PC_USER   2   /* reserved                                       */

typedef struct {
    double  tol;        /* relative tolerance (IterativeConfig.tol)         */
    double  atol;       /* absolute tolerance (IterativeConfig.atol)        */
    int32_t maxiter;    /* IterativeConfig.maxiter                          */
    int32_t pc;         /* DDG_PC_*                                          */
    double  alpha;      /* Helmholtz mass coefficient (0 = Poisson)         */
    double  shift;      /* extra  shift * I  (singular-Poisson eps-shift)   */
    int32_t precision;  /* DDG_FP64 or DDG_FP32 (vectors and operator)      */
    int32_t reserved;
} ddg_cg_config;

typedef struct {
    int32_t status;      /* DDG_SOLVE_*                                     */
    int32_t iterations;  /* CG iterations (mixed: float32 iterations)       */
    double  res_norm2;   /* final r.r (mixed: float64 true residual)        */
    double  b_norm2;     /* b.b                                             */
    int32_t updates;     /* mixed: float64 reliable updates performed       */
    int32_t reserved;
} ddg_solve_info;

/* CG on (alpha M + A + shift I) x = b with the stopping rule of
 * jax.scipy.sparse.linalg.cg as called at src/ddg/dg2d/sipg.py:604,910:
 * r.r <= max(tol^2 b.b, atol^2) checked before each iteration, at most
 * maxiter iterations.  b, x: device vectors of the config's precision;
 * x holds x0 on entry and the solution on exit.  The whole loop runs on the
 * device as a CUDA graph with a conditional while node; the call returns
 * after the stream has been synchronised and `info` filled.  With the
 * environment variable DDG_CG_EAGER=1 the same iteration kernels are
 * launched directly and the loop flag is read every 16 iterations (for
 * profilers, which cannot see kernels inside conditional graphs). */
int ddg_sipg_cg(ddg_sipg_op *op, const ddg_cg_config *cfg, const void *b,
                void *x, void *stream, ddg_solve_info *info);

/* Mixed-precision CG with reliable updates (extension; the reference solves
 * in float64 only).  float32 PCG iterations (operator, vectors and
 * block-Jacobi in float32, dot products accumulated in float64) keep their
 * search direction across float64 residual replacements: whenever the
 * float32 residual has dropped by `delta` (e.g. 0.1) since the last
 * replacement, x += x32, r = b - A x is recomputed in float64 and the
 * float32 iteration continues from it.  Stops when the float64 residual
 * satisfies the cfg tolerances (same rule as ddg_sipg_cg), after
 * cfg->maxiter float32 iterations, or when replacements stop reducing the
 * float64 residual (status DDG_SOLVE_STAGNATED).  cfg->precision is ignored.
 * b, x: float64 device vectors (x: x0 in, solution out). */
#define DDG_SOLVE_STAGNATED  4
int ddg_sipg_cg_mixed(ddg_sipg_op *op, const ddg_cg_config *cfg, double delta,
                      const double *b, double *x, void *stream, ddg_solve_info *info);

/* ---- per-element diffusivity and its adjoint gradient ------------------- */
/* Extension with no reference counterpart (ddg's SIPG form has no
 * coefficient): set (kappa: K host doubles > 0) or clear (NULL) a
 * per-element diffusivity.  The operator becomes volume kappa_k grad u.grad v,
 * face averages (kappa_M Dn_M + kappa_P Dn_P)/2 and penalty weight
 * (kappa_M + kappa_P)/2 (kappa_M on Dirichlet faces); symmetric, and equal to
 * the reference operator for kappa = 1.  Applies, CG (all precisions) and
 * the block-Jacobi preconditioner use it (rebuild the preconditioner after
 * setting it); multigrid and non-homogeneous Dirichlet loads do not. */
int ddg_sipg_set_kappa(ddg_sipg_op *op, const double *kappa);
/* g[k] = d a(u, lam; kappa) / d kappa_k for device float64 vectors u, lam;
 * the kappa-gradient contraction of the adjoint method: with A u = b and
 * A lam = dL/du, dL/dkappa = -g (a is linear in kappa). */
int ddg_sipg_grad_kappa(ddg_sipg_op *op, const double *u, const double *lam, double *g, void *stream);

/* ---- p / hp multigrid (src/ddg/dg2d/multigrid.py) ---------------------- */
typedef struct ddg_mg ddg_mg;                /* opaque, library-owned */

/* V-cycle description.  Level l = 0 is the finest.  Every level handle must
 * have its block-Jacobi smoother built with ddg_sipg_pc_build(alpha).
 * Between levels l and l+1 the transfer is either a p-transfer (same K,
 * prolongation I of shape (Np_l, Np_{l+1}), multigrid.py:106-134) or an
 * h-transfer (K_l = 4 K_{l+1}, fine element 4k+c = child c of k,
 * prolongation [I_0; I_1; I_2; I_3] of shape (4 Np, Np), :137-184).
 * Restriction is the transpose.  coarse_inv is the dense inverse of the
 * coarsest operator (the reference LU-factors it, :220-228; the caller
 * adds its eps*max|diag| shift first when regularising).  All HOST arrays,
 * read during the call. */
typedef struct {
    int32_t nlevels;
    int32_t precision;        /* DDG_FP32 or DDG_FP64: smoothing, transfers, coarse */
    int32_t nu;               /* pre/post smoothing sweeps (nu_smooth)      */
    int32_t reserved;
    double  omega;            /* smoother damping                            */
    double  alpha;            /* level operators are alpha M + A             */
    ddg_sipg_op *const *ops;  /* nlevels handles, finest first               */
    const double *const *prolong;   /* nlevels-1 host row-major matrices     */
    const int32_t *prolong_rows, *prolong_cols;
    const double *coarse_inv; /* (nc, nc) row-major, nc = K*Np of the coarsest */
} ddg_mg_desc;

int ddg_mg_create(const ddg_mg_desc *desc, ddg_mg **out);
int ddg_mg_destroy(ddg_mg *mg);
/* z = V-cycle(r) (multigrid.py:232-246), float64 device vectors of the
 * finest level (the M^-1(v_flat) callable of make_sipg_(hp)mg_preconditioner). */
int ddg_mg_apply(ddg_mg *mg, const double *r, double *z, void *stream);
/* float64 CG on (alpha M + A + shift I) x = b preconditioned by one V-cycle
 * per iteration; the whole loop, V-cycle included, runs as one device graph.
 * Stopping rule as ddg_sipg_cg (preconditioned: on r.r). */
int ddg_sipg_cg_mg(ddg_sipg_op *op, const ddg_cg_config *cfg, ddg_mg *mg,
                   const double *b, double *x, void *stream, ddg_solve_info *info);

/* ---- continuous-batching solve pool (serving) ------------------------- */
/* Extension (the reference solves one mesh per call).  A pool packs many
 * independent solves of one degree N into one element array; every CG
 * scalar is per request (segmented reductions), so a request's iterates are
 * the same whichever other requests share the launches.  The caller runs
 * the scheduling loop: admit arrivals while others iterate, iterate, poll,
 * retire finished requests (their element range is reused at once). */
typedef struct ddg_pool ddg_pool;

/* capacity: element slots (device memory is sized from it);
 * max_requests: concurrent requests; max_request_K: largest request. */
int ddg_pool_create(int N, int capacity, int max_requests, int max_request_K,
                    double tau_scale, int device, ddg_pool **out);
/* The same with the precision of the iteration vectors: DDG_FP64, or
 * DDG_FP32 (float32 vectors, geometry and block-Jacobi inverses, float64
 * reductions and CG scalars; for requests whose tolerance float32
 * iterations reach, such as 1e-6).  No reference counterpart. */
int ddg_pool_create_ex(int N, int capacity, int max_requests, int max_request_K,
                       double tau_scale, int precision, int device, ddg_pool **out);
int ddg_pool_destroy(ddg_pool *pool);
/* Admit one (alpha M + A) u = J M f solve on `mesh` (host arrays, its own
 * numbering; bc_types as in ddg_sipg_mesh_desc), source f (K x Np,
 * element-major, host), CG tolerances.  Returns the request slot, or
 * DDG_ERR_NOMEM when no slot / element range is free right now. */
int ddg_pool_admit(ddg_pool *pool, const ddg_sipg_mesh_desc *mesh, double alpha,
                   double tol, double atol, int maxiter, const double *f,
                   void *stream, int *slot);
/* 2*pairs block-Jacobi PCG iterations of every active request (one graph). */
int ddg_pool_iterate(ddg_pool *pool, int pairs, void *stream);
/* Tile shape of the pool's element kernels in later ddg_pool_iterate calls:
 * threads per block (64, 128 or 256), persistent 0 (one thread per element)
 * or 1 (a grid of at most 2048/threads blocks per SM looping over the
 * elements).  Results are identical for every shape; the serving
 * autotuner picks the fastest per (degree, element count).  No reference
 * counterpart (the reference has no serving layer). */
int ddg_pool_set_tile(ddg_pool *pool, int threads, int persistent);
/* Per slot: 1 while iterating, 0 when finished or empty; iteration counts. */
int ddg_pool_poll(ddg_pool *pool, int32_t *active, int32_t *iterations, void *stream);
/* Copy a finished request's solution (K x Np, host) and free its slot. */
int ddg_pool_retire(ddg_pool *pool, int slot, double *x, void *stream, ddg_solve_info *info);
/* Reference-element matrices of degree N into `device`'s constant memory
 * (ddg_sipg_create does this itself). */
int ddg_sipg_upload_reference(int N, const double *Dr, const double *Ds, const double *M,
                              const double *m1d, int device);

/* ---- curved elements (per-node geometry, cubature) --------------------- */
/* The operator of sipg_apply_2d on a Mesh2D whose geometric factors vary
 * node by node (curved boundary elements, src/ddg/dg2d/curved.py:93-236),
 * with either quadrature of sipg_bilinear_form: nodal (cub=None,
 * src/ddg/dg2d/sipg.py:188-189, 265-280) or the cubature branch
 * (cub=MeshCubature, src/ddg/dg2d/sipg.py:190-201, 281-299;
 * src/ddg/dg2d/cubature.py:73-223).  Float64 only. */
typedef struct ddg_curved_op ddg_curved_op;   /* opaque, library-owned */

#define DDG_QUAD_NODAL    0
#define DDG_QUAD_CUBATURE 1

/* All pointers HOST memory, read during ddg_curved_create only.  Volume
 * fields are the reference's (Np, K) row-major arrays, face fields
 * (3 Nfp, K), cubature fields (Ncub, K) / (3, Nfq, K) as MeshCubature holds
 * them. */
typedef struct {
    int32_t N, K, device;
    int32_t Ncub;            /* volume cubature points; 0: nodal quadrature only   */
    int32_t Nfq;             /* face cubature points (Ncub > 0)                   */
    int32_t reserved;
    double  tau_scale;       /* tau = tau_scale (N+1)^2 Fscale (first face node)  */
    const double *Dr, *Ds, *M, *m1d;   /* reference element, as ddg_sipg_mesh_desc */
    const int64_t *Fmask;    /* (Nfp, 3)                                          */
    const double *rx, *sx, *ry, *sy, *J;       /* (Np, K)  mesh.py:634-644        */
    const double *nx, *ny, *sJ, *Fscale;       /* (3 Nfp, K)  mesh.py:647-684     */
    const int64_t *EToE, *EToF;                /* (K, 3)                          */
    const int64_t *vmapM, *vmapP;              /* (3 Nfp K)                       */
    const int32_t *bc_types;                   /* (K, 3)                          */
    const double *cw;                          /* (Ncub)       MeshCubature.w     */
    const double *Drq, *Dsq, *Lq;              /* (Ncub, Np)                      */
    const double *cJ, *crx, *csx, *cry, *csy;  /* (Ncub, K)                       */
    const double *face_w;                      /* (Nfq)                           */
    const double *face_L1d;                    /* (3, Nfq, Nfp)                   */
    const double *face_sJ;                     /* (3, Nfq, K)                     */
} ddg_curved_desc;

int ddg_curved_create(const ddg_curved_desc *desc, ddg_curved_op **out);
int ddg_curved_destroy(ddg_curved_op *op);
int ddg_curved_set_bc(ddg_curved_op *op, const int32_t *bc_types);
/* y = A_quad u + alpha M_quad u (sipg_apply_2d with u_dir=None plus the
 * Helmholtz mass of sipg.py:593-601, cubature_mass_apply for quad 1);
 * element-major float64 device vectors. */
int ddg_curved_apply(ddg_curved_op *op, int quad, double alpha, const double *u, double *y, void *stream);
/* y = d a_quad(u, v; u_dir) / d v at v = 0: sipg_apply_2d with a
 * non-homogeneous Dirichlet ghost u_dir (sipg.py:216-233, 304-337), i.e.
 * A_quad u plus the Dirichlet load of u_dir by the same face rule.  u may be
 * null (zero): y is then the load alone (sipg.py:398-417 for quad 0). */
int ddg_curved_apply_dir(ddg_curved_op *op, int quad, const double *u, const double *u_dir, double *y,
                         void *stream);
/* y = M_quad f (mesh.J * (M_ref @ f) or cubature_mass_apply). */
int ddg_curved_mass(ddg_curved_op *op, int quad, const double *f, double *y, void *stream);
/* rhs = M_quad f - L_D(u_dir) + L_N(q_neu) (sipg.py:564-574, 851-864); the
 * loads use the nodal face rule, as sipg_dirichlet_load_2d /
 * sipg_neumann_load_2d do (sipg.py:398-453).  f, u_dir, q_neu may be null. */
int ddg_curved_rhs(ddg_curved_op *op, int quad, const double *f, const double *u_dir,
                   const double *q_neu, double *rhs, void *stream);
/* Block-Jacobi of (alpha M + A)_quad: diagonal blocks by coloured probing
 * of the apply (sipg.py:651-704), explicit inverses (sipg.py:707-715). */
int ddg_curved_pc_build(ddg_curved_op *op, int quad, double alpha, void *stream);
int ddg_curved_pc_apply(ddg_curved_op *op, const double *r, double *z, void *stream);
/* (K, Np, Np) row-major diagonal blocks of the last pc_build. */
int ddg_curved_pc_blocks(ddg_curved_op *op, double *blocks, void *stream);
/* float64 CG on (alpha M + A + shift I)_quad x = b, the stopping rule of
 * ddg_sipg_cg; cfg->pc = DDG_PC_JACOBI uses the last pc_build.  The loop
 * runs as a CUDA graph with a conditional while node. */
int ddg_curved_cg(ddg_curved_op *op, int quad, const ddg_cg_config *cfg, const double *b,
                  double *x, void *stream, ddg_solve_info *info);

/* ---- small vector helpers (device) ------------------------------------ */
/* y = a*x + b*y  (float64) */
int ddg_axpby(int64_t n, double a, const double *x, double b, double *y, void *stream);
/* out[0] = x.y  (float64 accumulation), out device double */
int ddg_dot(int64_t n, int precision, const void *x, const void *y, double *out, void *stream);
/* out[0] = x.y without allocating: no counterpart in the reference (an
 * addition for callers that cannot allocate device memory, e.g. code being
 * captured into a CUDA graph, or an embedding application that owns a fixed
 * device-memory budget).  Its scratch (block partials and a completion
 * counter, 512 KiB) is a static device array inside this library, present
 * on every GPU that has called it until the process exits.  n must not
 * exceed DDG_DOT_NOALLOC_MAX_N.  The first call on a device looks up that
 * array's address (do it before any stream capture); every call clears the
 * counter on `stream` first; calls that overlap on the GPU share the array
 * and race.  Same float64 accumulation as ddg_dot (summation order differs). */
#define DDG_DOT_NOALLOC_MAX_N 536870912LL
int ddg_dot_noalloc(int64_t n, int precision, const void *x, const void *y, double *out, void *stream);
/* float64 <-> float32 copies */
int ddg_cast(int64_t n, int to_precision, const void *src, void *dst, void *stream);

/* ---- mesh connectivity (host, C++) ------------------------------------ */
/* EToE/EToF as src/ddg/dg2d/mesh.py:520-571 (_ti_connect_2d), bit-exact:
 * face keys v_min*n_nodes+v_max, stable sort, adjacent equal keys pair,
 * boundary faces point to themselves.  EToV (K,3) int64 host.            */
int ddg_mesh_connect(int64_t K, const int64_t *EToV, int64_t *EToE, int64_t *EToF);
/* vmapM/vmapP as src/ddg/dg2d/mesh.py:574-627 (_build_maps_2d), bit-exact:
 * first face node of the partner within node_tol * edge length, fallback
 * vmapM.  x, y: (Np, K) row-major (the reference's arrays), Fmask (Nfp,3). */
int ddg_mesh_maps(int64_t K, int32_t N, const int64_t *Fmask,
                  const double *x, const double *y,
                  const int64_t *EToE, const int64_t *EToF,
                  const int64_t *EToV, const double *VX, const double *VY,
                  double node_tol, int64_t *vmapM, int64_t *vmapP);

/* Message of the last failure on this thread ("" if none). */
const char *ddg_last_error(void);
/* Library version string. */
const char *ddg_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DDG_SIPG_H */
