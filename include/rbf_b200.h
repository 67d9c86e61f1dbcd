/* rbf_b200.h -- C ABI of the B200 (sm_100a) RBF-FD operator assembly.
 *
 * This is the drop-in boundary for the assembly path of ivan-pi/gpu-assembly:
 * host C++ and Fortran (bind(c)) callers reach the sm_100a kernels through
 * these plain-C entry points instead of instantiating the reference's
 * cuSolverDx kernel template. Every entry point below names the reference
 * interface it replaces (paths relative to the reference repository).
 *
 * Conventions (the reference's, src/rbf_operators.h:292-316):
 *   - all array arguments are DEVICE pointers unless the name ends in _h;
 *   - indices are 0-based int32; a fixed-width stencil table ja holds the
 *     k neighbours of stencil s at ja[s*k .. s*k+k), self first;
 *   - a CSR stencil table holds row s at ja[ia[s] .. ia[s+1]);
 *   - the caller owns every buffer; entry points that need scratch take it
 *     from the context (rbfb_ctx) and never from the caller's buffers;
 *   - weights for right-hand side q go to values[q][row offset + j], the
 *     weight of neighbour ja[row offset + j] (src/rbf_operators.h:307-313);
 *   - per-stencil status info[s]: 0 = success, c+1 = zero pivot at
 *     elimination step c (LAPACK getrf convention, src/rbf_operators.h:315);
 *     the weights of such a stencil are written as quiet NaN;
 *   - `stream` is a cudaStream_t (NULL = legacy default stream); calls are
 *     asynchronous on it unless stated otherwise.
 *
 * Return values: 0 on success, a negative RBFB_E* code on argument or CUDA
 * errors (rbfb_status_string names it, rbfb_last_error gives details).
 * Synchronous calls that count singular stencils return that count (>= 0).
 */
#ifndef RBF_B200_H
#define RBF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define RBFB_OK 0
#define RBFB_EINVAL (-1)      /* bad argument (null pointer, k > n, ...)      */
#define RBFB_ECUDA (-2)       /* a CUDA runtime call failed                    */
#define RBFB_ENOMEM (-3)      /* device or pinned allocation failed            */
#define RBFB_EUNSUPPORTED (-4)/* no compiled kernel for this shape             */
#define RBFB_ETIMEOUT (-5)    /* a bounded wait ran out                        */
#define RBFB_EBUDGET (-6)     /* request larger than the server's HBM budget   */
#define RBFB_ENOTFOUND (-7)   /* unknown ticket                                */
#define RBFB_EBUSY (-8)       /* ticket not finished (non-blocking poll)       */
#define RBFB_ETOOBIG (-9)     /* beyond the fixed scratch of a no-allocation call */

/* ---- operators (right-hand sides) --------------------------------------
 * Right-hand-side columns, in output order: nc interpolation points first
 * (RBFB_OP_INTERP, the reference's fill_rhs, src/rbf_operators.h:156-185),
 * then each derivative operator set in `ops`, in bit order, evaluated at the
 * stencil centre. */
#define RBFB_OP_INTERP 1
#define RBFB_OP_LAPLACE 2
#define RBFB_OP_DX 4
#define RBFB_OP_DY 8
#define RBFB_OP_DXX 16
#define RBFB_OP_DYY 32
#define RBFB_OP_DXY 64

/* ---- precision ---------------------------------------------------------- */
#define RBFB_FP64 0     /* FP64 fill, FP64 elimination (the plain kernel)     */
#define RBFB_FP32_IR 1  /* FP64 fill, FP32 elimination, FP64 residual
                           iterative refinement, FP64 fallback per stencil   */

#define RBFB_MAX_RHS 8  /* right-hand sides per stencil                      */

typedef struct rbfb_ctx rbfb_ctx;
typedef struct rbfb_server rbfb_server;

/* Assembly descriptor: the run-time form of the reference's compile-time
 * interp_config<N, NRHS, P, Q, ARCH, T> (src/rbf_operators.h:187-290). */
typedef struct rbfb_desc {
    int degree;        /* P, total degree of the polynomial augmentation (0..4)   */
    int phs;           /* Q, odd PHS exponent phi(r) = r^Q; 0 = 2P-1 (per stencil)*/
    int ops;           /* RBFB_OP_* mask                                            */
    int precision;     /* RBFB_FP64 or RBFB_FP32_IR                                 */
    int scale;         /* 1: power-of-two radius scaling of each stencil (exact)    */
    int max_sweeps;    /* refinement sweeps before the FP64 fallback (0 = 6)        */
    double ir_tol;     /* converged when max|dx| <= ir_tol * max|x| (0 = 1e-11)     */
    double period[2];  /* box sides for minimum-image displacements; 0 = open axis  */
    int nc;            /* number of interpolation points (RBFB_OP_INTERP)           */
    const double* xc;  /* interpolation points in the stencil-local frame (device)  */
    const double* yc;
} rbfb_desc;

/* Counters of one assembly call (filled on synchronous calls). */
typedef struct rbfb_stats {
    long long stencils;       /* stencils assembled                                  */
    long long singular;       /* stencils with info != 0                             */
    long long fallback;       /* FP32_IR stencils re-solved in FP64                  */
    long long sweeps;         /* refinement sweeps summed over stencils              */
    int max_sweeps_used;      /* largest sweep count of any stencil                  */
    int buckets;              /* kernel shapes launched                              */
    float ms;                 /* device time of the call (CUDA events)               */
} rbfb_stats;

/* ---- context ------------------------------------------------------------ */
/* One context per host thread (or serialise calls on it). Holds the
 * workspace, the tuned launch table and the CUDA graphs of the batched path.
 * No reference counterpart: the reference keeps this state in template
 * constants and caller-owned buffers (src/rbf_operators.h:187-290). */
int rbfb_create(rbfb_ctx** ctx, int device);
int rbfb_destroy(rbfb_ctx* ctx);
const char* rbfb_status_string(int status);
const char* rbfb_last_error(const rbfb_ctx* ctx);
/* Number of this library's kernels launched by the context so far. */
long long rbfb_kernel_launches(const rbfb_ctx* ctx);

/* ---- stencil search ----------------------------------------------------- */
/* k nearest neighbours of every node, sorted by (squared distance, index),
 * self first: ja[s*k + t]. period == NULL or {0,0}: open plane, the
 * reference's NodeSet::stencils(k) (src/rbf_nodeset.h:155-181, nanoflann);
 * period = {Lx, Ly} > 0: periodic box, minimum-image metric, the reference's
 * KdTree::knn_stencils(k) (src/rbf_spatial.h:178-183, src/rbf_spatial.cpp:
 * 251-260, ckdtree). period is a HOST pointer. Equal to the reference's
 * result wherever no two candidates tie in distance. */
int rbfb_knn_stencils(rbfb_ctx* ctx, int n, const double* x, const double* y, int k,
                      const double* period_h, int* ja, void* stream);

/* k nearest nodes of nq arbitrary query points (xq, yq): the reference's
 * KdTree::knn_stencils(q, k) (src/rbf_spatial.h:173-178). */
int rbfb_knn_query(rbfb_ctx* ctx, int n, const double* x, const double* y, int nq,
                   const double* xq, const double* yq, int k, const double* period_h, int* ja,
                   void* stream);

/* The search of rbfb_knn_stencils without any allocation, for callers that
 * may not allocate device memory while they run: a solver loop that claimed
 * its device memory in a set-up phase and must not call cudaMalloc/cudaFree
 * afterwards (they can synchronise the device and fragment its pool), or a
 * host whose device memory belongs to another framework's allocator. No
 * counterpart in the reference (its searches run on the host).
 *
 * Needs no context: the scratch is a fixed array of about 3 MB in device
 * memory, held by every GPU that loads this library until the process exits.
 * Limit: n <= 65,536 nodes (and a cell grid of at most n/2 cells); larger
 * problems are rejected with RBFB_ETOOBIG. The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture. The address is
 * kept for the life of the process, so do not use these entry points across
 * a cudaDeviceReset. All calls share the one array: calls whose work
 * overlaps on the GPU (other streams, other host threads) race and must be
 * serialised by the caller. Same arguments, argument checks (and status
 * codes), result and ordering as rbfb_knn_stencils; like it, a query that
 * gives up widening its search leaves its row of ja unwritten, which
 * rbfb_knn_static_status reports. */
int rbfb_knn_stencils_static(int n, const double* x, const double* y, int k,
                             const double* period_h, int* ja, void* stream);

/* Completion status of the last rbfb_knn_stencils_static search on the
 * current device: 0 when every query finished, 1 when a query gave up (its
 * row of ja is then unwritten), negative on a CUDA error. Reads the status
 * word of the fixed array into host memory, allocating nothing, and
 * synchronises `stream`. No reference counterpart. */
int rbfb_knn_static_status(void* stream);

/* Completion status of the last search on this context: 0 when every query
 * finished, 1 when a query gave up widening its search (its row of ja is
 * then unwritten). Synchronises `stream`. No reference counterpart (the
 * reference's tree search cannot fail this way). */
int rbfb_knn_status(rbfb_ctx* ctx, void* stream);

/* ---- assembly ----------------------------------------------------------- */
/* Fixed-width stencils: the reference's assemble_interp_weights<Config>
 * (src/rbf_operators.h:320-376) and the planned assemble_laplace_weights
 * (src/main.cpp:15-16,44-45). values_h is a HOST array of nrhs DEVICE
 * pointers (the reference passes the same table in device memory, `A`),
 * each to nstencils*k doubles. info may be NULL. stats may be NULL; when
 * given, the call synchronises `stream` and fills it. */
int rbfb_assemble(rbfb_ctx* ctx, const rbfb_desc* desc, int nstencils, const double* x,
                  const double* y, int k, const int* ja, double* const* values_h, int* info,
                  rbfb_stats* stats, void* stream);

/* rbfb_assemble with the pointer table in DEVICE memory, as the reference's
 * kernel takes it: `T* const* A`, dereferenced on the device
 * (src/rbf_operators.h:324,370-375), filled by the caller and passed as
 * ptr(A_tab) (src/main.cpp:44-45). values_d holds nrhs device pointers; the
 * kernels read it, so the call stays asynchronous. */
int rbfb_assemble_dtab(rbfb_ctx* ctx, const rbfb_desc* desc, int nstencils, const double* x,
                       const double* y, int k, const int* ja, double* const* values_d, int* info,
                       rbfb_stats* stats, void* stream);

/* Stencils first .. first+count-1 of an n-node set (all n coordinates given):
 * ja_rows, values_rows[q] and info_rows hold only those rows (row first at
 * index 0). The unit of the multi-GPU split: each rank assembles a
 * contiguous node range against the full, replicated node set. The
 * reference's kernel has no range form (one launch covers all nstencils,
 * src/rbf_operators.h:317-328). */
int rbfb_assemble_range(rbfb_ctx* ctx, const rbfb_desc* desc, int first, int count, int n,
                        const double* x, const double* y, int k, const int* ja_rows,
                        double* const* values_rows, int* info_rows, rbfb_stats* stats,
                        void* stream);

/* Ragged stencils in CSR form (ia has nstencils+1 entries), optionally with a
 * per-stencil degree (int8, NULL = desc->degree): the uneven batch. FP64
 * with up to 3 right-hand sides: the whole batch in ONE persistent launch,
 * its warps taking the stencils in class order (system size descending,
 * then degree) from a list sorted on the device; systems of up to 96
 * unknowns. The refined form (and more right-hand sides): stencils bucketed
 * on the device by system size, one persistent launch per bucket of the
 * kernel shape that fits it. The call is a fixed launch sequence with no
 * host round trip; on a non-default stream it is captured in a CUDA graph
 * and replayed when the same batch comes again.
 * The Fortran module's fill_kernel (src/rbf_cuda.f90:36-99) is the
 * reference's only CSR-driven assembly. */
int rbfb_assemble_csr(rbfb_ctx* ctx, const rbfb_desc* desc, int nstencils, const double* x,
                      const double* y, const int* ia, const int* ja, const int8_t* degree,
                      double* const* values_h, int* info, rbfb_stats* stats, void* stream);

/* End to end from HOST memory: copies the nodes in, finds the k-NN stencils
 * (unless ja_h is given), assembles, and copies the stencils (ja_out_h, may
 * be NULL) and the weights (values_h: HOST array of nrhs HOST pointers) back,
 * pipelining the copies with the kernels in chunks. Synchronous. Returns the
 * number of singular stencils. */
int rbfb_assemble_host(rbfb_ctx* ctx, const rbfb_desc* desc, int n, const double* x_h,
                       const double* y_h, int k, const int* ja_h, int* ja_out_h,
                       double* const* values_h, int* info_h, rbfb_stats* stats);

/* ---- Fortran rbf_cuda module and solve_dp counterparts ------------------- */
/* The saddle-point matrix [A P; P^T 0] of every stencil, FP64, column-major
 * n x n (n = k_s + npoly(P)) with leading dimension ldm, stencil s in the
 * ldm x ldm slab at M + s*ldm*ldm (a stencil with n > ldm is skipped), in the shifted
 * (and, with desc->scale, scaled) frame: fill_matrix (src/rbf_operators.h:
 * 116-154) and the Fortran fill_kernel (src/rbf_cuda.f90:36-99). Uses
 * desc->degree, desc->phs, desc->scale and desc->period. */
int rbfb_fill_matrices(rbfb_ctx* ctx, const rbfb_desc* desc, int nstencils, const double* x,
                       const double* y, const int* ia, const int* ja, double* M, int ldm,
                       void* stream);

/* The Fortran fill_kernel (src/rbf_cuda.f90:36-99) with its arguments: the
 * degree-2, r^3 saddle-point matrix of each CSR stencil (0-based ia, ja), from
 * the ABSOLUTE node coordinates (no shift, no scaling), column-major with
 * leading dimension ldm, stencil s in the ldm x ldm slab at M + s*ldm*ldm
 * (a stencil with k_s + 6 > ldm is skipped). For nstencils = 1 this is the
 * reference's single output matrix (its kernel writes every stencil into the
 * same M). Arithmetic as there: (x_col - x_k)^2 + (y_col - y_k)^2, then
 * r2 * sqrt(r2). No context. */
int rbfb_fill_kernel(int nstencils, const double* x, const double* y, const int* ia,
                     const int* ja, double* M, int ldm, void* stream);

/* The Fortran fill_rhs (src/rbf_cuda.f90:101-136) with its arguments:
 * B(k, j) = |(xc_j, yc_j) - (x_k, y_k)|^3 for the n stencil nodes (x, y hold
 * the stencil's own coordinates) and B(n + i, j) = the i-th degree-2 monomial
 * at (xc_j, yc_j), for j < nc; column-major, ldb >= n + 6. No context. */
int rbfb_fill_rhs(int n, const double* x, const double* y, int nc, const double* xc,
                  const double* yc, double* B, int ldb, void* stream);

/* The Fortran store_to_csr (src/rbf_cuda.f90:139-157) with its arguments, for
 * one stencil idx: va[ia[idx] + k] = W(k,1) + W(k,2), k < ia[idx+1] - ia[idx],
 * W column-major with leading dimension ldw (p_xx + p_yy). The reference's is
 * a device subroutine; this is a host call launching one small kernel. */
int rbfb_store_to_csr_stencil(int nstencils, const int* ia, double* va, const double* W, int ldw,
                              int idx, void* stream);

/* va[ia[s] + j] = W[s][j][0] + W[s][j][1]: the Fortran store_to_csr, which
 * forms a Laplacian from the d2/dx2 and d2/dy2 weight columns (src/rbf_cuda.f90:
 * 139-157). wxx, wyy are CSR value arrays laid out like va. */
int rbfb_store_to_csr(int nstencils, const int* ia, const double* wxx, const double* wyy,
                      double* va, void* stream);

/* Launches solve_dp<<<1,32>>>: one 15x15 system with 9 right-hand sides,
 * FP64, A column-major (lda 15), B column-major (ldb 15), solved in place
 * with partial pivoting; ipiv receives 1-based LAPACK-style row interchanges,
 * *info the getrf status. The reference's demo kernel
 * (src/rbf_operators.cpp:7-11, launched from src/main.f90:57). */
int rbfb_solve_dp(double* A, int* ipiv, double* B, int* info, void* stream);

/* ---- applying the operator -------------------------------------------------- */
/* out[s] = sum_j values[s*k+j] * u[ja[s*k+j]] for s < n (fused multiply-adds
 * in row order from zero), then out[bnd[b]] = u[bnd[b]] for the nbnd listed
 * boundary rows (bnd may be NULL when nbnd = 0). The operator application and
 * boundary fix the reference sketches after its assembly (A.spmv and the
 * parallel_for over boundary nodes, src/main.cpp:57-66). */
int rbfb_spmv(int n, int k, const int* ja, const double* values, const double* u, double* out,
              const int* bnd, int nbnd, void* stream);

/* ---- solving with the assembled operator ------------------------------------
 * Solves A u = f by BiCGSTAB (van der Vorst, 1992; no preconditioner). A is
 * the operator rbfb_spmv applies: the stencil rows (fixed width k when ia is
 * NULL, else the CSR rows ja[ia[s] .. ia[s+1])) with the nbnd rows listed in
 * bnd replaced by identity rows, so that f holds the boundary values there.
 * The reference builds this operator as mv_op and leaves the solve after it
 * empty (src/main.cpp:57-68). Every ja entry must lie in [0, n).
 *
 * u holds the initial guess on entry and the last iterate on exit. The
 * iteration stops when the recursive residual satisfies
 * ||r||_2 <= tol * ||f||_2, after maxit iterations, or on a breakdown (a
 * zero or non-finite denominator). When f = 0, u is set to zero.
 * Synchronous on `stream`. Returns RBFB_OK when converged, RBFB_ENOCONV when
 * maxit ran out, RBFB_EBREAKDOWN on a breakdown, a negative argument or CUDA
 * code otherwise. *iters_h and *relres_h (host, either may be NULL) receive
 * the iterations taken and ||r||_2 / ||f||_2.
 *
 * The sums are deterministic: one thread per row, fused multiply-adds in row
 * order, and dot products reduced in a fixed order over a grid of
 * min(ceil(n / 256), 6 * SMs) blocks of 256 threads. */
#define RBFB_ENOCONV (-10)    /* iterative solve: maxit ran out              */
#define RBFB_EBREAKDOWN (-11) /* iterative solve: zero or non-finite pivot   */
int rbfb_solve_bicgstab(rbfb_ctx* ctx, int n, int k, const int* ia, const int* ja,
                        const double* values, const int* bnd, int nbnd, const double* f,
                        double* u, double tol, int maxit, int* iters_h, double* relres_h,
                        void* stream);

/* ---- D2Q9 lattice Boltzmann kernels that consume the operators -----------
 * The reference's feq_kernel, macros_kernel, bgk_kernel and bgk_kernel_split
 * (src/lbm/d2q9_kernels.cu:13-150, twins of src/lbm/d2q9_kernels.cuf:55-257),
 * one thread per node, for float (RBFB_LBM_FP32) and double (RBFB_LBM_FP64)
 * arrays. Lattice directions: 0 rest; 1-4 E, N, W, S; 5-8 NE, NW, SW, SE.
 * Storage is planar: direction a of node i at pdf[i + n*a]. Each product,
 * sum and quotient of the reference's expressions is rounded once, in its
 * order (no fused multiply-adds). Asynchronous on `stream`. */
#define RBFB_LBM_FP64 0
#define RBFB_LBM_FP32 1
/* pdf <- the equilibrium populations of (rho, ux, uy): feq_kernel. */
int rbfb_lbm_feq(int n, int precision, const void* rho, const void* ux, const void* uy, void* pdf,
                 void* stream);
/* rho, ux, uy <- the moments of pdf: macros_kernel. */
int rbfb_lbm_macros(int n, int precision, const void* pdf, void* rho, void* ux, void* uy,
                    void* stream);
/* BGK collision of pdf in place with relaxation rate omega; rho, ux, uy of
 * the pre-collision populations: bgk_kernel, or bgk_kernel_split when indp
 * (the direction-independent part of the equilibrium) is not NULL. */
int rbfb_lbm_bgk(int n, int precision, double omega, void* pdf, void* rho, void* ux, void* uy,
                 void* indp, void* stream);
/* One semi-Lagrangian time step: streaming of the post-collision field
 * pdf_in through the interpolation operators, then the BGK collision, into
 * pdf_out (must not alias pdf_in). Direction a (1..8) of node s becomes
 * sum_j W[(a-1)*n*k + s*k + j] * pdf_in[ja[s*k + j] + n*a], summed in j
 * order (the j = 0 product rounded, then a fused multiply-add per entry) -- the weights of
 * interpolation at the departure point x_s - c_a dt, as rbfb_assemble
 * returns them for RBFB_OP_INTERP at those 8 points (W: 8 consecutive arrays
 * of n*k doubles, FP64; rounded to float for RBFB_LBM_FP32); the rest
 * population stays. rho, ux, uy (each may be NULL) receive the moments of
 * the streamed populations. k <= 64. The reference assembles these
 * operators (src/rbf_operators.h:292-298) but ships no streaming kernel. */
int rbfb_lbm_stream_collide(int n, int precision, int k, const int* ja, const double* W,
                            double omega, const void* pdf_in, void* pdf_out, void* rho, void* ux,
                            void* uy, void* stream);

/* ---- node renumbering (locality) ------------------------------------------
 * A permutation is stored in gather form, as the reference's
 * rbf::Permutation (src/rbf_reorder.h:68-80): perm[i] is the OLD index of
 * the node at NEW position i; inv (old -> new) is optional everywhere. */

/* Space-filling-curve keys: curve 0 = Morton (Z order), 1 = Hilbert; ndiv
 * levels in 1..31 give 2*ndiv key bits. bbox_h is a HOST double[4] {xmin,
 * ymin, xmax, ymax} (the layout of rbf::BBox2<double>), or NULL for the
 * nodes' own bounding box. rbf_morton_keys / rbf_hilbert_keys with zidx /
 * hidx (src/rbf_ordering.F90:31-63,82-218; src/rbf_reorder.h:196-208). */
int rbfb_curve_keys(rbfb_ctx* ctx, int n, const double* x, const double* y, const double* bbox_h,
                    int ndiv, int curve, int64_t* keys, void* stream);
/* The nodes in curve order, stable (equal keys keep node order): morton_order
 * / hilbert_order (src/rbf_reorder.h:210-230). perm is required; keys (the
 * sorted keys) and inv may be NULL. */
int rbfb_curve_order(rbfb_ctx* ctx, int n, const double* x, const double* y, const double* bbox_h,
                     int ndiv, int curve, int64_t* keys, int* perm, int* inv, void* stream);
/* Nodes with nonzero flag last, both groups keeping their order:
 * boundary_last_by_flag (src/rbf_reorder.h:232-244). */
int rbfb_boundary_last(rbfb_ctx* ctx, int n, const int* flag, int* perm, int* inv, void* stream);
/* A' = P A P^T of a fixed-width stencil table: ja_out[s*k+j] =
 * inv[ja[perm[s]*k+j]] (renumber_stencils, src/rbf_reorder.h:256-281; here
 * out of place: ja_out must not alias ja). Self-first rows stay self-first. */
int rbfb_renumber_stencils(int n, int k, const int* ja, const int* perm, const int* inv,
                           int* ja_out, void* stream);
/* The same for CSR stencils (renumber_csr, src/rbf_reorder.h:283-303):
 * ia_out has n+1 entries; out of place. */
int rbfb_renumber_csr(rbfb_ctx* ctx, int n, const int* ia, const int* ja, const int* perm,
                      const int* inv, int* ia_out, int* ja_out, void* stream);
/* Node data into the new numbering: out[i] = in[perm[i]] for 4- or 8-byte
 * elements (Permutation::permute, src/rbf_reorder.h:68-80; out of place).
 * Also composes permutations: permuting p by q gives "p, then q". */
int rbfb_permute(int n, const int* perm, const void* in, void* out, int elem_bytes, void* stream);

/* ---- tuning --------------------------------------------------------------- */
/* Times the compiled kernel shapes for one system size and precision on the
 * given workload and records the fastest in the context's launch table
 * (lanes per stencil, CTA size, CTAs per SM). Returns the index of the
 * chosen shape, or a negative code. No reference counterpart (the
 * reference's block size comes from cuSolverDx, src/rbf_operators.h:280-281). */
int rbfb_autotune(rbfb_ctx* ctx, const rbfb_desc* desc, int nstencils, const double* x,
                  const double* y, int k, const int* ja, double* const* values_h);

/* Name of compiled kernel shape `index` (as returned by rbfb_autotune), e.g.
 * "mix_p3q5_n48_g16x2", or NULL past the last one. */
const char* rbfb_variant_name(int index);

/* Pins compiled shape `index` (and CTAs per SM, 0 = the occupancy maximum)
 * for the systems of desc's precision, degree and PHS exponent with k-node
 * stencils, as rbfb_autotune would record it. RBFB_EINVAL when the shape
 * does not serve that class. No reference counterpart (the reference fixes
 * its kernel at compile time, src/rbf_operators.h:187-290). */
int rbfb_select_variant(rbfb_ctx* ctx, const rbfb_desc* desc, int k, int index,
                        int blocks_per_sm);

/* ---- serving ---------------------------------------------------------------- */
/* Continuous-batching assembly server: requests (node sets of any size) are
 * admitted as slots and HBM budget free up, their k-NN and assembly overlap
 * on the device, and their nodes, stencils and weights stay resident on the
 * device until released. No reference counterpart. */
typedef struct rbfb_request {
    int n;               /* nodes                                                  */
    const double* x_h;   /* HOST coordinates (copied at submit)                    */
    const double* y_h;
    int k;               /* stencil size                                           */
    rbfb_desc desc;      /* operator description (xc/yc unused)                    */
} rbfb_request;

typedef struct rbfb_result {
    int status;              /* 0, or a negative code                              */
    int n, k, nrhs;
    long long singular;
    long long fallback;
    const int* ja;           /* DEVICE, n*k, resident until rbfb_server_release    */
    const double* values[RBFB_MAX_RHS]; /* DEVICE, n*k each                         */
    double submit_ms, start_ms, end_ms; /* host clock, relative to server creation  */
    double dev_start_ms, dev_end_ms;    /* device clock, same origin: when the request's
                                           kernels could start and when they finished
                                           (-1 until the request is done)             */
} rbfb_result;

int rbfb_server_create(rbfb_server** srv, int device, size_t hbm_budget_bytes, int max_slots);
int rbfb_server_submit(rbfb_server* srv, const rbfb_request* req, long long* ticket);
/* wait_ms < 0: block; 0: poll (RBFB_EBUSY while running); > 0: bounded wait
 * (RBFB_ETIMEOUT when it runs out). */
int rbfb_server_poll(rbfb_server* srv, long long ticket, int wait_ms, rbfb_result* res);
/* Copies a finished request's weights (and stencils if ja_h != NULL) to host. */
int rbfb_server_fetch(rbfb_server* srv, long long ticket, int* ja_h, double* const* values_h);
int rbfb_server_release(rbfb_server* srv, long long ticket);
int rbfb_server_destroy(rbfb_server* srv);
/* Bytes of device memory currently held by admitted requests. */
size_t rbfb_server_resident_bytes(const rbfb_server* srv);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#ifdef __CUDACC__
/* The reference's C-ABI kernel symbol, same signature
 * (src/rbf_operators.cpp:7): launch <<<1, 32>>>. */
extern "C" __global__ void solve_dp(double* A, int* ipiv, double* B, int* info);
#endif

#endif /* RBF_B200_H */
