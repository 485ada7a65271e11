/*
 * fiber3d_b200 — C ABI of the B200 (sm_100a) hydrodynamic hot path of fiber3d.
 *
 * Every entry point takes plain device pointers, element counts and a CUDA
 * stream (passed as void*; NULL = legacy default stream), launches
 * asynchronously on that stream and returns an f3d_status.  No entry point
 * allocates device memory: kernels that need scratch space take a caller
 * workspace whose size is returned by the matching *_workspace_bytes query.
 * A workspace must be zero-filled once when it is allocated; the kernels
 * leave its counter words at zero when they finish.
 *
 * Layout conventions follow python/kernels/kernels.py of fiber3d: points,
 * densities and normals are float64 arrays of shape (N, 3), row-major,
 * xyz-interleaved; outputs are flat float64 arrays of length 3*Nt.
 *
 * Device-side failures (a bounded wait that ran out) are recorded in a
 * per-device error word that f3d_get_device_error() reads and clears.
 */
#ifndef FIBER3D_B200_H
#define FIBER3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
typedef enum f3d_status {
  F3D_OK = 0,
  F3D_ERR_NULL = 1,          /* a required pointer is NULL                 */
  F3D_ERR_SHAPE = 2,         /* negative or inconsistent sizes             */
  F3D_ERR_ALIGN = 3,         /* a pointer is not 8-byte aligned            */
  F3D_ERR_WORKSPACE = 4,     /* workspace missing or too small             */
  F3D_ERR_ARG = 5,           /* unknown enum value / bad launch shape      */
  F3D_ERR_CUDA = 6,          /* a CUDA runtime call failed                 */
  F3D_ERR_NONFINITE = 7,     /* non-finite input detected (checking on)    */
  F3D_ERR_TIMEOUT = 8,       /* device-side bounded wait ran out           */
  F3D_ERR_SINGULAR = 9,      /* zero pivot in an LU factorisation          */
  F3D_ERR_TOO_LARGE = 10     /* size beyond a documented maximum           */
} f3d_status;

/* ---- enums ------------------------------------------------------------- */
typedef enum f3d_kernel {
  F3D_KERNEL_OSEEN = 0,      /* u_t = 1/(8 pi eta) sum_s [f/r + (r.f) r / r^3]      */
  F3D_KERNEL_STRESSLET = 1,  /* v_t = -3/(4 pi eta) sum_s (r.d)(r.n) r / r^5        */
  F3D_KERNEL_ROTLET = 2,     /* u_t = 1/(8 pi eta) sum_s tau x r / r^3              */
  F3D_KERNEL_TRACTION = 3    /* t_t = -3/(4 pi eta) sum_s (r.d_s)(r.n_t) r / r^5:
                                the normal is the TARGET's (kernels.py:1221-1264);
                                `normal` then holds nt target normals             */
} f3d_kernel;

typedef enum f3d_self_mode {
  /* every pair is summed; a pair with |r| < eps uses sqrt(r^2 + reg^2)
     (kernels.py:794-846, 856-908, 1186-1217)                                */
  F3D_SELF_REGULARISE = 0,
  /* the sources are the first ns targets (nt >= ns); the pair j == i is
     skipped, any other pair with |r| < eps is regularised (kernels.py:
     214-287, 1123-1183).  Targets past ns skip nothing.                     */
  F3D_SELF_SKIP_INDEX = 1,
  /* pairs whose int32 group ids are equal are skipped (same fiber);
     others are regularised as in F3D_SELF_REGULARISE. This fuses
     flow_fibers + self_flow_fibers (tstep/tstep_utils.py:653-700, 812-851) */
  F3D_SELF_SKIP_GROUP = 2,
  /* pairs with |r| < eps contribute exactly zero; no regularisation (the
     PyCUDA Oseen kernel, kernels/kernels_pycuda.py:22-66; with a tiny eps,
     the coincident-point exclusion of the STKFMM sums, kernels.py:1298-1485) */
  F3D_SELF_SKIP_CLOSE = 3
} f3d_self_mode;

typedef enum f3d_precision {
  F3D_FP64 = 0,              /* IEEE float64 everywhere                               */
  F3D_FP32C = 1              /* float32 pair terms from double-float coordinate
                                differences; float32 per-tile sums folded into a
                                two-sum (compensated) per-target accumulator; the
                                result is written as float64                         */
} f3d_precision;

/* Launch shape of a pair kernel.  All-zero means "library default". */
typedef struct f3d_pair_shape {
  int32_t tpt;     /* targets per thread: 1, 2 or 4 (4: FP64 only)           */
  int32_t sl;      /* source lanes per target group: 1, 8 or 32; or -1: the
                      symmetric form of a sum over one point set (each
                      unordered pair evaluated once, both directions
                      summed): FP64 Oseen or stresslet, F3D_SELF_SKIP_INDEX
                      or F3D_SELF_SKIP_GROUP, r_target the r_source pointer
                      itself (the sources are its first ns points; targets
                      past ns are summed one-sided in the same launch) and,
                      for SKIP_GROUP, trg_group the src_group pointer.
                      Its workspace holds 3072 T (T + T2) bytes of
                      partial sums, T = ceil(ns / 128), T2 =
                      ceil((nt - ns) / 128) (twice that for the
                      two-density Oseen pass), at most 2 GiB, and
                      T <= 1024 (131072 sources).  tpt, nsplit and
                      use_tma are then ignored.
                      Or -2: the tile form of a source -> target sum (the
                      symmetric kernel's target-side items: 128-point
                      tiles, two targets per thread, per-tile partials
                      summed in a fixed order): FP64 Oseen or stresslet,
                      F3D_SELF_REGULARISE; nsplit 1 (or 0) or 2 takes
                      the sources in tiles of 128 or 64 points (64:
                      twice the items, for sums too small to fill the
                      GPU); workspace 3072 S T2 bytes, S =
                      ceil(ns / 128) or ceil(ns / 64), T2 = ceil(nt /
                      128), ns <= 131072, at most 2 GiB (twice for the
                      two-density Oseen pass).                              */
  int32_t nsplit;  /* source splits (grid.y); 0 = derive from the SM count    */
  int32_t use_tma; /* 0 or 1: stage full source tiles with cp.async.bulk
                      (default); -1: stage them with plain loads            */
} f3d_pair_shape;

/* ---- library ----------------------------------------------------------- */
const char *f3d_version(void);
const char *f3d_status_string(int status);
/* Reads and clears the device error word of the current device (blocks on
   the given stream).  Returns F3D_OK or F3D_ERR_TIMEOUT. */
int f3d_get_device_error(void *stream);
/* Queues a copy of the device error word into *host_dst on `stream` without
   waiting and without clearing it (host_dst page-locked for the copy to be
   asynchronous).  After the stream has synchronised, a non-zero value means
   a kernel failed; f3d_get_device_error then reads and clears it.  Lets a
   caller that synchronises anyway (to read its results) check for failures
   in the same wait. */
int f3d_peek_device_error_async(int *host_dst, void *stream);

/* Bounded waits.  Every kernel that waits on an mbarrier (a bulk copy or a
   tensor-core MMA landing) gives up after a limit, records F3D_ERR_TIMEOUT in
   the device error word and returns, so the context stays usable.
   f3d_set_wait_limit_ns sets the limit that later calls pass to their
   kernels (0 restores the default, 2 s); f3d_wait_limit_ns reads it.
   No counterpart in fiber3d (its kernels run on the CPU). */
int f3d_set_wait_limit_ns(uint64_t limit_ns);
uint64_t f3d_wait_limit_ns(void);

/* Self-test of the bounded wait: one CTA waits, for limit_ns (1 ns .. 2 s),
   on an mbarrier that nothing arrives on (no copy is issued), then records
   F3D_ERR_TIMEOUT in the device error word.  It exercises the timeout
   reporting path without any fault.  No counterpart in fiber3d. */
int f3d_selftest_bounded_wait(uint64_t limit_ns, void *stream);

/* Launches an FMA-throughput probe (precision F3D_FP64 or F3D_FP32C = FP32;
   2 = FP64 tensor-core MMA, mma.sync m16n8k16) on `stream`; *flops receives
   the floating-point operations it performs (an FMA counts 2).  Timing it gives the measured pipe peak used as the
   roofline denominator of the pair kernels.  `sink` is an 8-byte device
   scratch word that is written only in a case that never occurs. */
int f3d_probe_fma(int precision, int iters, double *sink, double *flops, void *stream);

/* ---- all-pairs sums (A1, A2, A3, A4, A6) -------------------------------- */

/* Workspace bytes needed by f3d_pair_sum for these sizes and launch shape. */
int f3d_pair_workspace_bytes(int kernel, int precision, int64_t ns, int64_t nt,
                             const f3d_pair_shape *shape, size_t *bytes);

/* General source->target sum.  `normal` is read only for the stresslet.
   `src_group`/`trg_group` are read only for F3D_SELF_SKIP_GROUP.
   For F3D_SELF_SKIP_INDEX, the first ns points of r_target must be the
   sources (nt >= ns).  If `accumulate` is non-zero the result is added to `out`,
   otherwise `out` is overwritten. */
int f3d_pair_sum(int kernel, int precision, int self_mode,
                 const double *r_source, const double *r_target,
                 const double *density, const double *normal,
                 const int32_t *src_group, const int32_t *trg_group,
                 double *out, int64_t ns, int64_t nt,
                 double eta, double reg, double epsilon_distance,
                 int accumulate, const f3d_pair_shape *shape,
                 void *workspace, size_t workspace_bytes, void *stream);

/* The same sum from HOST memory in one call, for host-side bindings (the
   numpy-in, numpy-out functions of fiber3d's kernels.kernels,
   python/kernels/kernels.py:214-1264): r_source (ns x 3), r_target (nt x 3;
   pass the r_source pointer itself for a sum over one point set, whose
   max(ns, nt) points are then copied once), density (ns x 3), normal (stresslet: ns x 3 source
   normals; traction: nt x 3 target normals; else NULL) are copied to
   `device_buffer` (f3d_pair_host_bytes of them, 256-byte aligned), the sum
   runs on `stream` with `workspace` as f3d_pair_sum's, the result is copied
   into `out` (nt x 3, host) and the stream is synchronised.  Page-locked
   host buffers that the device can address (cudaHostAlloc, or
   cudaHostRegister under unified addressing) skip the copies: when every
   input is one, a single staging kernel reads them all, and such an `out`
   (8-byte aligned) is written by the pair kernel itself.  Other host
   memory is copied with cudaMemcpyAsync.  Returns F3D_OK, an argument
   status, or the first status a kernel recorded in the device error word
   (then cleared), e.g. F3D_ERR_TIMEOUT.  F3D_SELF_SKIP_GROUP is not
   accepted (no group ids on this path). */
int f3d_pair_host_bytes(int kernel, int64_t ns, int64_t nt, int same_points, size_t *bytes);
int f3d_pair_sum_host(int kernel, int precision, int self_mode, const double *r_source,
                      const double *r_target, const double *density, const double *normal, double *out,
                      int64_t ns, int64_t nt, double eta, double reg, double epsilon_distance,
                      const f3d_pair_shape *shape, void *device_buffer, size_t device_bytes,
                      void *workspace, size_t workspace_bytes, void *stream);

/* Resident CTAs per SM of the pair kernel that a sum of this kernel,
   precision, self mode (dual: the two-density FP64 Oseen pass) and launch
   shape would run (cudaOccupancyMaxActiveBlocksPerMultiprocessor), so that
   a tuner can size the source split to whole waves.  Launches nothing.
   No counterpart in fiber3d. */
int f3d_pair_occupancy(int kernel, int precision, int self_mode, int dual,
                       const f3d_pair_shape *shape, int *ctas_per_sm);

/* The same sum for callers that cannot allocate device memory (no workspace
   argument).  No counterpart in fiber3d.  Its scratch is a 32 MiB device
   array inside this library, held by every GPU that loads it until the
   process exits; sizes whose f3d_pair_workspace_bytes (default shape)
   exceeds 32 MiB return F3D_ERR_TOO_LARGE.  The first call on a device looks
   up that array's device address (make it before any stream capture).
   Each device has its own copy of the array, so calls on different devices
   never interfere; calls on the same device share it, and two of them that
   overlap on that GPU (different streams) race: order them on one stream.
   The cached address belongs to the device's current context: the library
   must not be used across a cudaDeviceReset of that device.  Allocates
   nothing. */
int f3d_pair_sum_noalloc(int kernel, int precision, int self_mode,
                         const double *r_source, const double *r_target,
                         const double *density, const double *normal,
                         const int32_t *src_group, const int32_t *trg_group,
                         double *out, int64_t ns, int64_t nt,
                         double eta, double reg, double epsilon_distance,
                         int accumulate, void *stream);

/* Two FP64 Oseen sums over the same sources, targets and self mode, with
   densities `density` -> `out` and `density2` -> `out2`, in one pass: each
   output carries exactly the arithmetic of f3d_pair_sum (F3D_KERNEL_OSEEN,
   F3D_FP64) with that density, the pair geometry being computed once.  No
   counterpart function in fiber3d; it evaluates in one pass the two Oseen
   sums a time step makes over the same fibers -- the explicit flow of the
   external forces (tstep.py:789-821) and the fiber forces of GMRES's initial
   guess in the first matvec (tstep.py:1003-1178).  Workspace from
   f3d_oseen_dual_workspace_bytes. */
int f3d_oseen_dual_workspace_bytes(int64_t ns, int64_t nt, const f3d_pair_shape *shape,
                                   size_t *bytes);
int f3d_oseen_dual(int self_mode, const double *r_source, const double *r_target,
                   const double *density, const double *density2, const int32_t *src_group,
                   const int32_t *trg_group, double *out, double *out2, int64_t ns, int64_t nt,
                   double eta, double reg, double epsilon_distance, int accumulate,
                   const f3d_pair_shape *shape, void *workspace, size_t workspace_bytes,
                   void *stream);

/* Named wrappers with the meaning of the fiber3d functions they replace. */

/* replaces oseen_kernel_source_target_numba, python/kernels/kernels.py:794-846 */
int f3d_oseen_source_target(const double *r_source, const double *r_target,
                            const double *density, double *u,
                            int64_t ns, int64_t nt, double eta, double reg,
                            double epsilon_distance, int precision,
                            void *workspace, size_t workspace_bytes, void *stream);

/* replaces oseen_kernel_times_density_numba, python/kernels/kernels.py:214-287 */
int f3d_oseen_times_density(const double *r_vectors, const double *density,
                            double *u, int64_t n, double eta, double reg,
                            double epsilon_distance, int precision,
                            void *workspace, size_t workspace_bytes, void *stream);

/* replaces rotlet_kernel_source_target_numba, python/kernels/kernels.py:856-908 */
int f3d_rotlet_source_target(const double *r_source, const double *r_target,
                             const double *density, double *u,
                             int64_t ns, int64_t nt, double eta, double reg,
                             double epsilon_distance, int precision,
                             void *workspace, size_t workspace_bytes, void *stream);

/* replaces stresslet_kernel_source_target_numba, python/kernels/kernels.py:1186-1217 */
int f3d_stresslet_source_target(const double *r_source, const double *r_target,
                                const double *normal, const double *density,
                                double *v, int64_t ns, int64_t nt, double eta,
                                double reg, double epsilon_distance, int precision,
                                void *workspace, size_t workspace_bytes, void *stream);

/* replaces stresslet_kernel_times_normal_times_density_numba,
   python/kernels/kernels.py:1123-1183 */
int f3d_stresslet_times_normal_times_density(const double *r_vectors,
                                             const double *normal,
                                             const double *density, double *v,
                                             int64_t n, double eta, double reg,
                                             double epsilon_distance, int precision,
                                             void *workspace, size_t workspace_bytes,
                                             void *stream);

/* ---- dense operator builders (A5 and friends) ---------------------------- */

/* replaces stresslet_kernel_times_normal_numba, python/kernels/kernels.py:1063-1120:
   M (3n x 3n, row-major, leading dimension ld >= 3n) with block
   S_ij = -3/(4 pi eta) (r.n_j)/|r|^5 r r^T, r = x_i - x_j, S_ii = 0. */
int f3d_stresslet_times_normal_dense(const double *r_vectors, const double *normal,
                                     double *M, int64_t n, int64_t ld, double eta,
                                     double reg, double epsilon_distance, void *stream);

/* replaces oseen_tensor (input_format 'r'), python/kernels/kernels.py:31-116:
   G (3n x 3n, row-major, ld >= 3n), block G_ij = f(r) I + g(r) r r^T with
   r = x_j - x_i, f = 1/(8 pi eta |r|), g = 1/(8 pi eta |r|^3); |r| <= eps is
   regularised (so the diagonal block is I/(8 pi eta reg)). */
int f3d_oseen_tensor_dense(const double *r_vectors, double *G, int64_t n, int64_t ld,
                           double eta, double reg, double epsilon_distance,
                           void *stream);

/* replaces oseen_tensor_source_target (input_format 'r'),
   python/kernels/kernels.py:119-211: G (3nt x 3ns, row-major, ld >= 3ns),
   block G_ts from r = x_s - x_t with the regularisation of oseen_tensor. */
int f3d_oseen_tensor_source_target_dense(const double *r_source, const double *r_target,
                                         double *G, int64_t ns, int64_t nt, int64_t ld,
                                         double eta, double reg, double epsilon_distance,
                                         void *stream);

/* The 3-index stresslet tensor of N points (replaces stresslet_kernel,
   python/kernels/kernels.py:911-992, input_format 'r'; the Python drop-in
   reorders 'xyz' input): S is (3N) x (3N) x 3, row-major, S[3i+a, 3j+b, c] =
   fr dr_a dr_b dr_c, dr = x_j - x_i, fr = -3/(4 pi eta dr^5) when dr > eps,
   else -3/(4 pi eta (dr^2 + reg^2)^(5/2)).  N <= 65535. */
int f3d_stresslet_tensor_dense(const double *r_vectors, double *S, int64_t n, double eta, double reg,
                               double epsilon_distance, void *stream);

/* replaces complementary_kernel, python/kernels/kernels.py:1286-1295:
   C = outer(normal.flat, normal.flat), 3n x 3n, row-major, ld >= 3n. */
int f3d_complementary_dense(const double *normal, double *C, int64_t n, int64_t ld,
                            void *stream);

/* ---- batched LU for the block-diagonal preconditioner (A13) --------------- */

/* Workspace bytes of the batched LU factor/solve (two queue counters each). */
int f3d_batched_lu_workspace_bytes(size_t *bytes);

/* Factors `count` row-major square matrices of uneven size in place, in one
   persistent launch.  Matrix b has size sizes[b], starts at
   A + matrix_offsets[b] (leading dimension sizes[b]); its pivots go to
   piv + vector_offsets[b] (0-based: row i was swapped with row piv[i]) and
   info[b] is 0 or the 1-based index of the first zero pivot.  `order`
   (optional) is the processing order (largest first balances the queue);
   max_n >= every size.  Replaces scipy.linalg.lu_factor per block
   (tstep/tstep_utils.py:1405-1419 fibers, :1341-1386 bodies). */
int f3d_batched_lu_factor(double *A, const int64_t *matrix_offsets,
                          const int64_t *vector_offsets, const int32_t *sizes,
                          const int32_t *order, int32_t count, int32_t max_n,
                          int32_t *piv, int32_t *info, void *workspace,
                          size_t workspace_bytes, void *stream);

/* f3d_batched_lu_factor with an explicit panel width (columns factored in
   shared memory per step): 8, 16 or 32, or 0 for the size-based default. */
int f3d_batched_lu_factor_panel(double *A, const int64_t *matrix_offsets,
                                const int64_t *vector_offsets, const int32_t *sizes,
                                const int32_t *order, int32_t count, int32_t max_n,
                                int32_t panel, int32_t *piv, int32_t *info, void *workspace,
                                size_t workspace_bytes, void *stream);

/* Solves every factored system in place: x + vector_offsets[b] holds the
   right-hand side on entry and the solution on exit.  Replaces
   scipy.linalg.lu_solve per block in P_inv (tstep/tstep.py:950-994). */
int f3d_batched_lu_solve(const double *LU, const int64_t *matrix_offsets,
                         const int64_t *vector_offsets, const int32_t *sizes,
                         const int32_t *order, int32_t count, int32_t max_n,
                         const int32_t *piv, double *x, void *workspace,
                         size_t workspace_bytes, void *stream);

/* Replaces every block of the packed buffer by its inverse (Gauss-Jordan with
   partial pivoting, one launch; same layout as f3d_batched_lu_factor), and
   when A32 is non-null also writes an FP32 copy at the same offsets.
   info[b] is 0 or the 1-based step of the first zero (or subnormal) pivot.
   Pivoting takes a row whose |a_pk| is within a factor 1 - 2^-20 of the
   column maximum (the first such row; blocks of more than 32 rows: within
   2^-16, on the FP64 tensor cores by blocked Gauss-Jordan).  max_n <= 128
   (else F3D_ERR_TOO_LARGE: use the LU).  With f3d_block_gemv this evaluates
   the fiber blocks of P_inv (tstep/tstep.py:950-994) as products with the
   explicit block inverses instead of per-block lu_solve. */
int f3d_batched_inverse(double *A, const int64_t *matrix_offsets, const int32_t *sizes,
                        int32_t count, int32_t max_n, float *A32, int32_t *info, void *stream);

/* Explicit inverse of one dense FP64 matrix, in place: blocked Gauss-Jordan
   elimination over 128-row blocks, each step an FP64 GEMM of rank 128 over
   the whole matrix (2 n^3 flops, as LU plus inversion), partial pivoting
   inside each 128 x 128 pivot block (no row exchange between blocks: stable
   for the second-kind operators inverted here, whose diagonal blocks carry
   the 1/w-scaled identity).  Replaces scipy.linalg.lu_factor of the dense
   shell operator (tstep/tstep.py:327-348) and of the rigid-body blocks
   (tstep/tstep_utils.py:1341-1386); the preconditioner then applies the
   inverse as a product.  A: row-major with leading dimension ld (even),
   at least np = n rounded up to a multiple of 128 rows of ld >= np
   doubles, 16-byte aligned, the matrix in its top-left n x n corner; the
   call sets the padding to the identity (which stays the identity) and
   leaves the inverse in the top-left corner.  workspace:
   f3d_dense_inverse_workspace_bytes(n, ld) bytes, 256-byte aligned.
   Synchronises `stream`.  F3D_ERR_SINGULAR when a pivot block is singular
   to working precision. */
int f3d_dense_inverse_workspace_bytes(int64_t n, int64_t ld, size_t *bytes);
int f3d_dense_inverse(double *A, int64_t n, int64_t ld, void *workspace, size_t workspace_bytes,
                      void *stream);

/* y + vector_offsets[b] = M_b (x + vector_offsets[b]) for every block, M_b
   row-major sizes[b] x sizes[b] at M + matrix_offsets[b]; M is double
   (F3D_FP64) or float (F3D_FP32C); x, y double, distinct.  FP64 sums. */
int f3d_block_gemv(int precision, const void *M, const int64_t *matrix_offsets,
                   const int64_t *vector_offsets, const int32_t *sizes, int32_t count,
                   int32_t max_n, const double *x, double *y, void *stream);

/* ---- fiber discretisation (A11, A12) ------------------------------------ */

/* A set of fibers on the device.  Points of all fibers are concatenated;
   fiber f has n[f] points starting at point pt_off[f], its 4n x 4n operator
   block at mat_off[f] (row-major) and its unknowns [X_x, X_y, X_z, T] at
   4*pt_off[f].  `mats` holds, per resolution N, the block
   [D1_0, D2_0, D3_0, D4_0 (N x N each, finite differences on
   alpha = linspace(-1,1,N)), P_X ((N-4) x N), P_T ((N-2) x N), w0 (N)]
   (tstep/fiber_matrices.py:38-104); res_off[f] is the offset of fiber f's
   block.  bc holds 4 codes per fiber (start translation, start rotation,
   end translation, end rotation): 0 force, 1 torque, 2 velocity,
   3 angular_velocity.  band = half-width of the finite-difference stencils
   (n_fd + 3). */
typedef struct f3d_fiber_set {
  int32_t nfib;
  const int32_t *n;
  const int64_t *pt_off;
  const int64_t *mat_off;
  const int64_t *res_off;
  const double *length;
  const int32_t *bc;
  const int32_t *pt_fib;   /* fiber index of every point */
  const double *mats;
  int32_t band;
} f3d_fiber_set;

/* geo[9p..9p+8] = (xs, xss, xsss) at every point p (D_k x, tstep.py:703-709). */
int f3d_fiber_geometry(const f3d_fiber_set *set, const double *x, double *geo,
                       int64_t npts, void *stream);

/* Per-fiber [P_cheb A; B] and [P_cheb RHS; B_RHS]: fiber.form_linear_operator,
   compute_RHS and apply_BC_rectangular (fiber/fiber.py:322-448, 473-582,
   810-961) with flow = background velocity on the fiber and force = external
   force per point.  Writes the blocks to A (and A_copy if non-NULL). */
int f3d_fiber_assemble(const f3d_fiber_set *set, double E, double dt, double c0,
                       double c1, double penalty, const double *x, const double *geo,
                       const double *flow, const double *force, double *A,
                       double *A_copy, double *rhs, int32_t max_n, void *stream);

/* fw = w * (-E X_ssss + xss T + xs T_s) from the fiber unknowns XT
   (fiber.force_operator, fiber/fiber.py:1399-1432, times the trapezoid
   weights of flow_fibers, tstep_utils.py:653-700, when weighted != 0). */
int f3d_fiber_forces(const f3d_fiber_set *set, double E, const double *geo,
                     const double *XT, double *fw, int64_t npts, int weighted,
                     void *stream);

/* fw = w * f: external point forces times the trapezoid weights. */
int f3d_fiber_weight(const f3d_fiber_set *set, const double *f, double *fw,
                     int64_t npts, void *stream);

/* Fiber rows of the matvec: res = A XT - [P_cheb [v; xs . D1 v]; 0]
   (tstep/tstep.py:1147-1173) with v the velocity on the fiber points. */
int f3d_fiber_residual(const f3d_fiber_set *set, const double *A, const double *geo,
                       const double *XT, const double *v, double *res, int32_t max_n,
                       void *stream);

/* ---- surfaces: periphery (shell) and rigid bodies (A7, body rows) ------- */

/* Workspace bytes of f3d_singularity_vectors for n nodes. */
int f3d_singularity_vectors_workspace_bytes(int64_t n, size_t *bytes);

/* Singularity-subtraction vectors e_c(i) = sum_{j != i} S_ij w_j e_c of one
   surface (periphery.get_singularity_subtraction_vectors,
   periphery/periphery.py:75-98; body.calc_vectors_singularity_subtraction,
   body/body.py:325-346), stored as E[9i + 3a + c] = e_c(i)_a. */
int f3d_singularity_vectors(const double *nodes, const double *normals,
                            const double *weights, double *E, int64_t n, double eta,
                            double reg, double epsilon_distance, void *workspace,
                            size_t workspace_bytes, void *stream);

/* Shell rows of the matvec (tstep/tstep.py:1097-1104 with the matrices of
   tstep.py:327-347): res_i = v_i - E_i mu_i - mu_i + n_i sum_j n_j.q_j,
   mu = q / w, where v already holds the double-layer sum of q (and every
   other source) at the shell nodes.  `scratch` is one device double. */
int f3d_shell_residual(const double *v, const double *E, const double *weights,
                       const double *normals, const double *q, double *res, int64_t n,
                       double *scratch, void *stream);

/* y_i = B_i x_i for n row-major 3 x 3 blocks (B: 9n doubles; x, y: 3n,
   distinct).  Applies the block-diagonal (node-local) periphery
   preconditioner, the inverses of the 3 x 3 diagonal blocks of the dense
   shell operator of tstep/tstep.py:327-347: a matrix-free alternative to
   its LU (tstep.py:348) for peripheries whose dense inverse does not fit. */
int f3d_block3_gemv(const double *B, const double *x, double *y, int64_t n, void *stream);

/* Binv (9n doubles, row-major 3 x 3 blocks) = the inverses of those diagonal
   blocks, B_i = -(E_i + I) / w_i + n_i n_i^T (E: 9n singularity vectors as
   f3d_singularity_vectors writes them; weights n; normals 3n), by adjugate
   over determinant.  When info (one device int32, zeroed by the caller) is
   non-NULL, every block whose determinant is zero or not finite adds 1. */
int f3d_shell_block_inverse(const double *E, const double *weights, const double *normals, double *Binv,
                            int64_t n, int32_t *info, void *stream);

/* Rigid-body rows of the matvec (tstep/tstep.py:1118-1143): for body b with
   unknowns x[x_off[b]..] = [lambda (3nb), U, Omega]:
   res = v - E mu - (U + Omega x r) on the nodes and -K^T lambda + (U, Omega). */
int f3d_body_residual(int32_t nbody, const int64_t *node_off, const int64_t *x_off,
                      const double *nodes, const double *centers, const double *E,
                      const double *weights, const double *v, const double *x, double *res,
                      void *stream);

/* Dense preconditioner block of a surface.  mode 0 (periphery, 3n x 3n):
   S - blockdiag(E_i/w_i + I/w_i) + n n^T (tstep/tstep.py:327-347).
   mode 1 (rigid body, (3n+6)^2): [[S - blockdiag(E_i/w_i), -K], [-K^T, I]]
   (tstep/tstep_utils.py:1341-1386), K = [I, rot] about `center`. */
int f3d_surface_dense(int mode, const double *nodes, const double *normals, const double *E,
                      const double *weights, const double *center, double *M, int64_t n,
                      int64_t ld, double eta, double reg, double epsilon_distance,
                      void *stream);

/* Rigid bodies at a new location/orientation (tstep.py:1392-1407 moves them;
   body.get_r_vectors / get_normals give the surfaces): node i of body
   b = body_of[i] gets nodes = R_b ref_nodes + loc_b, normals = R_b
   ref_normals and, when ref_E/E are non-NULL, E_i = R_b E_ref,i R_b^T (the
   singularity vectors of the rotated surface; 9 per node as
   f3d_singularity_vectors writes them).  R: nbody row-major 3 x 3. */
int f3d_rigid_body_update(const int32_t *body_of, const double *R, const double *loc,
                          const double *ref_nodes, const double *ref_normals, const double *ref_E,
                          int64_t nnodes, double *nodes, double *normals, double *E, void *stream);

/* Rigid-body time-step update on the device (tstep/tstep.py:1399-1407,
   quaternion/quaternion.py:14-53): body b's velocities are U = sol[vel_off[b]
   .. +3) and Omega = sol[vel_off[b]+3 .. +6); loc_b += dt U, quat_b <-
   q(dt Omega) quat_b (Hamilton product; quaternions (s, p1, p2, p3)) and
   R_b = R(quat_b), row-major.  loc (nbody x 3) and quat (nbody x 4) are the
   bodies' state, read and written; R (nbody x 9) is written. */
int f3d_body_advance(const double *sol, const int64_t *vel_off, int32_t nbody, double dt, double *loc,
                     double *quat, double *R, void *stream);

/* ---- velocity field at grid points (fiber3d's compute_velocity,
   tstep/tstep.py:1273-1381, post-processing :1414-1448) ---------------------
   The sums are f3d_pair_sum source -> target calls; these three entries are
   the rest. */

/* Self-flow of each fiber at its own nodes with uprate-fold upsampled
   quadrature (tstep.py:1352-1357): with M = uprate * n equispaced nodes,
   x_up = P_up x, f_up = (P_up f) * w_up * (L/2), vself_i = sum_u
   G(x_up,u - x_i) f_up,u, G the Oseen tensor with 1/r, 1/r^3 (r >
   epsilon_distance) or sqrt(r^2 + reg^2) in place of r (kernels.py:119-200).
   up_mats + up_off[k]: P_up (M x n row-major) then the unit-length trapezoid
   weights w_up (M) of fiber k's resolution (fiber_matrices.py:84-92).  f:
   the unweighted fiber force per point (npts, 3); vself (npts, 3).
   6 * max_n * (1 + uprate) doubles must fit 48 KiB (F3D_ERR_TOO_LARGE). */
int f3d_fiber_self_flow_up(const int32_t *npts, const int64_t *pt_off, const double *length, int32_t nfib,
                           int32_t max_n, const double *x, const double *f, const double *up_mats,
                           const int64_t *up_off, int32_t uprate, double eta, double reg,
                           double epsilon_distance, double *vself, void *stream);

/* For each grid point (ngrid, 3): if some node of fiber k lies within
   `near` (distance formed as fiber3d forms it), the point takes vself at
   k's nearest node (first minimum); the last such fiber wins
   (tstep.py:1341-1365).  Other rows of vfib are left as they are. */
int f3d_grid_near_fiber(const double *grid, int64_t ngrid, const double *x, const int64_t *pt_off,
                        int32_t nfib, const double *vself, double near, double *vfib, void *stream);

/* Rigid motion inside a sphere (tstep.py:1438-1448): grid points with
   |g - center|^2 <= radius^2 get v = U + W x (g - center), uw = (U, W). */
int f3d_grid_rigid_override(const double *grid, int64_t ngrid, const double *center, const double *uw,
                            double radius, double *v, void *stream);

/* Rigid-body frame change of preconditioner vectors: for body b the nvec[b]
   3-vectors at x + offsets[b] become R_b v (transpose 0) or R_b^T v
   (transpose 1), R_b row-major at R + 9b.  With the body block factored
   once in the body frame this applies the body preconditioner as fiber3d's
   precompute_body_PC path does (tstep/tstep.py:966-981, 227-252). */
int f3d_rotate_blocks(double *x, const int64_t *offsets, const int32_t *nvec, const double *R,
                      int32_t nbody, int transpose, void *stream);

/* dst[seg_dst[s] + k] = src[seg_src[s] + k] for k < seg_len[s] (max_len >= all). */
int f3d_gather_segments(const double *src, double *dst, const int64_t *seg_src,
                        const int64_t *seg_dst, const int64_t *seg_len, int32_t nseg,
                        int64_t max_len, void *stream);

/* ---- Krylov (GMRES) building blocks (A14) and the dense preconditioner ---- */
/* Replace scipy.sparse.linalg.gmres behind bpm_utilities/gmres.py:9-111.
   V is the Krylov basis, row-major, one vector of length n per row (ldv >= n).
   `k` points to a device int32: the number of basis rows in use, so that one
   captured CUDA graph serves every Arnoldi step.  kmax <= 256. */

int f3d_krylov_workspace_bytes(int64_t n, int32_t kmax, size_t *bytes);

/* h[i] (+)= V[i] . w for i < *k (two stages, fixed summation order). */
int f3d_krylov_multidot(const double *V, int64_t ldv, const double *w, const int32_t *k,
                        int32_t kmax, double *h, int64_t n, int accumulate,
                        void *workspace, size_t workspace_bytes, void *stream);

/* w -= sum_{i < *k} h[i] V[i]. */
int f3d_krylov_multiaxpy(const double *V, int64_t ldv, const double *h, const int32_t *k,
                         double *w, int64_t n, void *stream);

/* y (+)= sum_{i < k} c[i] V[i] (k given by value). */
int f3d_krylov_combine(const double *V, int64_t ldv, const double *c, int32_t k, double *y,
                       int64_t n, int accumulate, void *stream);

/* *beta = |w|_2; if hcol is non-NULL also hcol[*k] = |w|_2.  Workspace >= 2 KiB. */
int f3d_krylov_norm(const double *w, int64_t n, const int32_t *k, double *hcol,
                    double *beta, void *workspace, size_t workspace_bytes, void *stream);

/* Row (*k + offset) of dst (leading dimension ld) = src, n entries (the
   preconditioned basis vector z_k = P^-1 v_k kept for the update
   x += Z y; a negative row is skipped). */
int f3d_krylov_store(const double *src, const int32_t *k, int32_t offset, double *dst,
                     int64_t ld, int64_t n, void *stream);

/* V[*k] = w / *beta (zero if beta == 0) and also into `also` if non-NULL,
   then *k += 1 if bump. */
int f3d_krylov_scale_into(const double *w, const double *beta, int32_t *k, double *V,
                          int64_t ldv, int64_t n, int bump, double *also, void *stream);

/* count square FP64 products in one launch: y[y_off[b] ..] = M_b x[x_off[b] ..]
   with M_b the n[b] x n[b] row-major matrix at M + m_off[b] (offsets in
   doubles, device arrays; max_n >= every n[b]).  vec = 1 reads 16-byte
   pairs: every m_off[b] and n[b] even and M 16-byte aligned.  Applies the
   body-frame inverses of all rigid bodies' preconditioner blocks at once
   (fiber3d's A_inv_bodies, tstep/tstep.py:966-981). */
int f3d_gemv_batched(const double *M, const int64_t *m_off, const int64_t *n, const int64_t *x_off,
                     const int64_t *y_off, int32_t count, int64_t max_n, int vec, const double *x, double *y,
                     void *stream);

/* y = M x for a row-major rows x cols matrix stored as float64
   (precision F3D_FP64) or float32 (F3D_FP32C); the sum is float64.  Applies
   the explicit inverse of the periphery operator (tstep/tstep.py:957-958). */
int f3d_gemv(int precision, const void *M, int64_t ld, const double *x, double *y,
             int64_t rows, int64_t cols, void *stream);

/* FP16 copy of a row-major matrix for f3d_gemv_f16: row r is divided by
   row_scale[r], the smallest power of two >= max |M[r][c]| over the columns
   outside r's diagonal block, and rounded to FP16.  With diag_block = db > 0
   (square M, rows % db == 0) the entries of the db x db diagonal block that
   holds row r stay FP64 in diag[r*db + c] (zero in M16). */
int f3d_quantize_rows_f16(const double *M, int64_t ld, int64_t rows, int64_t cols,
                          int32_t diag_block, void *M16, int64_t ld16, float *row_scale,
                          double *diag, void *stream);

/* y = diag(row_scale) M16 x + blockdiag(diag) x for the output of
   f3d_quantize_rows_f16 (FP32 products and sums, FP64 result): the
   periphery preconditioner of the mixed-precision inner solves, read at
   2 bytes per entry. */
int f3d_gemv_f16(const void *M16, int64_t ld16, const float *row_scale, const double *diag,
                 int32_t diag_block, const double *x, double *y, int64_t rows, int64_t cols,
                 void *stream);

/* b = (float) a, elementwise. */
int f3d_cast_to_float(const double *a, float *b, int64_t n, void *stream);

/* ---- learned warm start: tensor-core GEMM and training kernels ----------- */
/* No counterpart in fiber3d (its GMRES always starts from zero,
   tstep/tstep.py:1209).  C (fp32, M x N, ldc) = alpha * A B^T on the 5th-gen
   tensor cores (tcgen05, BF16 operands rounded from the fp32 inputs, FP32
   accumulation in tensor memory).  Element (m, k) of A is
   A[m*a_rs + k*a_cs]; element (n, k) of B is B[n*b_rs + k*b_cs].  Optional
   epilogue: + bias[n], copy to pre[m*ldc+n], ReLU, multiply by
   (mask_src[m*ldm+n] > 0); accumulate adds into C.  N must be a multiple of
   16 and at most 256. */
int f3d_gemm_bf16(const float *A, int64_t a_rs, int64_t a_cs, const float *B, int64_t b_rs,
                  int64_t b_cs, float *C, int64_t ldc, int32_t M, int32_t N, int32_t K,
                  const float *bias, int relu, const float *mask_src, int64_t ldm, float *pre,
                  float alpha, int accumulate, void *stream);

/* Warm-start input for the per-fiber network from the last four solutions
   h0 (oldest) .. h3 (newest) of length n, fibers of npts = 32 points whose
   blocks start at o_fib (fiber3d's layout): per fiber 4 npts + 4 floats
   (second and third differences of positions and tensions, scaled by the
   RMS second difference, and four log10 ratios of difference RMS), each
   standardised as (v - mean[j]) / stdev[j] when mean/stdev are non-NULL;
   scale_x/scale_t receive the RMS second differences (the output units). */
int f3d_warmstart_features(const double *h0, const double *h1, const double *h2, const double *h3,
                           int64_t n, int64_t o_fib, int32_t nfib, int32_t npts, const float *mean,
                           const float *stdev, float *feats, double *scale_x, double *scale_t,
                           void *stream);

/* x0 = 3 h3 - 3 h2 + h1 (quadratic extrapolation) plus, when corr is
   non-NULL, the network's correction corr[f][k] (4 npts per fiber, rows X_x,
   X_y, X_z, T) times scale_x[f] (positions) or scale_t[f] (tensions) on
   fiber block f. */
int f3d_warmstart_guess(const double *h1, const double *h2, const double *h3, int64_t n,
                        int64_t o_fib, int32_t nfib, int32_t npts, const float *corr,
                        const double *scale_x, const double *scale_t, double *x0, void *stream);

/* out[n] (+)= sum_m G[m*ld + n]. */
int f3d_colsum(const float *G, int64_t ld, int32_t M, int32_t N, float *out, int accumulate,
               void *stream);

/* One bias-corrected Adam update of n fp32 parameters (step counts from 1). */
int f3d_adam(float *p, const float *g, float *m, float *v, int64_t n, float lr, float beta1,
             float beta2, float eps, int32_t step, void *stream);

/* D = 2 (Y - T) / (M N) and row_loss[m] = sum_n (Y - T)^2. */
int f3d_mse_grad(const float *Y, const float *T, float *D, float *row_loss, int32_t M, int32_t N,
                 void *stream);

/* ---- surface quadrature (set-up) ------------------------------------------
   Replaces Smooth_Closed_Surface_Quadrature_RBF(nodes, triangles, h, gradh)
   (python/quadratures/Smooth_Closed_Surface_Quadrature_RBF.py:3-470), the
   branch with the exact surface gradient that every fiber3d caller takes
   (tstep/tstep.py:297-300, body/body.py:104-107): phs RBF r^7 plus degree-7
   polynomials on the 80 nodes nearest each triangle, projected onto the
   triangle's plane.  nodes (n x 3), gradient (n x 3, gradh at the nodes),
   triangles (ntri x 3, any vertex order; a closed surface, every edge shared
   by exactly two triangles) -> weights (n).  neighbors (ntri x 80, nearest
   first) receives each triangle's nodes when non-NULL.  80 <= n <=
   715827882 (INT32_MAX / 3: node coordinates are indexed in 32-bit
   arithmetic), 1 <= ntri <= 2^24; larger n returns F3D_ERR_TOO_LARGE.
   Bad triangulations and zero pivots are reported through the device error
   word (F3D_ERR_ARG, F3D_ERR_SINGULAR; f3d_get_device_error). */
int f3d_surface_quadrature_workspace_bytes(int64_t n, int64_t ntri, size_t *bytes);
int f3d_surface_quadrature(const double *nodes, int64_t n, const int32_t *triangles, int64_t ntri,
                           const double *gradient, double *weights, int32_t *neighbors, void *workspace,
                           size_t workspace_bytes, void *stream);

/* ---- fast multipole method: the STKFMM PVel sums (kernels.py:1298-1485) --
   fiber3d's useFMM path (tstep/tstep.py:116-137) evaluates its Stokeslet
   (single layer) and stresslet (double layer) sums with the external STKFMM
   library (kernel-independent FMM, PVel kernel).  These entries are this
   library's own KIFMM on one GPU with the same inputs and outputs (velocity
   only): a uniform octree of depth 2..8, equivalent densities (Stokeslet +
   potential source) on cube surfaces of `order` points per edge, the
   near field (27 neighbour leaves) summed directly with coincident points
   (|r| < 1e-150) excluded, as STKFMM's kernels exclude them.
   All point and value arrays are device memory of the device that was
   current at f3d_fmm_create, which must be current for every call on the
   handle; the handle allocates its tree and expansions there itself
   (cudaMalloc in set_points / evaluate, kept for reuse) and frees them in
   f3d_fmm_destroy.  A handle is not safe for concurrent calls: give each
   host thread or stream its own.                                          */
typedef struct f3d_fmm f3d_fmm;

/* A handle for expansions of `order` (even, 4..16; n = 6 (order - 1)^2 + 2
   surface points) and leaves of about `max_pts` sources.  `surface` (n x 3:
   the unit cube's surface points of the order grid), `uc2ue` and `dc2de`
   (4n x 3n each, row-major: the pseudo-inverses that map a check potential
   on the surface at 2.95 (upward) or 1.05 (downward) half-widths to an
   equivalent density on the surface at 1.05 or 2.95) are host arrays the
   caller computes once per order (fiber3d_b200/fmm.py).  STKFMM(order,
   max_pts, ...) of the reference.                                         */
int f3d_fmm_create(int order, int max_pts, const double *surface, const double *uc2ue, const double *dc2de,
                   f3d_fmm **fmm);
int f3d_fmm_destroy(f3d_fmm *fmm);
/* The tree's cube: lower corner lo[3] and side `width` (stkfmm.setBox);
   every point must lie inside it.  Without it set_points takes the
   bounding cube of all points with a 10 % margin per side
   (kernels.py:1339-1348).                                                */
int f3d_fmm_set_box(f3d_fmm *fmm, const double *lo, double width);
/* Single-layer sources (nsl x 3), double-layer sources (ndl x 3) and
   targets (ntrg x 3); sorts them into the tree (stkfmm.setPoints +
   setupTree).  Counts up to 2^31 - 1 each.                               */
int f3d_fmm_set_points(f3d_fmm *fmm, int64_t nsl, const double *src_sl, int64_t ndl, const double *src_dl,
                       int64_t ntrg, const double *trg, void *stream);
/* out (ntrg x 3) = [single layer of sl_density (nsl x 3, forces) + double
   layer of the tensors D (ndl x 9, D_jk per source, the STKFMM layout; or,
   when dl_tensor is NULL, D = 2 n (x) d from dl_normal and dl_density,
   ndl x 3 each, fiber3d's convention at kernels.py:1410)] / eta:
   u_i = sum f_j / (8 pi) (delta_ij / r + r_i r_j / r^3)
         - 3 / (8 pi) sum r_i (r^T D r) / r^5,  r = target - source
   (stkfmm.evaluateFMM, velocity components).                             */
int f3d_fmm_evaluate(f3d_fmm *fmm, const double *sl_density, const double *dl_normal, const double *dl_density,
                     const double *dl_tensor, double *out, double eta, void *stream);
/* The tree of the last set_points: depth, non-empty source and target
   leaves, box (lo[3], width), and the number of non-empty entries of all
   target boxes' interaction lists (each one 3n x 4n block product of the
   far field); any output pointer but depth may be NULL.                   */
int f3d_fmm_tree_info(const f3d_fmm *fmm, int *depth, int64_t *src_leaves, int64_t *trg_leaves, double *box,
                      int64_t *m2l_pairs);
/* Kernels the last f3d_fmm_evaluate launched (for launch accounting). */
int f3d_fmm_last_launches(const f3d_fmm *fmm, int *launches);

#ifdef __cplusplus
}
#endif
#endif /* FIBER3D_B200_H */
