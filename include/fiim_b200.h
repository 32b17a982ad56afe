/* fiim_b200.h — C-ABI of the B200 (sm_100a) solve phase for factored approximate
 * inverse preconditioned BiCGSTAB, z = G * D^{-1} * (H * r).
 *
 * The reference (cfilelispapadopoulos/Computational-Mathematics) exports the solve phase
 * as C++ free functions linked from lib*.so with MKL underneath; it has no C or
 * foreign-function binding. Each entry point below replaces one of those functions,
 * with the same argument meaning, the same in/out convention (caller owns every
 * array; x is the initial guess in and the solution out; status through *info) and
 * the same termination logic, but computes on the GPU. All entry points return an
 * int status (FIIM_OK or a negative FIIM_E* code) in addition to the reference's
 * *info, since a GPU call can fail in ways the CPU one could not.
 *
 * Pointer spaces: the fiim_EPBiCGSTAB_* / fiim_PBiCGSTAB_* drop-ins take HOST arrays
 * and do the host->device upload, solve and download inside the call, as the
 * reference's blocking call does. Each host thread keeps the device copies of its last
 * system: a call stamps every matrix array and D^{-1} (address, size, 64-bit content
 * hash, recomputed on every call) and uploads them again only when a stamp differs;
 * b and x0 are uploaded on every call (see fiim_dropin_cache). The handle API (fiim_solver_*) takes host or
 * device arrays according to fiim_options.memory. The kernel-level entry points
 * (fiim_spmv, fiim_prec_apply) take DEVICE arrays and a cudaStream_t (as void*).
 */
#ifndef FIIM_B200_H
#define FIIM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define FIIM_OK 0
#define FIIM_EARG (-1)      /* invalid argument (sizes, null pointers, unsupported mode) */
#define FIIM_ECUDA (-2)     /* a CUDA runtime call failed; see fiim_last_error() */
#define FIIM_ENOMEM (-3)    /* device allocation failed */
#define FIIM_ENODEV (-4)    /* no CUDA device, or the device is not sm_100 */
#define FIIM_ETIMEOUT (-5)  /* the solve did not finish in time: the host-side iteration guard, or a
                               bounded device-side wait (grid barrier, bulk copy) that ran out */

/* ---- solver variants: whose control flow is reproduced --------------------- */
#define FIIM_AFIIM 0  /* AFIIM/src/bicgstab.cpp:87-297: maxmsteps = min(max(n,500)/50, 20)      */
#define FIIM_PDFIIM 1 /* PDFIIM/src/bicgstab.cpp:80-310: as AFIIM; symmetric A uses G^T for H  */
#define FIIM_ACIFIM 2 /* ACIFIM/src/bicgstab.cpp:97-327: min(max(n,2000)/50, 40), alpha guard  */

/* ---- precision of the preconditioner / inner solve -------------------------- */
#define FIIM_FP64 0        /* everything in FP64, as the reference                          */
#define FIIM_MIXED_FP32 1  /* FP64 iterative refinement around an FP32 inner BiCGSTAB       */
#define FIIM_MIXED_BF16 2  /* as FP32, with G, H stored in BF16 (FP32 accumulation)          */

#define FIIM_MEM_HOST 0
#define FIIM_MEM_DEVICE 1

/* Last error message of the calling thread (static storage, never NULL). */
const char *fiim_last_error(void);

/* Device-copy reuse of the drop-ins for the calling thread: enable != 0 (the default,
 * unless FIIM_DROPIN_CACHE=0 is set) skips the upload of matrix arrays whose address,
 * size and content hash are those of the previous call; 0 uploads every array on every
 * call. Returns the previous setting. No counterpart in the reference. */
int fiim_dropin_cache(int enable);

/* ===========================================================================
 * Reference-facing drop-ins (host arrays).
 * ======================================================================== */

/* Replaces EPBiCGSTAB of AFIIM (AFIIM/src/bicgstab.hpp:82-100, body bicgstab.cpp:87-297).
 * A: CSR (Av, Aj, Ai) 0-based; G: upper CSR incl. unit diagonal; IDv: D^{-1};
 * H: lower CSR incl. unit diagonal (layout of afiim, AFIIM/src/prec.cpp:682-740).
 * verbose != 0 prints the reference's termination messages. */
int fiim_EPBiCGSTAB_afiim(int n, double *Av, int *Aj, int *Ai, double *b, double tol, int NMAX,
                          double *Gv, int *Gj, int *Gi, double *IDv, double *Hv, int *Hj, int *Hi,
                          double *x, double *resval, int *iter, int verbose, int *info);

/* Replaces EPBiCGSTAB of PDFIIM (PDFIIM/src/bicgstab.hpp:75-86, body bicgstab.cpp:80-310),
 * with the sparseMatrix<int,int,double> members passed as raw CSR arrays
 * (sparseMatrix.hpp:68-75: v, j, i). issym != 0 is A.mtype == SYMMETRIC: A holds its
 * upper triangle only and the solver applies G^T where H would be (bicgstab.cpp:189-192);
 * H may then be NULL. */
int fiim_EPBiCGSTAB_pdfiim(int n, int issym, double *Av, int *Aj, int *Ai, double *b, double tol,
                           int NMAX, double *Gv, int *Gj, int *Gi, double *ID, double *Hv, int *Hj,
                           int *Hi, double *x, double *resval, int *iter, int verbose, int *info);

/* Replaces PBiCGSTAB of ACIFIM (ACIFIM/src/bicgstab.hpp:94-120, body bicgstab.cpp:97-327)
 * for mode 'E' (explicit G*D^{-1}*H, apply() at bicgstab.cpp:393-394,408-410) and mode
 * 'C' (Richardson-coupled with nr steps through L and U, bicgstab.cpp:395-404,411-420).
 * Modes 'I' and 'J' (triangular solves with L, U) return FIIM_EARG. */
int fiim_PBiCGSTAB_acifim(int n, double *Av, int *Aj, int *Ai, double *b, double tol, int NMAX,
                          double *Gv, int *Gj, int *Gi, double *IDv, double *Hv, int *Hj, int *Hi,
                          double *Lv, int *Lj, int *Li, double *Uv, int *Uj, int *Ui, int nr,
                          char mode, double *x, double *resval, int *iter, int verbose, int *info);

/* ===========================================================================
 * Handle API: set up once (upload, layout, tuning), solve many times.
 * ======================================================================== */
typedef struct fiim_solver_s *fiim_solver_t;

typedef struct {
    int variant;       /* FIIM_AFIIM / FIIM_PDFIIM / FIIM_ACIFIM                          */
    int issym;         /* PDFIIM symmetric input (see fiim_EPBiCGSTAB_pdfiim)              */
    int precision;     /* FIIM_FP64 / FIIM_MIXED_FP32 / FIIM_MIXED_BF16                    */
    int memory;        /* FIIM_MEM_HOST or FIIM_MEM_DEVICE for every array argument        */
    char mode;         /* ACIFIM preconditioner mode: 'E' (default) or 'C'                 */
    int nr;            /* ACIFIM mode 'C' relaxation steps                                 */
    int autotune;      /* 1: time candidate SpMV shapes at set-up and keep the fastest;    */
                       /* 0 (default): a fixed shape, so results repeat bit for bit across */
                       /* processes (the fused dot products' summation tree depends on it) */
    int verbose;       /* print the reference's termination messages                       */
    double inner_tol;  /* mixed: inner FP32 BiCGSTAB relative tolerance (default 1e-5)     */
    int inner_nmax;    /* mixed: inner iteration cap per refinement step (default 1000)    */
    int max_refine;    /* mixed: outer refinement steps cap (default 50)                   */
    int verified;      /* batched and block solves: 1 = a system (right-hand side) that     */
                       /* passes the reference's recurrence test must also have an FP64    */
                       /* true residual ||b - A x|| below tol * ||b - A x0||, or it restarts */
                       /* BiCGSTAB from its current x (masked, the others stay finished);   */
                       /* 0 (default): the recurrence test alone, as the reference stops    */
    int max_restarts;  /* verified: restart rounds cap (default 4)                         */
    double reliable;   /* mixed: delta in (0, 1) (default 0.01) = one FP32 BiCGSTAB whose  */
                       /* residual is replaced by the FP64 b - A x whenever it falls below  */
                       /* delta times its largest value since the last replacement         */
                       /* (reliable updates; the stop is the FP64 test, at most max_refine  */
                       /* verifications; inner_tol and inner_nmax unused); 0 = refinement   */
                       /* steps, each restarting the inner BiCGSTAB                        */
} fiim_options;

/* Defaults: FIIM_AFIIM, FP64, host memory, mode 'E', nr 1, autotune 0, verified 0,
 * reliable 0.01. */
void fiim_options_default(fiim_options *opt);

typedef struct {
    double resval;        /* reference-style ||r_k|| / ||r_0|| at termination (lagged, see docs) */
    double true_relres;   /* ||b - A x|| / ||b|| recomputed in FP64 after the solve              */
    int iter;             /* iterations (outer+inner total for mixed precision)                  */
    int info;             /* 0 converged, 1 diverged, 2 stagnated, 3 NMAX / non-finite alpha     */
    int refine_steps;     /* mixed precision: residual replacements (reliable updates) or outer  */
                          /* refinement steps taken                                              */
    double device_ms;     /* device time of the solve, CUDA events on the solve stream           */
    int launches;         /* kernels this solve launched (graph nodes included)                  */
} fiim_result;

/* Factors may be given as (G, IDv, H) for every variant; L and U only for ACIFIM 'C'.
 * For issym, H may be NULL. Arrays are read during the call only. */
int fiim_solver_create(fiim_solver_t *out, int n, const int *Ai, const int *Aj, const double *Av,
                       const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                       const int *Hi, const int *Hj, const double *Hv, const int *Li,
                       const int *Lj, const double *Lv, const int *Ui, const int *Uj,
                       const double *Uv, const fiim_options *opt);

/* Solve A x = b. b and x live in opt->memory space; x is the initial guess in and the
 * solution out. NMAX and tol mean what they mean in the reference; for mixed precision
 * tol is the outer FP64 relative-residual target. */
int fiim_solver_solve(fiim_solver_t s, const double *b, double *x, double tol, int NMAX,
                      fiim_result *res);

/* Bytes of device memory the solver holds. */
int64_t fiim_solver_device_bytes(fiim_solver_t s);

/* Row-block size (entries) and form of the SpMV for matrix `which` (0 A, 1 G, 2 H, 3 L,
   4 U). Forms: 0 CSR streams through registers, pipelined by one block; 1 bulk copies into
   two shared-memory buffers; 2 one warp per row block; 3 the sliced-diagonal copy (rows in
   slices of 32 that share at most 28 diagonals; built when the rows are sorted by column and
   it moves fewer bytes; FIIM_DIA=0 or FIIM_SPMV=rows/staged/warp keep the CSR streams). Every
   form gives the same bits. */
int fiim_solver_spmv_shape(fiim_solver_t s, int which, int *tile, int *form);

/* y = A x (op 0) or y = M x, the preconditioner application (op 1), with the solver's
 * own kernels; x, y in opt->memory space. Each row of every product is summed in
 * storage order with rounded products, as mkl_sparse_d_mv is restated by the oracle
 * (AFIIM/src/bicgstab.cpp:151,172-175), so the results are bit-identical to it. */
int fiim_solver_apply(fiim_solver_t s, int op, const double *x, double *y);

/* Profiling aid (no counterpart in the reference): replays each launch of the FP64
 * iteration body alone `reps` times between CUDA events on the solver's stream and
 * writes the mean ms per launch, its algorithmic bytes and (if names != NULL) its name
 * into names[i * name_len]. Call after a solve. Returns the number of kernels (<= max). */
int fiim_solver_kernel_times(fiim_solver_t s, int reps, int max_kernels, double *ms, double *bytes,
                             char *names, int name_len);

/* The same launches in the iteration body's order (both H products included), with a CUDA
 * event between consecutive launches: each launch's time as it follows the previous one.
 * *body_ms (if not NULL) receives the mean time of the same body without the events in
 * between, so their own cost is known. Returns the number of launches (<= max). */
int fiim_solver_kernel_times_seq(fiim_solver_t s, int reps, int max_kernels, double *ms, double *bytes,
                                 char *names, int name_len, double *body_ms);

/* How an FP64 solver runs its iteration loop: 0 a CUDA graph whose WHILE node repeats the
 * body on the device (the default), 1 a one-iteration graph relaunched by the host
 * (FIIM_GRAPH=host; also what a mixed-precision solver reports), 2 the whole solve as one
 * cooperative launch with grid barriers between its phases (FIIM_PERSIST=1, systems of at
 * most 65,536 rows), 3 the whole solve in one thread-block cluster of 16 CTAs whose shared
 * memory holds the solve vectors (the default for FP64 systems of at most 32,768 rows where
 * the device can run it; FIIM_PERSIST=0 keeps the WHILE graph). */
int fiim_solver_mode(fiim_solver_t s);

/* Bound on each grid-barrier wait of a one-launch solve, in polls (back-to-back acquire loads
 * of the barrier word, no sleep between them; default 2^21, about one to two seconds). A wait that runs out ends the solve with
 * FIIM_ETIMEOUT; the context stays usable. */
int fiim_solver_set_wait_limit(fiim_solver_t s, int polls);

/* Test hook for the bound above: the next solve of a one-launch solver starts with a barrier
 * that can never complete, so it must end with FIIM_ETIMEOUT after the wait limit. */
int fiim_solver_test_stall(fiim_solver_t s);

/* Algorithmic bytes of one FP64 iteration: 2 S(A) + 2 S(G) + 2 S(H) + 32 * 8n, where
 * S(M) = 12 nnz(M) + 4 (n + 1). */
double fiim_solver_iteration_bytes(fiim_solver_t s);

/* Bytes that one product with matrix `which` (0 A, 1 G, 2 H, 3 L, 4 U) reads from the
 * matrix in the form it is served in (fiim_solver_spmv_shape): 256 per diagonal of a slice
 * plus the slice records for the sliced-diagonal copy; the values, the column stream (2 or 4
 * bytes an entry), the row offsets and the row-block bounds for the CSR streams. -1 for a bad
 * handle or index. */
double fiim_solver_matrix_bytes(fiim_solver_t s, int which);

int fiim_solver_destroy(fiim_solver_t s);

/* ===========================================================================
 * Batched solve: many independent systems of uneven size in one device-driven loop.
 * No counterpart in the reference, whose drivers solve one system per call; each system
 * here runs the reference's loop (variant as in fiim_options) with its own scalars,
 * divergence window and termination.
 * The systems are passed concatenated as one block-diagonal CSR in global numbering:
 * system k owns rows and columns [sys_rows[k], sys_rows[k+1]) (sys_rows is a host
 * array of nsys + 1 offsets, sys_rows[0] = 0). opt->precision selects how G and H are
 * stored: FIIM_FP64, FIIM_MIXED_FP32 or FIIM_MIXED_BF16 (values widened to FP64 before
 * each product; A, D^{-1}, vectors and scalars stay FP64).
 * ======================================================================== */
typedef struct fiim_batch_s *fiim_batch_t;

int fiim_batch_create(fiim_batch_t *out, int nsys, const int *sys_rows, const int *Ai,
                      const int *Aj, const double *Av, const int *Gi, const int *Gj,
                      const double *Gv, const double *IDv, const int *Hi, const int *Hj,
                      const double *Hv, const fiim_options *opt);

/* Solves every system. Per-system outputs (host arrays of nsys, any may be NULL): iter,
 * info (reference codes), resval (rc/ro, lagged as in the reference) and the FP64 true
 * residual ||b_k - A_k x_k|| / ||b_k||. summary: max iterations, worst info, device time,
 * and in refine_steps the restart rounds of a verified solve (opt->verified). With
 * opt->verified, a system's iter counts the iterations of all its runs, and a system that
 * still misses the FP64 target after max_restarts rounds keeps info 0 and reports its
 * true residual. */
int fiim_batch_solve(fiim_batch_t s, const double *b, double *x, double tol, int NMAX,
                     int *iter, int *info, double *resval, double *true_relres,
                     fiim_result *summary);

int fiim_batch_destroy(fiim_batch_t s);

/* ===========================================================================
 * Multi-RHS block solve: 1..32 right-hand sides of one system. No counterpart in the
 * reference (one right-hand side per call); each right-hand side runs the reference's
 * loop with its own scalars and termination, and the sparse products are shared (SpMM).
 * B and X are n x nrhs, row-major (entry (i, j) at i * nrhs + j), in opt->memory space.
 * opt->precision: G, H stored in FP64 (FIIM_FP64) or FP32 (FIIM_MIXED_FP32).
 * ======================================================================== */
typedef struct fiim_block_s *fiim_block_t;

int fiim_block_create(fiim_block_t *out, int n, int nrhs, const int *Ai, const int *Aj,
                      const double *Av, const int *Gi, const int *Gj, const double *Gv,
                      const double *IDv, const int *Hi, const int *Hj, const double *Hv,
                      const fiim_options *opt);

/* Per-RHS outputs (host arrays of nrhs, any may be NULL) as for fiim_batch_solve. */
int fiim_block_solve(fiim_block_t s, const double *B, double *X, double tol, int NMAX,
                     int *iter, int *info, double *resval, double *true_relres,
                     fiim_result *summary);

/* Y = A X (op 0) or Y = G D^{-1} H X (op 1) on n x nrhs blocks with the solver's SpMM
 * kernels (in opt->memory space); each right-hand side's row sums are the reference's, in
 * storage order, whatever the shape. For inspection and tests. */
int fiim_block_apply(fiim_block_t s, int op, const double *X, double *Y);

/* SpMM shape of matrix `which` (0 A, 1 G, 2 H): lanes per row group (32 / lanes rows per
 * warp) and right-hand sides per lane (its load width: 1, or 2 or 4 as 16-byte pairs).
 * The default is one per lane in a group of the next power of two >= nrhs lanes, the same
 * for every matrix, so results repeat bit for bit across processes; opt->autotune = 1 times
 * every candidate shape on each matrix at set-up and keeps the fastest (the fused dot
 * products' summation tree follows the shape, so tuned results may differ in the last
 * bits from run to run). */
int fiim_block_spmm_shape(fiim_block_t s, int which, int *lanes, int *per_lane);

int fiim_block_destroy(fiim_block_t s);

/* ===========================================================================
 * Kernel-level entry points (device arrays, caller's stream; asynchronous).
 * ======================================================================== */

/* y = A x, FP64 CSR. vec = lanes per row (2,4,8,16,32) or 0 to choose from nnz/n.
 * Replaces mkl_sparse_d_mv(NON_TRANSPOSE, 1.0, A, GENERAL, x, 0.0, y)
 * (AFIIM/src/bicgstab.cpp:151,178,195). */
int fiim_spmv(int n, const int *Ai, const int *Aj, const double *Av, const double *x, double *y,
              int vec, void *stream);

/* z = G (IDv o (H r)), FP64; tm is caller scratch of n doubles. Replaces the explicit
 * preconditioner application (AFIIM/src/bicgstab.cpp:172-175; ACIFIM apply mode 'E').
 * G entries below the diagonal and H entries above it are ignored, as MKL's
 * TRIANGULAR descriptors do (AFIIM/src/bicgstab.cpp:140-147). */
int fiim_prec_apply(int n, const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                    const int *Hi, const int *Hj, const double *Hv, const double *r, double *z,
                    double *tm, void *stream);

/* Same product as fiim_prec_apply, but it allocates nothing and needs no caller scratch.
 * No counterpart in the reference (whose CPU code allocates freely). It is for callers
 * that cannot allocate device memory when they call: an application that gives all of
 * the GPU's memory to its own pool at start-up and forbids allocations behind it, or a
 * process held to a fixed device-memory budget. The intermediate vector lives in a
 * fixed array built into the library (1,048,576 doubles, 8 MiB), which every GPU that
 * loads the library's device code keeps until the process exits; n above 1,048,576 rows
 * returns FIIM_EARG. The first call on each device looks up that array's device address
 * (with the device current) and keeps it; make that first call before any stream
 * capture. The kept address belongs to the device's current context: after a
 * cudaDeviceReset of that device, do not call this entry point there again in the same
 * process (the array may be placed elsewhere in the new context). All calls on a device share the array, so calls that overlap on the GPU race
 * on it; each call overwrites all n entries it reads. Arrays and stream as for
 * fiim_prec_apply. */
int fiim_prec_apply_noalloc(int n, const int *Gi, const int *Gj, const double *Gv,
                            const double *IDv, const int *Hi, const int *Hj, const double *Hv,
                            const double *r, double *z, void *stream);

/* ===========================================================================
 * Problem generators (host; sizing pass with null arrays returns nnz).
 * ======================================================================== */
long fiim_gen_poisson2d(int nx, int ny, int *Ai, int *Aj, double *Av);
long fiim_gen_convdiff3d(int N, double peclet, int *Ai, int *Aj, double *Av);
long fiim_gen_convdiff2d(int N, double diff, double theta, double peclet, int *Ai, int *Aj,
                         double *Av);
void fiim_gen_batch_params(uint64_t seed, int k, int side_lo, int side_hi, double d_lo,
                           double d_hi, double pe_max, int *side, double *diff, double *theta,
                           double *peclet);
long fiim_gen_zipf(int n, double alpha, int cap, double scale, uint64_t seed, int *Ai, int *Aj,
                   double *Av);
double fiim_gen_zipf_mean(int n, double alpha, int cap, double scale, uint64_t seed, int sample);
void fiim_rand_normal(long n, uint64_t seed, double *out);
void fiim_model_rhs(int n, const int *Ai, const int *Aj, const double *Av, double *b);

/* ===========================================================================
 * Factor construction on the host (PDFIIM dynamic patterns), for callers and
 * benchmarks that need factors without the reference library. Produces the same
 * G, D^{-1}, H as pdfiim (PDFIIM/src/parPrec.cpp:95-588) for filttype/patt given.
 * Two calls: first with Gv == NULL returns sizes through nnzG/nnzH and keeps the
 * result in an internal buffer bound to the calling thread; the second copies it out.
 * ======================================================================== */
int fiim_pdfiim_build(int n, const int *Ai, const int *Aj, const double *Av, int prefill,
                      int lfill, int postfill, double ftol, int warpsize, char filttype,
                      char patt, int *nnzG, int *nnzH, double *Gv, int *Gj, int *Gi,
                      double *D, double *Hv, int *Hj, int *Hi);

/* The same construction on the GPU, with the same arguments, two-call protocol and
 * result, bit for bit: one warp per row, the row's pattern and its dense LU in the warp's
 * shared memory, two passes (counts, then entries at their offsets). A row whose pattern
 * outgrows 128 members in a solve (or 2048 in its set) returns FIIM_EARG; the host
 * construction has no such limit. Returns FIIM_ENODEV without an sm_100 device. */
int fiim_pdfiim_build_gpu(int n, const int *Ai, const int *Aj, const double *Av, int prefill,
                          int lfill, int postfill, double ftol, int warpsize, char filttype,
                          char patt, int *nnzG, int *nnzH, double *Gv, int *Gj, int *Gi,
                          double *D, double *Hv, int *Hj, int *Hi);

/* AFIIM factor construction on the host: the same G, D^{-1}, H as afiim
 * (AFIIM/src/prec.cpp:101-767, arguments as there; the example driver passes
 * elemPerRowCol 10, growth 5, eta 0, shift 0, AFIIM/example/example.cpp:37-39), bit for
 * bit. elemPerRowCol and growth only size the reference's buffers. The construction is
 * sequential in the rows, as the reference's is. Two calls, as fiim_pdfiim_build: the first
 * (Gv == NULL) builds and returns nnzG, nnzH; the second copies out. The result is kept per
 * calling thread, so threads may build different systems at once. */
int fiim_afiim_build(int n, const int *Ai, const int *Aj, const double *Av, double dtol,
                     int elemPerRowCol, int growth, double eta, double shift, int *nnzG,
                     int *nnzH, double *Gv, int *Gj, int *Gi, double *IDv, double *Hv, int *Hj,
                     int *Hi);

/* ACIFIM factor construction on the host: the same G, D^{-1}, H, L and U as acifim
 * (ACIFIM/src/prec.cpp:127-1052, arguments as there; the example driver passes
 * elemPerRowCol 30, growth 5, eta 0, shift 0, coeff 2, element_limit 200, filtit 30,
 * ACIFIM/example/example.cpp:42-47), bit for bit. elemPerRowCol and growth only size the
 * reference's buffers and do not change the result. Two calls: the first, with Gv == NULL,
 * builds and returns nnz[0..3] = nnz(G), nnz(H), nnz(L), nnz(U), keeping the result in a
 * buffer bound to the calling thread (so threads may build different systems at once);
 * the second copies it out (L and U are skipped when their pointers are NULL). A NaN
 * Schur complement, where the reference's acifim returns 1, returns FIIM_EARG. */
int fiim_acifim_build(int n, const int *Ai, const int *Aj, const double *Av, double dtol1,
                      double dtol2, int elemPerRowCol, int growth, double eta, double shift,
                      double coeff, int element_limit, int filtit, int *nnz, double *Gv, int *Gj,
                      int *Gi, double *IDv, double *Hv, int *Hj, int *Hi, double *Lv, int *Lj,
                      int *Li, double *Uv, int *Uj, int *Ui);

/* ===========================================================================
 * Row-partitioned solve of one system over several GPUs (one process per GPU).
 * No counterpart in the reference, whose solve runs on one node's cores.
 *
 * Rank r owns rows [row_starts[r], row_starts[r+1]) of A, G, D^{-1} and H and is given
 * exactly those rows, with GLOBAL column indices (row offsets 0-based at the block's first
 * row). Each iteration exchanges the halo entries each product needs (NCCL send/recv) and
 * gathers the ranks' partial dot products (NCCL all-gather); the gathered partials are
 * summed in rank order on every rank, so all ranks take the same termination decision.
 * Every rank's rows of every vector are computed as the single-GPU solve computes them;
 * the dot products differ from it in summation order only. Variants: AFIIM, PDFIIM with
 * the full (expanded) A and H, ACIFIM mode 'E'; FP64.
 * ======================================================================== */
#define FIIM_DIST_ID_BYTES 128
typedef struct fiim_dist_s *fiim_dist_t;

/* NCCL unique id for a new communicator (call on one rank, pass to all).
 * NCCL is loaded at run time: an already loaded libnccl.so.2 (PyTorch's) or the one named
 * by FIIM_NCCL_LIB; FIIM_ENODEV if none loads. */
int fiim_dist_unique_id(unsigned char *id);

/* Contiguous row blocks balancing each rank's streamed entries (rows of A, G, H; G and H
 * may be NULL): row_starts[0..world], each block at least one row. Host only. */
int fiim_dist_partition(int n, const int *Ai, const int *Gi, const int *Hi, int world,
                        int64_t *row_starts);

/* Host-only view of one matrix's plan on one rank (for inspection and tests): the rows
 * [row_starts[rank], +nloc) given by Mi (local offsets) and Mj (global columns); fill 1 keeps
 * col >= row (G), 2 keeps col <= row (H). Returns the halo (nbelow columns below the block,
 * then nabove above, ascending), the kept row offsets rp[nloc+1] and the renumbered columns
 * cols[nkept] (extended layout: halo below, owned rows, halo above). halo, rp, cols may be
 * NULL to query sizes. */
int fiim_dist_plan(int rank, int world, const int64_t *row_starts, const int *Mi, const int *Mj,
                   int fill, int *nbelow, int *nabove, int *nkept, int *halo, int *rp, int *cols);

/* Collective over all ranks: every rank calls it with the same id, world and row_starts.
 * device >= 0 selects the GPU (else the current one). Matrix arrays are host arrays, read
 * during the call; opt->memory says where solve's b and x live. Set-up errors are agreed
 * among the ranks, so that all of them return the same failure. */
int fiim_dist_create(fiim_dist_t *out, int rank, int world, const unsigned char *id, int device,
                     const int64_t *row_starts, const int *Ai, const int *Aj, const double *Av,
                     const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                     const int *Hi, const int *Hj, const double *Hv, const fiim_options *opt);

/* Collective: b and x are this rank's rows. res->device_ms is this rank's device time;
 * every other field is the same on all ranks. */
int fiim_dist_solve(fiim_dist_t h, const double *b, double *x, double tol, int NMAX,
                    fiim_result *res);
int fiim_dist_destroy(fiim_dist_t h);

/* All `world` row blocks of one system in this process, on the current GPU: the same
 * per-rank kernels, launch shapes and step order as fiim_dist_create/solve, with device
 * copies in place of NCCL, so its results are those of a world-GPU run, bit for bit. Global
 * host arrays; res->launches counts every block's kernels. */
int fiim_dist_emulate(int world, const int64_t *row_starts, int n, const int *Ai, const int *Aj,
                      const double *Av, const int *Gi, const int *Gj, const double *Gv,
                      const double *IDv, const int *Hi, const int *Hj, const double *Hv,
                      const double *b, double *x, double tol, int NMAX, const fiim_options *opt,
                      fiim_result *res);

/* ===========================================================================
 * Host input/output around the solve (no GPU needed).
 * ======================================================================== */

/* Reads a Matrix Market "coordinate real general|symmetric" square matrix into 0-based CSR
 * with each row sorted by column, giving the same arrays as the reference's readers:
 * form 0 as AFIIM/ACIFIM's read_coeff_matrix (AFIIM/src/rw_matrix.cpp:62-216: a symmetric
 * file is expanded to general), form 1 as PDFIIM's (PDFIIM/src/rw_matrix.cpp:60-150: a
 * symmetric file is kept as the upper triangle and *issym = 1). Two calls: first with
 * Ai == NULL returns *n and *nnz and keeps the matrix in a buffer bound to the calling
 * thread; the second (same *n, *nnz) copies it out. Unsupported types return FIIM_EARG. */
int fiim_read_mtx(const char *path, int form, int *n, int *nnz, int *issym, int *Ai, int *Aj,
                  double *Av);

/* Reads a Matrix Market "array real general" n x 1 vector (AFIIM/src/rw_matrix.cpp:246-309).
 * b == NULL: returns the length through *n; otherwise fills b[0..*n) (at most cap). */
int fiim_read_rhs(const char *path, int cap, double *b, int *n);

/* Binary factor file of G, D^{-1}, H (little-endian, checksummed), so that a factor
 * construction can be stored and reused. No counterpart in the reference. Load is two
 * calls: first with Gi == NULL returns *n, *nnzG, *nnzH (damaged or truncated files and
 * checksum mismatches return FIIM_EARG); the second copies the factors out. */
int fiim_factors_save(const char *path, int n, const int *Gi, const int *Gj, const double *Gv,
                      const double *IDv, const int *Hi, const int *Hj, const double *Hv);
int fiim_factors_load(const char *path, int *n, int *nnzG, int *nnzH, int *Gi, int *Gj, double *Gv,
                      double *IDv, int *Hi, int *Hj, double *Hv);

#ifdef __cplusplus
}
#endif
#endif /* FIIM_B200_H */
