/*
 * bcmgx.h -- C ABI of the B200 implementation of BootCMatchGX's single-rank
 * FCG + BCMG (matching-based aggregation AMG) path.
 *
 * Every entry point returns an int status (BCMGX_OK or a negative BCMGX_ERR_* code) and never
 * exits the process; bcmgx_last_error_string() describes the last failure of the calling thread.
 * All pointers are plain host or device pointers; sizes are in elements. Matrices are CSR with
 * int32 row offsets / column indices and FP64 values, rows column-sorted, the diagonal present
 * (the reference's struct CSR, BCMGX/src/datastruct/CSR.h:111-229, at np = 1).
 *
 * The reference library entry points this header replaces (BootCMatchGX, C++ not C):
 *   void prec_setup(handles*, CSR* Alocal, cgsprec*, const params&, PrecOut*)   prec_setup.h:55
 *   vector<vtype>* solve(handles*, CSR*, vector<vtype>* rhs, vector<vtype>* x0,
 *                        const params&, cgsprec&, SolverOut*)                    solve.h:30
 *   void prec_finalize(CSR*, cgsprec*, const params&, PrecOut*)                 prec_finalize.cu:8
 *   params Params::initFromPropertiesFile(const char* path)                     Params.cu:330
 */
#ifndef BCMGX_H
#define BCMGX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------ */
#define BCMGX_OK 0
#define BCMGX_ERR_INVALID_INPUT (-1)   /* bad argument, malformed matrix or settings file      */
#define BCMGX_ERR_UNSUPPORTED (-2)     /* option the reference has but this path does not run  */
#define BCMGX_ERR_NO_CONVERGENCE (-3)  /* itnlim reached (the reference's SolverOut.retv = -1) */
#define BCMGX_ERR_CUDA (-4)            /* a CUDA runtime call failed                           */
#define BCMGX_ERR_TIMEOUT (-5)         /* a bounded device loop or wait hit its limit          */
#define BCMGX_ERR_OOM (-6)             /* device or host allocation failed                     */
#define BCMGX_ERR_NOT_SPD (-7)         /* FCG met a non-positive curvature / non-finite value  */
#define BCMGX_ERR_INTERNAL (-8)

/* ---- enumerations (same values/order as BCMGX/src/config/Params.h) ----------------------- */
enum { BCMGX_SOLVER_CGHS = 0, BCMGX_SOLVER_FCG = 1, BCMGX_SOLVER_CGS = 2,
       BCMGX_SOLVER_PIPELINED_CGS = 3, BCMGX_SOLVER_CGS_CUBLAS = 4, BCMGX_SOLVER_INVALID = 5 };
enum { BCMGX_PREC_NONE = 0, BCMGX_PREC_L1_JACOBI = 1, BCMGX_PREC_BCMG = 2, BCMGX_PREC_AFSAI = 3,
       BCMGX_PREC_INVALID = 4 };
enum { BCMGX_BOOT_MULTIPLICATIVE = 0, BCMGX_BOOT_SYMMETRIZED_MULTIPLICATIVE = 1,
       BCMGX_BOOT_ADDITIVE = 2, BCMGX_BOOT_INVALID = 3 };
enum { BCMGX_MATCH_SUITOR = 0, BCMGX_MATCH_INVALID = 1 };
enum { BCMGX_CYCLE_V = 0, BCMGX_CYCLE_H = 1, BCMGX_CYCLE_W = 2, BCMGX_CYCLE_VARIABLE_V = 3,
       BCMGX_CYCLE_INVALID = 4 };
enum { BCMGX_L1_JACOBI = 0, BCMGX_RELAX_INVALID = 1 };
/* V-cycle arithmetic (extension; the reference is FP64 only) */
enum { BCMGX_VCYCLE_FP64 = 0, BCMGX_VCYCLE_FP32 = 1 };

/* Settings. Fields up to rec_res_int mirror struct params (BCMGX/src/config/Params.h:238-291),
 * same names, meaning and defaults. The fields after them are B200 extensions. */
typedef struct bcmgx_params {
    int solver;              /* "solver"          default CGHS (Params.h:253)        */
    int itnlim;              /* "itnlim"          default 2000                       */
    double rtol;             /* "rtol"            default 1e-6                       */
    int dispnorm;            /* "dispnorm"        default 1: print ||r|| per iteration */
    int preconditioner;      /* "preconditioner"  default NONE                       */
    int bootstrap_type;      /* "bootstrap_type"  default MULTIPLICATIVE             */
    int max_hrc;             /* "max_hrc"         default 1                          */
    double conv_ratio;       /* "conv_ratio"      default 0.8                        */
    int matchtype;           /* "matchtype"       default SUITOR                     */
    int aggrsweeps;          /* "aggrsweeps"      default 2 (=> 3 pairwise sweeps)   */
    int aggr_type;           /* "aggr_type"       default 0                          */
    int max_levels;          /* "max_levels"      default 39                         */
    int cycle_type;          /* "cycle_type"      default V_CYCLE                    */
    int coarse_solver;       /* "coarse_solver"   default L1_JACOBI                  */
    int relax_type;          /* "relax_type"      default L1_JACOBI                  */
    int relaxnumber_coarse;  /* "relaxnumber_coarse" default 20                      */
    int prerelax_sweeps;     /* "prerelax_sweeps" default 4                          */
    int postrelax_sweeps;    /* "postrelax_sweeps" default 4                         */
    int l1jacsweeps;         /* "l1jacsweeps"     default 4                          */
    int sstep;               /* "sstep"           default 1                          */
    int stop_criterion;      /* "stop_criterion"  default 1                          */
    int ru_res;              /* "ru_res"          default 1                          */
    int rec_res_int;         /* "rec_res_int"     default 0                          */
    int error;               /* set to 1 by the legacy reader for unsupported values  */
    /* ---- extensions ---- */
    int vcycle_precision;    /* BCMGX_VCYCLE_FP64 (default) or BCMGX_VCYCLE_FP32         */
    int record_sweeps;       /* keep every sweep's matching for inspection (default 0)   */
    int use_graph;           /* capture one FCG iteration in a CUDA graph (default 1)    */
    int device;              /* CUDA device ordinal (default: current device)           */
    int autotune;            /* time threads-per-row choices per level at set-up (default 1) */
    void* stream;            /* cudaStream_t to run on; NULL = library-owned stream      */
} bcmgx_params;

/* Stream order of device-resident inputs: with a library-owned stream (params.stream NULL),
 * every call that reads caller device buffers (set-up, solves, adjoint, preconditioner
 * application, batch solve) first waits for the work already queued on the legacy default
 * stream, so inputs written there (cudaMemcpy, torch's default stream) need no synchronisation.
 * Inputs written on other streams, or a stream passed in params.stream, are ordered by the
 * caller. Every such call returns only after its results are complete on the device. */

/* A CSR matrix handed to the library. The library copies it (from host or device). */
typedef struct bcmgx_csr {
    int n;                   /* rows                                        */
    int m;                   /* columns (== n for the solver)               */
    int64_t nnz;
    const int* row;          /* n + 1 offsets                               */
    const int* col;          /* nnz column indices, ascending in each row   */
    const double* val;       /* nnz values                                  */
    int on_device;           /* 1: pointers are device pointers             */
} bcmgx_csr;

/* Outcome of a solve; mirrors SolverOut (BCMGX/src/solver/SolverOut.h) plus timings. */
typedef struct bcmgx_solve_info {
    int retv;                /* 0, or -1 when itnlim was reached (FCG.cu:160-162) */
    int niter;               /* iterations, counted as the reference does (FCG.cu:164) */
    double delta0;           /* ||b - A x0||                                      */
    double exit_res;         /* final ||r||                                       */
    double solve_ms;         /* device time of the solve (CUDA events)            */
    int64_t full_n;
} bcmgx_solve_info;

#define BCMGX_MAX_LEVELS 64
/* Hierarchy summary; mirrors AMG::Hierarchy::printInfo (AMG.cu:167-179). */
typedef struct bcmgx_hierarchy_info {
    int num_levels;
    int n[BCMGX_MAX_LEVELS];
    int64_t nnz[BCMGX_MAX_LEVELS];
    double op_cmplx, op_wcmplx, avg_cratio;
    int maxcoarsesize, ftcoarse, num_sweep_records;
    double setup_ms;         /* device time of the set-up (CUDA events) */
    int tpr[BCMGX_MAX_LEVELS];   /* threads per row the solve kernels use on each level; negative: the
                                    staged kernel (matrix entries through shared memory) with -tpr;
                                    64: the sliced kernel (32-row slices, one thread per row) */
    int index_bytes[BCMGX_MAX_LEVELS]; /* column index bytes the solve kernels stream per entry
                                          (2: int16 offsets from the diagonal, 4: int32; 0: pattern-
                                          indexed rows, one byte per row naming the row's offsets) */
    int value_codes[BCMGX_MAX_LEVELS]; /* distinct values of a level whose solve kernels stream
                                          one-byte value codes (value-indexed CSR), else 0 */
} bcmgx_hierarchy_info;

typedef struct bcmgx_hierarchy bcmgx_hierarchy;

/* ---- settings ----------------------------------------------------------------------------- */
/* Defaults of struct params (Params.h:238-291) plus extension defaults. */
int bcmgx_params_default(bcmgx_params* p);
/* key = value file; '#' starts a comment; unknown keys ignored; a line without '=' is an error.
 * Replaces Params::initFromPropertiesFile (Params.cu:330-402, parser Params.cu:272-327). */
int bcmgx_params_from_properties(const char* path, bcmgx_params* p);
/* Legacy positional settings file. Replaces Params::initFromFile (Params.cu:406-474). */
int bcmgx_params_from_legacy_file(const char* path, bcmgx_params* p);
/* Writes the settings as Params::dump does (Params.cu:476-506). */
int bcmgx_params_dump(const bcmgx_params* p, const char* path_or_null_for_stdout);

/* ---- set-up / solve / finalize ------------------------------------------------------------ */
/* Builds the hierarchy. Replaces prec_setup -> bcmg_setup (prec_setup.cu:5-31, bcmg.cu:12-49). */
int bcmgx_setup(const bcmgx_csr* A, const bcmgx_params* p, bcmgx_hierarchy** out);
/* Solves A x = b with FCG (+ the V-cycle when preconditioner = BCMG). x holds x0 on entry and
 * the solution on return (the reference writes x0 in place, FCG.cu:199-207). b and x are host
 * pointers when on_device = 0, device pointers otherwise. Replaces solve -> solve_fcg
 * (solve.cu:11-51, FCG.cu:192-215). Returns BCMGX_ERR_NO_CONVERGENCE when itnlim is hit; x and
 * info are still filled. */
int bcmgx_solve(bcmgx_hierarchy* h, const double* b, double* x, int on_device, bcmgx_solve_info* info);
/* Solves A X = B for nrhs <= 32 right-hand sides at once (B, X row-major n x nrhs: entry (i, k)
 * at i*nrhs + k; X holds x0 on entry). Every sparse product is a CSR SpMM over the block, and
 * every column runs the FCG recurrence with its own scalars and stopping test; infos has nrhs
 * entries (or is NULL). The preconditioner is the hierarchy's own: the BCMG V-cycle, l1-Jacobi
 * sweeps, the AFSAI product G^T G, or none, each applied to the whole block. No counterpart in the
 * reference (its solve takes one vector, solve.cu:11-51); column k gives the result of bcmgx_solve
 * on column k up to rounding. */
int bcmgx_solve_multi(bcmgx_hierarchy* h, int nrhs, const double* B, double* X, int on_device,
    bcmgx_solve_info* infos);
/* Adjoint of x = A^{-1} b for a loss L(x): given g = dL/dx, solves A lambda = g with the same
 * hierarchy and FCG settings (A is SPD, so A^T = A) and returns dL/db = lambda and, when dA_val is
 * not NULL, dL/dA on A's sparsity pattern: dA_val[j] = -lambda_i x_{col[j]} for entry j of row i.
 * x is the forward solution. No counterpart in the reference (an extension of solve). */
int bcmgx_solve_adjoint(bcmgx_hierarchy* h, const double* g, const double* x, double* lambda, double* dA_val,
    int on_device, bcmgx_solve_info* info);
/* Releases everything the hierarchy owns. Replaces prec_finalize (prec_finalize.cu:8-31). */
int bcmgx_free(bcmgx_hierarchy* h);

int bcmgx_hierarchy_get_info(const bcmgx_hierarchy* h, bcmgx_hierarchy_info* info);
/* The AFSAI factor G of an AFSAI hierarchy (the preconditioner is G^T G): *nnz is set; the
 * n + 1 row offsets, columns and values are copied to the host arrays that are not NULL.
 * Inspection of afsai_setup's Aprec (preconditioner/afsai/afsai.cu:1016-1019). */
int bcmgx_hierarchy_get_afsai(const bcmgx_hierarchy* h, int64_t* nnz, int* row, int* col, double* val);
/* Copies level l's matrix to host arrays sized from bcmgx_hierarchy_get_info. */
int bcmgx_hierarchy_get_level(const bcmgx_hierarchy* h, int l, int* row, int* col, double* val);
/* Copies level l's composite prolongator (column agg[i], value p[i] of row i; l < levels-1) and
 * the l1-Jacobi divisor M (absolute row sums, relaxPrepare, matchingAggregation.cu:40-60). */
int bcmgx_hierarchy_get_prolongator(const bcmgx_hierarchy* h, int l, int* agg, double* p, double* M);
/* Sweep records (params.record_sweeps = 1): the suitor matching of sweep k. */
int bcmgx_hierarchy_get_sweep(const bcmgx_hierarchy* h, int k, int* level, int* sweep, int* n, int* nc,
    int* match, int* agg, double* p, double* w);
/* One preconditioner application v = B r (v zeroed first, as FCG does). Host or device pointers.
 * Replaces prec_apply -> bcmg_apply (prec_apply.cu:6-35, bcmg.cu:51-90). */
int bcmgx_prec_apply(bcmgx_hierarchy* h, const double* r, double* v, int on_device);

/* Average device time (ms, CUDA events on the hierarchy's stream, `reps` launches after one
 * warm-up) of level `level`'s solve kernels into out[0..5]: out[0] one l1-Jacobi sweep in the
 * cycle's precision, out[1] the residual, out[2] the FP64 SpMV, and on level 0 only (else 0):
 * out[3] the fused FCG SpMV + dots, out[4] the FP32 cycle's sweep that writes the FP64
 * preconditioned vector (0 for the FP64 cycle), out[5] the FCG update (two merged axpys and the
 * norm). The kernels run on fixed non-constant vectors (values in [0.5, 1.5)), as in a solve: on
 * zero vectors every sweep divides zero residuals, which times slower. No counterpart in the
 * reference: the measurement hook of the benchmarks. */
int bcmgx_time_kernels(bcmgx_hierarchy* h, int level, int reps, double* out_ms);
/* The same for the level-0 block kernels of a solve with nrhs (1..32) right-hand sides (blocks of
 * nrhs rounded up to a power of two columns): out[0] one block l1-Jacobi sweep in the cycle's
 * precision, out[1] the block residual, out[2] the FP64 block SpMM, out[3] the block FCG SpMV +
 * per-column dots. Allocates the multi-right-hand-side workspace. No counterpart in the
 * reference (its solve takes one vector). */
int bcmgx_time_block_kernels(bcmgx_hierarchy* h, int nrhs, int reps, double* out_ms);

/* ---- batched solves (no counterpart in the reference) ------------------------------------ */
/* Many independent systems solved together: their set-ups run concurrently (nthreads host
 * threads, one stream each; 0 = 8), and all their FCG solves run as ONE CUDA graph launch with one
 * device-driven loop per system. A holds nsys CSR descriptions. */
typedef struct bcmgx_batch bcmgx_batch;
int bcmgx_setup_batch(int nsys, const bcmgx_csr* A, const bcmgx_params* p, int nthreads, bcmgx_batch** out);
/* A batch over hierarchies built by bcmgx_setup (the caller keeps ownership of them). */
int bcmgx_batch_from_hierarchies(int nsys, bcmgx_hierarchy* const* hs, bcmgx_batch** out);
int bcmgx_batch_get_hierarchy(bcmgx_batch* B, int k, bcmgx_hierarchy** h);
/* b[k], x[k]: device vectors of system k (x: x0 in, solution out). infos: nsys entries or NULL. */
int bcmgx_batch_solve(bcmgx_batch* B, const double* const* b, double* const* x, bcmgx_solve_info* infos);
/* Lockstep form of the batch solve (on = 1, the default, when every member is BCMG with the same
 * cycle settings, rtol and itnlim): the members are grouped by their number of levels, each group's
 * hierarchy is the block-diagonal union of its members' (set up on the first solve), and every
 * V-cycle step and FCG step is one kernel over all members of a group; each member keeps its own
 * FCG scalars and stopping test, and the solution agrees with the member's single solve to
 * rounding. on = 0: one graph branch per member, whose iterates equal single solves bit for bit.
 * No counterpart in the reference. */
int bcmgx_batch_set_lockstep(bcmgx_batch* B, int on);
int bcmgx_batch_free(bcmgx_batch* B);

/* ---- row-partitioned multi-rank set-up and solve ------------------------------------------ */
/* The reference's np > 1 path: prec_setup / solve with the matrix split by rows over nranks ranks
 * (rank r holds rows offs[r] .. offs[r+1]-1 with global column ids; BCMGX/src/utility/
 * distribuite.cu, row_shift in CSR.h:173-176). Matching and aggregation are rank-local
 * (suitor.cu:95-100 skips other ranks' columns; makeAH writes 99999 for them, matching.cu:82-85;
 * each rank numbers its own aggregates after the lower ranks', matchingPairAggregation.cu:188-222);
 * every SpMV and l1-Jacobi sweep first brings the other ranks' entries of x that the local rows
 * use (the halo exchange, halo_communication/halo_communication.cu, CSR.cu:829-985,
 * l1jacobi.cu:94-342); the Galerkin product brings the prolongator rows of those columns
 * (spspmpi.cu:770-1120); FCG sums its dot products over ranks (triple_inner_product.cu:80-91).
 * The V-cycle runs in FP64 (the reference's arithmetic).
 * Two transports:
 *  - bcmgx_dist_setup_local: all nranks row blocks in this process on one device, the exchanges
 *    as device copies between the blocks' buffers and the sums over ranks as one small kernel;
 *  - bcmgx_dist_setup_nccl: one row block per process (one GPU each), exchanges as grouped
 *    ncclSend / ncclRecv and sums as ncclAllReduce on the hierarchy's stream; the communicator
 *    comes from bcmgx_nccl_comm_init. NCCL (libnccl.so.2) is loaded when first needed. */
typedef struct bcmgx_dist bcmgx_dist;
/* A: the whole matrix (host or device arrays); offs: nranks + 1 row offsets, offs[0] = 0,
 * offs[nranks] = A->n, every block non-empty. */
int bcmgx_dist_setup_local(const bcmgx_csr* A, int nranks, const int64_t* offs, const bcmgx_params* p,
    bcmgx_dist** out);
/* A_rows: this rank's rows (A_rows->n rows, A_rows->m = n_global columns, global column ids);
 * row_offset: the global id of its first row; ranks hold consecutive blocks in rank order. */
int bcmgx_dist_setup_nccl(const bcmgx_csr* A_rows, int64_t row_offset, int64_t n_global, void* nccl_comm,
    const bcmgx_params* p, bcmgx_dist** out);
/* FCG + the partitioned V-cycle. b, x: the rows this process holds (all rows in the local form,
 * this rank's block with NCCL); x holds x0 on entry and the solution on return. */
int bcmgx_dist_solve(bcmgx_dist* D, const double* b, double* x, int on_device, bcmgx_solve_info* info);
/* Global level sizes (n, nnz summed over ranks) and the hierarchy statistics. */
int bcmgx_dist_get_info(const bcmgx_dist* D, bcmgx_hierarchy_info* info);
/* The rows of level l that this process holds (all of them in the local form), with global
 * column ids: *rows and *nnz are set, and the arrays that are not NULL are filled (row: rows + 1
 * offsets). offs (nranks + 1 entries, may be NULL) receives the level's row partition. */
int bcmgx_dist_get_level(const bcmgx_dist* D, int l, int* rows, int64_t* nnz, int* row, int* col, double* val,
    int64_t* offs);
/* The composite prolongator of level l on this process's rows: global aggregate ids, values,
 * and the l1-Jacobi divisor M. */
int bcmgx_dist_get_prolongator(const bcmgx_dist* D, int l, int* agg, double* p, double* M);
int bcmgx_dist_free(bcmgx_dist* D);
/* NCCL plumbing for bcmgx_dist_setup_nccl: a unique id (128 bytes) made on one rank and shared
 * with the others by the caller, the communicator of nranks ranks on the current device, and its
 * release. */
int bcmgx_nccl_unique_id(unsigned char* id128);
int bcmgx_nccl_comm_init(int nranks, int rank, const unsigned char* id128, void** comm);
int bcmgx_nccl_comm_destroy(void* comm);

/* ---- kernels on caller-owned device memory ------------------------------------------------ */
/* y = alpha * A x + beta * y on device pointers (driverSpMV, driverSpMV.cu:219-235; kernel
 * CSRm::CSRVector_product_adaptive_miniwarp_witho, CSR.cu:829-846). threads_per_row = 0 picks
 * the autotuned choice. */
int bcmgx_spmv(int n, int m, int64_t nnz, const int* row, const int* col, const double* val,
    const double* x, double* y, double alpha, double beta, int threads_per_row, void* stream);
/* Y = alpha * A X + beta * Y for nrhs <= 32 vectors (X, Y row-major: m x nrhs and n x nrhs) on
 * device pointers: one warp per row, lane k on column k, A read once for all columns. No
 * counterpart in the reference (its SpMM, driverSpMM.cu:228, is a sparse x sparse product). */
int bcmgx_spmm(int n, int m, int64_t nnz, const int* row, const int* col, const double* val, int nrhs,
    const double* X, double* Y, double alpha, double beta, void* stream);
/* Edge weights of one pairwise sweep on A's pattern (diagonal slots 0). Replaces makeAH +
 * toMaximumProductMatrix + _write_T_warp (matching.cu:137-288). Device pointers. */
int bcmgx_edge_weights(int n, int64_t nnz, const int* row, const int* col, const double* val,
    const double* w, double* W, double* min_abs_out, void* stream);
/* Suitor half-approximate maximum-weight matching on weights W (A's pattern). M[v] = partner or
 * -1. Replaces approx_match_gpu_suitor (suitor.cu:303-329) (driverMWM, driverMWM.cu:251-263). */
int bcmgx_suitor_matching(int n, int64_t nnz, const int* row, const int* col, const double* W,
    int* M, void* stream);

/* Allocation-free variant of bcmgx_edge_weights. No counterpart in the reference. For callers
 * that cannot let the library allocate device memory -- a framework whose caching allocator
 * already holds (nearly) all of the GPU's memory, or a process under a fixed device-memory
 * budget. Same arguments and results as bcmgx_edge_weights; it calls no allocator (no cudaMalloc,
 * cudaMallocAsync, cudaFree or library allocator). Its scratch is a static device array of about
 * 8.5 MiB (per-row values and per-entry positions) that every GPU loading the library holds until
 * exit; matrices beyond 65536 rows or 2097152 non-zeros are rejected with
 * BCMGX_ERR_INVALID_INPUT. The first call on a device looks up that device's address of the
 * array (cudaGetSymbolAddress), so make that first call before any stream capture. With CUDA's
 * lazy module loading (the default since CUDA 12.2) the array's device memory is committed only
 * when the library's set-up module first loads on a device -- at that first call, or at the first
 * set-up call -- so a caller whose allocator will later take nearly all of the GPU's memory makes
 * one call (any size) before that, or runs with CUDA_MODULE_LOADING=EAGER. All calls share the
 * array: calls that overlap on the GPU (other streams, other host threads) race on it and must be
 * serialised by the caller. */
int bcmgx_edge_weights_noalloc(int n, int64_t nnz, const int* row, const int* col, const double* val,
    const double* w, double* W, double* min_abs_out, void* stream);

/* ---- input plumbing (host) ---------------------------------------------------------------- */
/* Size of the 7- or 27-point Laplacian on the (nx*P) x (ny*Q) x (nz*R) grid. */
int bcmgx_laplacian_3d_size(int stencil, int nx, int ny, int nz, int P, int Q, int R, int64_t* n, int64_t* nnz);
/* The Laplacian itself into caller arrays (row: n+1, col/val: nnz), in the reference's
 * rank-block-major global order. Replaces generateLocalLaplacian3D_7p/_27p
 * (laplacian.cu:119-777) stacked over P*Q*R ranks, and generateLocalLaplacian3D (-a n,
 * laplacian.cu:27-117) when P = Q = R = 1 and nx = ny = nz = n. */
int bcmgx_laplacian_3d(int stencil, int nx, int ny, int nz, int P, int Q, int R, int* row, int* col, double* val);
/* Reads nx ny nz P Q R from a laplacian .cfg file (read_laplacian_file, laplacian.cu:974-1017). */
int bcmgx_read_laplacian_cfg(const char* path, int* out6);
/* MatrixMarket coordinate real general/symmetric reader (readMTXDouble, CSR.cu:1973-2120).
 * The arrays are allocated by the library; release each with bcmgx_host_free. */
int bcmgx_read_matrix_market(const char* path, int* n, int* m, int64_t* nnz, int** row, int** col, double** val);
void bcmgx_host_free(void* p);
/* 7-point finite-volume diffusion with per-cell coefficient kappa (harmonic-mean faces,
 * Dirichlet boundary); no counterpart in the reference: the generator of the heterogeneous
 * benchmark problems. Arrays sized like bcmgx_laplacian_3d_size(7, nx, ny, nz, 1, 1, 1). */
int bcmgx_diffusion_7p(int nx, int ny, int nz, const double* kappa, int* row, int* col, double* val);

/* ---- errors ------------------------------------------------------------------------------- */
const char* bcmgx_last_error_string(void);
const char* bcmgx_version(void);
/* Number of kernels this library has launched in the process so far (all devices). */
int64_t bcmgx_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* BCMGX_H */
