// internal.h -- host-side types shared by the bcmgx library translation units.
#pragma once

#include "bcmgx.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace bcmgx {

struct Error : std::exception {
    int code;
    std::string msg;
    Error(int c, std::string m) : code(c), msg(std::move(m)) {}
    const char* what() const noexcept override { return msg.c_str(); }
};

void set_last_error(const std::string& s);
// Page-locked host blocks for the small host mirrors of device state. Released blocks are kept
// for reuse until the process exits: returning page-locked memory to the system can stall the
// calling thread for a long time, and solves are often set up and torn down repeatedly.
void* pinned_alloc(size_t bytes);
void pinned_free(void* p);
// counts every kernel launch of the library (reported by bcmgx_launch_count)
void note_launch();
void note_launches(long long k);
long long launch_count();
// Allocation-failure injection for the fault-path tests: while positive, every device allocation
// of the calling thread counts it down, and the one that brings it to zero fails as out of
// memory. bcmgx_setup arms it from the environment variable BCMGX_TEST_FAIL_ALLOC (k: fail the
// k-th allocation of that set-up) and disarms it on return. Zero in production.
extern thread_local long long t_fail_alloc_countdown;

#define BCMGX_CUDA(call)                                                                       \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw ::bcmgx::Error(BCMGX_ERR_CUDA, std::string(#call) + " failed: " +           \
                                                     cudaGetErrorString(e_) + " @" __FILE__); \
    } while (0)

#define BCMGX_CHECK_LAUNCH() BCMGX_CUDA(cudaGetLastError())

// Programmatic dependent launch of the solve path's kernels: a kernel launched through launch_dep
// with the attribute set may be scheduled while the kernel before it in the stream is still
// running, runs its prologue (reads of data that no kernel of a solve writes), then waits in
// dep_wait() (common.cuh) for its predecessor. Only kernels that call dep_wait() before any other
// global-memory access, and on every path, are launched this way. KIND: 0 = row kernels (plain,
// staged, sliced), 1 = element-wise cycle kernels, 2 = FCG kernels; BCMGX_PDL is a bit mask of the
// kinds that get the attribute, default 1 (row kernels only). Measured on one B200 (27-point 160^3,
// FP32 cycle): row kernels only, solve 31.4 -> 30.1 ms and one stream-launched cycle 1.19 -> 1.06 ms;
// adding the element-wise kernels made the graph solve slower (32.3 ms), adding the FCG kernels
// slowed the SpMV + dots pair (0.130 -> 0.144 ms).
bool dep_launch_enabled(int kind);
#ifdef __CUDACC__
template <int KIND = 1, typename... KA, typename... Args>
inline void launch_dep(void (*kernel)(KA...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = dep_launch_enabled(KIND) ? 1 : 0;
    note_launch();
    BCMGX_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KA>(args)...));
}
#endif

#define BCMGX_REQUIRE(cond, code, text)                                   \
    do {                                                                  \
        if (!(cond)) throw ::bcmgx::Error((code), std::string(text));     \
    } while (0)

// Stream-ordered device buffer (cudaMallocAsync from the device's default pool).
template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept { *this = std::move(o); }
    DBuf& operator=(DBuf&& o) noexcept
    {
        if (this != &o) {
            release();
            p = o.p;
            n = o.n;
            s = o.s;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    ~DBuf() { release(); }
    void alloc(size_t count, cudaStream_t stream)
    {
        release();
        s = stream;
        n = count;
        if (count == 0) return;
        if (t_fail_alloc_countdown > 0 && --t_fail_alloc_countdown == 0) {
            n = 0;
            throw Error(BCMGX_ERR_OOM, "device allocation of " + std::to_string(count * sizeof(T)) +
                    " bytes failed (injected by BCMGX_TEST_FAIL_ALLOC)");
        }
        // 64 bytes past the end: bulk copies of 16-byte granules (staged.cuh) may round the end
        // of a range up without leaving the allocation
        cudaError_t e = cudaMallocAsync((void**)&p, count * sizeof(T) + 64, stream);
        if (e != cudaSuccess) {
            p = nullptr;
            n = 0;
            (void)cudaGetLastError();
            throw Error(e == cudaErrorMemoryAllocation ? BCMGX_ERR_OOM : BCMGX_ERR_CUDA,
                std::string("device allocation of ") + std::to_string(count * sizeof(T)) +
                    " bytes failed: " + cudaGetErrorString(e));
        }
    }
    void release()
    {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    T* get() const { return p; }
};

// Device CSR with an optional FP32 copy of the values (FP32 V-cycle).
struct DevCsr {
    int n = 0, m = 0;
    int64_t nnz = 0;
    int max_row = 0;
    DBuf<int> row, col;
    DBuf<double> val;
    DBuf<float> val32;
    DBuf<short> dcol; // col - row as int16 when every entry is within 32767 of the diagonal, else empty
    DBuf<int> dpos;   // position of each row's diagonal entry (-1: none), where the producing kernel records it
    // value codes (value-indexed CSR, rowops.cuh Coded): when the matrix has at most 256 distinct
    // values, entry j's value is vtab64[vcode[j]] (and its FP32 copy vtab32[vcode[j]]); else empty
    DBuf<unsigned char> vcode;
    DBuf<double> vtab64;
    DBuf<float> vtab32;
    int nvalues = 0;  // distinct values in the table (0: not coded)
    int tpr = 0;      // threads per row for SpMV / smoother (autotuned)
    bool staged = false;  // row kernels stream the entries through shared-memory stages (staged.cuh)
    // sliced copy (sliced.cuh), built when the level's tuning picks the sliced kernels (tpr is then
    // 1: the CSR kernels that stand in for it, in a batch graph or a persistent cycle, sum each
    // row in the same order): slices of 32 rows, blocks of 4 entries per lane; int16 offsets when
    // dcol exists, else int32 columns; the value codes when the level is coded, else its FP32
    // (when val32 exists) and FP64 values
    bool sliced = false;
    DBuf<int> sl_ptr;
    DBuf<short> sl_off;
    DBuf<int> sl_col;
    DBuf<unsigned char> sl_code;
    DBuf<float> sl_val32;
    DBuf<double> sl_val64;
    // pattern-indexed rows (build_patterns): when the rows' column-offset sequences take at most
    // 255 distinct forms, sl_pid[r] is row r's form (rows past n take row n-1's) and sl_pat its
    // offsets, npat forms of patw int16 offsets each (zero past a form's length); else empty
    DBuf<unsigned char> sl_pid;
    DBuf<short> sl_pat;
    int npat = 0, patw = 0;
};

// tuning code of the sliced kernels (hierarchy info, BCMGX_TPR, the tuning cache); the staged
// kernels are coded as minus their threads per row
constexpr int kSlicedCode = 64;
void build_sliced(DevCsr& A, cudaStream_t s);
// Pattern-indexed rows of a coded level with int16 offsets and rows of at most 32 entries (one
// host round trip for the distinct forms, one for the check); leaves A.sl_pid empty when the level
// does not qualify. BCMGX_SLPAT=0 turns it off.
void build_patterns(DevCsr& A, cudaStream_t s);
void release_sliced(DevCsr& A);

struct Level {
    DevCsr A;
    DBuf<double> M;            // absolute row sums
    DBuf<float> M32;
    // composite prolongator to level + 1 (one entry per row) and its transpose
    DBuf<int> agg;
    DBuf<double> p;
    DBuf<float> p32;
    DBuf<int> rptr, ridx;
    DBuf<double> rval;
    DBuf<float> rval32;
    // V-cycle work vectors
    DBuf<double> rhs, x, x2;
    DBuf<float> rhs32, x32, x232;
};

struct SweepRecord {
    int level = 0, sweep = 0, n = 0, nc = 0;
    std::vector<int> match, agg;
    std::vector<double> p, w;
};

// Typed view of a device vector (or block of vectors) used by the V-cycle.
// A recorded persistent cycle program (persist.cuh) of one set of cycle arguments.
struct PStep;
struct PersistProgram {
    int level = -1;
    bool has_x = false;   // the call starts from the level's iterate (else from zero)
    DBuf<PStep> steps;
    int nsteps = 0;
};

struct Vec {
    void* p = nullptr;
    bool f32 = false;
    bool operator==(const Vec& o) const { return p == o.p; }
    bool operator!=(const Vec& o) const { return p != o.p; }
};

// Work buffers of one V-cycle application: per level the right-hand side (on level 0 of the FP32
// cycle: the FP32 copy of the incoming FP64 right-hand side), the two iterate buffers the
// sweeps alternate between (level 0 of the FP64 cycle uses the output and x2 only), and the
// level-0-sized residual. Block buffers hold K vectors row-major.
struct CycleBufs {
    struct L { Vec rhs, x, x2; };
    std::vector<L> lv;
    Vec res;
};

// Scratch of the multi-right-hand-side solve (multi.cu); opaque to the other units.
struct MultiWork;
void free_multi(MultiWork* w);
// Scratch, device state and captured graph of the CGHS / s-step solvers (krylov.cu).
struct KrylovWork;
void free_krylov(KrylovWork* w);

// FCG scalars that live on the device between kernels.
struct FcgState {
    double alpha, beta, gamma, delta;
    double rnorm2, delta0, tol;
    double theta, theta2;
    int iter, itnlim, done, bad;
    int ticket[4];
};

}  // namespace bcmgx

struct bcmgx_hierarchy {
    bcmgx_params prm{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<bcmgx::Level> lv;
    std::vector<bcmgx::SweepRecord> rec;
    int maxcoarsesize = 0, ftcoarse = 1;
    double op_cmplx = 0, op_wcmplx = 0, avg_cratio = 1, setup_ms = 0;
    std::vector<int> grid_sweeps;
    std::vector<std::pair<std::string, double>> prof;   // set-up phase times (BCMGX_PROFILE=1)
    // solve workspace
    bcmgx::DBuf<double> b, xv, r, v, w, d, q, res;
    bcmgx::DBuf<float> res32;
    bcmgx::DBuf<double> partials;
    bcmgx::DBuf<bcmgx::FcgState> st;
    bcmgx::FcgState* st_host = nullptr;   // pinned mirror
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t ws_n = -1;
    bcmgx::DBuf<double> hist;           // residual history, one entry per iteration
    cudaEvent_t ev_it[2] = { nullptr, nullptr };
    cudaEvent_t ev_in = nullptr;        // orders the library's stream after the caller's (after_caller)
    bool chain_in_block = false;        // small levels' sweep chains as one-block kernels (batch graphs)
    // captured solve (CUDA graph) and its own b / x buffers
    cudaGraphExec_t iter_graph = nullptr;
    bcmgx::DBuf<double> gb, gx;
    long long graph_startup_kernels = 0, graph_body_kernels = 0;
    bcmgx::CycleBufs cyc;                 // single-vector cycle buffers (views of lv[l] and res)
    // the persistent coarse cycle: first level it covers (-1: none), its barrier words, programs
    int persist_level = -1;
    bcmgx::DBuf<unsigned> persist_bar;
    std::vector<std::unique_ptr<bcmgx::PersistProgram>> persist;
    // multi-right-hand-side solve: its scratch and its captured graph (for multi_k columns)
    bcmgx::MultiWork* multi = nullptr;
    bcmgx::KrylovWork* krylov = nullptr;   // solvers other than FCG
    // standalone l1-Jacobi preconditioner: divisor a_ii + sum_{j != i} |a_ij| and a sweep buffer
    bcmgx::DBuf<double> l1d, l1tmp;
    // AFSAI preconditioner: the factor G of the scaled matrix, its transpose, and G r
    bcmgx::DevCsr afsai_G, afsai_GT;
    bcmgx::DBuf<double> afsai_tmp;
    ~bcmgx_hierarchy();
};

// A set of hierarchies whose solves run together as one CUDA graph launch.
namespace bcmgx {
struct LockGroup;
// one copy of a batch solve's vector list (lockstep.cu)
struct LockCopy {
    const double* src;
    double* dst;
    int n;
};
}  // namespace bcmgx

struct bcmgx_batch {
    std::vector<bcmgx_hierarchy*> hs;
    bool own = false;              // created by bcmgx_setup_batch: frees the hierarchies too
    bool own_stream = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    bcmgx::DBuf<unsigned char> copies, states_ptr;
    bcmgx::DBuf<bcmgx::FcgState> states;
    void* states_host = nullptr;
    void* copies_host = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_in = nullptr;
    // lockstep form (lockstep.cu, the default where the members share their cycle settings): the
    // members grouped by level count, each group one block-diagonal hierarchy, one graph for all
    int lockstep = 1;
    std::vector<bcmgx::LockGroup*> groups;   // owned; released by lock_free
    cudaGraphExec_t lock_exec = nullptr;
    bcmgx::DBuf<bcmgx::LockCopy> lock_copies;
    bcmgx::DBuf<bcmgx::FcgState> lock_states;
    void* lock_copies_host = nullptr;
    void* lock_states_host = nullptr;
    ~bcmgx_batch();
};

namespace bcmgx {

// ---- settings (params.cpp) ----
void params_default(bcmgx_params* p);
void params_from_properties(const char* path, bcmgx_params* p);
void params_from_legacy(const char* path, bcmgx_params* p);
void params_dump(const bcmgx_params* p, FILE* out);
const char* solver_name(int v);
const char* prec_name(int v);
const char* cycle_name(int v);
const char* boot_name(int v);

// ---- set-up (setup.cu) ----
void build_hierarchy(bcmgx_hierarchy* H, const bcmgx_csr* A);
// One sweep's matching + pairwise prolongator on a square matrix (see setup.cu).
struct SweepAgg {
    DBuf<int> agg, fine0, fine1;
    DBuf<double> p, wc;
    int nc = 0;
};
void sweep_aggregate(bcmgx_hierarchy* H, const DevCsr& A, const double* w, SweepAgg& out, int level, int sweep,
    double min_cap);
// C = P^T A P for the pairwise P given by agg / p over A's columns (coarse ids < ncols) and the fine
// rows fine0 / fine1 of the nc coarse rows.
void galerkin_dev(bcmgx_hierarchy* H, const DevCsr& A, const int* agg, const double* p, const int* fine0,
    const int* fine1, int nc, int ncols, DevCsr& C);
// Level finishing steps of build_hierarchy: int16 column offsets, divisor M (and the FP32 copies).
void finish_level_matrix(Level& V, bool want_f32, cudaStream_t s);
// R = P^T of a level's composite prolongator (agg with nc coarse rows).
void build_restriction(Level& V, int nc, bool want_f32, cudaStream_t s);
// P <- P * P_sweep on one-entry-per-row prolongators (first: P = P_sweep).
void compose_prolongator(int n, int* agg, double* p, const int* agg_s, const double* p_s, bool first, cudaStream_t s);
// Largest row length of a CSR (device arrays).
int row_max_dev(int n, const int* row, cudaStream_t s);
// Exclusive prefix sum on the device; out[n] = total (must fit int32). No host synchronisation.
void scan_exclusive_dev(const int* in, int* out, long n, cudaStream_t s);
// The same, returning the 64-bit total (synchronises the stream).
long long scan_exclusive(const int* in, int* out, long n, bool with_total, cudaStream_t s);
// Per-row lanes of the setup kernels and a grid-stride grid.
int setup_grid(long n, int threads = 256);

// ---- solve (solve.cu) ----
void ensure_solve_workspace(bcmgx_hierarchy* H);
int fcg_solve(bcmgx_hierarchy* H, const double* b_dev, double* x_dev, bcmgx_solve_info* info);
void prec_apply_dev(bcmgx_hierarchy* H, const double* r, double* v);
// resets the persistent cycle's barrier state (start of a solve of another driver)
void persist_reset_ext(bcmgx_hierarchy* H, cudaStream_t s);
void prec_apply_impl(bcmgx_hierarchy* H, const double* r, double* v, const int* skip);
// AFSAI preconditioner (afsai.cu): set-up of G and G^T, application v = G^T G r.
void afsai_build_dev(bcmgx_hierarchy* H);
void afsai_apply(bcmgx_hierarchy* H, const double* r, double* v, const int* skip);
// CGHS or the s-step CG (krylov.cu), for every solver but FCG.
int krylov_solve(bcmgx_hierarchy* H, const double* b, double* x, bcmgx_solve_info* info);
// FP64 row operations on level-0-like matrices with the autotuned shape; skip: see k_rowop.
void rowop_spmv(const DevCsr& A, const double* x, double* y, const int* skip, cudaStream_t s);
void rowop_resid(const DevCsr& A, const double* x, const double* f, double* y, const int* skip, cudaStream_t s);
// One V-cycle on 2^lk right-hand sides (row-major n0 x 2^lk blocks) with block buffers `bufs`.
void cycle_apply_block(bcmgx_hierarchy* H, const CycleBufs& bufs, int lk, const double* r, double* v, double* scratch,
    const int* skip);
// Block FCG for K right-hand sides of one system (multi.cu); B, X row-major n x K, device.
int multi_solve(bcmgx_hierarchy* H, int K, const double* B, double* X, bcmgx_solve_info* infos);
// Y = alpha A X + beta Y for row-major n x K blocks on device memory (K <= 32).
void launch_spmm(int n, int m, int K, const int* row, const int* col, const double* val, const double* X, double* Y,
    double alpha, double beta, cudaStream_t s);
// FP64 cycle steps of one level on caller-chosen vectors (x may hold halo entries after the
// level's own rows): one l1-Jacobi sweep, the residual, a sweep from zero, the restriction
// R res, the prolongation y = x + P xc, and plain copies / zeroing.
void step_jacobi64(const Level& V, const double* x, const double* f, double* y, cudaStream_t s);
void step_resid64(const Level& V, const double* x, const double* f, double* y, cudaStream_t s);
void step_first64(const Level& V, const double* f, double* u, cudaStream_t s);
void step_restrict64(const Level& V, int nc, const double* res, double* out, cudaStream_t s);
void step_prolong64(const Level& V, const double* xc, const double* x, double* y, cudaStream_t s);
void step_copy64(int n, const double* a, double* b, cudaStream_t s);
void step_zero64(int n, double* a, cudaStream_t s);
int num_sms();
void time_level_kernels(bcmgx_hierarchy* H, int l, int reps, double* out);
void time_block_kernels(bcmgx_hierarchy* H, int K, int reps, double* out);
double time_block_dots(bcmgx_hierarchy* H, int K, int reps);
void grad_pattern(const DevCsr& A, const double* lam, const double* x, double* dA, cudaStream_t s);
void batch_build(bcmgx_batch* B);
int batch_solve(bcmgx_batch* B, const double* const* b, double* const* x, bcmgx_solve_info* infos);
bool lock_supported(const bcmgx_batch* B);
void lock_build(bcmgx_batch* B);
int lock_solve(bcmgx_batch* B, const double* const* b, double* const* x, bcmgx_solve_info* infos);
void lock_free(bcmgx_batch* B);

// Blocks of `kernel` resident per SM with `threads` threads and `smem` bytes of dynamic shared
// memory on the current device (queried once per combination and device, then cached).
int blocks_per_sm(const void* kernel, int threads, size_t smem);
// Grid for a grid-stride kernel: min(need_blocks, blocks of this kernel resident on the GPU).
int fit_grid(const void* kernel, int threads, long need_blocks);
template <typename... A>
inline int fit_grid(void (*kernel)(A...), int threads, long need_blocks)
{
    return fit_grid((const void*)kernel, threads, need_blocks);
}

// Raises the kernel's dynamic shared-memory limit on the current device to at least `bytes`
// (never lowers it, so concurrent set-ups on other threads keep the room their launches need).
void ensure_smem_limit(const void* kernel, size_t bytes);
template <typename... A>
inline void ensure_smem_limit(void (*kernel)(A...), size_t bytes)
{
    ensure_smem_limit((const void*)kernel, bytes);
}

// ---- kernels usable on raw device memory (kernels.cu) ----
int autotune_tpr(Level& V, bool f32, cudaStream_t s);
void choose_level_kernels(bcmgx_hierarchy* H);
void stage_fault_init();
void stage_fault_check();
int default_tpr(int n, int64_t nnz);
void launch_spmv(int n, const int* row, const int* col, const double* val, const double* x, double* y,
    double alpha, double beta, int tpr, cudaStream_t s);
void edge_weights_dev(int n, int64_t nnz, const int* row, const int* col, const double* val,
    const double* w, double* W, int* tpos, double* min_out_host, cudaStream_t s);
void validate_csr_dev(int n, int m, int64_t nnz, const int* row, const int* col, bool need_diag, cudaStream_t s);
void tpos_dev(int n, int64_t nnz, const int* row, const int* col, int* tpos, cudaStream_t s);
// The edge weights formed inside the rank kernel (rows of at most 32 entries): the inputs of
// k_logw's expression instead of the stored weights.
struct FusedWeights {
    const double* val = nullptr;
    const double* w = nullptr;
    const double* C = nullptr;
    double zero_sub = 0.0;
    const double* zero_sub_dev = nullptr;   // when set, the substitute is read from here
};
// err_out: when given, the matching's error bits go to that device word and are not read back
// here (the caller reads them with its next round trip); otherwise they are checked on return.
void suitor_dev(int n, int64_t nnz, const int* row, const int* col, const double* W, const int* tpos, int* M, int max_row,
    cudaStream_t s, const FusedWeights* fw = nullptr, int* err_out = nullptr);

}  // namespace bcmgx
