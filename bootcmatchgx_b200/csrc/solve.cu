// solve.cu -- solve phase on the device: the l1-Jacobi V-cycle and flexible CG.
//
// V-cycle: GAMG_cycle (BCMGX/src/preconditioner/bcmg/GAMG_cycle.cu:58-236) at np = 1, with
// l1-Jacobi sweeps (l1jacobi.cu:345-479). FCG: flexibileConjugateGradients_v3
// (BCMGX/src/solver/fcg/FCG.cu:27-165). Differences in form, not in result:
//  * a sweep from a zero iterate is u = f / M (what the full sweep computes when u = 0), so
//    the first pre-smoothing sweep of every level and the first coarse sweep skip the SpMV;
//  * sweeps alternate between two level buffers and the prolongation writes out of place so
//    that no copy-back is needed (the reference copies when the sweep count is odd);
//  * the FCG dots and axpys are fused with the SpMV and with each other, and the scalars stay
//    on the device; reductions are two-stage and deterministic.
// FP32 V-cycle (vcycle_precision = FP32): levels 0..L-2 run on FP32 matrix values and vectors;
// the coarsest level, the outer residual, the dots and the direction updates stay FP64.
#include "internal.h"
#include <type_traits>
#include "rowops.cuh"
#include "staged.cuh"
#include "sliced.cuh"
#include "blockops.cuh"
#include "persist.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <unordered_map>
#include <tuple>

namespace bcmgx {

static int current_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        (void)cudaGetLastError();
        dev = 0;
    }
    return dev;
}

// SM count of the current device (cached per device).
int num_sms()
{
    static std::mutex mu;
    static std::unordered_map<int, int> cache;
    const int dev = current_device();
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = cache.find(dev);
        if (it != cache.end()) return it->second;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
        (void)cudaGetLastError();
        sms = 148;
    }
    std::lock_guard<std::mutex> g(mu);
    cache[dev] = sms;
    return sms;
}

void ensure_smem_limit(const void* kernel, size_t bytes)
{
    // the default limit covers 48 KB of static and dynamic shared memory together, so a kernel
    // with static shared memory needs the attribute already at 48 KB of dynamic memory
    if (bytes < 32 * 1024) return;
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> set;
    int dev = 0;
    BCMGX_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(mu);
    size_t& cur = set[std::make_pair(dev, kernel)];
    if (bytes <= cur) return;
    BCMGX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    cur = bytes;
}

// Grid of a grid-stride kernel: the blocks its work needs, but no more than fit on the GPU at
// once for this kernel (its registers and shared memory decide how many blocks an SM holds; the
// figure is queried once per kernel, block size, shared memory and device, and cached). Every
// block is then resident from the start: a grid larger than one wave would leave its last blocks
// to run after the first wave has finished all of its rows, on a mostly idle GPU.
int blocks_per_sm(const void* kernel, int threads, size_t smem)
{
    static std::mutex mu;
    static std::map<std::tuple<int, const void*, int, size_t>, int> cache;
    const auto key = std::make_tuple(current_device(), kernel, threads, smem);
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, smem) != cudaSuccess || b <= 0) {
        (void)cudaGetLastError();
        b = 1;
    }
    std::lock_guard<std::mutex> g(mu);
    cache[key] = b;
    return b;
}

bool dep_launch_enabled(int kind)
{
    static const int mask = [] {
        const char* e = std::getenv("BCMGX_PDL");
        return e && *e ? std::atoi(e) : 1;
    }();
    return (mask >> kind) & 1;
}

int fit_grid(const void* kernel, int threads, long need_blocks)
{
    const int b = blocks_per_sm(kernel, threads, 0);
    return (int)std::max<long>(1, std::min<long>(need_blocks, (long)num_sms() * b));
}

// VS: the matrix values (ValSrc: a `const T*`, or Coded<T> for a value-indexed matrix).
template <int OP, typename VS, typename XT, typename FT, typename MT, typename YT, typename IT>
static void launch_rowop(int tpr, int n, const int* row, const IT* col, VS val, const XT* x, const FT* f,
    const MT* M, YT* y, double alpha, double beta, const int* skip, cudaStream_t s)
{
    if (n <= 0) return;
    const long need = ((long)n * tpr + 255) / 256;
    auto go = [&](auto kern) {
        launch_dep<0>(kern, fit_grid(kern, 256, need), 256, 0, s, n, row, col, val, x, f, M, y, alpha, beta, skip);
    };
    switch (tpr) {
    case 1: go(k_rowop<1, OP, VS, XT, FT, MT, YT, IT>); break;
    case 2: go(k_rowop<2, OP, VS, XT, FT, MT, YT, IT>); break;
    case 4: go(k_rowop<4, OP, VS, XT, FT, MT, YT, IT>); break;
    case 8: go(k_rowop<8, OP, VS, XT, FT, MT, YT, IT>); break;
    case 16: go(k_rowop<16, OP, VS, XT, FT, MT, YT, IT>); break;
    default: go(k_rowop<32, OP, VS, XT, FT, MT, YT, IT>); break;
    }
    BCMGX_CHECK_LAUNCH();
}

// Deterministic values in [0.5, 1.5) for the vectors the timing hooks and the autotuner run the
// kernels on: a zero vector makes every sweep divide a zero residual, and FP32 division leaves
// its fast path for a zero numerator, so zero vectors time a case the solve does not see.
template <typename T>
__global__ void k_fill_probe(long n, T* __restrict__ a, unsigned salt)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        unsigned h = (unsigned)i * 0x9E3779B1u ^ salt;
        h ^= h >> 15;
        h *= 0x85EBCA77u;
        h ^= h >> 13;
        a[i] = (T)(0.5 + (double)(h & 0xFFFFFFu) / 16777216.0);
    }
}

template <typename T>
static void fill_probe(T* a, long n, unsigned salt, cudaStream_t s)
{
    if (n <= 0) return;
    auto k = k_fill_probe<T>;
    note_launch();
    k<<<fit_grid(k, 256, (n + 255) / 256), 256, 0, s>>>(n, a, salt);
    BCMGX_CHECK_LAUNCH();
}

// Fault word of the staged row kernels and the persistent cycle, in mapped pinned host memory:
// nonzero when one of their waits (on a shared-memory stage, at a grid barrier: code 8) gave up. The entry points read it after their final stream
// synchronisation (stage_fault_check), so the check costs no copy. It is one word for the
// process: with solves on several threads, the entry point that reads it first reports it.
static int* g_stage_fault = nullptr;
static std::once_flag g_stage_fault_once;

void stage_fault_init()
{
    std::call_once(g_stage_fault_once, [] {
        void* p = nullptr;
        BCMGX_CUDA(cudaHostAlloc(&p, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable));
        *(volatile int*)p = 0;
        g_stage_fault = (int*)p;
    });
}

void stage_fault_check()
{
    if (g_stage_fault && *(volatile int*)g_stage_fault) {
        const int code = *(volatile int*)g_stage_fault;
        *(volatile int*)g_stage_fault = 0;
        if (code == 8)
            throw Error(BCMGX_ERR_TIMEOUT, "persistent cycle: a wait at a grid barrier gave up (code 8)");
        throw Error(BCMGX_ERR_TIMEOUT, "staged row kernel: a wait on a shared-memory stage gave up (code " +
            std::to_string(code) + ")");
    }
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }
static bool al16(const void* p) { return aligned16(p); }

// Fault-path test hook of the staged kernels: BCMGX_TEST_STAGE_FAULT=<ns> in the environment makes
// the launches that follow (the variable is read at every launch; a captured graph keeps the value
// of its capture) drop block 0's first tile copy and wait at most <ns> for a stage, so that the
// timeout path runs and the entry point returns BCMGX_ERR_TIMEOUT. Unset in production.
static unsigned long long stage_test_wait_ns()
{
    const char* e = std::getenv("BCMGX_TEST_STAGE_FAULT");
    if (!e || !*e) return 0;
    const long long v = std::atoll(e);
    return v > 0 ? (unsigned long long)v : 0ull;
}

// The staged form of launch_rowop (staged.cuh): one resident wave of blocks over tiles of R rows.
template <int S, int OP, typename VS, typename XT, typename FT, typename MT, typename YT, typename IT>
static void launch_staged(int n, int64_t nnz, const int* row, const IT* col, VS val, const XT* x, const FT* f,
    const MT* M, YT* y, double alpha, double beta, const int* skip, cudaStream_t s)
{
    using C = StageCfg<VS, IT>;
    auto kern = k_rowop_staged<S, OP, VS, XT, FT, MT, YT, IT>;
    ensure_smem_limit(kern, C::SMEM);
    const int per_sm = blocks_per_sm((const void*)kern, kStageThreads, C::SMEM);
    stage_fault_init();
    const int R = stage_tile_rows<VS, IT>(n, nnz, S);
    const long ntiles = ((long)n + R - 1) / R;
    const int grid = (int)std::min<long>(ntiles, (long)per_sm * num_sms());
    const unsigned long long test_ns = stage_test_wait_ns();
    launch_dep<0>(kern, grid, kStageThreads, C::SMEM, s, n, R, row, col, val, x, f, M, y, alpha, beta, skip, g_stage_fault,
        test_ns ? test_ns : kStageWaitNs, test_ns ? 1 : 0);
    BCMGX_CHECK_LAUNCH();
}

// ------------------------------------------------------------------------------------------
// sliced form (sliced.cuh)
// ------------------------------------------------------------------------------------------
void release_sliced(DevCsr& A)
{
    A.sliced = false;
    A.sl_pid.release();
    A.sl_pat.release();
    A.npat = A.patw = 0;
    A.sl_ptr.release();
    A.sl_off.release();
    A.sl_col.release();
    A.sl_code.release();
    A.sl_val32.release();
    A.sl_val64.release();
}

// Builds A's sliced copy from its CSR arrays (one host round trip for the total). The codes are
// used when the level is coded and its table has a free (zero) slot for the padding.
void build_sliced(DevCsr& A, cudaStream_t s)
{
    if (A.sl_ptr.p || A.n <= 0) return;
    const long nsl = ((long)A.n + kSliceRows - 1) / kSliceRows;
    DBuf<int> cnt;
    cnt.alloc(nsl, s);
    auto kw = k_sl_width;
    note_launch();
    kw<<<fit_grid(kw, 256, ceil_div(nsl * 32, 256)), 256, 0, s>>>(A.n, A.row.p, cnt.p);
    BCMGX_CHECK_LAUNCH();
    A.sl_ptr.alloc(nsl + 1, s);
    const long long total = scan_exclusive(cnt.p, A.sl_ptr.p, nsl, true, s);
    const bool coded = A.vcode.p && A.nvalues > 0 && A.nvalues < kValueCodes;
    if (coded) A.sl_code.alloc(std::max<long long>(total, 1), s);
    else {
        A.sl_val64.alloc(std::max<long long>(total, 1), s);
        if (A.val32.p) A.sl_val32.alloc(std::max<long long>(total, 1), s);
    }
    auto fill = [&](auto kern, auto* cidx, auto* sidx) {
        note_launch();
        kern<<<fit_grid(kern, 256, ceil_div(nsl * 32, 256)), 256, 0, s>>>(A.n, A.row.p, cidx, A.sl_ptr.p, sidx,
            A.vcode.p, coded ? A.sl_code.p : nullptr, A.nvalues, A.val32.p, coded ? nullptr : A.sl_val32.p,
            A.val.p, coded ? nullptr : A.sl_val64.p);
        BCMGX_CHECK_LAUNCH();
    };
    if (A.dcol.p) {
        A.sl_off.alloc(std::max<long long>(total, 1), s);
        fill(k_sl_fill<short>, (const short*)A.dcol.p, A.sl_off.p);
    } else {
        A.sl_col.alloc(std::max<long long>(total, 1), s);
        fill(k_sl_fill<int>, (const int*)A.col.p, A.sl_col.p);
    }
    build_patterns(A, s);
    // the sliced kernels read the copy in their prologue, before their dependency wait (launch_dep),
    // so it is complete before the first of them is launched
    BCMGX_CUDA(cudaStreamSynchronize(s));
}

template <int OP, typename VS, typename XT, typename FT, typename MT, typename YT>
static void launch_sliced(const DevCsr& A, SlSrc<VS> sv, const XT* x, const FT* f, const MT* M, YT* y, double alpha,
    double beta, const int* skip, cudaStream_t s)
{
    const long nsl = ((long)A.n + kSliceRows - 1) / kSliceRows;
    if constexpr (ValSrc<VS>::coded) {
        if (A.sl_pid.p && A.npat > 0 && A.sl_code.p && sv.code == A.sl_code.p) {
            // pattern-indexed rows: codes and form bytes streamed, offsets from the form table
            using T = typename ValSrc<VS>::type;
            auto kern = k_rowop_slpat<OP, T, XT, FT, MT, YT>;
            const size_t smem = (((size_t)A.npat * A.patw * sizeof(short) + 15) & ~(size_t)15) +
                (size_t)kSlWarps * kSpStages * kSpStageBytes;
            ensure_smem_limit((const void*)kern, smem);
            const int per_sm = blocks_per_sm((const void*)kern, kSlWarps * 32, smem);
            const int grid = (int)std::max<long>(1, std::min<long>(ceil_div(nsl, kSlWarps), (long)per_sm * num_sms()));
            launch_dep<0>(kern, grid, kSlWarps * 32, smem, s, A.n, A.sl_ptr.p, (const unsigned char*)A.sl_pid.p,
                (const unsigned char*)sv.code, sv.tab, (const short*)A.sl_pat.p, A.npat, A.patw, x, f, M, y, alpha, beta,
                skip);
            BCMGX_CHECK_LAUNCH();
            return;
        }
    }
    auto go = [&](auto* idx) {
        using IT = std::remove_const_t<std::remove_pointer_t<decltype(idx)>>;
        using C = SlStage<IT, VS>;
        auto run = [&](auto kern) {
            ensure_smem_limit((const void*)kern, C::SMEM);
            const int per_sm = blocks_per_sm((const void*)kern, kSlWarps * 32, C::SMEM);
            const int grid = (int)std::max<long>(1, std::min<long>(ceil_div(nsl, kSlWarps), (long)per_sm * num_sms()));
            launch_dep<0>(kern, grid, kSlWarps * 32, C::SMEM, s, A.n, A.sl_ptr.p, idx, sv, x, f, M, y, alpha, beta, skip);
        };
        if (A.max_row > 0 && A.max_row <= C::NBMAX * kSliceG) run(k_rowop_sliced<OP, VS, XT, FT, MT, YT, IT, true>);
        else run(k_rowop_sliced<OP, VS, XT, FT, MT, YT, IT, false>);
    };
    if (A.sl_off.p) go((const short*)A.sl_off.p);
    else go((const int*)A.sl_col.p);
    BCMGX_CHECK_LAUNCH();
}

// The row operation on a level matrix, through its int16 column offsets when it has them, through
// its value codes when it has them and `val` is the level's own FP64 or FP32 value array (the
// codes index a table of those same values), and through the staged kernel when the level's
// tuning chose it (stage: -1 follows A.staged, 0 / 1 force it off / on). The staged kernel exists
// for 1, 2, 4 and 8 threads per row.
template <int OP, typename VS, typename XT, typename FT, typename MT, typename YT>
static void launch_rowop_vs(int tpr, const DevCsr& A, VS val, const void* val_ptr, const XT* x, const FT* f, const MT* M,
    YT* y, double alpha, double beta, const int* skip, cudaStream_t s, int stage)
{
    const bool staged = (stage < 0 ? A.staged : stage == 1) && (tpr == 1 || tpr == 2 || tpr == 4 || tpr == 8) &&
        aligned16(A.row.p) && aligned16(val_ptr) && aligned16(A.dcol.p ? (const void*)A.dcol.p : (const void*)A.col.p);
    if (staged) {
        auto go = [&](auto* colp) {
            switch (tpr) {
            case 1: launch_staged<1, OP>(A.n, A.nnz, A.row.p, colp, val, x, f, M, y, alpha, beta, skip, s); break;
            case 2: launch_staged<2, OP>(A.n, A.nnz, A.row.p, colp, val, x, f, M, y, alpha, beta, skip, s); break;
            case 4: launch_staged<4, OP>(A.n, A.nnz, A.row.p, colp, val, x, f, M, y, alpha, beta, skip, s); break;
            default: launch_staged<8, OP>(A.n, A.nnz, A.row.p, colp, val, x, f, M, y, alpha, beta, skip, s); break;
            }
        };
        if (A.dcol.p) go((const short*)A.dcol.p);
        else go((const int*)A.col.p);
        return;
    }
    if (A.dcol.p) launch_rowop<OP>(tpr, A.n, A.row.p, (const short*)A.dcol.p, val, x, f, M, y, alpha, beta, skip, s);
    else launch_rowop<OP>(tpr, A.n, A.row.p, (const int*)A.col.p, val, x, f, M, y, alpha, beta, skip, s);
}

// form (stage): -1 the level's tuned kernel (sliced, staged or plain), 0 the plain CSR kernel, 1 the
// staged kernel, 2 the sliced kernel. The sliced kernel runs when the level has its sliced copy
// and `val` is one of the level's own value arrays (else the CSR kernels do, with tpr).
template <int OP, typename VT, typename XT, typename FT, typename MT, typename YT>
static void launch_rowop_A(int tpr, const DevCsr& A, const VT* val, const XT* x, const FT* f, const MT* M, YT* y,
    double alpha, double beta, const int* skip, cudaStream_t s, int stage = -1)
{
    if (A.n <= 0) return;
    const VT* own = nullptr;
    const VT* tab = nullptr;
    const VT* slv = nullptr;
    if constexpr (std::is_same<VT, float>::value) {
        own = A.val32.p;
        tab = A.vtab32.p;
        slv = A.sl_val32.p;
    } else {
        own = A.val.p;
        tab = A.vtab64.p;
        slv = A.sl_val64.p;
    }
    if ((stage == 2 || (stage < 0 && A.sliced)) && A.sl_ptr.p && val == own) {
        if (A.sl_code.p && tab) {
            launch_sliced<OP>(A, SlSrc<Coded<VT>> { A.sl_code.p, tab }, x, f, M, y, alpha, beta, skip, s);
            return;
        }
        if (slv) {
            launch_sliced<OP>(A, SlSrc<const VT*> { slv }, x, f, M, y, alpha, beta, skip, s);
            return;
        }
    }
    if (A.vcode.p && tab && val == own) {
        launch_rowop_vs<OP>(tpr, A, Coded<VT> { A.vcode.p, tab }, (const void*)A.vcode.p, x, f, M, y, alpha, beta,
            skip, s, stage);
        return;
    }
    launch_rowop_vs<OP>(tpr, A, val, (const void*)val, x, f, M, y, alpha, beta, skip, s, stage);
}

// About 6-8 entries per lane: 27-point rows -> 4 lanes, 7-point rows -> 2 lanes.
int default_tpr(int n, int64_t nnz)
{
    const double avg = n > 0 ? (double)nnz / n : 1.0;
    if (avg <= 3) return 1;
    if (avg <= 12) return 2;
    if (avg <= 32) return 4;
    if (avg <= 64) return 8;
    if (avg <= 128) return 16;
    return 32;
}

void launch_spmv(int n, const int* row, const int* col, const double* val, const double* x, double* y,
    double alpha, double beta, int tpr, cudaStream_t s)
{
    launch_rowop<OP_AXPBY>(tpr, n, row, col, val, x, (const double*)nullptr, (const double*)nullptr, y, alpha, beta,
        nullptr, s);
}

void rowop_spmv(const DevCsr& A, const double* x, double* y, const int* skip, cudaStream_t s)
{
    launch_rowop_A<OP_AXPBY>(A.tpr, A, A.val.p, x, (const double*)nullptr, (const double*)nullptr, y,
        1.0, 0.0, skip, s);
}

void rowop_resid(const DevCsr& A, const double* x, const double* f, double* y, const int* skip, cudaStream_t s)
{
    launch_rowop_A<OP_RESID>(A.tpr, A, A.val.p, x, f, (const double*)nullptr, y, 1.0, 0.0, skip, s);
}

// ------------------------------------------------------------------------------------------
// element-wise kernels of the cycle
// ------------------------------------------------------------------------------------------
// Sweep from a zero iterate: u = f / M; optionally keeps a converted copy of f.
template <typename FT, typename MT, typename YT, typename CT>
__global__ void k_first_sweep(int n, const FT* __restrict__ f, const MT* __restrict__ M, YT* __restrict__ u,
    CT* __restrict__ fcopy, const int* __restrict__ skip)
{
    dep_wait();
    dep_release();
    if (skip && *skip) return;
    using AT = typename Wider<MT>::type;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        AT fi = (AT)f[i];
        if (fcopy) fcopy[i] = (CT)fi;
        u[i] = (YT)(fi / (AT)M[i]);
    }
}

// k l1-Jacobi sweeps of a small level in one block of kChainThreads threads: the sweeps of
// Cycle::chain (the first from a zero iterate when src is null), each followed by a block-wide
// barrier, so a chain is one launch instead of k. Sweep i writes out[i]: out[k-1] = dst, and
// out[i] = q0 for even k-2-i, q1 otherwise (the ping-pong order of chain). The row arithmetic is
// k_first_sweep's and k_rowop<S, OP_JACOBI>'s, so the iterates are the same; vectors written by
// the block are gathered with coherent loads.
constexpr int kChainThreads = 1024;
constexpr long kChainMaxNnz = 65536;   // larger levels keep one launch per sweep (32768: -2 %, 262144: -9 % on the batch benchmark)

template <int S, typename T, typename IT>
__global__ void __launch_bounds__(kChainThreads) k_chain_block(int n, const int* __restrict__ row, const IT* __restrict__ col,
    const T* __restrict__ val, const T* __restrict__ f, const T* __restrict__ M, const T* src, T* dst, T* q0, T* q1, int k,
    const int* __restrict__ skip)
{
    dep_wait();
    dep_release();
    if (skip && *skip) return;
    using AT = typename Acc<T>::type;
    using WT = typename Wider<T>::type;
    const int lane = threadIdx.x & (S - 1);
    const int sub = (threadIdx.x & 31) / S;
    const int rows_per_step = blockDim.x / S;
    const T* in = src;
    for (int i = 0; i < k; i++) {
        T* out = i == k - 1 ? dst : (((k - 2 - i) & 1) == 0 ? q0 : q1);
        if (in == nullptr) {
            for (int r = threadIdx.x; r < n; r += blockDim.x) out[r] = (T)((WT)f[r] / (WT)M[r]);
        } else {
            for (int base = (threadIdx.x & ~31) / S; base < n; base += rows_per_step) {
                const int r = base + sub;
                AT sum = 0;
                if (r < n) sum = row_partial<S, AT, false>(__ldg(row + r), __ldg(row + r + 1), lane, r, col, val, in);
                sum = subwarp_sum<S>(sum);
                if (r < n && lane == 0) out[r] = (T)(((-sum + (AT)f[r]) / (AT)M[r]) + (AT)in[r]);
            }
        }
        __syncthreads();
        in = out;
    }
}

template <typename T>
__global__ void k_zero(int n, T* __restrict__ a, const int* __restrict__ skip)
{
    dep_wait();
    dep_release();
    if (skip && *skip) return;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) a[i] = T(0);
}

template <typename ST, typename DT>
__global__ void k_convert(int n, const ST* __restrict__ a, DT* __restrict__ b, const int* __restrict__ skip)
{
    dep_wait();
    dep_release();
    if (skip && *skip) return;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) b[i] = (DT)a[i];
}

// out[c] = sum over the fine rows i of aggregate c (ascending) of p_i * res_i  (R = P^T).
template <typename RT, typename WT, typename OT>
__global__ void k_restrict(int nc, const int* __restrict__ rptr, const int* __restrict__ ridx,
    const WT* __restrict__ rval, const RT* __restrict__ res, OT* __restrict__ out, const int* __restrict__ skip)
{
    dep_wait();
    dep_release();
    if (skip && *skip) return;
    using AT = typename Wider<OT>::type;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (long)gridDim.x * blockDim.x) {
        AT s = 0;
        for (int t = rptr[c]; t < rptr[c + 1]; t++) s = mad_rn((AT)rval[t], (AT)res[ridx[t]], s);
        out[c] = (OT)s;
    }
}

// y = p .* xc[agg] + x  (P has one entry per row; y may alias x).
template <typename PT, typename CT, typename XT, typename YT>
__global__ void k_prolong(int n, const int* __restrict__ agg, const PT* __restrict__ p, const CT* __restrict__ xc,
    const XT* x, YT* y, const int* __restrict__ skip)
{
    dep_wait();
    dep_release();
    if (skip && *skip) return;
    using AT = typename Wider<YT>::type;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        y[i] = (YT)mad_rn((AT)p[i], (AT)xc[agg[i]], (AT)x[i]);
}

// grid for an element-wise kernel over n elements
template <typename Kern>
static int ew_grid(Kern kern, long n) { return fit_grid(kern, 256, (n + 255) / 256); }

// ------------------------------------------------------------------------------------------
// block launches (blockops.cuh)
// ------------------------------------------------------------------------------------------
static int ceil_log2(int k)
{
    int lg = 0;
    while ((1 << lg) < k) lg++;
    return lg;
}

static bool aligned_for(const void* p, int W, size_t elem)
{
    const size_t a = std::min<size_t>(16, W * elem);
    return p == nullptr || ((uintptr_t)p % a) == 0;
}

// Y = alpha A X + beta Y / F - A X / Jacobi sweep on blocks with leading dimension ld and K
// columns (X has m rows); vector loads and stores when the pointers and ld allow them, else one
// column per lane.
template <int OP, typename VT, typename XT, typename FT, typename MT, typename YT>
static void launch_blk_rowop(int n, int m, int ld, int K, const int* row, const int* col, const VT* val, const XT* x,
    const FT* f, const MT* M, YT* y, double alpha, double beta, const int* skip, cudaStream_t s)
{
    if (n <= 0) return;
    BlkShape sh = blk_shape(K, (int)sizeof(XT));
    if (sh.W > 1 && (ld % sh.W != 0 || !aligned_for(x, sh.W, sizeof(XT)) || !aligned_for(y, sh.W, sizeof(YT)) ||
                        !aligned_for(f, sh.W, sizeof(FT))))
        sh = BlkShape { 1, ceil_log2(K) };
    const long per_block = blk_rows_per_block<VT>(sh.lpe_log2, kBlkRowopThreads);
    const long need = ((long)n + per_block - 1) / per_block;
    const int stage_ok = (long)m * ld <= 0x7fffffffL ? 1 : 0;
    auto go = [&](auto kern) {
        note_launch();
        kern<<<fit_grid(kern, kBlkRowopThreads, need), kBlkRowopThreads, 0, s>>>(n, sh.lpe_log2, ld, K, row, col, val, x,
            f, M, y, alpha, beta, stage_ok, skip);
    };
    if constexpr (sizeof(XT) == 4) {
        if (sh.W == 4) {
            go(k_blk_rowop<OP, 4, VT, XT, FT, MT, YT>);
            BCMGX_CHECK_LAUNCH();
            return;
        }
    }
    if (sh.W == 2) go(k_blk_rowop<OP, 2, VT, XT, FT, MT, YT>);
    else go(k_blk_rowop<OP, 1, VT, XT, FT, MT, YT>);
    BCMGX_CHECK_LAUNCH();
}

// ------------------------------------------------------------------------------------------
// the cycle: one code path for a single vector (lk < 0: the sub-warp row kernels above) and for
// blocks of 2^lk right-hand sides (the block kernels of blockops.cuh)
// ------------------------------------------------------------------------------------------
template <typename T> static int tcode() { return std::is_same<T, float>::value ? 1 : 0; }

// Launches k_persist cooperatively (every block resident) with up to two blocks per SM; af, ax,
// ay: the vectors of the program's argument slots.
static void launch_persist(bcmgx_hierarchy* H, const PStep* steps, int nsteps, const int* skip, cudaStream_t s,
    const void* af, const void* ax, void* ay)
{
    stage_fault_init();
    int want = 2;
    if (const char* e = std::getenv("BCMGX_PERSIST_BLOCKS")) want = std::max(1, std::atoi(e));
    const int per_sm = std::min(want, blocks_per_sm((const void*)k_persist, kPersistThreads, 0));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(num_sms() * std::max(per_sm, 1)));
    cfg.blockDim = dim3(kPersistThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // fault-path test hook: BCMGX_TEST_PERSIST_FAULT=<ns> (read at every launch; a captured graph
    // keeps the value of its capture) shortens the barrier wait and drops block 0
    unsigned long long wait_ns = kPersistWaitNs;
    int drop = 0;
    if (const char* e = std::getenv("BCMGX_TEST_PERSIST_FAULT"))
        if (std::atoll(e) > 0) {
            wait_ns = (unsigned long long)std::atoll(e);
            drop = 1;
        }
    note_launch();
    BCMGX_CUDA(cudaLaunchKernelEx(&cfg, k_persist, steps, nsteps, H->persist_bar.p, g_stage_fault, skip, af, ax, ay,
        wait_ns, drop));
}

// Resets the persistent cycle's barrier words (and a poisoned state left by a timeout); once at
// the start of every solve or preconditioner application.
static void persist_reset(bcmgx_hierarchy* H, cudaStream_t s)
{
    if (H->persist_level >= 0) BCMGX_CUDA(cudaMemsetAsync(H->persist_bar.p, 0, 4 * sizeof(unsigned), s));
}

// Entries of the largest level that the persistent cycle takes; 0, the default, leaves it off:
// measured on one B200 it was slower than the graph-launched kernels it replaces (a grid barrier
// costs about what a graph kernel node does, and the cooperative launch inside the solve graph
// costs more: the 7-point 50^3 solve went from 2.6 to 4.9 ms, the 27-point 160^3 solve from 58.9
// to 64.8 ms). BCMGX_PERSIST_NNZ=<entries> turns it on.
constexpr int64_t kPersistMaxNnz = 0;

static int choose_persist_level(const bcmgx_hierarchy* H)
{
    int64_t limit = kPersistMaxNnz;
    if (const char* e = std::getenv("BCMGX_PERSIST_NNZ")) limit = std::atoll(e);
    if (limit <= 0 || H->prm.preconditioner != BCMGX_PREC_BCMG) return -1;
    int lc = -1;
    for (int l = (int)H->lv.size() - 1; l >= 0; l--) {
        if (H->lv[l].A.nnz > limit) break;
        lc = l;
    }
    return lc;
}

struct Cycle {
    bcmgx_hierarchy* H;
    const CycleBufs& B;
    cudaStream_t s;
    const int* skip;
    bool fp32;
    int L;
    int lk;   // -1: single vector; else the block has 2^lk columns (leading dimension 2^lk)
    // recording mode (persist.cuh): the steps are appended here instead of launched
    std::vector<PStep>* rec = nullptr;

    bool lf32(int l) const { return fp32 && l < L - 1; }
    Level& lv(int l) const { return H->lv[l]; }
    template <typename Kern>
    int grid(Kern kern, int n) const { return ew_grid(kern, lk < 0 ? (long)n : ((long)n << lk)); }

    // ---- kernel dispatch (single vector or block) ----
    template <int OP, typename VT, typename XT, typename FT, typename MT, typename YT>
    void rowop(const DevCsr& A, const VT* val, const XT* x, const FT* f, const MT* M, YT* y) const
    {
        if (rec) {
            PStep p {};
            p.op = OP == OP_JACOBI ? P_JACOBI : P_RESID;
            p.n = A.n;
            p.S = A.tpr;
            p.vt = tcode<VT>();
            const VT* own = std::is_same<VT, float>::value ? (const VT*)A.val32.p : (const VT*)A.val.p;
            const void* tab = std::is_same<VT, float>::value ? (const void*)A.vtab32.p : (const void*)A.vtab64.p;
            p.coded = (A.vcode.p && tab && val == own) ? 1 : 0;
            p.val = p.coded ? tab : (const void*)val;
            p.code = p.coded ? A.vcode.p : nullptr;
            p.col16 = A.dcol.p ? 1 : 0;
            p.col = A.dcol.p ? (const void*)A.dcol.p : (const void*)A.col.p;
            p.row = A.row.p;
            p.x = x;
            p.xt = tcode<XT>();
            p.f = f;
            p.ft = tcode<FT>();
            p.M = M;
            p.mt = tcode<MT>();
            p.y = y;
            p.yt = tcode<YT>();
            BCMGX_REQUIRE(OP != OP_AXPBY && p.xt == p.vt, BCMGX_ERR_INTERNAL, "cycle step without a persistent form");
            rec->push_back(p);
            return;
        }
        if (lk < 0) launch_rowop_A<OP>(A.tpr, A, val, x, f, M, y, 1.0, 0.0, skip, s);
        else launch_blk_rowop<OP>(A.n, A.m, 1 << lk, 1 << lk, A.row.p, A.col.p, val, x, f, M, y, 1.0, 0.0, skip, s);
    }
    template <typename FT, typename MT, typename YT, typename CT>
    void first(int n, const FT* f, const MT* M, YT* u, CT* fcopy) const
    {
        if (rec) {
            PStep p {};
            p.op = P_FIRST;
            p.n = n;
            p.f = f;
            p.ft = tcode<FT>();
            p.M = M;
            p.mt = tcode<MT>();
            p.y = u;
            p.yt = tcode<YT>();
            p.extra = fcopy;
            p.ct = tcode<CT>();
            rec->push_back(p);
            return;
        }
        if (lk >= 0) {
            auto k = k_blk_first_sweep<FT, MT, YT, CT>;
            note_launch();
            k<<<grid(k, n), 256, 0, s>>>(n, lk, f, M, u, fcopy, skip);
        } else {
            auto k = k_first_sweep<FT, MT, YT, CT>;
            launch_dep(k, grid(k, n), 256, 0, s, n, f, M, u, fcopy, skip);
        }
        BCMGX_CHECK_LAUNCH();
    }
    template <typename ST, typename DT>
    void convert(int n, const ST* a, DT* b) const
    {
        if (rec) {
            PStep p {};
            p.op = P_CONVERT;
            p.n = n;
            p.x = a;
            p.xt = tcode<ST>();
            p.y = b;
            p.yt = tcode<DT>();
            rec->push_back(p);
            return;
        }
        if (lk >= 0) {
            auto k = k_blk_convert<ST, DT>;
            note_launch();
            k<<<grid(k, n), 256, 0, s>>>(n, lk, a, b, skip);
        } else {
            auto k = k_convert<ST, DT>;
            launch_dep(k, grid(k, n), 256, 0, s, n, a, b, skip);
        }
        BCMGX_CHECK_LAUNCH();
    }
    template <typename T>
    void zero_n(int n, T* a) const
    {
        if (rec) {
            PStep p {};
            p.op = P_ZERO;
            p.n = n;
            p.y = a;
            p.yt = tcode<T>();
            rec->push_back(p);
            return;
        }
        if (lk >= 0) {
            auto k = k_blk_zero<T>;
            note_launch();
            k<<<grid(k, n), 256, 0, s>>>(n, lk, a, skip);
        } else {
            auto k = k_zero<T>;
            launch_dep(k, grid(k, n), 256, 0, s, n, a, skip);
        }
        BCMGX_CHECK_LAUNCH();
    }
    // out = P^T res: for a block, an SpMM with the stored transpose (rptr, ridx, rval)
    template <typename RT, typename WT, typename OT>
    void restrict_to(int nc, const Level& V, const WT* rval, const RT* res, OT* out) const
    {
        if (rec) {
            PStep p {};
            p.op = P_RESTRICT;
            p.n = nc;
            p.idx = V.rptr.p;
            p.idx2 = V.ridx.p;
            p.M = rval;
            p.mt = tcode<WT>();
            p.f = res;
            p.ft = tcode<RT>();
            p.y = out;
            p.yt = tcode<OT>();
            rec->push_back(p);
            return;
        }
        if (lk >= 0) {
            launch_blk_rowop<OP_AXPBY>(nc, V.A.n, 1 << lk, 1 << lk, V.rptr.p, V.ridx.p, rval, res, (const OT*)nullptr,
                (const OT*)nullptr, out, 1.0, 0.0, skip, s);
            return;
        }
        auto k = k_restrict<RT, WT, OT>;
        launch_dep(k, grid(k, nc), 256, 0, s, nc, V.rptr.p, V.ridx.p, rval, res, out, skip);
        BCMGX_CHECK_LAUNCH();
    }
    template <typename PT, typename CT, typename XT, typename YT>
    void prolong(int n, const Level& V, const PT* p, const CT* xc, const XT* x, YT* y) const
    {
        if (rec) {
            PStep q {};
            q.op = P_PROLONG;
            q.n = n;
            q.idx = V.agg.p;
            q.M = p;
            q.mt = tcode<PT>();
            q.xc = xc;
            q.ct = tcode<CT>();
            q.x = x;
            q.xt = tcode<XT>();
            q.y = y;
            q.yt = tcode<YT>();
            rec->push_back(q);
            return;
        }
        if (lk >= 0) {
            auto k = k_blk_prolong<PT, CT, XT, YT>;
            note_launch();
            k<<<grid(k, n), 256, 0, s>>>(n, lk, V.agg.p, p, xc, x, y, skip);
        } else {
            auto k = k_prolong<PT, CT, XT, YT>;
            launch_dep(k, grid(k, n), 256, 0, s, n, V.agg.p, p, xc, x, y, skip);
        }
        BCMGX_CHECK_LAUNCH();
    }

    // ---- cycle steps on typed views ----
    void sweep(int l, Vec f, Vec in, Vec out) const
    {
        Level& V = lv(l);
        const DevCsr& A = V.A;
        if (!lf32(l))
            rowop<OP_JACOBI>(A, A.val.p, (const double*)in.p, (const double*)f.p, V.M.p, (double*)out.p);
        else if (out.f32)
            rowop<OP_JACOBI>(A, A.val32.p, (const float*)in.p, (const float*)f.p, V.M32.p, (float*)out.p);
        else
            rowop<OP_JACOBI>(A, A.val32.p, (const float*)in.p, (const float*)f.p, V.M32.p, (double*)out.p);
    }

    // sweep from zero; if fcopy is given (level 0 of the FP32 cycle) f is double and is also
    // converted into fcopy.
    void first_sweep(int l, Vec f, Vec out, Vec fcopy) const
    {
        Level& V = lv(l);
        const int n = V.A.n;
        if (!lf32(l)) {
            first(n, (const double*)f.p, V.M.p, (double*)out.p, (double*)nullptr);
        } else if (f.f32) {
            if (out.f32) first(n, (const float*)f.p, V.M32.p, (float*)out.p, (float*)nullptr);
            else first(n, (const float*)f.p, V.M32.p, (double*)out.p, (float*)nullptr);
        } else {
            if (out.f32) first(n, (const double*)f.p, V.M32.p, (float*)out.p, (float*)fcopy.p);
            else first(n, (const double*)f.p, V.M32.p, (double*)out.p, (float*)fcopy.p);
        }
    }

    void copy(Vec a, Vec b, int n) const
    {
        if (a.f32 && b.f32) convert(n, (const float*)a.p, (float*)b.p);
        else if (!a.f32 && !b.f32) convert(n, (const double*)a.p, (double*)b.p);
        else if (a.f32) convert(n, (const float*)a.p, (double*)b.p);
        else convert(n, (const double*)a.p, (float*)b.p);
    }

    void zero(Vec a, int n) const
    {
        if (a.f32) zero_n(n, (float*)a.p);
        else zero_n(n, (double*)a.p);
    }

    // k sweeps from `src` (p == nullptr: zero iterate) ending in `dst`, using the level
    // buffers A and B as intermediates. fcopy: see first_sweep.
    void chain(int l, int k, Vec f, Vec src, Vec dst, Vec A, Vec Bf, Vec fcopy = Vec()) const
    {
        const int n = lv(l).A.n;
        if (k <= 0) {
            if (src.p == nullptr) zero(dst, n);
            else if (src != dst) copy(src, dst, n);
            return;
        }
        std::vector<Vec> out(k);
        out[k - 1] = dst;
        for (int i = k - 2; i >= 0; i--) out[i] = (out[i + 1] == A) ? Bf : A;
        if (src.p != nullptr && src == out[0]) {
            Vec other = (src == A) ? Bf : A;
            copy(src, other, n);
            src = other;
        }
        if (chain_in_block(l, k, f, src, dst, A, Bf, fcopy)) return;
        Vec fl = f;
        for (int i = 0; i < k; i++) {
            if (i == 0 && src.p == nullptr) {
                first_sweep(l, f, out[0], fcopy);
                if (fcopy.p) fl = fcopy;   // later sweeps read the converted right-hand side
            } else {
                sweep(l, fl, i == 0 ? src : out[i - 1], out[i]);
            }
        }
    }

    // While the batch graph is captured (H->chain_in_block), a chain of k >= 2 sweeps on a small
    // single-vector level whose vectors all have the level's precision runs as one k_chain_block
    // launch; returns false otherwise. A solve that has the GPU to itself keeps one launch per
    // sweep: one block works through a level far slower than a grid does, and only when hundreds
    // of systems run side by side is the number of kernels the bound.
    bool chain_in_block(int l, int k, Vec f, Vec src, Vec dst, Vec A, Vec Bf, Vec fcopy) const
    {
        const Level& V = lv(l);
        const DevCsr& Am = V.A;
        const bool f32 = lf32(l);
        if (rec || !H->chain_in_block || lk >= 0 || k < 2 || fcopy.p || Am.nnz > kChainMaxNnz) return false;
        for (const Vec& v : { f, dst, A, Bf })
            if (v.f32 != f32) return false;
        if (src.p && src.f32 != f32) return false;
        const Vec q0 = (dst == A) ? Bf : A;
        const Vec q1 = (q0 == A) ? Bf : A;
        auto go = [&](auto kern, auto val, auto M, auto* tp, auto* colp) {
            using T = std::remove_pointer_t<decltype(tp)>;
            note_launch();
            kern<<<1, kChainThreads, 0, s>>>(Am.n, Am.row.p, colp, val, (const T*)f.p, M, (const T*)src.p, (T*)dst.p,
                (T*)q0.p, (T*)q1.p, k, skip);
            BCMGX_CHECK_LAUNCH();
        };
        auto dispatch = [&](auto* tp, auto val, auto M) {
            using T = std::remove_pointer_t<decltype(tp)>;
            auto with_col = [&](auto* colp) {
                using IT = std::remove_const_t<std::remove_pointer_t<decltype(colp)>>;
                switch (Am.tpr) {
                case 1: go(k_chain_block<1, T, IT>, val, M, tp, colp); break;
                case 2: go(k_chain_block<2, T, IT>, val, M, tp, colp); break;
                case 4: go(k_chain_block<4, T, IT>, val, M, tp, colp); break;
                case 8: go(k_chain_block<8, T, IT>, val, M, tp, colp); break;
                case 16: go(k_chain_block<16, T, IT>, val, M, tp, colp); break;
                default: go(k_chain_block<32, T, IT>, val, M, tp, colp); break;
                }
            };
            if (Am.dcol.p) with_col((const short*)Am.dcol.p);
            else with_col((const int*)Am.col.p);
        };
        if (f32) dispatch((float*)nullptr, (const float*)Am.val32.p, (const float*)V.M32.p);
        else dispatch((double*)nullptr, (const double*)Am.val.p, (const double*)V.M.p);
        return true;
    }

    // One cycle on level l for right-hand side f, starting from x_cur (nullptr: zero),
    // leaving the result in dst.
    // The cycle on the levels from l down as one persistent launch (persist.cuh), with the program
    // recorded for this form of the call (ensure_solve_workspace).
    void run_persistent(int l, Vec f, Vec x_cur, Vec dst) const
    {
        const PersistProgram* prog = nullptr;
        for (auto& pp : H->persist)
            if (pp->level == l && pp->has_x == (x_cur.p != nullptr)) prog = pp.get();
        BCMGX_REQUIRE(prog != nullptr, BCMGX_ERR_INTERNAL, "no recorded persistent cycle for this call");
        launch_persist(H, prog->steps.p, prog->nsteps, skip, s, f.p, x_cur.p, dst.p);
    }

    void run(int l, Vec f, Vec x_cur, Vec dst) const
    {
        if (!rec && lk < 0 && !H->chain_in_block && H->persist_level >= 0 && l == H->persist_level) {
            run_persistent(l, f, x_cur, dst);
            return;
        }
        Level& V = lv(l);
        const int n = V.A.n;
        const bool f32 = lf32(l);
        const CycleBufs::L& Lb = B.lv[l];
        const Vec A = (l == 0 && !f32) ? dst : Lb.x;
        const Vec Bf = Lb.x2;
        const bcmgx_params& P = H->prm;
        // level-0 FP32: f arrives in FP64 and is converted once into the level's FP32 rhs
        Vec fcopy;
        if (f32 && !f.f32) fcopy = Lb.rhs;
        if (l == L - 1) {
            chain(l, P.relaxnumber_coarse, f, x_cur, dst, A, Bf, fcopy);
            return;
        }
        const int coeff = P.cycle_type == BCMGX_CYCLE_VARIABLE_V ? (1 << l) : 1;
        const int kpre = P.prerelax_sweeps * coeff, kpost = P.postrelax_sweeps * coeff;
        Vec pre_dst = (dst.f32 == f32) ? dst : A;
        Vec fl = f;
        if (fcopy.p) {
            if (x_cur.p == nullptr && kpre > 0) {
                chain(l, kpre, f, x_cur, pre_dst, A, Bf, fcopy);
            } else {
                copy(f, fcopy, n);
                chain(l, kpre, fcopy, x_cur, pre_dst, A, Bf);
            }
            fl = fcopy;
        } else {
            chain(l, kpre, f, x_cur, pre_dst, A, Bf);
        }
        Vec xpre = pre_dst;
        // residual and restriction
        const DevCsr& Am = V.A;
        Level& C = lv(l + 1);
        const bool cf32 = lf32(l + 1);
        const Vec fc = B.lv[l + 1].rhs;
        const Vec xc_dst = B.lv[l + 1].x;
        if (f32) {
            float* res = (float*)B.res.p;
            rowop<OP_RESID>(Am, Am.val32.p, (const float*)xpre.p, (const float*)fl.p, (const float*)nullptr, res);
            if (cf32) restrict_to(C.A.n, V, V.rval32.p, (const float*)res, (float*)fc.p);
            else restrict_to(C.A.n, V, V.rval.p, (const float*)res, (double*)fc.p);
        } else {
            double* res = (double*)B.res.p;
            rowop<OP_RESID>(Am, Am.val.p, (const double*)xpre.p, (const double*)fl.p, (const double*)nullptr, res);
            restrict_to(C.A.n, V, V.rval.p, (const double*)res, (double*)fc.p);
        }
        Vec xc;   // nullptr: coarse correction is zero
        if (L > 2 || P.relaxnumber_coarse > 0) {
            int visits = l < (int)H->grid_sweeps.size() ? H->grid_sweeps[l] : 1;
            for (int i = 1; i <= visits; i++) {
                run(l + 1, fc, xc, xc_dst);
                xc = xc_dst;
                if (l + 1 == L - 1) break;
            }
        }
        // prolongation into the buffer the post-smoothing chain starts from
        Vec pdst;
        if (kpost <= 0) {
            pdst = dst;
        } else {
            Vec o0 = dst;
            for (int i = kpost - 2; i >= 0; i--) o0 = (o0 == A) ? Bf : A;
            pdst = (o0 == A) ? Bf : A;
        }
        if (xc.p != nullptr) {
            if (!f32) {
                prolong(n, V, V.p.p, (const double*)xc.p, (const double*)xpre.p, (double*)pdst.p);
            } else if (xc.f32) {
                if (pdst.f32) prolong(n, V, V.p32.p, (const float*)xc.p, (const float*)xpre.p, (float*)pdst.p);
                else prolong(n, V, V.p32.p, (const float*)xc.p, (const float*)xpre.p, (double*)pdst.p);
            } else {
                if (pdst.f32) prolong(n, V, V.p32.p, (const double*)xc.p, (const float*)xpre.p, (float*)pdst.p);
                else prolong(n, V, V.p32.p, (const double*)xc.p, (const float*)xpre.p, (double*)pdst.p);
            }
        } else if (pdst != xpre) {
            copy(xpre, pdst, n);
        }
        chain(l, kpost, fl, pdst, dst, A, Bf);
    }
};

// Standalone l1-Jacobi preconditioner: l1jacsweeps sweeps u <- u + (r - A u) / D from u = 0, with
// D = a_ii + sum_{j != i} |a_ij| (l1jacobi_apply, l1jacobi.cu:513-523, and set_l1j, :484-493).
// The sweeps alternate between v and a scratch vector so that the last one writes v.
static void l1jacobi_apply(bcmgx_hierarchy* H, const double* r, double* v, const int* skip)
{
    const DevCsr& A = H->lv[0].A;
    const int n = A.n, k = H->prm.l1jacsweeps;
    cudaStream_t s = H->stream;
    std::vector<double*> out(k);
    out[k - 1] = v;
    for (int i = k - 2; i >= 0; i--) out[i] = (out[i + 1] == v) ? H->l1tmp.p : v;
    auto first = k_first_sweep<double, double, double, double>;
    launch_dep(first, ew_grid(first, n), 256, 0, s, n, r, H->l1d.p, out[0], (double*)nullptr, skip);
    BCMGX_CHECK_LAUNCH();
    for (int i = 1; i < k; i++)
        launch_rowop_A<OP_JACOBI>(A.tpr, A, A.val.p, (const double*)out[i - 1], r, (const double*)H->l1d.p,
            out[i], 1.0, 0.0, skip, s);
}

void prec_apply_impl(bcmgx_hierarchy* H, const double* r, double* v, const int* skip)
{
    const int n0 = H->lv[0].A.n;
    if (H->prm.preconditioner == BCMGX_PREC_L1_JACOBI) {
        l1jacobi_apply(H, r, v, skip);
        return;
    }
    if (H->prm.preconditioner == BCMGX_PREC_AFSAI) {
        afsai_apply(H, r, v, skip);
        return;
    }
    if (H->prm.preconditioner != BCMGX_PREC_BCMG) {
        note_launch();
        auto k = k_convert<double, double>;
        k<<<ew_grid(k, n0), 256, 0, H->stream>>>(n0, r, v, skip);
        BCMGX_CHECK_LAUNCH();
        return;
    }
    Cycle c { H, H->cyc, H->stream, skip, H->prm.vcycle_precision == BCMGX_VCYCLE_FP32, (int)H->lv.size(), -1 };
    c.run(0, Vec { (void*)r, false }, Vec(), Vec { v, false });
}

// The preconditioner on a block of 2^lk right-hand sides (scratch: an n x 2^lk block, needed by
// l1-Jacobi and AFSAI): the block V-cycle, the standalone l1-Jacobi sweeps (l1jacobi_apply on
// every column: the first from zero, the last into v), AFSAI's G^T (G r) as two block SpMMs
// (afsai_apply), or the identity.
void cycle_apply_block(bcmgx_hierarchy* H, const CycleBufs& bufs, int lk, const double* r, double* v, double* scratch,
    const int* skip)
{
    const int n0 = H->lv[0].A.n;
    const int kp = 1 << lk;
    cudaStream_t s = H->stream;
    if (H->prm.preconditioner == BCMGX_PREC_L1_JACOBI) {
        const DevCsr& A = H->lv[0].A;
        const int k = H->prm.l1jacsweeps;
        std::vector<double*> out(k);
        out[k - 1] = v;
        for (int i = k - 2; i >= 0; i--) out[i] = (out[i + 1] == v) ? scratch : v;
        auto first = k_blk_first_sweep<double, double, double, double>;
        note_launch();
        first<<<ew_grid(first, (long)n0 << lk), 256, 0, s>>>(n0, lk, r, H->l1d.p, out[0], (double*)nullptr, skip);
        BCMGX_CHECK_LAUNCH();
        for (int i = 1; i < k; i++)
            launch_blk_rowop<OP_JACOBI>(n0, n0, kp, kp, A.row.p, A.col.p, A.val.p, (const double*)out[i - 1], r,
                (const double*)H->l1d.p, out[i], 1.0, 0.0, skip, s);
        return;
    }
    if (H->prm.preconditioner == BCMGX_PREC_AFSAI) {
        const DevCsr& G = H->afsai_G;
        const DevCsr& GT = H->afsai_GT;
        launch_blk_rowop<OP_AXPBY>(n0, n0, kp, kp, G.row.p, G.col.p, G.val.p, r, (const double*)nullptr,
            (const double*)nullptr, scratch, 1.0, 0.0, skip, s);
        launch_blk_rowop<OP_AXPBY>(n0, n0, kp, kp, GT.row.p, GT.col.p, GT.val.p, (const double*)scratch,
            (const double*)nullptr, (const double*)nullptr, v, 1.0, 0.0, skip, s);
        return;
    }
    if (H->prm.preconditioner != BCMGX_PREC_BCMG) {
        note_launch();
        auto k = k_blk_convert<double, double>;
        k<<<ew_grid(k, (long)n0 << lk), 256, 0, H->stream>>>(n0, lk, r, v, skip);
        BCMGX_CHECK_LAUNCH();
        return;
    }
    Cycle c { H, bufs, H->stream, skip, H->prm.vcycle_precision == BCMGX_VCYCLE_FP32, (int)H->lv.size(), lk };
    c.run(0, Vec { (void*)r, false }, Vec(), Vec { v, false });
}

void launch_spmm(int n, int m, int K, const int* row, const int* col, const double* val, const double* X, double* Y,
    double alpha, double beta, cudaStream_t s)
{
    launch_blk_rowop<OP_AXPBY>(n, m, K, K, row, col, val, X, (const double*)nullptr, (const double*)nullptr, Y, alpha,
        beta, nullptr, s);
}

void prec_apply_dev(bcmgx_hierarchy* H, const double* r, double* v)
{
    ensure_solve_workspace(H);
    persist_reset(H, H->stream);
    prec_apply_impl(H, r, v, nullptr);
}

void persist_reset_ext(bcmgx_hierarchy* H, cudaStream_t s) { persist_reset(H, s); }

// ------------------------------------------------------------------------------------------
// FP64 cycle steps on caller-chosen vectors (the row-partitioned cycle, dist.cu)
// ------------------------------------------------------------------------------------------
void step_jacobi64(const Level& V, const double* x, const double* f, double* y, cudaStream_t s)
{
    launch_rowop_A<OP_JACOBI>(V.A.tpr, V.A, V.A.val.p, x, f, V.M.p, y, 1.0, 0.0, nullptr, s);
}

void step_resid64(const Level& V, const double* x, const double* f, double* y, cudaStream_t s)
{
    launch_rowop_A<OP_RESID>(V.A.tpr, V.A, V.A.val.p, x, f, (const double*)nullptr, y, 1.0, 0.0, nullptr, s);
}

void step_first64(const Level& V, const double* f, double* u, cudaStream_t s)
{
    const int n = V.A.n;
    if (n <= 0) return;
    auto k = k_first_sweep<double, double, double, double>;
    note_launch();
    k<<<ew_grid(k, n), 256, 0, s>>>(n, f, V.M.p, u, (double*)nullptr, nullptr);
    BCMGX_CHECK_LAUNCH();
}

void step_restrict64(const Level& V, int nc, const double* res, double* out, cudaStream_t s)
{
    if (nc <= 0) return;
    auto k = k_restrict<double, double, double>;
    note_launch();
    k<<<ew_grid(k, nc), 256, 0, s>>>(nc, V.rptr.p, V.ridx.p, V.rval.p, res, out, nullptr);
    BCMGX_CHECK_LAUNCH();
}

void step_prolong64(const Level& V, const double* xc, const double* x, double* y, cudaStream_t s)
{
    const int n = V.A.n;
    if (n <= 0) return;
    auto k = k_prolong<double, double, double, double>;
    note_launch();
    k<<<ew_grid(k, n), 256, 0, s>>>(n, V.agg.p, V.p.p, xc, x, y, nullptr);
    BCMGX_CHECK_LAUNCH();
}

void step_copy64(int n, const double* a, double* b, cudaStream_t s)
{
    if (n <= 0 || a == b) return;
    BCMGX_CUDA(cudaMemcpyAsync(b, a, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
}

void step_zero64(int n, double* a, cudaStream_t s)
{
    if (n <= 0) return;
    BCMGX_CUDA(cudaMemsetAsync(a, 0, sizeof(double) * n, s));
}

// ------------------------------------------------------------------------------------------
// FCG kernels
// ------------------------------------------------------------------------------------------
constexpr int kRedBlocksPerSM = 8;
constexpr int kRedThreads = 256;

// grid of the FCG kernels: at most kRedBlocksPerSM blocks per SM (the size of the partials)
template <typename Kern>
static int red_grid(Kern kern, long work_threads)
{
    const long need = (work_threads + kRedThreads - 1) / kRedThreads;
    return std::min(fit_grid(kern, kRedThreads, need), num_sms() * kRedBlocksPerSM);
}

// r = b - A x and ||r||^2 -> delta0, tolerance (FCG.cu:46-51).
template <int S, typename IT>
__global__ void __launch_bounds__(kRedThreads) k_fcg_resid0(int n, const int* __restrict__ row, const IT* __restrict__ col,
    const double* __restrict__ val, const double* __restrict__ x, const double* __restrict__ b, double* __restrict__ r,
    FcgState* st, double* partials)
{
    dep_wait();
    dep_release();
    const int lane = threadIdx.x & (S - 1);
    const int sub = (threadIdx.x & 31) / S;
    const long stride = (long)gridDim.x * blockDim.x / S;
    double acc[1] = { 0.0 };
    for (long base = ((long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / S; base < n; base += stride) {
        const long r0 = base + sub;
        double s = 0;
        if (r0 < n) s = row_partial<S, double>(row[r0], row[r0 + 1], lane, (int)r0, col, val, x);
        s = subwarp_sum<S>(s);
        if (r0 < n && lane == 0) {
            double ri = -1.0 * s + 1.0 * b[r0];
            r[r0] = ri;
            acc[0] += ri * ri;
        }
    }
    double out[1];
    if (grid_sum<1>(acc, partials, &st->ticket[0], out) && threadIdx.x == 0) {
        st->delta0 = sqrt(out[0]);
        st->tol = st->tol * st->delta0;   // tol holds rtol on entry
        st->iter = 0;
        st->done = 0;
        st->bad = 0;
    }
}

// The dots of the step after pw = A pv (the level-0 FP64 row kernel, launched before): start-up
// (mode 0): alpha = r.pv, beta = pw.pv, delta = beta, theta = alpha / delta (FCG.cu:59-86); loop
// (mode 1): alpha = r.pv, beta = pw.pv, gamma = oq.pv (triple_innerproduct,
// triple_inner_product.cu:7-101) followed by the scalar recurrence theta = gamma/delta, delta =
// beta - gamma^2/delta, theta2 = alpha/delta (FCG.cu:132-136). The sums run in a fixed order
// whichever row kernel formed pw (so staged and plain solves agree bit for bit); VEC: 16-byte
// loads on aligned vectors.
template <int MODE, bool VEC>
__global__ void __launch_bounds__(kRedThreads, 4) k_fcg_dots(int n, const double* __restrict__ pv,
    const double* __restrict__ pw, const double* __restrict__ r, const double* __restrict__ oq, FcgState* st,
    double* partials, const int* __restrict__ skip)
{
    dep_wait();
    dep_release();
    if (skip && *skip) return;
    double acc[3] = { 0.0, 0.0, 0.0 };
    auto one = [&](long i) {
        const double vi = pv[i];
        acc[0] += r[i] * vi;
        acc[1] += pw[i] * vi;
        if (MODE == 1) acc[2] += oq[i] * vi;
    };
    if (VEC) {
        const long n2 = n >> 1;
        const double2* pv2 = reinterpret_cast<const double2*>(pv);
        const double2* pw2 = reinterpret_cast<const double2*>(pw);
        const double2* r2 = reinterpret_cast<const double2*>(r);
        const double2* oq2 = reinterpret_cast<const double2*>(oq);
        for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += (long)gridDim.x * blockDim.x) {
            const double2 v = pv2[i], w = pw2[i], rr = r2[i];
            acc[0] += rr.x * v.x;
            acc[0] += rr.y * v.y;
            acc[1] += w.x * v.x;
            acc[1] += w.y * v.y;
            if (MODE == 1) {
                const double2 q = oq2[i];
                acc[2] += q.x * v.x;
                acc[2] += q.y * v.y;
            }
        }
        if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) one(n - 1);
    } else {
        for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) one(i);
    }
    double out[3];
    if (grid_sum<3>(acc, partials, &st->ticket[1], out) && threadIdx.x == 0) {
        st->alpha = out[0];
        st->beta = out[1];
        if (MODE == 0) {
            st->delta = out[1];
            st->theta = out[0] / out[1];
        } else {
            st->gamma = out[2];
            const double th = out[2] / st->delta;
            const double dn = out[1] - ((out[2] * out[2]) / st->delta);
            st->theta = th;
            st->delta = dn;
            st->theta2 = out[0] / dn;
        }
        if (!(st->delta > 0.0) || !isfinite(st->theta)) st->bad = 1;
    }
}

// Start-up update x += theta v, r -= theta w, d = v, q = w, ||r||^2 (FCG.cu:88-100).
__global__ void __launch_bounds__(kRedThreads) k_fcg_update0(int n, const double* __restrict__ v, const double* __restrict__ w,
    double* __restrict__ x, double* __restrict__ r, double* __restrict__ d, double* __restrict__ q, FcgState* st, double* partials,
    double* hist)
{
    dep_wait();
    dep_release();
    if (st->bad) return;
    const double th = st->theta;
    double acc[1] = { 0.0 };
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double vi = v[i], wi = w[i];
        x[i] = th * vi + 1.0 * x[i];
        const double ri = -th * wi + 1.0 * r[i];
        r[i] = ri;
        d[i] = vi;
        q[i] = wi;
        acc[0] += ri * ri;
    }
    double out[1];
    if (grid_sum<1>(acc, partials, &st->ticket[2], out) && threadIdx.x == 0) {
        st->rnorm2 = out[0];
        if (hist) hist[0] = sqrt(out[0]);
    }
}

// Loop update: pv = -theta od + pv; x += theta2 pv; pw = -theta oq + pw; r -= theta2 pw
// (double_merged_axpy x2, FCG.cu:138-144), ||r|| and the stopping test (FCG.cu:146-156).
// VEC: all six vectors 16-byte aligned; each thread then moves two entries per 16-byte load and
// store (a streaming kernel wants bytes in flight), the odd last entry going to thread 0. At most
// 64 registers, so that four blocks of 256 threads stay resident per SM.
template <bool VEC>
__global__ void __launch_bounds__(kRedThreads, 4) k_fcg_update(int n, double* __restrict__ pv, const double* __restrict__ od,
    double* __restrict__ x, double* __restrict__ pw, const double* __restrict__ oq, double* __restrict__ r, FcgState* st,
    double* partials, double* hist, const int* __restrict__ skip)
{
    dep_wait();
    dep_release();
    if (skip && *skip) return;
    // a breakdown found by the dots kernel leaves x at the last valid iterate
    if (st->bad) {
        if (blockIdx.x == 0 && threadIdx.x == 0) st->done = 1;
        return;
    }
    const double th = st->theta, th2 = st->theta2;
    double acc[1] = { 0.0 };
    auto one = [&](long i) {
        const double nv = -th * od[i] + pv[i];
        pv[i] = nv;
        x[i] = th2 * nv + x[i];
        const double nw = -th * oq[i] + pw[i];
        pw[i] = nw;
        const double ri = -th2 * nw + r[i];
        r[i] = ri;
        acc[0] += ri * ri;
    };
    if (VEC) {
        const long n2 = n >> 1;
        double2* pv2 = reinterpret_cast<double2*>(pv);
        const double2* od2 = reinterpret_cast<const double2*>(od);
        double2* x2 = reinterpret_cast<double2*>(x);
        double2* pw2 = reinterpret_cast<double2*>(pw);
        const double2* oq2 = reinterpret_cast<const double2*>(oq);
        double2* r2 = reinterpret_cast<double2*>(r);
        for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += (long)gridDim.x * blockDim.x) {
            const double2 a = od2[i], b = pv2[i], c = oq2[i], d = pw2[i], e = x2[i], f = r2[i];
            double2 nv, nw, nx, nr;
            nv.x = -th * a.x + b.x;
            nv.y = -th * a.y + b.y;
            nx.x = th2 * nv.x + e.x;
            nx.y = th2 * nv.y + e.y;
            nw.x = -th * c.x + d.x;
            nw.y = -th * c.y + d.y;
            nr.x = -th2 * nw.x + f.x;
            nr.y = -th2 * nw.y + f.y;
            pv2[i] = nv;
            x2[i] = nx;
            pw2[i] = nw;
            r2[i] = nr;
            acc[0] += nr.x * nr.x;
            acc[0] += nr.y * nr.y;
        }
        if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) one(n - 1);
    } else {
        for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) one(i);
    }
    double out[1];
    if (grid_sum<1>(acc, partials, &st->ticket[3], out) && threadIdx.x == 0) {
        st->rnorm2 = out[0];
        const double l2 = sqrt(out[0]);
        st->iter += 1;
        if (hist) hist[st->iter] = l2;
        if (!isfinite(l2)) st->bad = 1;
        st->done = (!(l2 > st->tol) || st->iter >= st->itnlim || st->bad) ? 1 : 0;
    }
}

// The loop update on the hierarchy's stream (the vector form when every vector allows it).
static void fcg_update(int n, double* pv, const double* od, double* x, double* pw, const double* oq, double* r,
    FcgState* st, double* part, double* hist, const int* skip, cudaStream_t s)
{
    if (al16(pv) && al16(od) && al16(x) && al16(pw) && al16(oq) && al16(r)) {
        auto k = k_fcg_update<true>;
        launch_dep<2>(k, red_grid(k, ((long)n + 1) / 2), kRedThreads, 0, s, n, pv, od, x, pw, oq, r, st, part, hist, skip);
    } else {
        auto k = k_fcg_update<false>;
        launch_dep<2>(k, red_grid(k, n), kRedThreads, 0, s, n, pv, od, x, pw, oq, r, st, part, hist, skip);
    }
    BCMGX_CHECK_LAUNCH();
}

template <int S>
static void launch_resid0(const DevCsr& A, const double* x, const double* b, double* r, FcgState* st, double* part, cudaStream_t s)
{
    if (A.dcol.p) {
        auto k = k_fcg_resid0<S, short>;
        launch_dep<2>(k, red_grid(k, (long)A.n * S), kRedThreads, 0, s, A.n, A.row.p, A.dcol.p, A.val.p, x, b, r, st, part);
    } else {
        auto k = k_fcg_resid0<S, int>;
        launch_dep<2>(k, red_grid(k, (long)A.n * S), kRedThreads, 0, s, A.n, A.row.p, A.col.p, A.val.p, x, b, r, st, part);
    }
}
// ||r||^2 -> delta0 and the tolerance, as k_fcg_resid0 finishes, for an r formed by the level's
// row kernel
__global__ void __launch_bounds__(kRedThreads) k_fcg_norm0(int n, const double* __restrict__ r, FcgState* st,
    double* partials)
{
    dep_wait();
    dep_release();
    double acc[1] = { 0.0 };
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        acc[0] += r[i] * r[i];
    double out[1];
    if (grid_sum<1>(acc, partials, &st->ticket[0], out) && threadIdx.x == 0) {
        st->delta0 = sqrt(out[0]);
        st->tol = st->tol * st->delta0;   // tol holds rtol on entry
        st->iter = 0;
        st->done = 0;
        st->bad = 0;
    }
}

static void fcg_resid0(const DevCsr& A, const double* x, const double* b, double* r, FcgState* st, double* part, cudaStream_t s)
{
    if (A.sliced) {
        // the sliced kernel forms r = b - A x with the one-thread-per-row kernel's row sums; the
        // norm follows in a kernel of its own
        rowop_resid(A, x, b, r, nullptr, s);
        auto k = k_fcg_norm0;
        launch_dep<2>(k, red_grid(k, A.n), kRedThreads, 0, s, A.n, r, st, part);
        BCMGX_CHECK_LAUNCH();
        return;
    }
    switch (A.tpr) {
    case 1: launch_resid0<1>(A, x, b, r, st, part, s); break;
    case 2: launch_resid0<2>(A, x, b, r, st, part, s); break;
    case 4: launch_resid0<4>(A, x, b, r, st, part, s); break;
    case 8: launch_resid0<8>(A, x, b, r, st, part, s); break;
    case 16: launch_resid0<16>(A, x, b, r, st, part, s); break;
    default: launch_resid0<32>(A, x, b, r, st, part, s); break;
    }
    BCMGX_CHECK_LAUNCH();
}

// pw = A pv (the level's row kernel in FP64: the staged one when the tuning chose it) and the
// step's dots and scalars (k_fcg_dots).
template <int MODE>
static void fcg_dots(const DevCsr& A, const double* pv, double* pw, const double* r, const double* oq, FcgState* st,
    double* part, const int* skip, cudaStream_t s)
{
    launch_rowop_A<OP_AXPBY>(A.tpr, A, A.val.p, pv, (const double*)nullptr, (const double*)nullptr, pw, 1.0, 0.0, skip, s);
    const int n = A.n;
    if (al16(pv) && al16(pw) && al16(r) && (MODE == 0 || al16(oq))) {
        auto k = k_fcg_dots<MODE, true>;
        launch_dep<2>(k, red_grid(k, ((long)n + 1) / 2), kRedThreads, 0, s, n, pv, pw, r, oq, st, part, skip);
    } else {
        auto k = k_fcg_dots<MODE, false>;
        launch_dep<2>(k, red_grid(k, n), kRedThreads, 0, s, n, pv, pw, r, oq, st, part, skip);
    }
    BCMGX_CHECK_LAUNCH();
}

// Records the persistent programs of the hierarchy's cycle: the call on its first persistent level
// from a zero iterate and, for cycles that visit a level more than once, from the level's iterate.
// A program of the whole cycle (level 0) takes its right-hand side, iterate and output as argument
// slots (placeholders while recording, replaced by the launch's vectors).
static void record_persist_programs(bcmgx_hierarchy* H)
{
    cudaStream_t s = H->stream;
    const int lc = H->persist_level;
    const bool f32 = H->prm.vcycle_precision == BCMGX_VCYCLE_FP32;
    const int L = (int)H->lv.size();
    static char placeholders[3][16];
    void* const PF = placeholders[0];
    void* const PX = placeholders[1];
    void* const PD = placeholders[2];
    const bool multi_visit = lc > 0 && lc - 1 < (int)H->grid_sweeps.size() && H->grid_sweeps[lc - 1] > 1;
    for (int has_x = 0; has_x <= (multi_visit ? 1 : 0); has_x++) {
        Vec f, x, dst;
        if (lc == 0) {
            f = Vec { PF, false };
            dst = Vec { PD, false };
            if (has_x) x = Vec { PX, false };
        } else {
            f = H->cyc.lv[lc].rhs;
            dst = H->cyc.lv[lc].x;
            if (has_x) x = dst;
        }
        std::vector<PStep> steps;
        Cycle c { H, H->cyc, s, nullptr, f32, L, -1 };
        c.rec = &steps;
        c.run(lc, f, x, dst);
        auto slot = [&](const void*& ptr, unsigned char& sl) {
            sl = 0;
            if (ptr == PF) sl = 1;
            else if (ptr == PX) sl = 2;
            else if (ptr == PD) sl = 3;
            if (sl) ptr = nullptr;
        };
        for (PStep& p : steps) {
            slot(p.x, p.sx);
            slot(p.f, p.sf);
            const void* y = p.y;
            slot(y, p.sy);
            p.y = (void*)y;
            const void* e = p.extra;
            slot(e, p.se);
            p.extra = (void*)e;
            slot(p.xc, p.sc);
        }
        std::unique_ptr<PersistProgram> pp(new PersistProgram());
        pp->level = lc;
        pp->has_x = has_x != 0;
        pp->nsteps = (int)steps.size();
        pp->steps.alloc(steps.size(), s);
        BCMGX_CUDA(cudaMemcpyAsync(pp->steps.p, steps.data(), sizeof(PStep) * steps.size(), cudaMemcpyHostToDevice, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
        H->persist.push_back(std::move(pp));
    }
}

void ensure_solve_workspace(bcmgx_hierarchy* H)
{
    const int n0 = H->lv[0].A.n;
    cudaStream_t s = H->stream;
    if (H->ws_n == n0) return;
    H->r.alloc(n0, s);
    H->v.alloc(n0, s);
    H->w.alloc(n0, s);
    H->d.alloc(n0, s);
    H->q.alloc(n0, s);
    H->res.alloc(n0, s);
    if (H->prm.vcycle_precision == BCMGX_VCYCLE_FP32) H->res32.alloc(n0, s);
    H->partials.alloc((size_t)num_sms() * kRedBlocksPerSM * 4, s);
    H->st.alloc(1, s);
    BCMGX_CUDA(cudaMemsetAsync(H->st.p, 0, sizeof(FcgState), s));
    if (!H->st_host) H->st_host = (FcgState*)pinned_alloc(2 * sizeof(FcgState));
    const bool f32 = H->prm.vcycle_precision == BCMGX_VCYCLE_FP32;
    const int L = (int)H->lv.size();
    for (int l = 0; l < L; l++) {
        Level& V = H->lv[l];
        const int n = V.A.n;
        const bool lf = f32 && l < L - 1;
        if (lf) {
            V.x32.alloc(n, s);
            V.x232.alloc(n, s);
            V.rhs32.alloc(n, s);
        } else {
            if (l > 0) {
                V.x.alloc(n, s);
                V.rhs.alloc(n, s);
            }
            V.x2.alloc(n, s);
        }
    }
    H->cyc.lv.assign(L, CycleBufs::L());
    for (int l = 0; l < L; l++) {
        Level& V = H->lv[l];
        if (f32 && l < L - 1) H->cyc.lv[l] = { Vec { V.rhs32.p, true }, Vec { V.x32.p, true }, Vec { V.x232.p, true } };
        else H->cyc.lv[l] = { Vec { V.rhs.p, false }, Vec { V.x.p, false }, Vec { V.x2.p, false } };
    }
    H->cyc.res = f32 ? Vec { H->res32.p, true } : Vec { H->res.p, false };
    if (H->prm.preconditioner == BCMGX_PREC_L1_JACOBI) H->l1tmp.alloc(n0, s);
    H->persist.clear();
    H->persist_level = choose_persist_level(H);
    if (H->persist_level >= 0) {
        H->persist_bar.alloc(4, s);
        BCMGX_CUDA(cudaMemsetAsync(H->persist_bar.p, 0, 4 * sizeof(unsigned), s));
        record_persist_programs(H);
    }
    H->ws_n = n0;
}

// Average device time of one launch of each solve-phase kernel of level l, timed with CUDA
// events on the hierarchy's stream over `reps` back-to-back launches after one warm-up:
// out[0] l1-Jacobi sweep (in the cycle's precision), out[1] residual, out[2] FP64 y = A x,
// out[3] the FCG SpMV + dot products, out[4] the FP32 cycle's sweep that writes an FP64 result,
// out[5] the FCG update (two merged axpys and the norm) (out[3..5] on level 0 only, else 0).
void time_level_kernels(bcmgx_hierarchy* H, int l, int reps, double* out)
{
    ensure_solve_workspace(H);
    cudaStream_t s = H->stream;
    Level& V = H->lv[l];
    const DevCsr& A = V.A;
    const int n = A.n;
    const int L = (int)H->lv.size();
    const bool f32 = H->prm.vcycle_precision == BCMGX_VCYCLE_FP32 && l < L - 1;
    DBuf<double> a, b, c;
    DBuf<float> a32, b32, c32;
    a.alloc(n, s);
    b.alloc(n, s);
    c.alloc(n, s);
    fill_probe(a.p, n, 1u, s);
    fill_probe(c.p, n, 2u, s);
    if (f32) {
        a32.alloc(n, s);
        b32.alloc(n, s);
        c32.alloc(n, s);
        fill_probe(a32.p, n, 1u, s);
        fill_probe(c32.p, n, 2u, s);
    }
    cudaEvent_t e0, e1;
    BCMGX_CUDA(cudaEventCreate(&e0));
    BCMGX_CUDA(cudaEventCreate(&e1));
    auto timeit = [&](auto&& launch) {
        launch();
        BCMGX_CUDA(cudaEventRecord(e0, s));
        for (int i = 0; i < reps; i++) launch();
        BCMGX_CUDA(cudaEventRecord(e1, s));
        BCMGX_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        BCMGX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return (double)ms / reps;
    };
    if (f32) {
        out[0] = timeit([&] { launch_rowop_A<OP_JACOBI>(A.tpr, A, A.val32.p, (const float*)a32.p, (const float*)c32.p, V.M32.p, b32.p, 1.0, 0.0, nullptr, s); });
        out[1] = timeit([&] { launch_rowop_A<OP_RESID>(A.tpr, A, A.val32.p, (const float*)a32.p, (const float*)c32.p, (const float*)nullptr, b32.p, 1.0, 0.0, nullptr, s); });
    } else {
        out[0] = timeit([&] { launch_rowop_A<OP_JACOBI>(A.tpr, A, A.val.p, (const double*)a.p, (const double*)c.p, V.M.p, b.p, 1.0, 0.0, nullptr, s); });
        out[1] = timeit([&] { launch_rowop_A<OP_RESID>(A.tpr, A, A.val.p, (const double*)a.p, (const double*)c.p, (const double*)nullptr, b.p, 1.0, 0.0, nullptr, s); });
    }
    // the public SpMV (bcmgx_spmv) on the stored CSR arrays, with its default threads per row
    out[2] = timeit([&] { launch_spmv(n, A.row.p, A.col.p, A.val.p, a.p, b.p, 1.0, 0.0, default_tpr(n, A.nnz), s); });
    out[3] = 0;
    out[4] = 0;
    out[5] = 0;
    if (l == 0) {
        FcgState init {};
        init.delta = 1.0;
        BCMGX_CUDA(cudaMemcpyAsync(H->st.p, &init, sizeof(FcgState), cudaMemcpyHostToDevice, s));
        out[3] = timeit([&] { fcg_dots<1>(A, a.p, b.p, c.p, c.p, H->st.p, H->partials.p, nullptr, s); });
        // the cycle's last level-0 sweep writes the FP64 preconditioned vector
        if (f32)
            out[4] = timeit([&] { launch_rowop_A<OP_JACOBI>(A.tpr, A, A.val32.p, (const float*)a32.p, (const float*)c32.p,
                                      V.M32.p, b.p, 1.0, 0.0, nullptr, s); });
        DBuf<double> d4, d5, d6;
        d4.alloc(n, s);
        d5.alloc(n, s);
        d6.alloc(n, s);
        fill_probe(d4.p, n, 3u, s);
        fill_probe(d5.p, n, 4u, s);
        fill_probe(d6.p, n, 5u, s);
        init.theta = 1e-3;
        init.theta2 = 1e-3;
        init.tol = 0.0;
        init.itnlim = 1 << 30;
        BCMGX_CUDA(cudaMemcpyAsync(H->st.p, &init, sizeof(FcgState), cudaMemcpyHostToDevice, s));
        out[5] = timeit([&] { fcg_update(n, a.p, c.p, b.p, d4.p, d5.p, d6.p, H->st.p, H->partials.p, nullptr, nullptr, s); });
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

// Average device time (CUDA events on the hierarchy's stream, reps launches after one warm-up)
// of the level-0 block kernels for blocks of KP columns (K rounded up to a power of two, the
// multi-right-hand-side solve's padded width): out[0] one block l1-Jacobi sweep in the cycle's
// precision, out[1] the block residual, out[2] the FP64 block SpMM Y = A X, out[3] the block
// FCG SpMV + per-column dots (time_block_dots). Inputs are zero blocks.
void time_block_kernels(bcmgx_hierarchy* H, int K, int reps, double* out)
{
    ensure_solve_workspace(H);
    cudaStream_t s = H->stream;
    Level& V = H->lv[0];
    const DevCsr& A = V.A;
    const int L = (int)H->lv.size();
    const bool f32 = H->prm.vcycle_precision == BCMGX_VCYCLE_FP32 && L > 1;
    const int kp = 1 << ceil_log2(K);
    const size_t nk = (size_t)A.n * kp;
    DBuf<double> x, f, y;
    x.alloc(nk, s);
    y.alloc(nk, s);
    fill_probe(x.p, (long)nk, 1u, s);
    cudaEvent_t e0, e1;
    BCMGX_CUDA(cudaEventCreate(&e0));
    BCMGX_CUDA(cudaEventCreate(&e1));
    auto timeit = [&](auto&& launch) {
        launch();
        BCMGX_CUDA(cudaEventRecord(e0, s));
        for (int i = 0; i < reps; i++) launch();
        BCMGX_CUDA(cudaEventRecord(e1, s));
        BCMGX_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        BCMGX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return (double)ms / reps;
    };
    if (f32) {
        DBuf<float> x32, f32b, y32;
        x32.alloc(nk, s);
        f32b.alloc(nk, s);
        y32.alloc(nk, s);
        fill_probe(x32.p, (long)nk, 1u, s);
        fill_probe(f32b.p, (long)nk, 2u, s);
        out[0] = timeit([&] { launch_blk_rowop<OP_JACOBI>(A.n, A.m, kp, kp, A.row.p, A.col.p, A.val32.p,
                                  (const float*)x32.p, (const float*)f32b.p, V.M32.p, y32.p, 1.0, 0.0, nullptr, s); });
        out[1] = timeit([&] { launch_blk_rowop<OP_RESID>(A.n, A.m, kp, kp, A.row.p, A.col.p, A.val32.p,
                                  (const float*)x32.p, (const float*)f32b.p, (const float*)nullptr, y32.p, 1.0, 0.0, nullptr, s); });
        BCMGX_CUDA(cudaStreamSynchronize(s));
    } else {
        f.alloc(nk, s);
        fill_probe(f.p, (long)nk, 2u, s);
        out[0] = timeit([&] { launch_blk_rowop<OP_JACOBI>(A.n, A.m, kp, kp, A.row.p, A.col.p, A.val.p,
                                  (const double*)x.p, (const double*)f.p, V.M.p, y.p, 1.0, 0.0, nullptr, s); });
        out[1] = timeit([&] { launch_blk_rowop<OP_RESID>(A.n, A.m, kp, kp, A.row.p, A.col.p, A.val.p,
                                  (const double*)x.p, (const double*)f.p, (const double*)nullptr, y.p, 1.0, 0.0, nullptr, s); });
    }
    out[2] = timeit([&] { launch_blk_rowop<OP_AXPBY>(A.n, A.m, kp, kp, A.row.p, A.col.p, A.val.p, (const double*)x.p,
                              (const double*)nullptr, (const double*)nullptr, y.p, 1.0, 0.0, nullptr, s); });
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BCMGX_CUDA(cudaStreamSynchronize(s));
    out[3] = time_block_dots(H, K, reps);
}

// Threads-per-row autotuner: for a level with at least kTuneMinRows rows, one l1-Jacobi sweep
// in the cycle's precision is timed (CUDA events, 3 launches after a warm-up) for every
// candidate 1..16 of the plain kernel and 1, 2, 4, 8 of the staged one, and the fastest is kept.
// The result is a code: the threads per row, negative for the staged kernel (the two kernels
// sum a row in the same order, so that choice does not change results). Codes are cached per
// (rows, nnz, precision) for the life of the process, so repeated set-ups of same-shaped
// matrices reuse them; when the environment variable BCMGX_TUNE_CACHE names a file, the cache is
// also read from it at the first use and every new result is appended to it (one "rows nnz
// precision code" line each).
constexpr int kTuneMinRows = 20000;
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int64_t, int>, int> g_tune_cache;
static bool g_tune_loaded = false;

static void tune_cache_load()
{
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = std::getenv("BCMGX_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    long long z;
    int n, prec, t;
    while (std::fscanf(f, "%d %lld %d %d", &n, &z, &prec, &t) == 4)
        if (t == 1 || t == 2 || t == 4 || t == 8 || t == 16 || t == 32 || t == -1 || t == -2 || t == -4 || t == -8 ||
            t == kSlicedCode)
            g_tune_cache[std::make_tuple(n, (int64_t)z, prec)] = t;
    std::fclose(f);
}

static void tune_cache_store(const std::tuple<int, int64_t, int>& key, int t)
{
    const char* path = std::getenv("BCMGX_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "a");
    if (!f) return;
    std::fprintf(f, "%d %lld %d %d\n", std::get<0>(key), (long long)std::get<1>(key), std::get<2>(key), t);
    std::fclose(f);
}

int autotune_tpr(Level& V, bool f32, cudaStream_t s)
{
    DevCsr& A = V.A;
    const int n = A.n;
    if (n < kTuneMinRows) return default_tpr(n, A.nnz);
    const auto key = std::make_tuple(n, A.nnz, f32 ? 1 : 0);
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        tune_cache_load();
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) return it->second;
    }
    DBuf<double> a, b, c;
    DBuf<float> a32, b32, c32;
    if (f32) {
        a32.alloc(n, s);
        b32.alloc(n, s);
        c32.alloc(n, s);
        fill_probe(a32.p, n, 1u, s);
        fill_probe(c32.p, n, 2u, s);
    } else {
        a.alloc(n, s);
        b.alloc(n, s);
        c.alloc(n, s);
        fill_probe(a.p, n, 1u, s);
        fill_probe(c.p, n, 2u, s);
    }
    cudaEvent_t e0, e1;
    BCMGX_CUDA(cudaEventCreate(&e0));
    BCMGX_CUDA(cudaEventCreate(&e1));
    int best = default_tpr(n, A.nnz);
    float best_ms = 1e30f;
    // candidates: 1..16 threads per row, the staged kernel with 1, 2, 4 and 8 (coded negative),
    // and the sliced kernel (its copy of the matrix is built for the trial and kept if it wins)
    build_sliced(A, s);
    for (int t : {1, 2, 4, 8, 16, -1, -2, -4, -8, kSlicedCode}) {
        if (t == kSlicedCode && !A.sl_ptr.p) continue;
        const int tp = t == kSlicedCode ? 1 : t < 0 ? -t : t, stage = t == kSlicedCode ? 2 : t < 0 ? 1 : 0;
        auto launch = [&] {
            if (f32)
                launch_rowop_A<OP_JACOBI>(tp, A, A.val32.p, (const float*)a32.p, (const float*)c32.p, V.M32.p, b32.p, 1.0, 0.0, nullptr, s, stage);
            else
                launch_rowop_A<OP_JACOBI>(tp, A, A.val.p, (const double*)a.p, (const double*)c.p, V.M.p, b.p, 1.0, 0.0, nullptr, s, stage);
        };
        launch();
        BCMGX_CUDA(cudaEventRecord(e0, s));
        for (int r = 0; r < 3; r++) launch();
        BCMGX_CUDA(cudaEventRecord(e1, s));
        BCMGX_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        BCMGX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) {
            best_ms = ms;
            best = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best != kSlicedCode) release_sliced(A);
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune_cache[key] = best;
    tune_cache_store(key, best);
    return best;
}

// Gradient of L with respect to the stored entries of A for x = A^{-1} b: with the adjoint
// lambda = A^{-T} dL/dx = A^{-1} dL/dx (A symmetric), dL/da_ij = -lambda_i x_j on A's pattern.
// One sub-warp per row; the entries of the row are written in place of their values.
template <int S>
__global__ void __launch_bounds__(256) k_grad_pattern(int n, const int* __restrict__ row, const int* __restrict__ col,
    const double* __restrict__ lam, const double* __restrict__ x, double* __restrict__ dA)
{
    const int lane = threadIdx.x & (S - 1);
    const long stride = (long)gridDim.x * blockDim.x / S;
    for (long r = ((long)blockIdx.x * blockDim.x + threadIdx.x) / S; r < n; r += stride) {
        const double li = -lam[r];
        for (int j = row[r] + lane; j < row[r + 1]; j += S) dA[j] = li * __ldg(x + __ldcs(col + j));
    }
}

void grad_pattern(const DevCsr& A, const double* lam, const double* x, double* dA, cudaStream_t s)
{
    auto k = k_grad_pattern<4>;
    note_launch();
    k<<<fit_grid(k, 256, ((long)A.n * 4 + 255) / 256), 256, 0, s>>>(A.n, A.row.p, A.col.p, lam, x, dA);
    BCMGX_CHECK_LAUNCH();
}

// Initial FCG state (replaces a host copy so the start-up can be captured in a graph).
__global__ void k_fcg_init(FcgState* st, double rtol, int itnlim)
{
    dep_wait();
    dep_release();
    FcgState z {};
    z.tol = rtol;
    z.itnlim = itnlim;
    *st = z;
}

__global__ void k_set_while(cudaGraphConditionalHandle h, const FcgState* st)
{
    dep_wait();
    dep_release();
    cudaGraphSetConditional(h, st->done ? 0u : 1u);
}

// FCG start-up (FCG.cu:46-100): r = b - A x, delta0, v = B r, w = A v, alpha, beta, x += theta v,
// r -= theta w, d = v, q = w.
static void fcg_startup(bcmgx_hierarchy* H, const double* b, double* x, double* hist)
{
    cudaStream_t s = H->stream;
    const DevCsr& A = H->lv[0].A;
    const int n = A.n;
    FcgState* st = H->st.p;
    double* part = H->partials.p;
    double *r = H->r.p, *v = H->v.p, *w = H->w.p, *d = H->d.p, *q = H->q.p;
    persist_reset(H, s);
    launch_dep<2>(k_fcg_init, 1, 1, 0, s, st, H->prm.rtol, H->prm.itnlim);
    fcg_resid0(A, x, b, r, st, part, s);
    prec_apply_impl(H, r, v, nullptr);
    fcg_dots<0>(A, v, w, r, nullptr, st, part, nullptr, s);
    launch_dep<2>(k_fcg_update0, red_grid(k_fcg_update0, n), kRedThreads, 0, s, n, v, w, x, r, d, q, st, part, hist);
    BCMGX_CHECK_LAUNCH();
}

// One FCG iteration (FCG.cu:102-156); the roles of (v, w) and (d, q) alternate with the parity.
// Every kernel returns at once when *skip is set (the solve has converged).
static void fcg_iteration(bcmgx_hierarchy* H, bool even, double* x, double* hist, const int* skip)
{
    cudaStream_t s = H->stream;
    const DevCsr& A = H->lv[0].A;
    const int n = A.n;
    FcgState* st = H->st.p;
    double* part = H->partials.p;
    double *r = H->r.p, *v = H->v.p, *w = H->w.p, *d = H->d.p, *q = H->q.p;
    double* pv = even ? v : d;
    double* pw = even ? w : q;
    const double* od = even ? d : v;
    const double* oq = even ? q : w;
    prec_apply_impl(H, r, pv, skip);
    fcg_dots<1>(A, pv, pw, r, oq, st, part, skip, s);
    fcg_update(n, pv, od, x, pw, oq, r, st, part, hist, skip, s);
}

// Adds the whole solve of hierarchy H to graph g as an independent branch: the start-up, then a
// WHILE conditional node whose body is two iterations (the second skips itself once the first
// converges) followed by a kernel that sets the loop condition from the device-side `done` flag.
// The branch works on the hierarchy's own b / x buffers (gb, gx).
static void add_solve_to_graph(bcmgx_hierarchy* H, cudaGraph_t g)
{
    cudaStream_t s = H->stream;
    const int n = H->lv[0].A.n;
    if (!H->gb.p) {
        H->gb.alloc(n, s);
        H->gx.alloc(n, s);
    }
    if (!H->hist.p) H->hist.alloc((size_t)std::max(H->prm.itnlim, 1) + 2, s);
    BCMGX_CUDA(cudaStreamSynchronize(s));
    const long long c0 = launch_count();
    BCMGX_CUDA(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    fcg_startup(H, H->gb.p, H->gx.p, H->hist.p);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    BCMGX_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &ndeps));
    std::vector<cudaGraphNode_t> tail(deps, deps + ndeps);
    cudaGraph_t gg = g;
    BCMGX_CUDA(cudaStreamEndCapture(s, &gg));
    const long long c1 = launch_count();
    cudaGraphConditionalHandle h;
    BCMGX_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wn;
    BCMGX_CUDA(cudaGraphAddNode(&wn, g, tail.data(), tail.size(), &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    BCMGX_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    fcg_iteration(H, true, H->gx.p, H->hist.p, &H->st.p->done);
    fcg_iteration(H, false, H->gx.p, H->hist.p, &H->st.p->done);
    launch_dep<2>(k_set_while, 1, 1, 0, s, h, (const FcgState*)H->st.p);
    BCMGX_CHECK_LAUNCH();
    BCMGX_CUDA(cudaStreamEndCapture(s, &body));
    const long long c2 = launch_count();
    H->graph_startup_kernels = c1 - c0;
    H->graph_body_kernels = c2 - c1;
    note_launches(-(c2 - c0));   // captured, not launched
}

static void build_solve_graph(bcmgx_hierarchy* H)
{
    cudaGraph_t g = nullptr;
    BCMGX_CUDA(cudaGraphCreate(&g, 0));
    add_solve_to_graph(H, g);
    BCMGX_CUDA(cudaGraphInstantiate(&H->iter_graph, g, 0));
    BCMGX_CUDA(cudaGraphDestroy(g));
}

// Kernels launched by one graph solve of H that ran `iters` iterations.
static long long graph_launches(const bcmgx_hierarchy* H, int iters, int bad)
{
    const long long bodies = std::max(1LL, (long long)(iters + 1) / 2 + (bad ? 1 : 0));
    return H->graph_startup_kernels + H->graph_body_kernels * bodies;
}

// ------------------------------------------------------------------------------------------
// batched solves: many hierarchies in one graph launch
// ------------------------------------------------------------------------------------------
struct BatchCopy {
    const double* src;
    double* dst;
    int n;
};

// One block per vector: dst = src for every (src, dst, n) of the list.
__global__ void k_batch_copy(int m, const BatchCopy* __restrict__ list)
{
    for (int k = blockIdx.x; k < m; k += gridDim.x) {
        const BatchCopy c = list[k];
        for (int i = threadIdx.x; i < c.n; i += blockDim.x) c.dst[i] = c.src[i];
    }
}

__global__ void k_batch_states(int m, FcgState* const* __restrict__ st, FcgState* __restrict__ out)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) out[k] = *st[k];
}

// While one system's solve is captured into the batch graph: sweep chains of small levels as one
// block (fewer, longer kernels per system), and the plain row kernels instead of the staged ones
// (a staged kernel's resident grid of large shared-memory blocks would hold the SMs that the other
// systems' branches run on). The hierarchy's own settings come back when the capture ends.
struct BatchCaptureMode {
    bcmgx_hierarchy* H;
    std::vector<char> staged;
    explicit BatchCaptureMode(bcmgx_hierarchy* h) : H(h)
    {
        H->chain_in_block = true;
        for (Level& V : H->lv) {
            staged.push_back((V.A.staged ? 1 : 0) | (V.A.sliced ? 2 : 0));
            V.A.staged = false;
            V.A.sliced = false;
        }
    }
    ~BatchCaptureMode()
    {
        H->chain_in_block = false;
        for (size_t l = 0; l < staged.size(); l++) {
            H->lv[l].A.staged = (staged[l] & 1) != 0;
            H->lv[l].A.sliced = (staged[l] & 2) != 0;
        }
    }
};

void batch_build(bcmgx_batch* B)
{
    cudaGraph_t g = nullptr;
    BCMGX_CUDA(cudaGraphCreate(&g, 0));
    for (bcmgx_hierarchy* H : B->hs) {
        ensure_solve_workspace(H);
        BatchCaptureMode mode(H);
        add_solve_to_graph(H, g);
    }
    BCMGX_CUDA(cudaGraphInstantiate(&B->exec, g, 0));
    BCMGX_CUDA(cudaGraphDestroy(g));
    const int m = (int)B->hs.size();
    cudaStream_t s = B->stream;
    B->copies.alloc(sizeof(BatchCopy) * 2 * (size_t)m, s);
    B->states_ptr.alloc(sizeof(FcgState*) * (size_t)m, s);
    B->states.alloc(m, s);
    std::vector<FcgState*> sp(m);
    for (int k = 0; k < m; k++) sp[k] = B->hs[k]->st.p;
    BCMGX_CUDA(cudaMemcpyAsync(B->states_ptr.p, sp.data(), sizeof(FcgState*) * m, cudaMemcpyHostToDevice, s));
    B->states_host = pinned_alloc(sizeof(FcgState) * m);
    B->copies_host = pinned_alloc(sizeof(BatchCopy) * 2 * m);
    BCMGX_CUDA(cudaStreamSynchronize(s));
}

// b[k], x[k]: device vectors of system k; x holds x0 on entry and the solution on return.
int batch_solve(bcmgx_batch* B, const double* const* b, double* const* x, bcmgx_solve_info* infos)
{
    const int m = (int)B->hs.size();
    cudaStream_t s = B->stream;
    // every system's stream must have finished its own work before the batch graph runs on B's stream
    for (bcmgx_hierarchy* H : B->hs) BCMGX_CUDA(cudaStreamSynchronize(H->stream));
    BatchCopy* in = (BatchCopy*)B->copies_host;
    for (int k = 0; k < m; k++) {
        in[2 * k] = BatchCopy { b[k], B->hs[k]->gb.p, B->hs[k]->lv[0].A.n };
        in[2 * k + 1] = BatchCopy { x[k], B->hs[k]->gx.p, B->hs[k]->lv[0].A.n };
    }
    BCMGX_CUDA(cudaMemcpyAsync(B->copies.p, in, sizeof(BatchCopy) * 2 * m, cudaMemcpyHostToDevice, s));
    note_launch();
    k_batch_copy<<<std::min(2 * m, 65535), 256, 0, s>>>(2 * m, (const BatchCopy*)B->copies.p);
    BCMGX_CHECK_LAUNCH();
    BCMGX_CUDA(cudaEventRecord(B->ev0, s));
    BCMGX_CUDA(cudaGraphLaunch(B->exec, s));
    BCMGX_CUDA(cudaEventRecord(B->ev1, s));
    BCMGX_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < m; k++) in[k] = BatchCopy { B->hs[k]->gx.p, x[k], B->hs[k]->lv[0].A.n };
    BCMGX_CUDA(cudaMemcpyAsync(B->copies.p, in, sizeof(BatchCopy) * m, cudaMemcpyHostToDevice, s));
    note_launch();
    k_batch_copy<<<std::min(m, 65535), 256, 0, s>>>(m, (const BatchCopy*)B->copies.p);
    note_launch();
    k_batch_states<<<ceil_div(m, 128), 128, 0, s>>>(m, (FcgState* const*)B->states_ptr.p, B->states.p);
    BCMGX_CHECK_LAUNCH();
    BCMGX_CUDA(cudaMemcpyAsync(B->states_host, B->states.p, sizeof(FcgState) * m, cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaStreamSynchronize(s));
    float ms = 0;
    BCMGX_CUDA(cudaEventElapsedTime(&ms, B->ev0, B->ev1));
    const FcgState* S = (const FcgState*)B->states_host;
    int status = BCMGX_OK;
    for (int k = 0; k < m; k++) {
        const bcmgx_params& P = B->hs[k]->prm;
        note_launches(graph_launches(B->hs[k], S[k].iter, S[k].bad));
        if (infos) {
            infos[k].niter = S[k].iter + 1;
            infos[k].retv = S[k].iter >= P.itnlim ? -1 : 0;
            infos[k].delta0 = S[k].delta0;
            infos[k].exit_res = std::sqrt(S[k].rnorm2);
            infos[k].solve_ms = ms;
            infos[k].full_n = B->hs[k]->lv[0].A.n;
        }
        if (S[k].bad) status = BCMGX_ERR_NOT_SPD;
        else if (S[k].iter >= P.itnlim && status == BCMGX_OK) status = BCMGX_ERR_NO_CONVERGENCE;
    }
    return status;
}

static int finish_solve(bcmgx_hierarchy* H, bcmgx_solve_info* info, int n)
{
    const bcmgx_params& P = H->prm;
    float ms = 0;
    BCMGX_CUDA(cudaEventElapsedTime(&ms, H->ev0, H->ev1));
    const FcgState& S = *H->st_host;
    if (info) {
        info->niter = S.iter + 1;
        info->retv = S.iter >= P.itnlim ? -1 : 0;
        info->delta0 = S.delta0;
        info->exit_res = std::sqrt(S.rnorm2);
        info->solve_ms = ms;
        info->full_n = n;
    }
    if (S.bad) return BCMGX_ERR_NOT_SPD;
    return S.iter >= P.itnlim ? BCMGX_ERR_NO_CONVERGENCE : BCMGX_OK;
}

// Flexible CG (FCG.cu:27-165) on device vectors b, x (x: x0 in, solution out).
// Stream path: iterations are enqueued one ahead of the convergence test (the extra iteration skips
// itself on the device once `done` is set), so the GPU never waits for the host between
// iterations. Graph path (use_graph, not with dispnorm): one launch of the captured solve.
int fcg_solve(bcmgx_hierarchy* H, const double* b, double* x, bcmgx_solve_info* info)
{
    ensure_solve_workspace(H);
    cudaStream_t s = H->stream;
    const int n = H->lv[0].A.n;
    const bcmgx_params& P = H->prm;
    if (P.use_graph == 1 && !P.dispnorm) {
        if (!H->iter_graph) build_solve_graph(H);
        BCMGX_CUDA(cudaMemcpyAsync(H->gb.p, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        BCMGX_CUDA(cudaMemcpyAsync(H->gx.p, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        BCMGX_CUDA(cudaEventRecord(H->ev0, s));
        BCMGX_CUDA(cudaGraphLaunch(H->iter_graph, s));
        BCMGX_CUDA(cudaEventRecord(H->ev1, s));
        BCMGX_CUDA(cudaMemcpyAsync(x, H->gx.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        BCMGX_CUDA(cudaMemcpyAsync(H->st_host, H->st.p, sizeof(FcgState), cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
        note_launches(graph_launches(H, H->st_host->iter, H->st_host->bad));
        return finish_solve(H, info, n);
    }
    if (!H->hist.p) H->hist.alloc((size_t)std::max(P.itnlim, 1) + 2, s);
    BCMGX_CUDA(cudaEventRecord(H->ev0, s));
    fcg_startup(H, b, x, H->hist.p);
    FcgState* ring = H->st_host;   // two pinned slots
    const int* done_flag = &H->st.p->done;
    auto enqueue = [&](int k) {
        fcg_iteration(H, (k % 2) == 0, x, H->hist.p, done_flag);
        BCMGX_CUDA(cudaMemcpyAsync(ring + (k % 2), H->st.p, sizeof(FcgState), cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaEventRecord(H->ev_it[k % 2], s));
    };
    enqueue(0);
    int k = 0;
    for (;;) {
        enqueue(k + 1);
        BCMGX_CUDA(cudaEventSynchronize(H->ev_it[k % 2]));
        const FcgState& S = ring[k % 2];
        if (P.dispnorm && !S.bad) std::printf("%d) r norm: %.10lf\n", S.iter - 1, std::sqrt(S.rnorm2));
        if (S.done) break;
        k++;
    }
    BCMGX_CUDA(cudaEventRecord(H->ev1, s));
    BCMGX_CUDA(cudaMemcpyAsync(H->st_host, H->st.p, sizeof(FcgState), cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaStreamSynchronize(s));
    return finish_solve(H, info, n);
}

}  // namespace bcmgx
