// api.cpp -- the C ABI (include/bcmgx.h). Every entry point converts exceptions into status
// codes and records the message for bcmgx_last_error_string(); nothing calls exit().
#include "internal.h"

#include <atomic>
#include <map>
#include <mutex>
#include <thread>
#include <cstdlib>
#include <cmath>
#include <cstdio>

namespace bcmgx {

static thread_local std::string g_last_error;
thread_local long long t_fail_alloc_countdown = 0;

// Arms the allocation-failure injection of the calling thread for one set-up (see internal.h)
// and disarms it when the set-up returns or throws.
struct FailAllocScope {
    FailAllocScope()
    {
        const char* e = std::getenv("BCMGX_TEST_FAIL_ALLOC");
        t_fail_alloc_countdown = (e && *e) ? std::max(0LL, std::atoll(e)) : 0;
    }
    ~FailAllocScope() { t_fail_alloc_countdown = 0; }
};

// A CUDA event owned for the duration of a scope.
struct ScopedEvent {
    cudaEvent_t e = nullptr;
    ScopedEvent() { BCMGX_CUDA(cudaEventCreate(&e)); }
    ~ScopedEvent()
    {
        if (e) cudaEventDestroy(e);
    }
};

void set_last_error(const std::string& s) { g_last_error = s; }

static std::atomic<long long> g_launches { 0 };

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void note_launches(long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(); }

template <typename F>
static int guarded(F&& f)
{
    try {
        f();
        return BCMGX_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return BCMGX_ERR_OOM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return BCMGX_ERR_INTERNAL;
    } catch (...) {
        set_last_error("unknown failure");
        return BCMGX_ERR_INTERNAL;
    }
}

// Device guard: makes the hierarchy's device current for the duration of a call.
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int dev)
    {
        cudaGetDevice(&prev);
        if (dev >= 0 && dev != prev) BCMGX_CUDA(cudaSetDevice(dev));
    }
    ~DeviceScope()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

static void check_params(const bcmgx_params* p)
{
    BCMGX_REQUIRE(p != nullptr, BCMGX_ERR_INVALID_INPUT, "params is NULL");
    BCMGX_REQUIRE(p->error == 0, BCMGX_ERR_INVALID_INPUT, "settings carry an error flag (unsupported legacy option)");
    BCMGX_REQUIRE(p->solver >= BCMGX_SOLVER_CGHS && p->solver < BCMGX_SOLVER_INVALID, BCMGX_ERR_INVALID_INPUT,
        "invalid solver");
    BCMGX_REQUIRE(p->preconditioner >= BCMGX_PREC_NONE && p->preconditioner < BCMGX_PREC_INVALID, BCMGX_ERR_INVALID_INPUT,
        "invalid preconditioner");
    if (p->solver == BCMGX_SOLVER_CGS || p->solver == BCMGX_SOLVER_PIPELINED_CGS || p->solver == BCMGX_SOLVER_CGS_CUBLAS)
        BCMGX_REQUIRE(p->sstep >= 1 && p->sstep <= 8, BCMGX_ERR_INVALID_INPUT, "sstep must be 1..8");
    if (p->preconditioner == BCMGX_PREC_L1_JACOBI)
        BCMGX_REQUIRE(p->l1jacsweeps >= 1, BCMGX_ERR_INVALID_INPUT, "l1jacsweeps must be >= 1");
    BCMGX_REQUIRE(p->cycle_type >= 0 && p->cycle_type < BCMGX_CYCLE_INVALID, BCMGX_ERR_INVALID_INPUT, "invalid cycle_type");
    BCMGX_REQUIRE(p->matchtype == BCMGX_MATCH_SUITOR, BCMGX_ERR_INVALID_INPUT, "invalid matchtype");
    BCMGX_REQUIRE(p->relax_type == BCMGX_L1_JACOBI && p->coarse_solver == BCMGX_L1_JACOBI, BCMGX_ERR_INVALID_INPUT,
        "invalid relax_type / coarse_solver");
    BCMGX_REQUIRE(p->bootstrap_type == BCMGX_BOOT_MULTIPLICATIVE, BCMGX_ERR_UNSUPPORTED,
        "only the MULTIPLICATIVE bootstrap composition is implemented by the reference (bcmg.cu:63-86)");
    BCMGX_REQUIRE(p->max_hrc == 1, BCMGX_ERR_UNSUPPORTED, "max_hrc > 1 (bootstrap) is not supported (Params.cu:463)");
    BCMGX_REQUIRE(p->aggr_type == 0, BCMGX_ERR_UNSUPPORTED, "aggr_type != 0 is not supported (Params.cu:467)");
    BCMGX_REQUIRE(p->aggrsweeps >= 0 && p->aggrsweeps < 30, BCMGX_ERR_INVALID_INPUT, "aggrsweeps out of range");
    BCMGX_REQUIRE(p->max_levels >= 1 && p->max_levels <= BCMGX_MAX_LEVELS, BCMGX_ERR_INVALID_INPUT, "max_levels out of range");
    BCMGX_REQUIRE(p->itnlim >= 1, BCMGX_ERR_INVALID_INPUT, "itnlim < 1");
    BCMGX_REQUIRE(p->prerelax_sweeps >= 0 && p->postrelax_sweeps >= 0 && p->relaxnumber_coarse >= 0,
        BCMGX_ERR_INVALID_INPUT, "negative sweep count");
    BCMGX_REQUIRE(p->vcycle_precision == BCMGX_VCYCLE_FP64 || p->vcycle_precision == BCMGX_VCYCLE_FP32,
        BCMGX_ERR_INVALID_INPUT, "invalid vcycle_precision");
}

// solve() dispatch on the solver type (solver/solve.cu:11-51)
static int solve_dispatch(bcmgx_hierarchy* h, const double* b, double* x, bcmgx_solve_info* info)
{
    return h->prm.solver == BCMGX_SOLVER_FCG ? fcg_solve(h, b, x, info) : krylov_solve(h, b, x, info);
}

static std::mutex g_pin_mu;
static std::multimap<size_t, void*> g_pin_free;
constexpr size_t kPinHeader = 64;   // the block's size, stored in front of the returned pointer

void* pinned_alloc(size_t bytes)
{
    const size_t b = (bytes + 63) & ~(size_t)63;
    {
        std::lock_guard<std::mutex> g(g_pin_mu);
        auto it = g_pin_free.find(b);
        if (it != g_pin_free.end()) {
            void* p = it->second;
            g_pin_free.erase(it);
            return p;
        }
    }
    void* base = nullptr;
    BCMGX_CUDA(cudaMallocHost(&base, b + kPinHeader));
    *(size_t*)base = b;
    return (char*)base + kPinHeader;
}

void pinned_free(void* p)
{
    if (!p) return;
    const size_t b = *(size_t*)((char*)p - kPinHeader);
    std::lock_guard<std::mutex> g(g_pin_mu);
    g_pin_free.emplace(b, p);
}

// Builds one hierarchy (the body of bcmgx_setup). own_stream forces a library-owned stream even
// when params name one (batch set-ups run concurrently, one stream each).
// Device-resident inputs are written by the caller's own work, normally on the legacy default
// stream (torch's default stream, plain cudaMemcpy). A library-owned stream is non-blocking and
// does not wait for that stream by itself, so every entry that reads caller buffers on it first
// orders it after the work already issued there. A stream passed in bcmgx_params.stream is the
// caller's to order.
static void after_caller(cudaStream_t s, cudaEvent_t ev, bool own)
{
    if (!own) return;
    BCMGX_CUDA(cudaEventRecord(ev, cudaStreamLegacy));
    BCMGX_CUDA(cudaStreamWaitEvent(s, ev, 0));
}

// The row kernel of every level: BCMGX_TPR forces the codes (one code for every level, "-2", or
// one per level, "-2,-2,4"; levels past the list take its last code); else the autotuner times
// them (levels of at least 20,000 rows) or the default threads per row apply.
void choose_level_kernels(bcmgx_hierarchy* H)
{
    const bcmgx_params* p = &H->prm;
    std::vector<int> force;
    if (const char* env = std::getenv("BCMGX_TPR")) {
        for (const char* q = env; *q;) {
            char* end = nullptr;
            const long v = std::strtol(q, &end, 10);
            BCMGX_REQUIRE(end != q, BCMGX_ERR_INVALID_INPUT, "BCMGX_TPR: expected comma-separated integers");
            force.push_back((int)v);
            q = *end == ',' ? end + 1 : end;
            BCMGX_REQUIRE(*q == 0 || *end == ',', BCMGX_ERR_INVALID_INPUT, "BCMGX_TPR: expected comma-separated integers");
        }
    }
    const int L = (int)H->lv.size();
    for (int l = 0; l < L; l++) {
        Level& V = H->lv[l];
        const bool f32 = p->vcycle_precision == BCMGX_VCYCLE_FP32 && l < L - 1;
        int code;
        if (!force.empty()) code = force[std::min(l, (int)force.size() - 1)];
        else if (p->autotune) code = autotune_tpr(V, f32, H->stream);
        else code = default_tpr(V.A.n, V.A.nnz);
        // negative: the staged kernel with -code threads per row (1, 2, 4 or 8); kSlicedCode: the
        // sliced kernel (one lane per row: the CSR kernels stand in for it with 1 thread per row)
        if (code == kSlicedCode) {
            build_sliced(V.A, H->stream);
            V.A.sliced = V.A.sl_ptr.p != nullptr;
            V.A.staged = false;
            V.A.tpr = 1;
            continue;
        }
        release_sliced(V.A);
        V.A.staged = code < 0;
        V.A.tpr = code < 0 ? -code : code;
        if (V.A.tpr < 1) V.A.tpr = default_tpr(V.A.n, V.A.nnz);
    }
}

static bcmgx_hierarchy* setup_one(const bcmgx_csr* A, const bcmgx_params* p, int device, bool own_stream)
{
    check_params(p);
    BCMGX_REQUIRE(A->n > 0 && A->n == A->m, BCMGX_ERR_INVALID_INPUT, "matrix must be square with n > 0");
    BCMGX_REQUIRE(A->nnz > 0 && A->nnz <= 0x7fffffffLL, BCMGX_ERR_INVALID_INPUT, "nnz must be in [1, 2^31-1]");
    BCMGX_REQUIRE(A->row && A->col && A->val, BCMGX_ERR_INVALID_INPUT, "NULL CSR array");
    FailAllocScope inject;
    std::unique_ptr<bcmgx_hierarchy> H(new bcmgx_hierarchy());
    H->prm = *p;
    int dev = device >= 0 ? device : p->device;
    if (dev < 0) BCMGX_CUDA(cudaGetDevice(&dev));
    H->device = dev;
    H->prm.device = dev;
    DeviceScope ds(dev);
    if (p->stream && !own_stream) {
        H->stream = (cudaStream_t)p->stream;
    } else {
        BCMGX_CUDA(cudaStreamCreateWithFlags(&H->stream, cudaStreamNonBlocking));
        H->own_stream = true;
        H->prm.stream = H->stream;
    }
    // keep freed blocks in the pool: repeated set-ups reuse them without cudaMalloc
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    BCMGX_CUDA(cudaEventCreate(&H->ev0));
    BCMGX_CUDA(cudaEventCreate(&H->ev1));
    BCMGX_CUDA(cudaEventCreateWithFlags(&H->ev_it[0], cudaEventDisableTiming));
    BCMGX_CUDA(cudaEventCreateWithFlags(&H->ev_it[1], cudaEventDisableTiming));
    BCMGX_CUDA(cudaEventCreateWithFlags(&H->ev_in, cudaEventDisableTiming));
    if (A->on_device) after_caller(H->stream, H->ev_in, H->own_stream);
    ScopedEvent t0, t1;
    BCMGX_CUDA(cudaEventRecord(t0.e, H->stream));
    stage_fault_init();
    build_hierarchy(H.get(), A);
    choose_level_kernels(H.get());
    BCMGX_CUDA(cudaEventRecord(t1.e, H->stream));
    BCMGX_CUDA(cudaEventSynchronize(t1.e));
    float ms = 0;
    cudaEventElapsedTime(&ms, t0.e, t1.e);
    stage_fault_check();
    H->setup_ms = ms;
    return H.release();
}

static void finish_batch(bcmgx_batch* B, const bcmgx_params* p)
{
    DeviceScope ds(B->device);
    if (p && p->stream) {
        B->stream = (cudaStream_t)p->stream;
    } else {
        BCMGX_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
        B->own_stream = true;
    }
    BCMGX_CUDA(cudaEventCreate(&B->ev0));
    BCMGX_CUDA(cudaEventCreate(&B->ev1));
    BCMGX_CUDA(cudaEventCreateWithFlags(&B->ev_in, cudaEventDisableTiming));
}

}  // namespace bcmgx

using namespace bcmgx;

bcmgx_batch::~bcmgx_batch()
{
    if (stream) cudaStreamSynchronize(stream);
    bcmgx::lock_free(this);
    bcmgx::pinned_free(lock_copies_host);
    bcmgx::pinned_free(lock_states_host);
    if (exec) cudaGraphExecDestroy(exec);
    copies.release();
    states_ptr.release();
    states.release();
    if (stream) cudaStreamSynchronize(stream);
    bcmgx::pinned_free(states_host);
    bcmgx::pinned_free(copies_host);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_in) cudaEventDestroy(ev_in);
    if (own)
        for (auto* h : hs) delete h;
    if (own_stream && stream) cudaStreamDestroy(stream);
}

bcmgx_hierarchy::~bcmgx_hierarchy()
{
    if (iter_graph) cudaGraphExecDestroy(iter_graph);
    bcmgx::free_multi(multi);
    multi = nullptr;
    bcmgx::free_krylov(krylov);
    krylov = nullptr;
    l1d.release();
    l1tmp.release();
    afsai_G = bcmgx::DevCsr();
    afsai_GT = bcmgx::DevCsr();
    afsai_tmp.release();
    lv.clear();
    b.release();
    xv.release();
    r.release();
    v.release();
    w.release();
    d.release();
    q.release();
    res.release();
    res32.release();
    partials.release();
    st.release();
    hist.release();
    gb.release();
    gx.release();
    // every stream-ordered buffer goes before the stream does (members left to their own
    // destructors would free on a destroyed stream)
    persist.clear();
    persist_bar.release();
    if (stream) cudaStreamSynchronize(stream);
    bcmgx::pinned_free(st_host);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_in) cudaEventDestroy(ev_in);
    for (auto& e : ev_it)
        if (e) cudaEventDestroy(e);
    if (own_stream && stream) cudaStreamDestroy(stream);
}

extern "C" {

const char* bcmgx_last_error_string(void) { return g_last_error.c_str(); }

const char* bcmgx_version(void) { return "bcmgx-b200 0.1 (sm_100a)"; }

int64_t bcmgx_launch_count(void) { return g_launches.load(); }

int bcmgx_params_default(bcmgx_params* p)
{
    return guarded([&] {
        BCMGX_REQUIRE(p != nullptr, BCMGX_ERR_INVALID_INPUT, "params is NULL");
        params_default(p);
    });
}

int bcmgx_params_from_properties(const char* path, bcmgx_params* p)
{
    return guarded([&] {
        BCMGX_REQUIRE(path && p, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        params_from_properties(path, p);
    });
}

int bcmgx_params_from_legacy_file(const char* path, bcmgx_params* p)
{
    return guarded([&] {
        BCMGX_REQUIRE(path && p, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        params_from_legacy(path, p);
    });
}

int bcmgx_params_dump(const bcmgx_params* p, const char* path)
{
    return guarded([&] {
        BCMGX_REQUIRE(p != nullptr, BCMGX_ERR_INVALID_INPUT, "params is NULL");
        FILE* f = path ? std::fopen(path, "w") : stdout;
        BCMGX_REQUIRE(f != nullptr, BCMGX_ERR_INVALID_INPUT, "cannot open output file");
        params_dump(p, f);
        if (path) std::fclose(f);
    });
}

int bcmgx_setup(const bcmgx_csr* A, const bcmgx_params* p, bcmgx_hierarchy** out)
{
    return guarded([&] {
        BCMGX_REQUIRE(A && out, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        *out = nullptr;
        *out = setup_one(A, p, -1, false);
    });
}

int bcmgx_setup_batch(int nsys, const bcmgx_csr* A, const bcmgx_params* p, int nthreads, bcmgx_batch** out)
{
    return guarded([&] {
        BCMGX_REQUIRE(nsys > 0 && A && p && out, BCMGX_ERR_INVALID_INPUT, "bad argument");
        BCMGX_REQUIRE(p->solver == BCMGX_SOLVER_FCG, BCMGX_ERR_UNSUPPORTED, "batched solves need FCG");
        *out = nullptr;
        check_params(p);
        int dev = p->device;
        if (dev < 0) BCMGX_CUDA(cudaGetDevice(&dev));
        std::unique_ptr<bcmgx_batch> B(new bcmgx_batch());
        B->own = true;
        B->device = dev;
        B->hs.assign(nsys, nullptr);
        const int T = std::max(1, std::min(nthreads > 0 ? nthreads : 8, nsys));
        std::vector<std::string> errs(T);
        std::vector<int> codes(T, BCMGX_OK);
        std::vector<std::thread> pool;
        for (int t = 0; t < T; t++) {
            pool.emplace_back([&, t] {
                try {
                    BCMGX_CUDA(cudaSetDevice(dev));
                    for (int k = t; k < nsys; k += T) B->hs[k] = setup_one(&A[k], p, dev, true);
                } catch (const Error& e) {
                    codes[t] = e.code;
                    errs[t] = e.msg;
                } catch (const std::exception& e) {
                    codes[t] = BCMGX_ERR_INTERNAL;
                    errs[t] = e.what();
                }
            });
        }
        for (auto& th : pool) th.join();
        for (int t = 0; t < T; t++)
            if (codes[t] != BCMGX_OK) throw Error(codes[t], "batch set-up: " + errs[t]);
        finish_batch(B.get(), p);
        *out = B.release();
    });
}

int bcmgx_batch_from_hierarchies(int nsys, bcmgx_hierarchy* const* hs, bcmgx_batch** out)
{
    return guarded([&] {
        BCMGX_REQUIRE(nsys > 0 && hs && out, BCMGX_ERR_INVALID_INPUT, "bad argument");
        *out = nullptr;
        std::unique_ptr<bcmgx_batch> B(new bcmgx_batch());
        B->hs.assign(hs, hs + nsys);
        B->device = hs[0]->device;
        for (auto* h : B->hs) BCMGX_REQUIRE(h && h->device == B->device, BCMGX_ERR_INVALID_INPUT, "hierarchies must share one device");
        for (auto* h : B->hs) BCMGX_REQUIRE(h->prm.solver == BCMGX_SOLVER_FCG, BCMGX_ERR_UNSUPPORTED, "batched solves need FCG");
        finish_batch(B.get(), &hs[0]->prm);
        *out = B.release();
    });
}

int bcmgx_batch_get_hierarchy(bcmgx_batch* B, int k, bcmgx_hierarchy** h)
{
    return guarded([&] {
        BCMGX_REQUIRE(B && h && k >= 0 && k < (int)B->hs.size(), BCMGX_ERR_INVALID_INPUT, "bad argument");
        *h = B->hs[k];
    });
}

int bcmgx_batch_solve(bcmgx_batch* B, const double* const* b, double* const* x, bcmgx_solve_info* infos)
{
    int status = BCMGX_OK;
    int rc = guarded([&] {
        BCMGX_REQUIRE(B && b && x, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        DeviceScope ds(B->device);
        if (B->lockstep && lock_supported(B)) {
            if (!B->lock_exec) lock_build(B);
            after_caller(B->stream, B->ev_in, B->own_stream);
            status = lock_solve(B, b, x, infos);
        } else {
            if (!B->exec) batch_build(B);
            after_caller(B->stream, B->ev_in, B->own_stream);
            status = batch_solve(B, b, x, infos);
        }
        if (status == BCMGX_ERR_NO_CONVERGENCE) set_last_error("batch solve: a system reached itnlim");
        if (status == BCMGX_ERR_NOT_SPD) set_last_error("batch solve: FCG breakdown in a system");
        stage_fault_check();
    });
    return rc != BCMGX_OK ? rc : status;
}

int bcmgx_batch_set_lockstep(bcmgx_batch* B, int on)
{
    return guarded([&] {
        BCMGX_REQUIRE(B, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        B->lockstep = on ? 1 : 0;
    });
}

int bcmgx_batch_free(bcmgx_batch* B)
{
    return guarded([&] {
        if (!B) return;
        DeviceScope ds(B->device);
        delete B;
    });
}

int bcmgx_solve(bcmgx_hierarchy* h, const double* b, double* x, int on_device, bcmgx_solve_info* info)
{
    int status = BCMGX_OK;
    int rc = guarded([&] {
        BCMGX_REQUIRE(h && b && x, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        DeviceScope ds(h->device);
        const int n = h->lv[0].A.n;
        cudaStream_t s = h->stream;
        if (on_device) {
            after_caller(s, h->ev_in, h->own_stream);
            status = solve_dispatch(h, b, x, info);
        } else {
            h->b.alloc(n, s);
            h->xv.alloc(n, s);
            BCMGX_CUDA(cudaMemcpyAsync(h->b.p, b, sizeof(double) * n, cudaMemcpyHostToDevice, s));
            BCMGX_CUDA(cudaMemcpyAsync(h->xv.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, s));
            status = solve_dispatch(h, h->b.p, h->xv.p, info);
            BCMGX_CUDA(cudaMemcpyAsync(x, h->xv.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
            BCMGX_CUDA(cudaStreamSynchronize(s));
        }
        if (status == BCMGX_ERR_NO_CONVERGENCE) set_last_error("itnlim reached before the tolerance");
        if (status == BCMGX_ERR_NOT_SPD) set_last_error("FCG breakdown: non-positive or non-finite curvature");
        stage_fault_check();
    });
    return rc != BCMGX_OK ? rc : status;
}

int bcmgx_solve_multi(bcmgx_hierarchy* h, int nrhs, const double* B, double* X, int on_device, bcmgx_solve_info* infos)
{
    int status = BCMGX_OK;
    int rc = guarded([&] {
        BCMGX_REQUIRE(h && B && X, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        BCMGX_REQUIRE(nrhs >= 1 && nrhs <= 32, BCMGX_ERR_INVALID_INPUT, "nrhs must be 1..32");
        BCMGX_REQUIRE(h->prm.solver == BCMGX_SOLVER_FCG, BCMGX_ERR_UNSUPPORTED, "multiple right-hand sides need FCG");
        DeviceScope ds(h->device);
        const size_t nk = (size_t)h->lv[0].A.n * nrhs;
        cudaStream_t s = h->stream;
        if (on_device) {
            after_caller(s, h->ev_in, h->own_stream);
            status = multi_solve(h, nrhs, B, X, infos);
        } else {
            DBuf<double> bd, xd;
            bd.alloc(nk, s);
            xd.alloc(nk, s);
            BCMGX_CUDA(cudaMemcpyAsync(bd.p, B, sizeof(double) * nk, cudaMemcpyHostToDevice, s));
            BCMGX_CUDA(cudaMemcpyAsync(xd.p, X, sizeof(double) * nk, cudaMemcpyHostToDevice, s));
            status = multi_solve(h, nrhs, bd.p, xd.p, infos);
            BCMGX_CUDA(cudaMemcpyAsync(X, xd.p, sizeof(double) * nk, cudaMemcpyDeviceToHost, s));
            BCMGX_CUDA(cudaStreamSynchronize(s));
        }
        if (status == BCMGX_ERR_NO_CONVERGENCE) set_last_error("itnlim reached before the tolerance (some column)");
        if (status == BCMGX_ERR_NOT_SPD) set_last_error("FCG breakdown in some column: non-positive or non-finite curvature");
        stage_fault_check();
    });
    return rc != BCMGX_OK ? rc : status;
}

int bcmgx_solve_adjoint(bcmgx_hierarchy* h, const double* g, const double* x, double* lambda, double* dA_val,
    int on_device, bcmgx_solve_info* info)
{
    int status = BCMGX_OK;
    int rc = guarded([&] {
        BCMGX_REQUIRE(h && g && lambda, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        BCMGX_REQUIRE(!dA_val || x, BCMGX_ERR_INVALID_INPUT, "dA needs the forward solution x");
        DeviceScope ds(h->device);
        const DevCsr& A = h->lv[0].A;
        const int n = A.n;
        cudaStream_t s = h->stream;
        if (on_device) {
            after_caller(s, h->ev_in, h->own_stream);
            BCMGX_CUDA(cudaMemsetAsync(lambda, 0, sizeof(double) * n, s));
            status = solve_dispatch(h, g, lambda, info);
            if (dA_val) grad_pattern(A, lambda, x, dA_val, s);
            BCMGX_CUDA(cudaStreamSynchronize(s));
        } else {
            DBuf<double> gd, ld, xd, dd;
            gd.alloc(n, s);
            ld.alloc(n, s);
            BCMGX_CUDA(cudaMemcpyAsync(gd.p, g, sizeof(double) * n, cudaMemcpyHostToDevice, s));
            BCMGX_CUDA(cudaMemsetAsync(ld.p, 0, sizeof(double) * n, s));
            status = solve_dispatch(h, gd.p, ld.p, info);
            BCMGX_CUDA(cudaMemcpyAsync(lambda, ld.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
            if (dA_val) {
                xd.alloc(n, s);
                dd.alloc(std::max<int64_t>(A.nnz, 1), s);
                BCMGX_CUDA(cudaMemcpyAsync(xd.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, s));
                grad_pattern(A, ld.p, xd.p, dd.p, s);
                BCMGX_CUDA(cudaMemcpyAsync(dA_val, dd.p, sizeof(double) * A.nnz, cudaMemcpyDeviceToHost, s));
            }
            BCMGX_CUDA(cudaStreamSynchronize(s));
        }
        if (status == BCMGX_ERR_NO_CONVERGENCE) set_last_error("adjoint solve: itnlim reached before the tolerance");
        stage_fault_check();
    });
    return rc != BCMGX_OK ? rc : status;
}

int bcmgx_free(bcmgx_hierarchy* h)
{
    return guarded([&] {
        if (!h) return;
        DeviceScope ds(h->device);
        delete h;
    });
}

int bcmgx_hierarchy_get_info(const bcmgx_hierarchy* h, bcmgx_hierarchy_info* info)
{
    return guarded([&] {
        BCMGX_REQUIRE(h && info, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        std::memset(info, 0, sizeof(*info));
        info->num_levels = (int)h->lv.size();
        for (int l = 0; l < info->num_levels && l < BCMGX_MAX_LEVELS; l++) {
            info->n[l] = h->lv[l].A.n;
            info->nnz[l] = h->lv[l].A.nnz;
            info->tpr[l] = h->lv[l].A.sliced ? kSlicedCode : h->lv[l].A.staged ? -h->lv[l].A.tpr : h->lv[l].A.tpr;
            info->index_bytes[l] = h->lv[l].A.sl_pid.p ? 0 : h->lv[l].A.dcol.p ? 2 : 4;
            info->value_codes[l] = h->lv[l].A.vcode.p ? h->lv[l].A.nvalues : 0;
        }
        info->op_cmplx = h->op_cmplx;
        info->op_wcmplx = h->op_wcmplx;
        info->avg_cratio = h->avg_cratio;
        info->maxcoarsesize = h->maxcoarsesize;
        info->ftcoarse = h->ftcoarse;
        info->num_sweep_records = (int)h->rec.size();
        info->setup_ms = h->setup_ms;
    });
}

int bcmgx_hierarchy_get_level(const bcmgx_hierarchy* h, int l, int* row, int* col, double* val)
{
    return guarded([&] {
        BCMGX_REQUIRE(h && l >= 0 && l < (int)h->lv.size(), BCMGX_ERR_INVALID_INPUT, "bad level");
        DeviceScope ds(h->device);
        const DevCsr& A = h->lv[l].A;
        cudaStream_t s = h->stream;
        if (row) BCMGX_CUDA(cudaMemcpyAsync(row, A.row.p, sizeof(int) * ((size_t)A.n + 1), cudaMemcpyDeviceToHost, s));
        if (col) BCMGX_CUDA(cudaMemcpyAsync(col, A.col.p, sizeof(int) * A.nnz, cudaMemcpyDeviceToHost, s));
        if (val) BCMGX_CUDA(cudaMemcpyAsync(val, A.val.p, sizeof(double) * A.nnz, cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
    });
}

int bcmgx_hierarchy_get_afsai(const bcmgx_hierarchy* h, int64_t* nnz, int* row, int* col, double* val)
{
    return guarded([&] {
        BCMGX_REQUIRE(h && nnz, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        BCMGX_REQUIRE(h->prm.preconditioner == BCMGX_PREC_AFSAI, BCMGX_ERR_INVALID_INPUT, "not an AFSAI hierarchy");
        DeviceScope ds(h->device);
        const DevCsr& G = h->afsai_G;
        cudaStream_t s = h->stream;
        *nnz = G.nnz;
        if (row) BCMGX_CUDA(cudaMemcpyAsync(row, G.row.p, sizeof(int) * ((size_t)G.n + 1), cudaMemcpyDeviceToHost, s));
        if (col) BCMGX_CUDA(cudaMemcpyAsync(col, G.col.p, sizeof(int) * G.nnz, cudaMemcpyDeviceToHost, s));
        if (val) BCMGX_CUDA(cudaMemcpyAsync(val, G.val.p, sizeof(double) * G.nnz, cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
    });
}

int bcmgx_hierarchy_get_prolongator(const bcmgx_hierarchy* h, int l, int* agg, double* p, double* M)
{
    return guarded([&] {
        BCMGX_REQUIRE(h && l >= 0 && l < (int)h->lv.size(), BCMGX_ERR_INVALID_INPUT, "bad level");
        DeviceScope ds(h->device);
        const Level& V = h->lv[l];
        cudaStream_t s = h->stream;
        const size_t n = V.A.n;
        if (agg || p) BCMGX_REQUIRE(l + 1 < (int)h->lv.size(), BCMGX_ERR_INVALID_INPUT, "coarsest level has no prolongator");
        if (agg) BCMGX_CUDA(cudaMemcpyAsync(agg, V.agg.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
        if (p) BCMGX_CUDA(cudaMemcpyAsync(p, V.p.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        if (M) BCMGX_CUDA(cudaMemcpyAsync(M, V.M.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
    });
}

int bcmgx_hierarchy_get_sweep(const bcmgx_hierarchy* h, int k, int* level, int* sweep, int* n, int* nc, int* match,
    int* agg, double* p, double* w)
{
    return guarded([&] {
        BCMGX_REQUIRE(h && k >= 0 && k < (int)h->rec.size(), BCMGX_ERR_INVALID_INPUT, "bad sweep record index");
        const SweepRecord& r = h->rec[k];
        if (level) *level = r.level;
        if (sweep) *sweep = r.sweep;
        if (n) *n = r.n;
        if (nc) *nc = r.nc;
        if (match) std::memcpy(match, r.match.data(), sizeof(int) * r.n);
        if (agg) std::memcpy(agg, r.agg.data(), sizeof(int) * r.n);
        if (p) std::memcpy(p, r.p.data(), sizeof(double) * r.n);
        if (w) std::memcpy(w, r.w.data(), sizeof(double) * r.n);
    });
}

int bcmgx_prec_apply(bcmgx_hierarchy* h, const double* r, double* v, int on_device)
{
    return guarded([&] {
        BCMGX_REQUIRE(h && r && v, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        DeviceScope ds(h->device);
        const int n = h->lv[0].A.n;
        cudaStream_t s = h->stream;
        if (on_device) {
            after_caller(s, h->ev_in, h->own_stream);
            prec_apply_dev(h, r, v);
            BCMGX_CUDA(cudaStreamSynchronize(s));
        } else {
            DBuf<double> rd, vd;
            rd.alloc(n, s);
            vd.alloc(n, s);
            BCMGX_CUDA(cudaMemcpyAsync(rd.p, r, sizeof(double) * n, cudaMemcpyHostToDevice, s));
            prec_apply_dev(h, rd.p, vd.p);
            BCMGX_CUDA(cudaMemcpyAsync(v, vd.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
            BCMGX_CUDA(cudaStreamSynchronize(s));
        }
        stage_fault_check();
    });
}

int bcmgx_time_kernels(bcmgx_hierarchy* h, int level, int reps, double* out_ms)
{
    return guarded([&] {
        BCMGX_REQUIRE(h && out_ms && level >= 0 && level < (int)h->lv.size() && reps > 0, BCMGX_ERR_INVALID_INPUT, "bad argument");
        DeviceScope ds(h->device);
        time_level_kernels(h, level, reps, out_ms);
        stage_fault_check();
    });
}

int bcmgx_time_block_kernels(bcmgx_hierarchy* h, int nrhs, int reps, double* out_ms)
{
    return guarded([&] {
        BCMGX_REQUIRE(h && out_ms && nrhs >= 1 && nrhs <= 32 && reps > 0, BCMGX_ERR_INVALID_INPUT, "bad argument");
        DeviceScope ds(h->device);
        time_block_kernels(h, nrhs, reps, out_ms);
    });
}

int bcmgx_spmv(int n, int m, int64_t nnz, const int* row, const int* col, const double* val, const double* x, double* y,
    double alpha, double beta, int threads_per_row, void* stream)
{
    return guarded([&] {
        BCMGX_REQUIRE(n >= 0 && m >= 0 && nnz >= 0, BCMGX_ERR_INVALID_INPUT, "negative size");
        BCMGX_REQUIRE(row && (nnz == 0 || (col && val)) && x && y, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        int t = threads_per_row;
        if (t <= 0) t = default_tpr(n, nnz);
        BCMGX_REQUIRE(t == 1 || t == 2 || t == 4 || t == 8 || t == 16 || t == 32, BCMGX_ERR_INVALID_INPUT,
            "threads_per_row must be a power of two <= 32");
        if (n > 0) validate_csr_dev(n, m, nnz, row, col, false, (cudaStream_t)stream);
        launch_spmv(n, row, col, val, x, y, alpha, beta, t, (cudaStream_t)stream);
    });
}

int bcmgx_spmm(int n, int m, int64_t nnz, const int* row, const int* col, const double* val, int nrhs, const double* X,
    double* Y, double alpha, double beta, void* stream)
{
    return guarded([&] {
        BCMGX_REQUIRE(n >= 0 && m >= 0 && nnz >= 0, BCMGX_ERR_INVALID_INPUT, "negative size");
        BCMGX_REQUIRE(nrhs >= 1 && nrhs <= 32, BCMGX_ERR_INVALID_INPUT, "nrhs must be 1..32");
        BCMGX_REQUIRE(row && (nnz == 0 || (col && val)) && X && Y, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        if (n > 0) validate_csr_dev(n, m, nnz, row, col, false, (cudaStream_t)stream);
        launch_spmm(n, m, nrhs, row, col, val, X, Y, alpha, beta, (cudaStream_t)stream);
    });
}

int bcmgx_edge_weights(int n, int64_t nnz, const int* row, const int* col, const double* val, const double* w, double* W,
    double* min_abs_out, void* stream)
{
    return guarded([&] {
        BCMGX_REQUIRE(n > 0 && nnz > 0 && row && col && val && w && W, BCMGX_ERR_INVALID_INPUT, "bad argument");
        cudaStream_t s = (cudaStream_t)stream;
        validate_csr_dev(n, n, nnz, row, col, true, s);
        DBuf<int> tpos;
        tpos.alloc(nnz, s);
        double mn = 0;
        edge_weights_dev(n, nnz, row, col, val, w, W, tpos.p, &mn, s);
        BCMGX_CUDA(cudaStreamSynchronize(s));
        if (min_abs_out) *min_abs_out = mn;
    });
}

int bcmgx_suitor_matching(int n, int64_t nnz, const int* row, const int* col, const double* W, int* M, void* stream)
{
    return guarded([&] {
        BCMGX_REQUIRE(n > 0 && nnz > 0 && row && col && W && M, BCMGX_ERR_INVALID_INPUT, "bad argument");
        cudaStream_t s = (cudaStream_t)stream;
        validate_csr_dev(n, n, nnz, row, col, false, s);
        DBuf<int> tpos;
        tpos.alloc(nnz, s);
        tpos_dev(n, nnz, row, col, tpos.p, s);
        suitor_dev(n, nnz, row, col, W, tpos.p, M, 0, s);
        BCMGX_CUDA(cudaStreamSynchronize(s));
    });
}

}  // extern "C"
