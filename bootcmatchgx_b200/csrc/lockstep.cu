// lockstep.cu -- many independent FCG + BCMG solves in lockstep: one kernel per step over all
// systems at once.
//
// The batch graph of solve.cu gives every system its own branch, so a launch holds one kernel node
// per system, level and step (about 116k nodes for 256 small systems), and the node count, not the
// bytes, bounds it. Here the systems whose hierarchies have the same number of levels form a group,
// and the group's hierarchy is the block-diagonal union of its members' hierarchies, level by
// level: the matrices side by side (columns shifted by the member's row offset), the composite
// prolongators with their aggregate ids shifted by the member's coarse offset. A block-diagonal
// level keeps every member's rows and their sums unchanged, so one V-cycle of the group applies
// every member's own V-cycle at once with the group's row kernels. FCG runs per member on the
// concatenated vectors: its dot products and norms are summed per member (each member's rows are
// cut into chunks of kLockChunk rows, one block per chunk, and the last chunk of a member to finish
// adds the member's chunk sums in chunk order, so the sums are deterministic), every member keeps
// its own scalars and stopping test, and a member that has stopped is left alone by the updates.
// The group iterates while any member is still running: a WHILE graph node per group, the groups
// as independent branches of one graph, one launch per batch solve.
//
// The V-cycle arithmetic of a member is its own solve's (same rows, same operations); the per-member
// sums add the same terms in another order than a solve of the member alone, so the iterates
// agree with single solves to rounding, not bit for bit.
#include "internal.h"
#include "common.cuh"

#include <algorithm>
#include <cstdlib>
#include <map>

namespace bcmgx {

constexpr int kLockChunk = 2048;   // rows per block of the FCG kernels
constexpr int kLockThreads = 256;
constexpr int kLockGroup = 32;     // members per group at most (BCMGX_LOCK_GROUP overrides)

struct LockGroup {
    std::vector<int> sys;                   // batch indices of the members
    std::vector<int> off;                   // level-0 row offset of every member (members + 1)
    std::unique_ptr<bcmgx_hierarchy> H;     // the block-diagonal hierarchy of the members
    int m = 0, nchunks = 0;
    DBuf<int> ck_sys, ck_r0, ck_r1;         // per chunk: member, first row, end row
    DBuf<int> mem_ck0, mem_nck;             // per member: first chunk, number of chunks
    DBuf<FcgState> st;                      // per member
    DBuf<double> part;                      // per chunk: up to 3 partial sums
    DBuf<int> flags;                        // [0] members still running, [1] 1 once none is
    DBuf<int> sysd;                         // the members' batch indices (device copy of sys)
    long long startup_kernels = 0, body_kernels = 0;
    ~LockGroup()
    {
        ck_sys.release();
        ck_r0.release();
        ck_r1.release();
        mem_ck0.release();
        mem_nck.release();
        st.release();
        part.release();
        flags.release();
        sysd.release();
        H.reset();
    }
};

// ------------------------------------------------------------------------------------------
// building the group hierarchy
// ------------------------------------------------------------------------------------------
struct CatSeg {
    const void* src;
    void* dst;
    long long n;
    int add;    // added to every int (kind 0)
    int kind;   // 0: int + add, 1: 8-byte copy
};

__global__ void k_cat(int nseg, const CatSeg* __restrict__ segs)
{
    for (int k = blockIdx.x; k < nseg; k += gridDim.x) {
        const CatSeg g = segs[k];
        if (g.kind == 0) {
            const int* s = (const int*)g.src;
            int* d = (int*)g.dst;
            for (long long i = threadIdx.x; i < g.n; i += blockDim.x) d[i] = s[i] + g.add;
        } else {
            const double* s = (const double*)g.src;
            double* d = (double*)g.dst;
            for (long long i = threadIdx.x; i < g.n; i += blockDim.x) d[i] = s[i];
        }
    }
}

static void run_cat(const std::vector<CatSeg>& segs, cudaStream_t s)
{
    if (segs.empty()) return;
    DBuf<CatSeg> d;
    d.alloc(segs.size(), s);
    BCMGX_CUDA(cudaMemcpyAsync(d.p, segs.data(), sizeof(CatSeg) * segs.size(), cudaMemcpyHostToDevice, s));
    note_launch();
    k_cat<<<(int)std::min<size_t>(segs.size(), 65535), 256, 0, s>>>((int)segs.size(), d.p);
    BCMGX_CHECK_LAUNCH();
    BCMGX_CUDA(cudaStreamSynchronize(s));   // segs (host memory) is read by the copy above
}

// The block-diagonal union of hierarchies with the same number of levels and the same settings.
static std::unique_ptr<bcmgx_hierarchy> concat_hierarchies(const std::vector<bcmgx_hierarchy*>& hs, int device,
    cudaStream_t s)
{
    std::unique_ptr<bcmgx_hierarchy> H(new bcmgx_hierarchy());
    const bcmgx_hierarchy& h0 = *hs[0];
    H->prm = h0.prm;
    H->prm.stream = s;
    H->prm.dispnorm = 0;
    H->device = device;
    H->stream = s;
    H->own_stream = false;
    H->grid_sweeps = h0.grid_sweeps;
    H->maxcoarsesize = h0.maxcoarsesize;
    H->ftcoarse = h0.ftcoarse;
    const int L = (int)h0.lv.size();
    const bool f32 = H->prm.vcycle_precision == BCMGX_VCYCLE_FP32;
    H->lv.resize(L);
    std::vector<std::vector<long long>> roff(L), zoff(L);
    for (int l = 0; l < L; l++) {
        roff[l].assign(hs.size() + 1, 0);
        zoff[l].assign(hs.size() + 1, 0);
        for (size_t k = 0; k < hs.size(); k++) {
            roff[l][k + 1] = roff[l][k] + hs[k]->lv[l].A.n;
            zoff[l][k + 1] = zoff[l][k] + hs[k]->lv[l].A.nnz;
        }
        BCMGX_REQUIRE(roff[l].back() <= 0x7fffffffLL && zoff[l].back() <= 0x7fffffffLL, BCMGX_ERR_UNSUPPORTED,
            "lockstep batch: a level of the union exceeds 2^31-1 rows or entries");
    }
    for (int l = 0; l < L; l++) {
        Level& V = H->lv[l];
        DevCsr& A = V.A;
        A.n = A.m = (int)roff[l].back();
        A.nnz = zoff[l].back();
        A.row.alloc((size_t)A.n + 1, s);
        A.col.alloc(std::max<int64_t>(A.nnz, 1), s);
        A.val.alloc(std::max<int64_t>(A.nnz, 1), s);
        std::vector<CatSeg> segs;
        for (size_t k = 0; k < hs.size(); k++) {
            const Level& S = hs[k]->lv[l];
            A.max_row = std::max(A.max_row, S.A.max_row);
            segs.push_back({ S.A.row.p, A.row.p + roff[l][k], S.A.n, (int)zoff[l][k], 0 });
            segs.push_back({ S.A.col.p, A.col.p + zoff[l][k], S.A.nnz, (int)roff[l][k], 0 });
            segs.push_back({ S.A.val.p, A.val.p + zoff[l][k], S.A.nnz, 0, 1 });
        }
        if (l + 1 < L) {
            V.agg.alloc(A.n, s);
            V.p.alloc(A.n, s);
            for (size_t k = 0; k < hs.size(); k++) {
                const Level& S = hs[k]->lv[l];
                segs.push_back({ S.agg.p, V.agg.p + roff[l][k], S.A.n, (int)roff[l + 1][k], 0 });
                segs.push_back({ S.p.p, V.p.p + roff[l][k], S.A.n, 0, 1 });
            }
        }
        const int nnz32 = (int)A.nnz;
        BCMGX_CUDA(cudaMemcpyAsync(A.row.p + A.n, &nnz32, sizeof(int), cudaMemcpyHostToDevice, s));
        run_cat(segs, s);
    }
    // the derived arrays as the set-up makes them: divisors, FP32 copies, int16 offsets, value
    // codes, the transposed prolongators; the coarsest level stays FP64
    for (int l = 0; l < L; l++) {
        finish_level_matrix(H->lv[l], f32 && l < L - 1, s);
        if (l + 1 < L) build_restriction(H->lv[l], H->lv[l + 1].A.n, f32, s);
    }
    BCMGX_CUDA(cudaEventCreate(&H->ev0));
    BCMGX_CUDA(cudaEventCreate(&H->ev1));
    choose_level_kernels(H.get());
    BCMGX_CUDA(cudaStreamSynchronize(s));
    return H;
}

// ------------------------------------------------------------------------------------------
// per-member FCG kernels (one block per chunk of a member's rows)
// ------------------------------------------------------------------------------------------
struct LockTabs {
    const int* ck_sys;
    const int* ck_r0;
    const int* ck_r1;
    const int* mem_ck0;
    const int* mem_nck;
};

__global__ void k_lock_init(int m, FcgState* st, double rtol, int itnlim, int* flags)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        FcgState z {};
        z.tol = rtol;
        z.itnlim = itnlim;
        st[k] = z;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        flags[0] = m;
        flags[1] = 0;
    }
}

// The chunk's K sums (valid in thread 0 of every block) go to part[chunk]; the member's last chunk
// to arrive adds its chunks' sums in chunk order and returns true (in all of its threads) with the
// totals in out[] (valid in thread 0). The ticket is reset for the next use.
template <int K>
__device__ __forceinline__ bool member_sum(double (&v)[K], int chunk, int first, int nck, double* part, int* ticket,
    double (&out)[K])
{
    block_sum<K>(v);
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) part[(size_t)chunk * 3 + k] = v[k];
        __threadfence();
        last = atomicAdd(ticket, 1) == nck - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = 0.0;
    for (int c = threadIdx.x; c < nck; c += blockDim.x)
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] += __ldcg(part + (size_t)(first + c) * 3 + k);
    block_sum<K>(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) out[k] = acc[k];
        *ticket = 0;
    }
    return true;
}

// A member stops (done, and its running count is taken off the group's)
__device__ __forceinline__ void member_stop(FcgState& S, int* flags)
{
    S.done = 1;
    if (atomicSub(flags, 1) == 1) flags[1] = 1;
}

// r = b - A x was formed by the row kernel; ||r|| -> delta0 and the tolerance (FCG.cu:46-51)
__global__ void __launch_bounds__(kLockThreads) k_lock_norm0(LockTabs t, const double* __restrict__ r, FcgState* st,
    double* part)
{
    const int c = blockIdx.x, k = t.ck_sys[c];
    double acc[1] = { 0.0 };
    for (int i = t.ck_r0[c] + threadIdx.x; i < t.ck_r1[c]; i += blockDim.x) acc[0] += r[i] * r[i];
    double out[1];
    if (member_sum<1>(acc, c, t.mem_ck0[k], t.mem_nck[k], part, &st[k].ticket[0], out) && threadIdx.x == 0) {
        FcgState& S = st[k];
        S.delta0 = sqrt(out[0]);
        S.tol = S.tol * S.delta0;
        S.iter = 0;
        S.done = 0;
        S.bad = 0;
    }
}

// The member's dots after pw = A pv and its scalar recurrence (the start-up with MODE 0, the loop
// with MODE 1), as k_fcg_dots computes them.
template <int MODE>
__global__ void __launch_bounds__(kLockThreads) k_lock_dots(LockTabs t, const double* __restrict__ pv,
    const double* __restrict__ pw, const double* __restrict__ r, const double* __restrict__ oq, FcgState* st,
    double* part, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    const int c = blockIdx.x, k = t.ck_sys[c];
    if (st[k].done) return;
    double acc[3] = { 0.0, 0.0, 0.0 };
    for (int i = t.ck_r0[c] + threadIdx.x; i < t.ck_r1[c]; i += blockDim.x) {
        const double vi = pv[i];
        acc[0] += r[i] * vi;
        acc[1] += pw[i] * vi;
        if (MODE == 1) acc[2] += oq[i] * vi;
    }
    double out[3];
    if (member_sum<3>(acc, c, t.mem_ck0[k], t.mem_nck[k], part, &st[k].ticket[1], out) && threadIdx.x == 0) {
        FcgState& S = st[k];
        S.alpha = out[0];
        S.beta = out[1];
        if (MODE == 0) {
            S.delta = out[1];
            S.theta = out[0] / out[1];
        } else {
            S.gamma = out[2];
            const double th = out[2] / S.delta;
            const double dn = out[1] - ((out[2] * out[2]) / S.delta);
            S.theta = th;
            S.delta = dn;
            S.theta2 = out[0] / dn;
        }
        if (!(S.delta > 0.0) || !isfinite(S.theta)) S.bad = 1;
    }
}

// Start-up update x += theta v, r -= theta w, d = v, q = w, ||r||^2 (FCG.cu:88-100); a member whose
// start-up broke down stops here.
__global__ void __launch_bounds__(kLockThreads) k_lock_update0(LockTabs t, const double* __restrict__ v,
    const double* __restrict__ w, double* __restrict__ x, double* __restrict__ r, double* __restrict__ d,
    double* __restrict__ q, FcgState* st, double* part, int* flags)
{
    const int c = blockIdx.x, k = t.ck_sys[c];
    if (st[k].bad) {
        if (c == t.mem_ck0[k] && threadIdx.x == 0) member_stop(st[k], flags);
        return;
    }
    const double th = st[k].theta;
    double acc[1] = { 0.0 };
    for (int i = t.ck_r0[c] + threadIdx.x; i < t.ck_r1[c]; i += blockDim.x) {
        const double vi = v[i], wi = w[i];
        x[i] = th * vi + 1.0 * x[i];
        const double ri = -th * wi + 1.0 * r[i];
        r[i] = ri;
        d[i] = vi;
        q[i] = wi;
        acc[0] += ri * ri;
    }
    double out[1];
    if (member_sum<1>(acc, c, t.mem_ck0[k], t.mem_nck[k], part, &st[k].ticket[2], out) && threadIdx.x == 0)
        st[k].rnorm2 = out[0];
}

// Loop update (double_merged_axpy twice, FCG.cu:138-144), ||r|| and the member's stopping test
// (FCG.cu:146-156); a member that stopped keeps its iterate.
__global__ void __launch_bounds__(kLockThreads) k_lock_update(LockTabs t, double* __restrict__ pv,
    const double* __restrict__ od, double* __restrict__ x, double* __restrict__ pw, const double* __restrict__ oq,
    double* __restrict__ r, FcgState* st, double* part, int* flags)
{
    if (flags[1]) return;
    const int c = blockIdx.x, k = t.ck_sys[c];
    if (st[k].done) return;
    if (st[k].bad) {
        if (c == t.mem_ck0[k] && threadIdx.x == 0) member_stop(st[k], flags);
        return;
    }
    const double th = st[k].theta, th2 = st[k].theta2;
    double acc[1] = { 0.0 };
    for (int i = t.ck_r0[c] + threadIdx.x; i < t.ck_r1[c]; i += blockDim.x) {
        const double nv = -th * od[i] + pv[i];
        pv[i] = nv;
        x[i] = th2 * nv + x[i];
        const double nw = -th * oq[i] + pw[i];
        pw[i] = nw;
        const double ri = -th2 * nw + r[i];
        r[i] = ri;
        acc[0] += ri * ri;
    }
    double out[1];
    if (member_sum<1>(acc, c, t.mem_ck0[k], t.mem_nck[k], part, &st[k].ticket[3], out) && threadIdx.x == 0) {
        FcgState& S = st[k];
        S.rnorm2 = out[0];
        const double l2 = sqrt(out[0]);
        S.iter += 1;
        if (!isfinite(l2)) S.bad = 1;
        if (!(l2 > S.tol) || S.iter >= S.itnlim || S.bad) member_stop(S, flags);
    }
}

__global__ void k_lock_set_while(cudaGraphConditionalHandle h, const int* flags)
{
    cudaGraphSetConditional(h, flags[1] ? 0u : 1u);
}

// ------------------------------------------------------------------------------------------
// groups, graph and solve
// ------------------------------------------------------------------------------------------
static LockTabs tabs(const LockGroup& G)
{
    return LockTabs { G.ck_sys.p, G.ck_r0.p, G.ck_r1.p, G.mem_ck0.p, G.mem_nck.p };
}

// Members whose settings let them share one cycle: same levels, cycle, sweeps and precision.
static bool same_cycle(const bcmgx_hierarchy* a, const bcmgx_hierarchy* b)
{
    const bcmgx_params &p = a->prm, &q = b->prm;
    return a->lv.size() == b->lv.size() && p.preconditioner == BCMGX_PREC_BCMG && q.preconditioner == BCMGX_PREC_BCMG &&
        p.cycle_type == q.cycle_type && p.prerelax_sweeps == q.prerelax_sweeps &&
        p.postrelax_sweeps == q.postrelax_sweeps && p.relaxnumber_coarse == q.relaxnumber_coarse &&
        p.vcycle_precision == q.vcycle_precision && p.rtol == q.rtol && p.itnlim == q.itnlim;
}

bool lock_supported(const bcmgx_batch* B)
{
    for (const bcmgx_hierarchy* h : B->hs)
        if (h->prm.preconditioner != BCMGX_PREC_BCMG || h->prm.rtol != B->hs[0]->prm.rtol ||
            h->prm.itnlim != B->hs[0]->prm.itnlim || h->prm.vcycle_precision != B->hs[0]->prm.vcycle_precision ||
            h->prm.cycle_type != B->hs[0]->prm.cycle_type || h->prm.prerelax_sweeps != B->hs[0]->prm.prerelax_sweeps ||
            h->prm.postrelax_sweeps != B->hs[0]->prm.postrelax_sweeps ||
            h->prm.relaxnumber_coarse != B->hs[0]->prm.relaxnumber_coarse)
            return false;
    return true;
}

static void add_group_to_graph(LockGroup& G, cudaGraph_t g, cudaStream_t s)
{
    bcmgx_hierarchy* H = G.H.get();
    const DevCsr& A = H->lv[0].A;
    const LockTabs t = tabs(G);
    const int nc = G.nchunks;
    double *x = H->gx.p, *b = H->gb.p, *r = H->r.p, *v = H->v.p, *w = H->w.p, *d = H->d.p, *q = H->q.p;
    FcgState* st = G.st.p;
    double* part = G.part.p;
    int* flags = G.flags.p;
    const long long c0 = launch_count();
    BCMGX_CUDA(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    note_launch();
    k_lock_init<<<ceil_div(G.m, 256), 256, 0, s>>>(G.m, st, H->prm.rtol, H->prm.itnlim, flags);
    rowop_resid(A, x, b, r, nullptr, s);
    note_launch();
    k_lock_norm0<<<nc, kLockThreads, 0, s>>>(t, r, st, part);
    prec_apply_impl(H, r, v, nullptr);
    rowop_spmv(A, v, w, nullptr, s);
    note_launch();
    k_lock_dots<0><<<nc, kLockThreads, 0, s>>>(t, v, w, r, nullptr, st, part, nullptr);
    note_launch();
    k_lock_update0<<<nc, kLockThreads, 0, s>>>(t, v, w, x, r, d, q, st, part, flags);
    BCMGX_CHECK_LAUNCH();
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
    // two iterations per pass (the roles of (v, w) and (d, q) alternate); the second skips itself
    // once every member has stopped
    for (int it = 0; it < 2; it++) {
        const bool even = it == 0;
        double* pv = even ? v : d;
        double* pw = even ? w : q;
        const double* od = even ? d : v;
        const double* oq = even ? q : w;
        prec_apply_impl(H, r, pv, flags + 1);
        rowop_spmv(A, pv, pw, flags + 1, s);
        note_launch();
        k_lock_dots<1><<<nc, kLockThreads, 0, s>>>(t, pv, pw, r, oq, st, part, flags + 1);
        note_launch();
        k_lock_update<<<nc, kLockThreads, 0, s>>>(t, pv, od, x, pw, oq, r, st, part, flags);
    }
    note_launch();
    k_lock_set_while<<<1, 1, 0, s>>>(h, flags);
    BCMGX_CHECK_LAUNCH();
    BCMGX_CUDA(cudaStreamEndCapture(s, &body));
    const long long c2 = launch_count();
    G.startup_kernels = c1 - c0;
    G.body_kernels = c2 - c1;
    note_launches(-(c2 - c0));   // captured, not launched
}

void lock_build(bcmgx_batch* B)
{
    cudaStream_t s = B->stream;
    const int nsys = (int)B->hs.size();
    for (bcmgx_hierarchy* H : B->hs) BCMGX_CUDA(cudaStreamSynchronize(H->stream));
    // members grouped by their number of levels, then by size: groups of at most kLockGroup
    // members of neighbouring sizes, which tend to stop after similar numbers of iterations (a
    // group iterates until its last member stops; the groups run side by side)
    int per = kLockGroup;
    if (const char* e = std::getenv("BCMGX_LOCK_GROUP")) per = std::max(1, std::atoi(e));
    std::map<size_t, std::vector<int>> bylev;
    for (int k = 0; k < nsys; k++) bylev[B->hs[k]->lv.size()].push_back(k);
    std::vector<std::vector<int>> groups;
    for (auto& kv : bylev) {
        std::vector<int> v = kv.second;
        std::stable_sort(v.begin(), v.end(), [&](int a, int b) { return B->hs[a]->lv[0].A.n < B->hs[b]->lv[0].A.n; });
        const int ng = (int)((v.size() + per - 1) / per);
        for (int g = 0; g < ng; g++) {
            const size_t a = v.size() * g / ng, b = v.size() * (g + 1) / ng;
            groups.emplace_back(v.begin() + a, v.begin() + b);
        }
    }
    lock_free(B);
    for (auto& members : groups) {
        std::unique_ptr<LockGroup> G(new LockGroup());
        G->sys = members;
        G->m = (int)G->sys.size();
        std::vector<bcmgx_hierarchy*> hs;
        for (int k : G->sys) {
            BCMGX_REQUIRE(same_cycle(B->hs[G->sys[0]], B->hs[k]), BCMGX_ERR_INTERNAL, "lockstep group with mixed settings");
            hs.push_back(B->hs[k]);
        }
        G->H = concat_hierarchies(hs, B->device, s);
        bcmgx_hierarchy* H = G->H.get();
        ensure_solve_workspace(H);
        const int n = H->lv[0].A.n;
        H->gb.alloc(n, s);
        H->gx.alloc(n, s);
        // chunks of every member's rows
        G->off.assign(G->m + 1, 0);
        std::vector<int> cs, c0, c1, m0(G->m), mn(G->m);
        for (int i = 0; i < G->m; i++) {
            const int nk = hs[i]->lv[0].A.n;
            G->off[i + 1] = G->off[i] + nk;
            m0[i] = (int)cs.size();
            for (int r = 0; r < nk; r += kLockChunk) {
                cs.push_back(i);
                c0.push_back(G->off[i] + r);
                c1.push_back(G->off[i] + std::min(nk, r + kLockChunk));
            }
            mn[i] = (int)cs.size() - m0[i];
        }
        G->nchunks = (int)cs.size();
        auto up = [&](DBuf<int>& d, const std::vector<int>& h) {
            d.alloc(h.size(), s);
            BCMGX_CUDA(cudaMemcpyAsync(d.p, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, s));
        };
        up(G->ck_sys, cs);
        up(G->ck_r0, c0);
        up(G->ck_r1, c1);
        up(G->mem_ck0, m0);
        up(G->mem_nck, mn);
        up(G->sysd, G->sys);
        G->st.alloc(G->m, s);
        BCMGX_CUDA(cudaMemsetAsync(G->st.p, 0, sizeof(FcgState) * G->m, s));
        G->part.alloc((size_t)G->nchunks * 3, s);
        G->flags.alloc(2, s);
        BCMGX_CUDA(cudaMemsetAsync(G->flags.p, 0, 2 * sizeof(int), s));
        BCMGX_CUDA(cudaStreamSynchronize(s));   // the host vectors above are read by the copies
        B->groups.push_back(G.release());
    }
    cudaGraph_t g = nullptr;
    BCMGX_CUDA(cudaGraphCreate(&g, 0));
    for (LockGroup* G : B->groups) add_group_to_graph(*G, g, s);
    BCMGX_CUDA(cudaGraphInstantiate(&B->lock_exec, g, 0));
    BCMGX_CUDA(cudaGraphDestroy(g));
    B->lock_copies.alloc(3 * (size_t)nsys, s);
    B->lock_states.alloc((size_t)nsys, s);
    if (!B->lock_copies_host) B->lock_copies_host = pinned_alloc(sizeof(LockCopy) * 3 * (size_t)nsys);
    if (!B->lock_states_host) B->lock_states_host = pinned_alloc(sizeof(FcgState) * (size_t)nsys);
    BCMGX_CUDA(cudaStreamSynchronize(s));
}

void lock_free(bcmgx_batch* B)
{
    if (B->lock_exec) cudaGraphExecDestroy(B->lock_exec);
    B->lock_exec = nullptr;
    for (LockGroup* G : B->groups) delete G;
    B->groups.clear();
    B->lock_copies.release();
    B->lock_states.release();
}

// dst[i] = src[i] for every (src, dst, n) of the list, one block per entry
__global__ void k_lock_copy(int m, const LockCopy* __restrict__ list)
{
    for (int k = blockIdx.x; k < m; k += gridDim.x) {
        const LockCopy c = list[k];
        for (int i = threadIdx.x; i < c.n; i += blockDim.x) c.dst[i] = c.src[i];
    }
}

// member k's state into the batch-ordered array
__global__ void k_lock_states(int m, const FcgState* __restrict__ st, const int* __restrict__ sys, FcgState* out)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) out[sys[k]] = st[k];
}

int lock_solve(bcmgx_batch* B, const double* const* b, double* const* x, bcmgx_solve_info* infos)
{
    const int nsys = (int)B->hs.size();
    cudaStream_t s = B->stream;
    // (the graph reads the groups' own copies of the members' hierarchies, made and synchronised
    // by lock_build: the members' streams need no wait here)
    // one list for both directions: the 2 m copies in (b and x0), then the m copies out (x)
    LockCopy* in = (LockCopy*)B->lock_copies_host;
    int nc = 0;
    for (LockGroup* G : B->groups)
        for (int i = 0; i < G->m; i++) {
            const int k = G->sys[i], nk = G->off[i + 1] - G->off[i];
            in[nc++] = LockCopy { b[k], G->H->gb.p + G->off[i], nk };
            in[nc++] = LockCopy { x[k], G->H->gx.p + G->off[i], nk };
        }
    int no = nc;
    for (LockGroup* G : B->groups)
        for (int i = 0; i < G->m; i++) {
            const int k = G->sys[i], nk = G->off[i + 1] - G->off[i];
            in[no++] = LockCopy { G->H->gx.p + G->off[i], x[k], nk };
        }
    BCMGX_CUDA(cudaMemcpyAsync(B->lock_copies.p, in, sizeof(LockCopy) * no, cudaMemcpyHostToDevice, s));
    note_launch();
    k_lock_copy<<<std::min(nc, 65535), 256, 0, s>>>(nc, (const LockCopy*)B->lock_copies.p);
    BCMGX_CHECK_LAUNCH();
    BCMGX_CUDA(cudaEventRecord(B->ev0, s));
    BCMGX_CUDA(cudaGraphLaunch(B->lock_exec, s));
    BCMGX_CUDA(cudaEventRecord(B->ev1, s));
    note_launch();
    k_lock_copy<<<std::min(no - nc, 65535), 256, 0, s>>>(no - nc, (const LockCopy*)B->lock_copies.p + nc);
    for (LockGroup* G : B->groups) {
        note_launch();
        k_lock_states<<<ceil_div(G->m, 128), 128, 0, s>>>(G->m, G->st.p, G->sysd.p, B->lock_states.p);
    }
    BCMGX_CHECK_LAUNCH();
    BCMGX_CUDA(cudaMemcpyAsync(B->lock_states_host, B->lock_states.p, sizeof(FcgState) * nsys, cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaStreamSynchronize(s));
    float ms = 0;
    BCMGX_CUDA(cudaEventElapsedTime(&ms, B->ev0, B->ev1));
    const FcgState* S = (const FcgState*)B->lock_states_host;
    // launches of the graph: every group's start-up, and its loop body once per two iterations of
    // its longest-running member
    for (LockGroup* G : B->groups) {
        int most = 0;
        for (int k : G->sys) most = std::max(most, S[k].iter);
        note_launches(G->startup_kernels + G->body_kernels * std::max(1, (most + 1) / 2));
    }
    int status = BCMGX_OK;
    for (int k = 0; k < nsys; k++) {
        const bcmgx_params& P = B->hs[k]->prm;
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

}  // namespace bcmgx
