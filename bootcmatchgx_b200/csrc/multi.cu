// multi.cu -- K <= 32 right-hand sides of one system in one solve: block FCG around the block
// V-cycle (the V-cycle of solve.cu run on n x K blocks with the kernels of blockops.cuh).
//
// Every column k runs the recurrence of flexibileConjugateGradients_v3 (FCG.cu:27-165) with its
// own scalars: the dot products of all K columns come out of one fused kernel (SpMM + K triples
// of dots), reduced deterministically per column. A column stops on its own tolerance
// rtol * ||b_k - A x0_k|| or on itnlim; from then on its x and r are left unchanged, and the loop
// ends when every column has stopped. A column with a zero initial residual stops at once with
// x = x0. The whole solve is one CUDA graph: the start-up, then a WHILE conditional node over
// two iterations per body, as the single-vector graph solve. Internally the block has KP columns
// (the next power of two >= K, leading dimension KP); the padding columns are zero and stopped
// from the start.
#include "internal.h"
#include "blockops.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace bcmgx {

int num_sms();

namespace {

constexpr int kBlkThreads = 256;
constexpr int kBlkBlocksPerSM = 8;

struct BlockState {
    double alpha[kMaxRhs], beta[kMaxRhs], gamma[kMaxRhs], delta[kMaxRhs];
    double theta[kMaxRhs], theta2[kMaxRhs], rnorm2[kMaxRhs], delta0[kMaxRhs], tol[kMaxRhs];
    int iter[kMaxRhs], done[kMaxRhs], bad[kMaxRhs];
    int all_done, itnlim;
    int ticket[4];
};

// Per-column sums: thread values v[q][w] belong to column (lane % lpe) * W + w (lpe * W <= 32,
// a power of two; threads without a column hold zeros). Warps meet in shared memory, blocks in
// `partials` (block-major), and the last block to arrive adds the partials in block order, so
// the result does not depend on scheduling. Returns true in every thread of the last block;
// out[] is valid in its warp 0, lane k holding column k. blockDim.x <= 256.
template <int NV, int W>
__device__ __forceinline__ bool blk_colsum(const double (&v)[NV][W], int lpe, double* partials, int* ticket, double (&out)[NV])
{
    __shared__ double sh[NV][8][32][W];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++)
#pragma unroll
        for (int w = 0; w < W; w++) sh[q][wid][lane][w] = v[q][w];
    __syncthreads();
    if (wid == 0) {
        const int g = (lane / W) & (lpe - 1), w = lane % W;   // lanes of column `lane`: g, g + lpe, ...
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double t = 0.0;
            for (int wi = 0; wi < (int)(blockDim.x >> 5); wi++)
                for (int l = g; l < 32; l += lpe) t += sh[q][wi][l][w];
            partials[((size_t)blockIdx.x * NV + q) * 32 + lane] = t;
        }
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!last) return false;
    __threadfence();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double t = 0.0;
            for (int b = 0; b < (int)gridDim.x; b++) t += __ldcg(partials + ((size_t)b * NV + q) * 32 + lane);
            out[q] = t;
        }
        if (lane == 0) *ticket = 0;
    }
    return true;
}

__global__ void k_blk_init(BlockState* st, int K, double rtol, int itnlim)
{
    const int k = threadIdx.x;
    if (k < kMaxRhs) {
        st->iter[k] = 0;
        st->done[k] = k < K ? 0 : 1;
        st->bad[k] = 0;
        st->tol[k] = rtol;
        st->rnorm2[k] = 0.0;
        st->delta0[k] = 0.0;
    }
    if (k == 0) {
        st->all_done = 0;
        st->itnlim = itnlim;
        for (int t = 0; t < 4; t++) st->ticket[t] = 0;
    }
}

// R = B - A X and per column delta0 = ||r||, tol = rtol * delta0 (FCG.cu:46-51).
template <int W>
__global__ void __launch_bounds__(kBlkThreads, 4) k_blk_resid0(int n, int lpe_log2, int kp, const int* __restrict__ row,
    const int* __restrict__ col, const double* __restrict__ val, const double* __restrict__ X, const double* __restrict__ B,
    double* __restrict__ R, BlockState* st, double* partials, int stage_ok)
{
    __shared__ BlkEnt<double> stage[kBlkThreads / 32][BlkStage<double>::cap];
    const int lane = threadIdx.x & 31;
    double acc[1][W] = {};
    blk_rows<W>(n, lpe_log2, kp, kp, row, col, val, X, stage_ok, stage[threadIdx.x >> 5],
        [&](long, long o, const double (&s)[W]) {
            double bb[W], rr[W];
            ldw<W>(B + o, bb);
#pragma unroll
            for (int w = 0; w < W; w++) {
                rr[w] = -1.0 * s[w] + 1.0 * bb[w];
                acc[0][w] += rr[w] * rr[w];
            }
            stv<W>(R + o, rr);
        });
    double out[1];
    if (blk_colsum<1, W>(acc, 1 << lpe_log2, partials, &st->ticket[0], out) && threadIdx.x < kp) {
        const double d0 = sqrt(out[0]);
        st->delta0[lane] = d0;
        st->tol[lane] = st->tol[lane] * d0;
        if (d0 == 0.0) st->done[lane] = 1;   // x0 solves this column exactly
    }
}

// PW = A PV with the per-column dots alpha = r.pv, beta = pw.pv (and gamma = oq.pv in the loop),
// then the scalar recurrence of each running column (FCG.cu:59-86, 121-136).
template <int MODE, int W>
__global__ void __launch_bounds__(kBlkThreads, 4) k_blk_spmv_dots(int n, int lpe_log2, int kp, const int* __restrict__ row,
    const int* __restrict__ col, const double* __restrict__ val, const double* __restrict__ PV, double* __restrict__ PW,
    const double* __restrict__ R, const double* __restrict__ OQ, BlockState* st, double* partials, int stage_ok,
    const int* __restrict__ skip)
{
    if (skip && *skip) return;
    __shared__ BlkEnt<double> stage[kBlkThreads / 32][BlkStage<double>::cap];
    const int lane = threadIdx.x & 31;
    double acc[3][W] = {};
    blk_rows<W>(n, lpe_log2, kp, kp, row, col, val, PV, stage_ok, stage[threadIdx.x >> 5],
        [&](long, long o, const double (&s)[W]) {
            double vi[W], ri[W], qi[W];
            stv<W>(PW + o, s);
            ldw<W>(PV + o, vi);
            ldw<W>(R + o, ri);
            if (MODE == 1) ldw<W>(OQ + o, qi);
#pragma unroll
            for (int w = 0; w < W; w++) {
                acc[0][w] += ri[w] * vi[w];
                acc[1][w] += s[w] * vi[w];
                if (MODE == 1) acc[2][w] += qi[w] * vi[w];
            }
        });
    double out[3];
    if (blk_colsum<3, W>(acc, 1 << lpe_log2, partials, &st->ticket[1], out) && threadIdx.x < kp && !st->done[lane]) {
        const int k = lane;
        st->alpha[k] = out[0];
        st->beta[k] = out[1];
        if (MODE == 0) {
            st->delta[k] = out[1];
            st->theta[k] = out[0] / out[1];
        } else {
            st->gamma[k] = out[2];
            const double th = out[2] / st->delta[k];
            const double dn = out[1] - ((out[2] * out[2]) / st->delta[k]);
            st->theta[k] = th;
            st->delta[k] = dn;
            st->theta2[k] = out[0] / dn;
        }
        if (!(st->delta[k] > 0.0) || !isfinite(st->theta[k])) st->bad[k] = 1;
    }
}

// Start-up update of each running column (FCG.cu:88-100): X += theta V, R -= theta W, D = V,
// Q = W, ||r||^2. Element loop: a thread always sees the same column, lane % kp.
__global__ void __launch_bounds__(kBlkThreads) k_blk_update0(int n, int lk, const double* __restrict__ V,
    const double* __restrict__ W, double* __restrict__ X, double* __restrict__ R, double* __restrict__ D,
    double* __restrict__ Q, BlockState* st, double* partials)
{
    const int kp = 1 << lk;
    const int c = threadIdx.x & (kp - 1);
    const bool live = !st->done[c] && !st->bad[c];
    const double th = live ? st->theta[c] : 0.0;
    double acc[1][1] = { { 0.0 } };
    if (live) {
        BCMGX_BLOCK_ELEMS(o, n, lk)
        {
            const double vi = V[o], wi = W[o];
            X[o] = th * vi + 1.0 * X[o];
            const double ri = -th * wi + 1.0 * R[o];
            R[o] = ri;
            D[o] = vi;
            Q[o] = wi;
            acc[0][0] += ri * ri;
        }
    }
    double out[1];
    if (blk_colsum<1, 1>(acc, kp, partials, &st->ticket[2], out) && threadIdx.x < kp && !st->done[c] && !st->bad[c])
        st->rnorm2[c] = out[0];
}

// Loop update of each running column (FCG.cu:138-156): PV = -theta OD + PV, X += theta2 PV,
// PW = -theta OQ + PW, R -= theta2 PW, then ||r|| and the column's stopping test. A column that
// broke down (bad) stops with its last valid iterate. all_done = every column stopped.
__global__ void __launch_bounds__(kBlkThreads) k_blk_update(int n, int lk, double* __restrict__ PV,
    const double* __restrict__ OD, double* __restrict__ X, double* __restrict__ PW, const double* __restrict__ OQ,
    double* __restrict__ R, BlockState* st, double* partials, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    const int kp = 1 << lk;
    const int c = threadIdx.x & (kp - 1);
    const bool live = !st->done[c] && !st->bad[c];
    const double th = live ? st->theta[c] : 0.0, th2 = live ? st->theta2[c] : 0.0;
    double acc[1][1] = { { 0.0 } };
    if (live) {
        BCMGX_BLOCK_ELEMS(o, n, lk)
        {
            const double nv = -th * OD[o] + PV[o];
            PV[o] = nv;
            X[o] = th2 * nv + X[o];
            const double nw = -th * OQ[o] + PW[o];
            PW[o] = nw;
            const double ri = -th2 * nw + R[o];
            R[o] = ri;
            acc[0][0] += ri * ri;
        }
    }
    double out[1];
    if (blk_colsum<1, 1>(acc, kp, partials, &st->ticket[3], out) && threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int stopped = 1;
        if (lane < kp) {
            if (live) {
                st->rnorm2[lane] = out[0];
                st->iter[lane] += 1;
                const double l2 = sqrt(out[0]);
                if (!isfinite(l2)) st->bad[lane] = 1;
                if (!(l2 > st->tol[lane]) || st->iter[lane] >= st->itnlim || st->bad[lane]) st->done[lane] = 1;
            } else if (st->bad[lane]) {
                st->done[lane] = 1;
            }
            stopped = st->done[lane];
        }
        stopped = __all_sync(0xffffffffu, stopped);
        if (lane == 0) st->all_done = stopped;
    }
}

__global__ void k_blk_set_while(cudaGraphConditionalHandle h, const BlockState* st)
{
    cudaGraphSetConditional(h, st->all_done ? 0u : 1u);
}

}  // namespace

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
struct MultiWork {
    int K = 0, lk = 0;                      // columns, log2 of the padded width KP
    std::vector<DBuf<unsigned char>> raw;   // cycle buffers
    CycleBufs cyc;
    DBuf<double> B, X, R, V, W, D, Q, part;
    DBuf<double> P;                         // scratch block of the l1-Jacobi / AFSAI preconditioners
    DBuf<BlockState> st;
    BlockState* st_host = nullptr;
    cudaGraphExec_t graph = nullptr;
    long long startup_kernels = 0, body_kernels = 0;
    ~MultiWork()
    {
        if (graph) cudaGraphExecDestroy(graph);
        pinned_free(st_host);
    }
};

void free_multi(MultiWork* w) { delete w; }

namespace {

Vec cycle_buf(MultiWork& wk, size_t n, bool f32, cudaStream_t s)
{
    wk.raw.emplace_back();
    wk.raw.back().alloc((n << wk.lk) * (f32 ? sizeof(float) : sizeof(double)), s);
    return Vec { wk.raw.back().p, f32 };
}

// (Re)allocates the block workspace for K columns (padded to KP): the cycle buffers of every
// level in the cycle's precision (as ensure_solve_workspace does for one vector) and the FCG
// block vectors. A new K also drops the captured graph.
void ensure_multi(bcmgx_hierarchy* H, MultiWork& wk, int K)
{
    if (wk.K == K) return;
    cudaStream_t s = H->stream;
    if (wk.graph) {
        BCMGX_CUDA(cudaStreamSynchronize(s));
        cudaGraphExecDestroy(wk.graph);
        wk.graph = nullptr;
    }
    int lk = 0;
    while ((1 << lk) < K) lk++;
    const bool same_width = wk.K > 0 && wk.lk == lk;
    wk.K = K;
    if (same_width) return;   // same padded width: buffers stay
    wk.lk = lk;
    wk.raw.clear();
    wk.raw.reserve(4 * H->lv.size() + 1);   // no reallocation: the views keep raw pointers only
    const int L = (int)H->lv.size();
    const bool f32 = H->prm.vcycle_precision == BCMGX_VCYCLE_FP32;
    wk.cyc.lv.assign(L, CycleBufs::L());
    for (int l = 0; l < L; l++) {
        const size_t n = (size_t)H->lv[l].A.n;
        const bool lf = f32 && l < L - 1;
        CycleBufs::L& b = wk.cyc.lv[l];
        // level 0 of the FP64 cycle reads the FCG block and sweeps into the output block
        if (l > 0 || lf) {
            b.rhs = cycle_buf(wk, n, lf, s);
            b.x = cycle_buf(wk, n, lf, s);
        }
        b.x2 = cycle_buf(wk, n, lf, s);
    }
    wk.cyc.res = cycle_buf(wk, (size_t)H->lv[0].A.n, f32 && L > 1, s);
    const size_t nk = (size_t)H->lv[0].A.n << lk;
    wk.B.alloc(nk, s);
    wk.X.alloc(nk, s);
    wk.R.alloc(nk, s);
    wk.V.alloc(nk, s);
    wk.W.alloc(nk, s);
    wk.D.alloc(nk, s);
    wk.Q.alloc(nk, s);
    wk.part.alloc((size_t)num_sms() * kBlkBlocksPerSM * 3 * 32, s);
    const int pc = H->prm.preconditioner;
    if (pc == BCMGX_PREC_L1_JACOBI || pc == BCMGX_PREC_AFSAI) wk.P.alloc(nk, s);
    wk.st.alloc(1, s);
    if (!wk.st_host) wk.st_host = (BlockState*)pinned_alloc(2 * sizeof(BlockState));
}

// grid of a row-slot SpMM kernel over n rows (at most kBlkBlocksPerSM blocks per SM: the size
// of the partials)
template <typename Kern>
int rows_grid(Kern kern, long n, BlkShape sh)
{
    const long rows_per_block = blk_rows_per_block<double>(sh.lpe_log2, kBlkThreads);
    return std::min(fit_grid(kern, kBlkThreads, (n + rows_per_block - 1) / rows_per_block), num_sms() * kBlkBlocksPerSM);
}

// the staged 32-bit entry offsets (col * kp) hold for blocks of fewer than 2^31 elements
int stage_ok(const DevCsr& A, int kp) { return (long)A.m * kp <= 0x7fffffffL ? 1 : 0; }

// the level-0 SpMM shape of the FCG kernels (FP64 blocks of KP columns)
BlkShape fcg_shape(const MultiWork& wk) { return blk_shape(1 << wk.lk, (int)sizeof(double)); }

void launch_resid0(const DevCsr& A, const MultiWork& wk, cudaStream_t s)
{
    const BlkShape sh = fcg_shape(wk);
    const int kp = 1 << wk.lk;
    auto go = [&](auto kern) {
        note_launch();
        kern<<<rows_grid(kern, A.n, sh), kBlkThreads, 0, s>>>(A.n, sh.lpe_log2, kp, A.row.p, A.col.p, A.val.p, wk.X.p,
            wk.B.p, wk.R.p, wk.st.p, wk.part.p, stage_ok(A, kp));
    };
    if (sh.W == 2) go(k_blk_resid0<2>);
    else go(k_blk_resid0<1>);
    BCMGX_CHECK_LAUNCH();
}

template <int MODE>
void launch_dots(const DevCsr& A, const MultiWork& wk, const double* pv, double* pw, const double* oq, const int* skip,
    cudaStream_t s)
{
    const BlkShape sh = fcg_shape(wk);
    const int kp = 1 << wk.lk;
    auto go = [&](auto kern) {
        note_launch();
        kern<<<rows_grid(kern, A.n, sh), kBlkThreads, 0, s>>>(A.n, sh.lpe_log2, kp, A.row.p, A.col.p, A.val.p, pv, pw,
            wk.R.p, oq, wk.st.p, wk.part.p, stage_ok(A, kp), skip);
    };
    if (sh.W == 2) go(k_blk_spmv_dots<MODE, 2>);
    else go(k_blk_spmv_dots<MODE, 1>);
    BCMGX_CHECK_LAUNCH();
}

// grid of an element-wise kernel over an n x 2^lk block (at most kBlkBlocksPerSM blocks per SM:
// the size of the partials)
template <typename Kern>
int elem_grid(Kern kern, long n, int lk)
{
    return std::min(fit_grid(kern, kBlkThreads, ((n << lk) + kBlkThreads - 1) / kBlkThreads), num_sms() * kBlkBlocksPerSM);
}

void blk_startup(bcmgx_hierarchy* H, MultiWork& wk)
{
    cudaStream_t s = H->stream;
    const DevCsr& A = H->lv[0].A;
    note_launch();
    k_blk_init<<<1, 32, 0, s>>>(wk.st.p, wk.K, H->prm.rtol, H->prm.itnlim);
    BCMGX_CHECK_LAUNCH();
    launch_resid0(A, wk, s);
    cycle_apply_block(H, wk.cyc, wk.lk, wk.R.p, wk.V.p, wk.P.p, nullptr);
    launch_dots<0>(A, wk, wk.V.p, wk.W.p, nullptr, nullptr, s);
    note_launch();
    k_blk_update0<<<elem_grid(k_blk_update0, A.n, wk.lk), kBlkThreads, 0, s>>>(A.n, wk.lk, wk.V.p, wk.W.p, wk.X.p, wk.R.p, wk.D.p, wk.Q.p,
        wk.st.p, wk.part.p);
    BCMGX_CHECK_LAUNCH();
}

// one block iteration; (V, W) and (D, Q) swap roles with the parity, as in the single solve
void blk_iteration(bcmgx_hierarchy* H, MultiWork& wk, bool even, const int* skip)
{
    cudaStream_t s = H->stream;
    const DevCsr& A = H->lv[0].A;
    double* pv = even ? wk.V.p : wk.D.p;
    double* pw = even ? wk.W.p : wk.Q.p;
    const double* od = even ? wk.D.p : wk.V.p;
    const double* oq = even ? wk.Q.p : wk.W.p;
    cycle_apply_block(H, wk.cyc, wk.lk, wk.R.p, pv, wk.P.p, skip);
    launch_dots<1>(A, wk, pv, pw, oq, skip, s);
    note_launch();
    k_blk_update<<<elem_grid(k_blk_update, A.n, wk.lk), kBlkThreads, 0, s>>>(A.n, wk.lk, pv, od, wk.X.p, pw, oq, wk.R.p, wk.st.p,
        wk.part.p, skip);
    BCMGX_CHECK_LAUNCH();
}

void build_multi_graph(bcmgx_hierarchy* H, MultiWork& wk)
{
    cudaStream_t s = H->stream;
    BCMGX_CUDA(cudaStreamSynchronize(s));
    cudaGraph_t g = nullptr;
    BCMGX_CUDA(cudaGraphCreate(&g, 0));
    const long long c0 = launch_count();
    BCMGX_CUDA(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    blk_startup(H, wk);
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
    blk_iteration(H, wk, true, &wk.st.p->all_done);
    blk_iteration(H, wk, false, &wk.st.p->all_done);
    note_launch();
    k_blk_set_while<<<1, 1, 0, s>>>(h, wk.st.p);
    BCMGX_CHECK_LAUNCH();
    BCMGX_CUDA(cudaStreamEndCapture(s, &body));
    const long long c2 = launch_count();
    wk.startup_kernels = c1 - c0;
    wk.body_kernels = c2 - c1;
    note_launches(-(c2 - c0));   // captured, not launched
    BCMGX_CUDA(cudaGraphInstantiate(&wk.graph, g, 0));
    BCMGX_CUDA(cudaGraphDestroy(g));
}

// n x K block (leading dimension K) <-> n x KP block (leading dimension KP, zero padding)
void copy_block(double* dst, size_t dld, const double* src, size_t sld, int n, int K, cudaStream_t s)
{
    if (dld == sld)
        BCMGX_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * (size_t)n * sld, cudaMemcpyDeviceToDevice, s));
    else
        BCMGX_CUDA(cudaMemcpy2DAsync(dst, sizeof(double) * dld, src, sizeof(double) * sld, sizeof(double) * K, n,
            cudaMemcpyDeviceToDevice, s));
}

// Stream path (use_graph = 0): the start-up, then iterations enqueued one ahead of the host's
// look at the stopping flag (the extra iteration skips itself on the device once all_done is
// set), as the single-vector stream solve.
void multi_stream_solve(bcmgx_hierarchy* H, MultiWork& wk)
{
    cudaStream_t s = H->stream;
    blk_startup(H, wk);
    BlockState* ring = wk.st_host;
    auto enqueue = [&](int k) {
        blk_iteration(H, wk, (k % 2) == 0, &wk.st.p->all_done);
        BCMGX_CUDA(cudaMemcpyAsync(ring + (k % 2), wk.st.p, sizeof(BlockState), cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaEventRecord(H->ev_it[k % 2], s));
    };
    enqueue(0);
    int k = 0;
    for (;;) {
        enqueue(k + 1);
        BCMGX_CUDA(cudaEventSynchronize(H->ev_it[k % 2]));
        if (ring[k % 2].all_done) break;
        k++;
    }
}

}  // namespace

// B, X: device, row-major n x K (X: x0 in, solution out). infos: K entries or null.
// Average device time of the level-0 block FCG SpMV + dots (loop form) for K columns, on the
// solve's block workspace filled with zeros (CUDA events, reps launches after one warm-up).
double time_block_dots(bcmgx_hierarchy* H, int K, int reps)
{
    ensure_solve_workspace(H);
    if (!H->multi) H->multi = new MultiWork();
    MultiWork& wk = *H->multi;
    ensure_multi(H, wk, K);
    cudaStream_t s = H->stream;
    const DevCsr& A = H->lv[0].A;
    const size_t nk = (size_t)A.n << wk.lk;
    for (DBuf<double>* b : { &wk.V, &wk.W, &wk.R, &wk.Q }) BCMGX_CUDA(cudaMemsetAsync(b->p, 0, sizeof(double) * nk, s));
    note_launch();
    k_blk_init<<<1, 32, 0, s>>>(wk.st.p, wk.K, 1.0, 1);
    BCMGX_CHECK_LAUNCH();
    cudaEvent_t e0, e1;
    BCMGX_CUDA(cudaEventCreate(&e0));
    BCMGX_CUDA(cudaEventCreate(&e1));
    launch_dots<1>(A, wk, wk.V.p, wk.W.p, wk.Q.p, nullptr, s);
    BCMGX_CUDA(cudaEventRecord(e0, s));
    for (int i = 0; i < reps; i++) launch_dots<1>(A, wk, wk.V.p, wk.W.p, wk.Q.p, nullptr, s);
    BCMGX_CUDA(cudaEventRecord(e1, s));
    BCMGX_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    BCMGX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return (double)ms / reps;
}

int multi_solve(bcmgx_hierarchy* H, int K, const double* B, double* X, bcmgx_solve_info* infos)
{
    BCMGX_REQUIRE(K >= 1 && K <= kMaxRhs, BCMGX_ERR_INVALID_INPUT, "the number of right-hand sides must be 1..32");
    ensure_solve_workspace(H);
    if (!H->multi) H->multi = new MultiWork();
    MultiWork& wk = *H->multi;
    ensure_multi(H, wk, K);
    const bool graph = H->prm.use_graph == 1;
    if (graph && !wk.graph) build_multi_graph(H, wk);
    cudaStream_t s = H->stream;
    const int n = H->lv[0].A.n;
    const size_t kp = (size_t)1 << wk.lk;
    if (kp != (size_t)K) {
        BCMGX_CUDA(cudaMemsetAsync(wk.B.p, 0, sizeof(double) * n * kp, s));
        BCMGX_CUDA(cudaMemsetAsync(wk.X.p, 0, sizeof(double) * n * kp, s));
    }
    copy_block(wk.B.p, kp, B, K, n, K, s);
    copy_block(wk.X.p, kp, X, K, n, K, s);
    BCMGX_CUDA(cudaEventRecord(H->ev0, s));
    if (graph) BCMGX_CUDA(cudaGraphLaunch(wk.graph, s));
    else multi_stream_solve(H, wk);
    BCMGX_CUDA(cudaEventRecord(H->ev1, s));
    copy_block(X, K, wk.X.p, kp, n, K, s);
    BCMGX_CUDA(cudaMemcpyAsync(wk.st_host, wk.st.p, sizeof(BlockState), cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaStreamSynchronize(s));
    float ms = 0;
    BCMGX_CUDA(cudaEventElapsedTime(&ms, H->ev0, H->ev1));
    const BlockState& S = *wk.st_host;
    int maxit = 0, anybad = 0, status = BCMGX_OK;
    for (int k = 0; k < K; k++) {
        maxit = std::max(maxit, S.iter[k]);
        anybad |= S.bad[k];
        if (infos) {
            infos[k].niter = S.iter[k] + 1;
            infos[k].retv = S.iter[k] >= S.itnlim ? -1 : 0;
            infos[k].delta0 = S.delta0[k];
            infos[k].exit_res = std::sqrt(S.rnorm2[k]);
            infos[k].solve_ms = ms;
            infos[k].full_n = n;
        }
        if (S.bad[k]) status = BCMGX_ERR_NOT_SPD;
        else if (S.iter[k] >= S.itnlim && status == BCMGX_OK) status = BCMGX_ERR_NO_CONVERGENCE;
    }
    if (graph) {
        const long long bodies = std::max(1LL, (long long)(maxit + 1) / 2 + (anybad ? 1 : 0));
        note_launches(wk.startup_kernels + wk.body_kernels * bodies);
    }
    return status;
}

}  // namespace bcmgx
