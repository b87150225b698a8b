// dist.cu -- the row-partitioned multi-rank path: the reference's prec_setup / solve at np > 1.
//
// Every rank holds a block of consecutive rows of each level (rank r: rows offs[r] ..
// offs[r+1]-1), stored with local column ids: its own columns first (global id - offs[r]), then
// its halo, the columns of other ranks that its rows touch, in ascending global order (so that
// every other rank's entries form one contiguous segment). A vector of the level keeps the same
// layout: its own entries, then room for the halo, which the exchange fills before every kernel
// that reads x through the matrix (the reference's halo exchange, halo_communication.cu and
// CSR.cu:829-985; l1jacobi.cu:94-342). Set-up per pairwise sweep, as the reference does it:
//  * the matching on the rank's diagonal block only (suitor.cu:95-100; makeAH's 99999 for other
//    ranks' columns caps the block's minimum |a_hat|, matching.cu:82-85, 231-251), aggregates
//    numbered locally (matchingPairAggregation.cu:24-170) and shifted by the lower ranks' counts
//    (:188-222);
//  * the Galerkin product on the rank's full rows, with the aggregate id and prolongator value of
//    every halo column brought by one exchange (the rows of P that nsparseMGPU_commu_new fetches,
//    spspmpi.cu:770-1120);
//  * coarsening tests on the global sizes (full_n, matchingAggregation.cu:158-206, 400-416).
// The solve is FCG with its dot products summed over ranks (triple_inner_product.cu:80-91,
// vector.cu:492-516) and the FP64 V-cycle (GAMG_cycle.cu:58-236) whose sweeps and residuals
// exchange halos, while restriction and prolongation stay rank-local (R_local / P_local).
//
// Transports: the local form keeps all ranks' blocks in this process on one device and on one
// stream, so that each step runs rank after rank, an exchange is a device copy from the sending
// block's packed buffer into the receiving block's halo, and a sum over ranks is one small kernel
// adding the ranks' partials in rank order. The NCCL form holds one block per process: an
// exchange is one group of ncclSend / ncclRecv, a sum an ncclAllReduce, a gather of set-up counts
// an ncclAllGather, all on the hierarchy's stream. No kernel waits on another rank's memory.
#include "internal.h"
#include "rowops.cuh"

#include <nccl.h>
#include <dlfcn.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>

namespace bcmgx {

// ------------------------------------------------------------------------------------------
// NCCL, loaded at run time (the library itself does not link it)
// ------------------------------------------------------------------------------------------
struct NcclApi {
    ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
    ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
    ncclResult_t (*GroupStart)() = nullptr;
    ncclResult_t (*GroupEnd)() = nullptr;
    ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*AllGather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*CommCount)(const ncclComm_t, int*) = nullptr;
    ncclResult_t (*CommUserRank)(const ncclComm_t, int*) = nullptr;
    const char* (*GetErrorString)(ncclResult_t) = nullptr;
};

static const NcclApi& nccl()
{
    static NcclApi api;
    static std::once_flag once;
    static std::string failure;
    std::call_once(once, [] {
        void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            failure = std::string("NCCL is not available: ") + dlerror();
            return;
        }
        auto get = [&](auto& fn, const char* name) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
            if (!fn) failure = std::string("NCCL symbol missing: ") + name;
        };
        get(api.GetUniqueId, "ncclGetUniqueId");
        get(api.CommInitRank, "ncclCommInitRank");
        get(api.CommDestroy, "ncclCommDestroy");
        get(api.GroupStart, "ncclGroupStart");
        get(api.GroupEnd, "ncclGroupEnd");
        get(api.Send, "ncclSend");
        get(api.Recv, "ncclRecv");
        get(api.AllReduce, "ncclAllReduce");
        get(api.AllGather, "ncclAllGather");
        get(api.CommCount, "ncclCommCount");
        get(api.CommUserRank, "ncclCommUserRank");
        get(api.GetErrorString, "ncclGetErrorString");
    });
    if (!failure.empty()) throw Error(BCMGX_ERR_UNSUPPORTED, failure);
    return api;
}

#define BCMGX_NCCL(call)                                                                        \
    do {                                                                                        \
        ncclResult_t r_ = (call);                                                               \
        if (r_ != ncclSuccess)                                                                  \
            throw ::bcmgx::Error(BCMGX_ERR_CUDA, std::string("NCCL call failed: ") +           \
                                                     nccl().GetErrorString(r_));                \
    } while (0)

// ------------------------------------------------------------------------------------------
// kernels
// ------------------------------------------------------------------------------------------
// flag[c] = 1 for every column c of rows [0, n) outside [r0, r1)
__global__ void k_mark_halo(int n, const int* __restrict__ row, const int* __restrict__ col, int r0, int r1,
    int* __restrict__ flag)
{
    const int lane = threadIdx.x & 31;
    for (long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += ((long)gridDim.x * blockDim.x) >> 5)
        for (int j = row[i] + lane; j < row[i + 1]; j += 32) {
            const int c = col[j];
            if (c < r0 || c >= r1) flag[c] = 1;
        }
}

// gid[pos[c]] = c for every flagged column (ascending: pos is the exclusive scan of the flags)
__global__ void k_halo_list(int m, const int* __restrict__ flag, const int* __restrict__ pos, int* __restrict__ gid)
{
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < m; c += (long)gridDim.x * blockDim.x)
        if (flag[c]) gid[pos[c]] = (int)c;
}

// global column ids -> local ones: own columns c - r0, halo columns n + pos[c]
__global__ void k_localize(int n, const int* __restrict__ row, int* __restrict__ col, int r0, int r1,
    const int* __restrict__ pos)
{
    const int lane = threadIdx.x & 31;
    for (long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += ((long)gridDim.x * blockDim.x) >> 5)
        for (int j = row[i] + lane; j < row[i + 1]; j += 32) {
            const int c = col[j];
            col[j] = (c >= r0 && c < r1) ? c - r0 : n + pos[c];
        }
}

// the rank's diagonal block (columns < n) of a localized matrix: entry counts, then the copy
__global__ void k_block_count(int n, const int* __restrict__ row, const int* __restrict__ col, int* __restrict__ cnt)
{
    const int lane = threadIdx.x & 31;
    for (long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += ((long)gridDim.x * blockDim.x) >> 5) {
        int k = 0;
        for (int j = row[i] + lane; j < row[i + 1]; j += 32) k += col[j] < n ? 1 : 0;
        k = warp_sum(k);
        if (lane == 0) cnt[i] = k;
    }
}

__global__ void k_block_copy(int n, const int* __restrict__ row, const int* __restrict__ col, const double* __restrict__ val,
    const int* __restrict__ brow, int* __restrict__ bcol, double* __restrict__ bval)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        int o = brow[i];
        for (int j = row[i]; j < row[i + 1]; j++) {
            const int c = col[j];
            if (c < n) {
                bcol[o] = c;
                bval[o] = val[j];
                o++;
            }
        }
    }
}

template <typename T>
__global__ void k_pack(int m, const int* __restrict__ idx, const T* __restrict__ x, T* __restrict__ buf)
{
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (long)gridDim.x * blockDim.x) buf[k] = x[idx[k]];
}

// ext[i] = agg[i] + shift for the rank's own rows (global aggregate ids); p copied alongside
__global__ void k_extend(int n, const int* __restrict__ agg, const double* __restrict__ p, int shift,
    int* __restrict__ agg_ext, double* __restrict__ p_ext)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        agg_ext[i] = agg[i] + shift;
        p_ext[i] = p[i];
    }
}

__global__ void k_fill1(long n, double* a)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) a[i] = 1.0;
}

// sums over ranks in the local form: out = parts[0][k] + parts[1][k] + ... (rank order), written
// back to every rank's slot
__global__ void k_combine(int nparts, double* const* __restrict__ parts, int k)
{
    const int i = threadIdx.x;
    if (i >= k) return;
    double s = 0.0;
    for (int p = 0; p < nparts; p++) s += parts[p][i];
    for (int p = 0; p < nparts; p++) parts[p][i] = s;
}

// ---- FCG on the rank's rows: the kernels leave the rank's partial sums in sums[], the scalar
// ---- kernel (k_dfcg_scalars) applies the recurrence to the sums over ranks
constexpr int kDThreads = 256;
constexpr int kDBlocksPerSM = 8;

// r = b - A x, sums[0] = ||r||^2 over the rank's rows (FCG.cu:46-51)
template <int S, typename IT>
__global__ void __launch_bounds__(kDThreads) k_dfcg_resid0(int n, const int* __restrict__ row, const IT* __restrict__ col,
    const double* __restrict__ val, const double* __restrict__ x, const double* __restrict__ b, double* __restrict__ r,
    double* sums, double* partials, int* ticket)
{
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
            const double ri = -1.0 * s + 1.0 * b[r0];
            r[r0] = ri;
            acc[0] += ri * ri;
        }
    }
    double out[1];
    if (grid_sum<1>(acc, partials, ticket, out) && threadIdx.x == 0) sums[0] = out[0];
}

// pw = A pv over the rank's rows with the partial dots r.pv, pw.pv (and oq.pv in MODE 1)
template <int S, int MODE, typename IT>
__global__ void __launch_bounds__(kDThreads) k_dfcg_dots(int n, const int* __restrict__ row, const IT* __restrict__ col,
    const double* __restrict__ val, const double* __restrict__ pv, double* __restrict__ pw, const double* __restrict__ r,
    const double* __restrict__ oq, double* sums, double* partials, int* ticket)
{
    const int lane = threadIdx.x & (S - 1);
    const int sub = (threadIdx.x & 31) / S;
    const long stride = (long)gridDim.x * blockDim.x / S;
    double acc[3] = { 0.0, 0.0, 0.0 };
    for (long base = ((long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / S; base < n; base += stride) {
        const long r0 = base + sub;
        double s = 0;
        if (r0 < n) s = row_partial<S, double>(row[r0], row[r0 + 1], lane, (int)r0, col, val, pv);
        s = subwarp_sum<S>(s);
        if (r0 < n && lane == 0) {
            pw[r0] = s;
            const double vi = pv[r0];
            acc[0] += r[r0] * vi;
            acc[1] += s * vi;
            if (MODE == 1) acc[2] += oq[r0] * vi;
        }
    }
    double out[3];
    if (grid_sum<3>(acc, partials, ticket, out) && threadIdx.x == 0) {
        sums[0] = out[0];
        sums[1] = out[1];
        sums[2] = MODE == 1 ? out[2] : 0.0;
    }
}

// start-up update x += theta v, r -= theta w, d = v, q = w; sums[0] = ||r||^2 (FCG.cu:88-100)
__global__ void __launch_bounds__(kDThreads) k_dfcg_update0(int n, const double* __restrict__ v, const double* __restrict__ w,
    double* __restrict__ x, double* __restrict__ r, double* __restrict__ d, double* __restrict__ q, const FcgState* st,
    double* sums, double* partials, int* ticket)
{
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
    if (grid_sum<1>(acc, partials, ticket, out) && threadIdx.x == 0) sums[0] = out[0];
}

// loop update (double_merged_axpy x2, FCG.cu:138-144); sums[0] = ||r||^2
__global__ void __launch_bounds__(kDThreads) k_dfcg_update(int n, double* __restrict__ pv, const double* __restrict__ od,
    double* __restrict__ x, double* __restrict__ pw, const double* __restrict__ oq, double* __restrict__ r,
    const FcgState* st, double* sums, double* partials, int* ticket)
{
    if (st->bad) return;
    const double th = st->theta, th2 = st->theta2;
    double acc[1] = { 0.0 };
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
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
    if (grid_sum<1>(acc, partials, ticket, out) && threadIdx.x == 0) sums[0] = out[0];
}

// The FCG scalars from the sums over ranks. stage 0: delta0 and the tolerance; 1: the start-up
// dots; 2: ||r|| after the start-up update; 3: the loop dots and recurrence (FCG.cu:132-136);
// 4: ||r|| after a loop update and the stopping test (FCG.cu:146-156).
__global__ void k_dfcg_scalars(int stage, FcgState* st, const double* sums, double rtol, int itnlim)
{
    if (stage == 0) {
        FcgState z {};
        z.delta0 = sqrt(sums[0]);
        z.tol = rtol * z.delta0;
        z.itnlim = itnlim;
        *st = z;
    } else if (stage == 1) {
        st->alpha = sums[0];
        st->beta = sums[1];
        st->delta = sums[1];
        st->theta = sums[0] / sums[1];
        if (!(st->delta > 0.0) || !isfinite(st->theta)) st->bad = 1;
    } else if (stage == 2) {
        st->rnorm2 = sums[0];
    } else if (stage == 3) {
        st->alpha = sums[0];
        st->beta = sums[1];
        st->gamma = sums[2];
        const double th = sums[2] / st->delta;
        const double dn = sums[1] - ((sums[2] * sums[2]) / st->delta);
        st->theta = th;
        st->delta = dn;
        st->theta2 = sums[0] / dn;
        if (!(st->delta > 0.0) || !isfinite(st->theta)) st->bad = 1;
    } else {
        if (st->bad) {
            st->done = 1;
            return;
        }
        st->rnorm2 = sums[0];
        const double l2 = sqrt(sums[0]);
        st->iter += 1;
        if (!isfinite(l2)) st->bad = 1;
        st->done = (!(l2 > st->tol) || st->iter >= st->itnlim || st->bad) ? 1 : 0;
    }
}

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
// The halo of one level on one rank.
struct Halo {
    int n = 0, nh = 0;                  // own rows, halo entries
    std::vector<int> rcnt, roff;        // per rank: halo entries it owns, their first position
    std::vector<int> scnt, soff;        // per rank: entries sent to it, their first position in sidx
    DBuf<int> sidx;                     // own rows to send, grouped by destination rank
    std::vector<int> gid;               // global ids of the halo entries (ascending)
};

struct Part {
    bcmgx_hierarchy* H = nullptr;       // the rank's levels (local column ids); shares the stream
    int rank = 0;
    std::vector<Halo> halo;             // per level
    DBuf<double> sendbuf;               // packed entries of the next exchange
    DBuf<double> xh, r, v, w, d, q;     // FCG vectors (x, v, d with halo room)
    DBuf<double> b;                     // right-hand side staging
    DBuf<double> sums, partials;
    DBuf<int> tickets;
    DBuf<FcgState> st;
    DBuf<double> res;                   // the cycle's residual (level-0 rows)
    ~Part() { delete H; }
    Part() = default;
    Part(Part&& o) noexcept { *this = std::move(o); }
    Part& operator=(Part&& o) noexcept
    {
        if (this != &o) {
            delete H;
            H = o.H;
            o.H = nullptr;
            rank = o.rank;
            halo = std::move(o.halo);
            sendbuf = std::move(o.sendbuf);
            xh = std::move(o.xh);
            r = std::move(o.r);
            v = std::move(o.v);
            w = std::move(o.w);
            d = std::move(o.d);
            q = std::move(o.q);
            b = std::move(o.b);
            sums = std::move(o.sums);
            partials = std::move(o.partials);
            tickets = std::move(o.tickets);
            st = std::move(o.st);
            res = std::move(o.res);
        }
        return *this;
    }
};

}  // namespace bcmgx

struct bcmgx_dist {
    bcmgx_params prm {};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int nranks = 1;
    bool local = true;
    ncclComm_t comm = nullptr;
    std::vector<bcmgx::Part> parts;            // all ranks (local form) or this rank (NCCL form)
    std::vector<std::vector<int64_t>> offs;    // per level: the ranks' row offsets
    std::vector<int64_t> level_nnz;            // per level: entries summed over ranks
    int maxcoarsesize = 0, ftcoarse = 1;
    double op_cmplx = 1, op_wcmplx = 1, avg_cratio = 1, setup_ms = 0;
    std::vector<int> grid_sweeps;
    bcmgx::DBuf<double*> part_sums;            // local form: every rank's sums[] (k_combine)
    bcmgx::FcgState* st_host = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~bcmgx_dist();
};

namespace bcmgx {

static int dgrid(long n, int threads = 256) { return setup_grid(n, threads); }

// ---- collectives over the ranks --------------------------------------------------------------
// every rank's value of a per-rank count (vals: one per part of this process)
static std::vector<long long> gather_counts(bcmgx_dist* D, const std::vector<long long>& mine)
{
    if (D->local) return mine;
    DBuf<long long> in, out;
    in.alloc(1, D->stream);
    out.alloc(D->nranks, D->stream);
    BCMGX_CUDA(cudaMemcpyAsync(in.p, mine.data(), sizeof(long long), cudaMemcpyHostToDevice, D->stream));
    BCMGX_NCCL(nccl().AllGather(in.p, out.p, 1, ncclInt64, D->comm, D->stream));
    std::vector<long long> all(D->nranks);
    BCMGX_CUDA(cudaMemcpyAsync(all.data(), out.p, sizeof(long long) * D->nranks, cudaMemcpyDeviceToHost, D->stream));
    BCMGX_CUDA(cudaStreamSynchronize(D->stream));
    return all;
}

// the first k entries of every rank's sums[] replaced by their sum over the ranks
static void sum_over_ranks(bcmgx_dist* D, int k)
{
    if (D->local) {
        note_launch();
        k_combine<<<1, 32, 0, D->stream>>>((int)D->parts.size(), D->part_sums.p, k);
        BCMGX_CHECK_LAUNCH();
        return;
    }
    double* s = D->parts[0].sums.p;
    BCMGX_NCCL(nccl().AllReduce(s, s, k, ncclDouble, ncclSum, D->comm, D->stream));
}

// Fills the halo entries of x (per part: x[n .. n + nh)) from their owners: pack, then move.
template <typename T>
static void exchange(bcmgx_dist* D, int l, const std::vector<T*>& x)
{
    cudaStream_t s = D->stream;
    for (size_t i = 0; i < D->parts.size(); i++) {
        Part& P = D->parts[i];
        const Halo& h = P.halo[l];
        const int m = (int)h.sidx.n;
        if (m <= 0) continue;
        note_launch();
        k_pack<T><<<dgrid(m), 256, 0, s>>>(m, h.sidx.p, x[i], (T*)P.sendbuf.p);
        BCMGX_CHECK_LAUNCH();
    }
    if (D->local) {
        for (size_t i = 0; i < D->parts.size(); i++) {
            Part& P = D->parts[i];
            const Halo& h = P.halo[l];
            for (int q = 0; q < D->nranks; q++) {
                if (h.rcnt[q] == 0) continue;
                const Part& Q = D->parts[q];
                const Halo& hq = Q.halo[l];
                BCMGX_REQUIRE(hq.scnt[P.rank] == h.rcnt[q], BCMGX_ERR_INTERNAL, "halo plans disagree");
                BCMGX_CUDA(cudaMemcpyAsync(x[i] + h.n + h.roff[q], (const T*)Q.sendbuf.p + hq.soff[P.rank],
                    sizeof(T) * h.rcnt[q], cudaMemcpyDeviceToDevice, s));
            }
        }
        return;
    }
    Part& P = D->parts[0];
    const Halo& h = P.halo[l];
    const ncclDataType_t t = sizeof(T) == 8 ? ncclDouble : ncclInt32;
    BCMGX_NCCL(nccl().GroupStart());
    for (int q = 0; q < D->nranks; q++) {
        if (q == P.rank) continue;
        if (h.scnt[q] > 0) BCMGX_NCCL(nccl().Send((const T*)P.sendbuf.p + h.soff[q], h.scnt[q], t, q, D->comm, s));
        if (h.rcnt[q] > 0) BCMGX_NCCL(nccl().Recv(x[0] + h.n + h.roff[q], h.rcnt[q], t, q, D->comm, s));
    }
    BCMGX_NCCL(nccl().GroupEnd());
}

// Halo plan of a level whose matrices (one per part, n rows, global column ids < m) hold the
// rows offs[rank] .. offs[rank + 1] - 1; rewrites their columns to local ids.
static void build_halo(bcmgx_dist* D, int l, const std::vector<DevCsr*>& A, const std::vector<int64_t>& offs, long m)
{
    cudaStream_t s = D->stream;
    const int R = D->nranks;
    DBuf<int> flag, pos;
    flag.alloc(m, s);
    pos.alloc((size_t)m + 1, s);
    for (size_t i = 0; i < D->parts.size(); i++) {
        Part& P = D->parts[i];
        DevCsr& M = *A[i];
        const int r0 = (int)offs[P.rank], r1 = (int)offs[P.rank + 1];
        Halo h;
        h.n = M.n;
        BCMGX_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int) * m, s));
        if (M.n > 0) {
            note_launch();
            k_mark_halo<<<dgrid((long)M.n * 32), 256, 0, s>>>(M.n, M.row.p, M.col.p, r0, r1, flag.p);
            BCMGX_CHECK_LAUNCH();
        }
        h.nh = (int)scan_exclusive(flag.p, pos.p, m, true, s);
        DBuf<int> gid;
        gid.alloc(std::max(h.nh, 1), s);
        note_launch();
        k_halo_list<<<dgrid(m), 256, 0, s>>>((int)m, flag.p, pos.p, gid.p);
        if (M.n > 0) {
            note_launch();
            k_localize<<<dgrid((long)M.n * 32), 256, 0, s>>>(M.n, M.row.p, M.col.p, r0, r1, pos.p);
        }
        BCMGX_CHECK_LAUNCH();
        M.m = M.n + h.nh;
        h.gid.resize(h.nh);
        if (h.nh) BCMGX_CUDA(cudaMemcpyAsync(h.gid.data(), gid.p, sizeof(int) * h.nh, cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
        // owners: ranks hold consecutive blocks, the halo is ascending
        h.rcnt.assign(R, 0);
        h.roff.assign(R, 0);
        for (int q = 0; q < R; q++) {
            const auto lo = std::lower_bound(h.gid.begin(), h.gid.end(), (int)offs[q]);
            const auto hi = std::lower_bound(h.gid.begin(), h.gid.end(), (int)offs[q + 1]);
            h.roff[q] = (int)(lo - h.gid.begin());
            h.rcnt[q] = (int)(hi - lo);
        }
        P.halo.resize(std::max((size_t)l + 1, P.halo.size()));
        P.halo[l] = std::move(h);
    }
    // what every rank sends: the entries of its block in the other ranks' halos
    if (D->local) {
        for (size_t i = 0; i < D->parts.size(); i++) {
            Part& P = D->parts[i];
            Halo& h = P.halo[l];
            const int r0 = (int)offs[P.rank];
            h.scnt.assign(R, 0);
            h.soff.assign(R, 0);
            std::vector<int> idx;
            for (int q = 0; q < R; q++) {
                const Halo& hq = D->parts[q].halo[l];
                h.soff[q] = (int)idx.size();
                h.scnt[q] = hq.rcnt[P.rank];
                for (int k = 0; k < hq.rcnt[P.rank]; k++) idx.push_back(hq.gid[hq.roff[P.rank] + k] - r0);
            }
            h.sidx.alloc(idx.size(), s);
            if (!idx.empty())
                BCMGX_CUDA(cudaMemcpyAsync(h.sidx.p, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice, s));
        }
    } else {
        Part& P = D->parts[0];
        Halo& h = P.halo[l];
        // the ranks' receive counts (an R x R table), then the requested ids rank to rank
        DBuf<int> mine, all;
        mine.alloc(R, s);
        all.alloc((size_t)R * R, s);
        BCMGX_CUDA(cudaMemcpyAsync(mine.p, h.rcnt.data(), sizeof(int) * R, cudaMemcpyHostToDevice, s));
        BCMGX_NCCL(nccl().AllGather(mine.p, all.p, R, ncclInt32, D->comm, s));
        std::vector<int> table((size_t)R * R);
        BCMGX_CUDA(cudaMemcpyAsync(table.data(), all.p, sizeof(int) * R * R, cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
        h.scnt.assign(R, 0);
        h.soff.assign(R, 0);
        int tot = 0;
        for (int q = 0; q < R; q++) {
            h.soff[q] = tot;
            h.scnt[q] = q == P.rank ? 0 : table[(size_t)q * R + P.rank];
            tot += h.scnt[q];
        }
        DBuf<int> want;
        want.alloc(std::max(h.nh, 1), s);
        if (h.nh) BCMGX_CUDA(cudaMemcpyAsync(want.p, h.gid.data(), sizeof(int) * h.nh, cudaMemcpyHostToDevice, s));
        h.sidx.alloc(tot, s);
        BCMGX_NCCL(nccl().GroupStart());
        for (int q = 0; q < R; q++) {
            if (q == P.rank) continue;
            if (h.rcnt[q] > 0) BCMGX_NCCL(nccl().Send(want.p + h.roff[q], h.rcnt[q], ncclInt32, q, D->comm, s));
            if (h.scnt[q] > 0) BCMGX_NCCL(nccl().Recv(h.sidx.p + h.soff[q], h.scnt[q], ncclInt32, q, D->comm, s));
        }
        BCMGX_NCCL(nccl().GroupEnd());
        std::vector<int> idx(tot);
        if (tot) BCMGX_CUDA(cudaMemcpyAsync(idx.data(), h.sidx.p, sizeof(int) * tot, cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
        const int r0 = (int)offs[P.rank];
        for (int& v : idx) v -= r0;
        if (tot) BCMGX_CUDA(cudaMemcpyAsync(h.sidx.p, idx.data(), sizeof(int) * tot, cudaMemcpyHostToDevice, s));
    }
    for (Part& P : D->parts) {
        const size_t need = std::max<size_t>(P.halo[l].sidx.n, 1);
        if (P.sendbuf.n < need) P.sendbuf.alloc(need, s);
    }
    BCMGX_CUDA(cudaStreamSynchronize(s));
}

// The rank's diagonal block (its own columns) of a localized matrix.
static void diagonal_block(const DevCsr& A, DevCsr& B, cudaStream_t s)
{
    const int n = A.n;
    B.n = B.m = n;
    B.row.alloc((size_t)n + 1, s);
    DBuf<int> cnt;
    cnt.alloc(std::max(n, 1), s);
    note_launch();
    k_block_count<<<dgrid((long)n * 32), 256, 0, s>>>(n, A.row.p, A.col.p, cnt.p);
    BCMGX_CHECK_LAUNCH();
    B.nnz = scan_exclusive(cnt.p, B.row.p, n, true, s);
    B.col.alloc(std::max<int64_t>(B.nnz, 1), s);
    B.val.alloc(std::max<int64_t>(B.nnz, 1), s);
    note_launch();
    k_block_copy<<<dgrid(n), 256, 0, s>>>(n, A.row.p, A.col.p, A.val.p, B.row.p, B.col.p, B.val.p);
    BCMGX_CHECK_LAUNCH();
    B.max_row = row_max_dev(n, B.row.p, s);
}

static std::vector<int64_t> offsets_of(const std::vector<long long>& counts)
{
    std::vector<int64_t> o(counts.size() + 1, 0);
    for (size_t q = 0; q < counts.size(); q++) o[q + 1] = o[q] + counts[q];
    return o;
}

// The partitioned set-up (matchingAggregation / adaptiveCoarsening at np > 1). On entry every
// part holds its level-0 rows with global column ids in H->lv[0].A.
static void dist_build(bcmgx_dist* D, int64_t n_global)
{
    cudaStream_t s = D->stream;
    const bcmgx_params& Pm = D->prm;
    const int R = D->nranks;
    std::vector<DevCsr*> mats;
    for (Part& P : D->parts) mats.push_back(&P.H->lv[0].A);
    build_halo(D, 0, mats, D->offs[0], n_global);
    D->grid_sweeps.assign(std::max(Pm.max_levels - 1, 0), 1);
    if (Pm.cycle_type == BCMGX_CYCLE_H) {
        for (size_t i = 0; i < D->grid_sweeps.size(); i++)
            if (i % 2 == 0) D->grid_sweeps[i] = 2;
    } else if (Pm.cycle_type == BCMGX_CYCLE_W) {
        for (size_t i = 0; i + 1 < D->grid_sweeps.size(); i++) D->grid_sweeps[i] = 2;
    }
    D->ftcoarse = 1;
    D->maxcoarsesize = (int)(40 * std::pow((double)n_global, 1.0 / 3.0));   // AMG.cu:238-241
    std::vector<DBuf<double>> w(D->parts.size());
    for (size_t i = 0; i < D->parts.size(); i++) {
        const int n = D->parts[i].H->lv[0].A.n;
        w[i].alloc(n, s);
        note_launch();
        k_fill1<<<dgrid(n), 256, 0, s>>>(n, w[i].p);
    }
    BCMGX_CHECK_LAUNCH();
    const int sweepnumber = Pm.aggrsweeps + 1;
    double avcoarseratio = 0;
    int level;
    int64_t nglob = n_global;
    for (level = 1; level < Pm.max_levels;) {
        const size_t np = D->parts.size();
        // the running sweep's matrices (level matrix, then each sweep's coarse matrix) and halos
        std::vector<DevCsr> cur(np);
        std::vector<const DevCsr*> Ai(np);
        std::vector<Halo> sweep_halo(np);
        for (size_t i = 0; i < np; i++) Ai[i] = &D->parts[i].H->lv[level - 1].A;
        std::vector<DBuf<int>> Pagg(np);
        std::vector<DBuf<double>> Pval(np);
        for (size_t i = 0; i < np; i++) {
            Pagg[i].alloc(Ai[i]->n, s);
            Pval[i].alloc(Ai[i]->n, s);
        }
        std::vector<int64_t> coff;
        int64_t nfine = nglob, ncoarse = 0;
        for (int sw = 0; sw < sweepnumber; sw++) {
            std::vector<SweepAgg> ag(np);
            std::vector<long long> ncs(np);
            for (size_t i = 0; i < np; i++) {
                Part& P = D->parts[i];
                const Halo& h = sw == 0 ? P.halo[level - 1] : sweep_halo[i];
                DevCsr blk;
                diagonal_block(*Ai[i], blk, s);
                // a rank whose rows reach other ranks' columns has makeAH's 99999 in its minimum
                sweep_aggregate(P.H, blk, w[i].p, ag[i], level - 1, sw, h.nh > 0 ? 99999.0 : DBL_MAX);
                ncs[i] = ag[i].nc;
            }
            const std::vector<long long> all = gather_counts(D, ncs);
            coff = offsets_of(all);
            ncoarse = coff[R];
            // aggregate ids and prolongator values of every column the rank's rows touch
            std::vector<DBuf<int>> aext(np);
            std::vector<DBuf<double>> pext(np);
            std::vector<int*> ap(np);
            std::vector<double*> pp(np);
            for (size_t i = 0; i < np; i++) {
                Part& P = D->parts[i];
                const int n = Ai[i]->n, m = Ai[i]->m;
                aext[i].alloc(std::max(m, 1), s);
                pext[i].alloc(std::max(m, 1), s);
                note_launch();
                k_extend<<<dgrid(n), 256, 0, s>>>(n, ag[i].agg.p, ag[i].p.p, (int)coff[P.rank], aext[i].p, pext[i].p);
                BCMGX_CHECK_LAUNCH();
                ap[i] = aext[i].p;
                pp[i] = pext[i].p;
            }
            // the exchange runs on the plan of the sweep's matrix: swap it in as level-(level-1)'s
            // plan for the sweep, then restore
            std::vector<Halo> saved(np);
            if (sw > 0)
                for (size_t i = 0; i < np; i++) {
                    saved[i] = std::move(D->parts[i].halo[level - 1]);
                    D->parts[i].halo[level - 1] = std::move(sweep_halo[i]);
                }
            exchange<int>(D, level - 1, ap);
            exchange<double>(D, level - 1, pp);
            if (sw > 0)
                for (size_t i = 0; i < np; i++) {
                    sweep_halo[i] = std::move(D->parts[i].halo[level - 1]);
                    D->parts[i].halo[level - 1] = std::move(saved[i]);
                }
            std::vector<DevCsr> C(np);
            for (size_t i = 0; i < np; i++)
                galerkin_dev(D->parts[i].H, *Ai[i], aext[i].p, pext[i].p, ag[i].fine0.p, ag[i].fine1.p, ag[i].nc,
                    (int)ncoarse, C[i]);
            const double coarse_ratio = (double)nfine / (double)ncoarse;
            if (coarse_ratio <= 1.2) D->ftcoarse = 100;   // matchingAggregation.cu:165-167
            for (size_t i = 0; i < np; i++)
                compose_prolongator((int)Pagg[i].n, Pagg[i].p, Pval[i].p, ag[i].agg.p, ag[i].p.p, sw == 0, s);
            // C's halo (its columns are global coarse ids); C becomes the next sweep's matrix
            std::vector<DevCsr*> cm(np);
            for (size_t i = 0; i < np; i++) cm[i] = &C[i];
            {
                // build the plan into a scratch level slot, then keep it as the sweep's plan
                std::vector<Halo> keep(np);
                for (size_t i = 0; i < np; i++)
                    if ((int)D->parts[i].halo.size() > level) keep[i] = std::move(D->parts[i].halo[level]);
                build_halo(D, level, cm, coff, ncoarse);
                for (size_t i = 0; i < np; i++) {
                    sweep_halo[i] = std::move(D->parts[i].halo[level]);
                    D->parts[i].halo[level] = std::move(keep[i]);
                }
            }
            for (size_t i = 0; i < np; i++) {
                cur[i] = std::move(C[i]);
                Ai[i] = &cur[i];
                w[i] = std::move(ag[i].wc);
            }
            nfine = ncoarse;
            if ((double)ncoarse <= (double)D->ftcoarse * D->maxcoarsesize || sw + 1 == sweepnumber) break;
        }
        // the level: composite prolongator and restriction (rank-local), the coarse matrix and its halo
        for (size_t i = 0; i < np; i++) {
            Part& P = D->parts[i];
            Level& F = P.H->lv[level - 1];
            F.agg = std::move(Pagg[i]);
            F.p = std::move(Pval[i]);
            build_restriction(F, cur[i].n, false, s);
            if (level == 1) finish_level_matrix(F, false, s);
            Level NL;
            NL.A = std::move(cur[i]);
            P.H->lv.push_back(std::move(NL));
            if ((int)P.halo.size() <= level) P.halo.resize(level + 1);
            P.halo[level] = std::move(sweep_halo[i]);
        }
        D->offs.push_back(coff);
        avcoarseratio += (double)nglob / (double)ncoarse;
        nglob = ncoarse;
        level++;
        if ((double)ncoarse <= (double)D->ftcoarse * D->maxcoarsesize) break;
    }
    const int L = (int)D->parts[0].H->lv.size();
    for (Part& P : D->parts) {
        if (L == 1) finish_level_matrix(P.H->lv[0], false, s);
        for (int l = 1; l < L; l++) finish_level_matrix(P.H->lv[l], false, s);
        for (int l = 0; l < L; l++) {
            Level& V = P.H->lv[l];
            V.A.tpr = default_tpr(V.A.n, V.A.nnz);
            V.A.staged = false;
        }
    }
    // level sizes over ranks and the complexities (AMG.cu:144-165)
    D->level_nnz.assign(L, 0);
    for (int l = 0; l < L; l++) {
        std::vector<long long> z(D->parts.size());
        for (size_t i = 0; i < D->parts.size(); i++) z[i] = D->parts[i].H->lv[l].A.nnz;
        const std::vector<long long> all = gather_counts(D, z);
        for (long long v : all) D->level_nnz[l] += v;
    }
    double c = 0, wc = 0;
    for (int l = 0; l < L; l++) {
        c += (double)D->level_nnz[l];
        wc += std::pow(2.0, (double)l) * (double)D->level_nnz[l];
    }
    D->op_cmplx = c / (double)D->level_nnz[0];
    D->op_wcmplx = wc / (double)D->level_nnz[0];
    D->avg_cratio = level > 1 ? avcoarseratio / (level - 1) : 1;
}

// Work vectors of the solve: cycle buffers with halo room, the FCG vectors, the sums.
static void dist_workspace(bcmgx_dist* D)
{
    cudaStream_t s = D->stream;
    const int L = (int)D->parts[0].H->lv.size();
    std::vector<double*> sp;
    for (Part& P : D->parts) {
        for (int l = 0; l < L; l++) {
            Level& V = P.H->lv[l];
            const size_t nx = (size_t)V.A.n + P.halo[l].nh;
            V.x.alloc(std::max<size_t>(nx, 1), s);
            V.x2.alloc(std::max<size_t>(nx, 1), s);
            V.rhs.alloc(std::max(V.A.n, 1), s);
        }
        const int n = P.H->lv[0].A.n;
        const size_t nx = (size_t)n + P.halo[0].nh;
        P.xh.alloc(nx, s);
        P.v.alloc(nx, s);
        P.d.alloc(nx, s);
        P.r.alloc(n, s);
        P.w.alloc(n, s);
        P.q.alloc(n, s);
        P.b.alloc(n, s);
        P.res.alloc(std::max(n, 1), s);
        P.sums.alloc(4, s);
        P.partials.alloc((size_t)num_sms() * kDBlocksPerSM * 4, s);
        P.tickets.alloc(4, s);
        BCMGX_CUDA(cudaMemsetAsync(P.tickets.p, 0, sizeof(int) * 4, s));
        P.st.alloc(1, s);
        BCMGX_CUDA(cudaMemsetAsync(P.st.p, 0, sizeof(FcgState), s));
        sp.push_back(P.sums.p);
    }
    if (D->local) {
        D->part_sums.alloc(sp.size(), s);
        BCMGX_CUDA(cudaMemcpyAsync(D->part_sums.p, sp.data(), sizeof(double*) * sp.size(), cudaMemcpyHostToDevice, s));
    }
    if (!D->st_host) D->st_host = (FcgState*)pinned_alloc(sizeof(FcgState));
    BCMGX_CUDA(cudaStreamSynchronize(s));
}

// ---- the partitioned V-cycle (FP64) ----------------------------------------------------------
// Vectors of a cycle step: per part, a pointer (level-0 right-hand side and output come from FCG).
using PV = std::vector<double*>;

struct DistCycle {
    bcmgx_dist* D;
    int L;
    cudaStream_t s;
    PV of(int l, int which) const   // 0: rhs, 1: x, 2: x2
    {
        PV v;
        for (Part& P : D->parts) {
            Level& V = P.H->lv[l];
            v.push_back(which == 0 ? V.rhs.p : which == 1 ? V.x.p : V.x2.p);
        }
        return v;
    }
    PV res() const
    {
        PV v;
        for (Part& P : D->parts) v.push_back(P.res.p);
        return v;
    }
    void sweep(int l, const PV& f, const PV& in, const PV& out) const
    {
        exchange<double>(D, l, in);
        for (size_t i = 0; i < D->parts.size(); i++) step_jacobi64(D->parts[i].H->lv[l], in[i], f[i], out[i], s);
    }
    void first(int l, const PV& f, const PV& out) const
    {
        for (size_t i = 0; i < D->parts.size(); i++) step_first64(D->parts[i].H->lv[l], f[i], out[i], s);
    }
    void copy(int l, const PV& a, const PV& b) const
    {
        for (size_t i = 0; i < D->parts.size(); i++) step_copy64(D->parts[i].H->lv[l].A.n, a[i], b[i], s);
    }
    void zero(int l, const PV& a) const
    {
        for (size_t i = 0; i < D->parts.size(); i++) step_zero64(D->parts[i].H->lv[l].A.n, a[i], s);
    }
    // k sweeps from src (empty: zero iterate) into dst through the buffers A and B (Cycle::chain)
    void chain(int l, int k, const PV& f, const PV& src_in, const PV& dst, const PV& A, const PV& B) const
    {
        PV src = src_in;
        if (k <= 0) {
            if (src.empty()) zero(l, dst);
            else if (src != dst) copy(l, src, dst);
            return;
        }
        std::vector<PV> out(k);
        out[k - 1] = dst;
        for (int i = k - 2; i >= 0; i--) out[i] = (out[i + 1] == A) ? B : A;
        if (!src.empty() && src == out[0]) {
            const PV other = (src == A) ? B : A;
            copy(l, src, other);
            src = other;
        }
        for (int i = 0; i < k; i++) {
            if (i == 0 && src.empty()) first(l, f, out[0]);
            else sweep(l, f, i == 0 ? src : out[i - 1], out[i]);
        }
    }
    void run(int l, const PV& f, const PV& xcur, const PV& dst) const
    {
        const bcmgx_params& P = D->prm;
        const PV A = l == 0 ? dst : of(l, 1);
        const PV B = of(l, 2);
        if (l == L - 1) {
            chain(l, P.relaxnumber_coarse, f, xcur, dst, A, B);
            return;
        }
        const int coeff = P.cycle_type == BCMGX_CYCLE_VARIABLE_V ? (1 << l) : 1;
        const int kpre = P.prerelax_sweeps * coeff, kpost = P.postrelax_sweeps * coeff;
        chain(l, kpre, f, xcur, dst, A, B);
        const PV xpre = dst;
        const PV r = res();
        exchange<double>(D, l, xpre);
        for (size_t i = 0; i < D->parts.size(); i++) step_resid64(D->parts[i].H->lv[l], xpre[i], f[i], r[i], s);
        const PV fc = of(l + 1, 0);
        for (size_t i = 0; i < D->parts.size(); i++)
            step_restrict64(D->parts[i].H->lv[l], D->parts[i].H->lv[l + 1].A.n, r[i], fc[i], s);
        PV xc;
        if (L > 2 || P.relaxnumber_coarse > 0) {
            const int visits = l < (int)D->grid_sweeps.size() ? D->grid_sweeps[l] : 1;
            for (int i = 1; i <= visits; i++) {
                run(l + 1, fc, xc, of(l + 1, 1));
                xc = of(l + 1, 1);
                if (l + 1 == L - 1) break;
            }
        }
        PV pdst;
        if (kpost <= 0) {
            pdst = dst;
        } else {
            PV o0 = dst;
            for (int i = kpost - 2; i >= 0; i--) o0 = (o0 == A) ? B : A;
            pdst = (o0 == A) ? B : A;
        }
        if (!xc.empty()) {
            for (size_t i = 0; i < D->parts.size(); i++) step_prolong64(D->parts[i].H->lv[l], xc[i], xpre[i], pdst[i], s);
        } else if (pdst != xpre) {
            copy(l, xpre, pdst);
        }
        chain(l, kpost, f, pdst, dst, A, B);
    }
};

template <typename Kern>
static int dred_grid(Kern kern, long work_threads)
{
    const long need = (work_threads + kDThreads - 1) / kDThreads;
    return std::min(fit_grid(kern, kDThreads, need), num_sms() * kDBlocksPerSM);
}

template <int S>
static void launch_dresid0(Part& P, cudaStream_t s)
{
    const DevCsr& A = P.H->lv[0].A;
    note_launch();
    if (A.dcol.p) {
        auto k = k_dfcg_resid0<S, short>;
        k<<<dred_grid(k, (long)A.n * S), kDThreads, 0, s>>>(A.n, A.row.p, A.dcol.p, A.val.p, P.xh.p, P.b.p, P.r.p,
            P.sums.p, P.partials.p, P.tickets.p);
    } else {
        auto k = k_dfcg_resid0<S, int>;
        k<<<dred_grid(k, (long)A.n * S), kDThreads, 0, s>>>(A.n, A.row.p, A.col.p, A.val.p, P.xh.p, P.b.p, P.r.p,
            P.sums.p, P.partials.p, P.tickets.p);
    }
    BCMGX_CHECK_LAUNCH();
}

template <int S, int MODE>
static void launch_ddots(Part& P, const double* pv, double* pw, const double* oq, cudaStream_t s)
{
    const DevCsr& A = P.H->lv[0].A;
    note_launch();
    if (A.dcol.p) {
        auto k = k_dfcg_dots<S, MODE, short>;
        k<<<dred_grid(k, (long)A.n * S), kDThreads, 0, s>>>(A.n, A.row.p, A.dcol.p, A.val.p, pv, pw, P.r.p, oq,
            P.sums.p, P.partials.p, P.tickets.p + 1);
    } else {
        auto k = k_dfcg_dots<S, MODE, int>;
        k<<<dred_grid(k, (long)A.n * S), kDThreads, 0, s>>>(A.n, A.row.p, A.col.p, A.val.p, pv, pw, P.r.p, oq,
            P.sums.p, P.partials.p, P.tickets.p + 1);
    }
    BCMGX_CHECK_LAUNCH();
}

static void dresid0(Part& P, cudaStream_t s)
{
    switch (P.H->lv[0].A.tpr) {
    case 1: launch_dresid0<1>(P, s); break;
    case 2: launch_dresid0<2>(P, s); break;
    case 4: launch_dresid0<4>(P, s); break;
    case 8: launch_dresid0<8>(P, s); break;
    case 16: launch_dresid0<16>(P, s); break;
    default: launch_dresid0<32>(P, s); break;
    }
}

template <int MODE>
static void ddots(Part& P, const double* pv, double* pw, const double* oq, cudaStream_t s)
{
    switch (P.H->lv[0].A.tpr) {
    case 1: launch_ddots<1, MODE>(P, pv, pw, oq, s); break;
    case 2: launch_ddots<2, MODE>(P, pv, pw, oq, s); break;
    case 4: launch_ddots<4, MODE>(P, pv, pw, oq, s); break;
    case 8: launch_ddots<8, MODE>(P, pv, pw, oq, s); break;
    case 16: launch_ddots<16, MODE>(P, pv, pw, oq, s); break;
    default: launch_ddots<32, MODE>(P, pv, pw, oq, s); break;
    }
}

static void scalars(bcmgx_dist* D, int stage)
{
    for (Part& P : D->parts) {
        note_launch();
        k_dfcg_scalars<<<1, 1, 0, D->stream>>>(stage, P.st.p, P.sums.p, D->prm.rtol, D->prm.itnlim);
    }
    BCMGX_CHECK_LAUNCH();
}

// FCG over the ranks (flexibileConjugateGradients_v3, FCG.cu:27-165, at np > 1). b, x: this
// process's rows (device); x holds x0 on entry.
static int dist_fcg(bcmgx_dist* D, const double* b, double* x, bcmgx_solve_info* info)
{
    cudaStream_t s = D->stream;
    const int L = (int)D->parts[0].H->lv.size();
    DistCycle cyc { D, L, s };
    int64_t off = 0;
    for (Part& P : D->parts) {
        const int n = P.H->lv[0].A.n;
        BCMGX_CUDA(cudaMemcpyAsync(P.b.p, b + off, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        BCMGX_CUDA(cudaMemcpyAsync(P.xh.p, x + off, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        off += n;
    }
    BCMGX_CUDA(cudaEventRecord(D->ev0, s));
    PV xs, vs, ds, rs;
    for (Part& P : D->parts) {
        xs.push_back(P.xh.p);
        vs.push_back(P.v.p);
        ds.push_back(P.d.p);
        rs.push_back(P.r.p);
    }
    // start-up (FCG.cu:46-100)
    exchange<double>(D, 0, xs);
    for (Part& P : D->parts) dresid0(P, s);
    sum_over_ranks(D, 1);
    scalars(D, 0);
    cyc.run(0, rs, PV(), vs);
    exchange<double>(D, 0, vs);
    for (Part& P : D->parts) ddots<0>(P, P.v.p, P.w.p, nullptr, s);
    sum_over_ranks(D, 2);
    scalars(D, 1);
    for (Part& P : D->parts) {
        const int n = P.H->lv[0].A.n;
        note_launch();
        k_dfcg_update0<<<dred_grid(k_dfcg_update0, n), kDThreads, 0, s>>>(n, P.v.p, P.w.p, P.xh.p, P.r.p, P.d.p, P.q.p,
            P.st.p, P.sums.p, P.partials.p, P.tickets.p + 2);
    }
    BCMGX_CHECK_LAUNCH();
    sum_over_ranks(D, 1);
    scalars(D, 2);
    // loop (FCG.cu:102-156): the roles of (v, w) and (d, q) alternate
    FcgState& S = *D->st_host;
    for (int k = 0;; k++) {
        const bool even = (k % 2) == 0;
        const PV& pv = even ? vs : ds;
        cyc.run(0, rs, PV(), pv);
        exchange<double>(D, 0, pv);
        for (Part& P : D->parts) {
            double* ppv = even ? P.v.p : P.d.p;
            double* ppw = even ? P.w.p : P.q.p;
            ddots<1>(P, ppv, ppw, even ? P.q.p : P.w.p, s);
        }
        sum_over_ranks(D, 3);
        scalars(D, 3);
        for (Part& P : D->parts) {
            const int n = P.H->lv[0].A.n;
            double* ppv = even ? P.v.p : P.d.p;
            double* ppw = even ? P.w.p : P.q.p;
            const double* od = even ? P.d.p : P.v.p;
            const double* oq = even ? P.q.p : P.w.p;
            note_launch();
            k_dfcg_update<<<dred_grid(k_dfcg_update, n), kDThreads, 0, s>>>(n, ppv, od, P.xh.p, ppw, oq, P.r.p, P.st.p,
                P.sums.p, P.partials.p, P.tickets.p + 3);
        }
        BCMGX_CHECK_LAUNCH();
        sum_over_ranks(D, 1);
        scalars(D, 4);
        BCMGX_CUDA(cudaMemcpyAsync(&S, D->parts[0].st.p, sizeof(FcgState), cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
        if (D->prm.dispnorm && !S.bad) std::printf("%d) r norm: %.10lf\n", S.iter - 1, std::sqrt(S.rnorm2));
        if (S.done) break;
    }
    BCMGX_CUDA(cudaEventRecord(D->ev1, s));
    off = 0;
    for (Part& P : D->parts) {
        const int n = P.H->lv[0].A.n;
        BCMGX_CUDA(cudaMemcpyAsync(x + off, P.xh.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        off += n;
    }
    BCMGX_CUDA(cudaStreamSynchronize(s));
    float ms = 0;
    BCMGX_CUDA(cudaEventElapsedTime(&ms, D->ev0, D->ev1));
    if (info) {
        info->niter = S.iter + 1;
        info->retv = S.iter >= D->prm.itnlim ? -1 : 0;
        info->delta0 = S.delta0;
        info->exit_res = std::sqrt(S.rnorm2);
        info->solve_ms = ms;
        info->full_n = D->offs[0].back();
    }
    if (S.bad) return BCMGX_ERR_NOT_SPD;
    return S.iter >= D->prm.itnlim ? BCMGX_ERR_NO_CONVERGENCE : BCMGX_OK;
}

// The settings the partitioned path runs: FCG + BCMG with the FP64 V-cycle.
static void check_dist_params(const bcmgx_params* p)
{
    BCMGX_REQUIRE(p != nullptr, BCMGX_ERR_INVALID_INPUT, "params is NULL");
    BCMGX_REQUIRE(p->solver == BCMGX_SOLVER_FCG && p->preconditioner == BCMGX_PREC_BCMG, BCMGX_ERR_UNSUPPORTED,
        "the row-partitioned path runs FCG with the BCMG preconditioner");
    BCMGX_REQUIRE(p->vcycle_precision == BCMGX_VCYCLE_FP64, BCMGX_ERR_UNSUPPORTED,
        "the row-partitioned path runs the FP64 V-cycle");
    BCMGX_REQUIRE(p->matchtype == BCMGX_MATCH_SUITOR && p->bootstrap_type == BCMGX_BOOT_MULTIPLICATIVE &&
            p->max_hrc == 1 && p->aggr_type == 0 && p->error == 0,
        BCMGX_ERR_UNSUPPORTED, "unsupported BCMG settings");
    BCMGX_REQUIRE(p->cycle_type >= 0 && p->cycle_type < BCMGX_CYCLE_INVALID, BCMGX_ERR_INVALID_INPUT, "invalid cycle_type");
    BCMGX_REQUIRE(p->aggrsweeps >= 0 && p->aggrsweeps < 30 && p->max_levels >= 1 && p->max_levels <= BCMGX_MAX_LEVELS &&
            p->itnlim >= 1 && p->prerelax_sweeps >= 0 && p->postrelax_sweeps >= 0 && p->relaxnumber_coarse >= 0,
        BCMGX_ERR_INVALID_INPUT, "settings out of range");
}

static bcmgx_dist* dist_new(const bcmgx_params* p)
{
    std::unique_ptr<bcmgx_dist> D(new bcmgx_dist());
    D->prm = *p;
    int dev = p->device;
    if (dev < 0) BCMGX_CUDA(cudaGetDevice(&dev));
    D->device = dev;
    BCMGX_CUDA(cudaSetDevice(dev));
    if (p->stream) {
        D->stream = (cudaStream_t)p->stream;
    } else {
        BCMGX_CUDA(cudaStreamCreateWithFlags(&D->stream, cudaStreamNonBlocking));
        D->own_stream = true;
    }
    BCMGX_CUDA(cudaEventCreate(&D->ev0));
    BCMGX_CUDA(cudaEventCreate(&D->ev1));
    return D.release();
}

static Part new_part(bcmgx_dist* D, int rank)
{
    Part P;
    P.rank = rank;
    P.H = new bcmgx_hierarchy();
    P.H->prm = D->prm;
    P.H->prm.record_sweeps = 0;
    P.H->device = D->device;
    P.H->stream = D->stream;
    P.H->own_stream = false;
    P.H->lv.emplace_back();
    return P;
}

// copy of rows [r0, r1) of A (host or device arrays) into a device CSR with global column ids
static void load_rows(const bcmgx_csr* A, int64_t r0, int64_t r1, int m, DevCsr& M, cudaStream_t s)
{
    const int n = (int)(r1 - r0);
    std::vector<int> rh(2);
    const cudaMemcpyKind kind = A->on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
    BCMGX_CUDA(cudaMemcpy(&rh[0], A->row + r0, sizeof(int), kind));
    BCMGX_CUDA(cudaMemcpy(&rh[1], A->row + r1, sizeof(int), kind));
    const int64_t e0 = rh[0], e1 = rh[1];
    M.n = n;
    M.m = m;
    M.nnz = e1 - e0;
    M.row.alloc((size_t)n + 1, s);
    M.col.alloc(std::max<int64_t>(M.nnz, 1), s);
    M.val.alloc(std::max<int64_t>(M.nnz, 1), s);
    const cudaMemcpyKind k2 = A->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    BCMGX_CUDA(cudaMemcpyAsync(M.row.p, A->row + r0, sizeof(int) * ((size_t)n + 1), k2, s));
    BCMGX_CUDA(cudaMemcpyAsync(M.col.p, A->col + e0, sizeof(int) * M.nnz, k2, s));
    BCMGX_CUDA(cudaMemcpyAsync(M.val.p, A->val + e0, sizeof(double) * M.nnz, k2, s));
    // row offsets relative to the block
    if (e0 != 0) {
        std::vector<int> rows((size_t)n + 1);
        BCMGX_CUDA(cudaMemcpyAsync(rows.data(), M.row.p, sizeof(int) * rows.size(), cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
        for (int& v : rows) v -= (int)e0;
        BCMGX_CUDA(cudaMemcpyAsync(M.row.p, rows.data(), sizeof(int) * rows.size(), cudaMemcpyHostToDevice, s));
    }
    validate_csr_dev(n, m, M.nnz, M.row.p, M.col.p, false, s);
    M.max_row = row_max_dev(n, M.row.p, s);
}

}  // namespace bcmgx

using namespace bcmgx;

bcmgx_dist::~bcmgx_dist()
{
    if (stream) cudaStreamSynchronize(stream);
    parts.clear();
    part_sums.release();
    if (stream) cudaStreamSynchronize(stream);
    pinned_free(st_host);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (own_stream && stream) cudaStreamDestroy(stream);
}

namespace {
template <typename F>
int dist_guarded(F&& f)
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
    }
}

struct TimedEvents {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TimedEvents()
    {
        BCMGX_CUDA(cudaEventCreate(&e0));
        BCMGX_CUDA(cudaEventCreate(&e1));
    }
    ~TimedEvents()
    {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
    float ms() const
    {
        BCMGX_CUDA(cudaEventSynchronize(e1));
        float v = 0;
        BCMGX_CUDA(cudaEventElapsedTime(&v, e0, e1));
        return v;
    }
};

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (dev >= 0 && dev != prev) BCMGX_CUDA(cudaSetDevice(dev));
    }
    ~DevGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};
}  // namespace

extern "C" {

int bcmgx_dist_setup_local(const bcmgx_csr* A, int nranks, const int64_t* offs, const bcmgx_params* p, bcmgx_dist** out)
{
    return dist_guarded([&] {
        BCMGX_REQUIRE(A && offs && out && nranks >= 1, BCMGX_ERR_INVALID_INPUT, "bad argument");
        *out = nullptr;
        check_dist_params(p);
        BCMGX_REQUIRE(A->n > 0 && A->n == A->m && A->nnz > 0 && A->nnz <= 0x7fffffffLL && A->row && A->col && A->val,
            BCMGX_ERR_INVALID_INPUT, "matrix must be square, non-empty, with int32 offsets");
        BCMGX_REQUIRE(offs[0] == 0 && offs[nranks] == A->n, BCMGX_ERR_INVALID_INPUT, "offsets must run from 0 to n");
        for (int r = 0; r < nranks; r++)
            BCMGX_REQUIRE(offs[r + 1] > offs[r], BCMGX_ERR_INVALID_INPUT, "every rank needs at least one row");
        DevGuard g(p->device);
        std::unique_ptr<bcmgx_dist> D(dist_new(p));
        D->nranks = nranks;
        D->local = true;
        D->offs.push_back(std::vector<int64_t>(offs, offs + nranks + 1));
        TimedEvents te;
        BCMGX_CUDA(cudaEventRecord(te.e0, D->stream));
        for (int r = 0; r < nranks; r++) {
            D->parts.push_back(new_part(D.get(), r));
            load_rows(A, offs[r], offs[r + 1], A->n, D->parts.back().H->lv[0].A, D->stream);
        }
        dist_build(D.get(), A->n);
        dist_workspace(D.get());
        BCMGX_CUDA(cudaEventRecord(te.e1, D->stream));
        D->setup_ms = te.ms();
        *out = D.release();
    });
}

int bcmgx_dist_setup_nccl(const bcmgx_csr* A_rows, int64_t row_offset, int64_t n_global, void* nccl_comm,
    const bcmgx_params* p, bcmgx_dist** out)
{
    return dist_guarded([&] {
        BCMGX_REQUIRE(A_rows && out && nccl_comm, BCMGX_ERR_INVALID_INPUT, "bad argument");
        *out = nullptr;
        check_dist_params(p);
        BCMGX_REQUIRE(A_rows->n > 0 && A_rows->m == n_global && n_global <= 0x7fffffffLL && A_rows->nnz > 0 &&
                A_rows->nnz <= 0x7fffffffLL && A_rows->row && A_rows->col && A_rows->val && row_offset >= 0 &&
                row_offset + A_rows->n <= n_global,
            BCMGX_ERR_INVALID_INPUT, "this rank's rows must be non-empty and lie inside the global matrix");
        DevGuard g(p->device);
        std::unique_ptr<bcmgx_dist> D(dist_new(p));
        D->local = false;
        D->comm = (ncclComm_t)nccl_comm;
        int R = 0, me = 0;
        BCMGX_NCCL(nccl().CommCount(D->comm, &R));
        BCMGX_NCCL(nccl().CommUserRank(D->comm, &me));
        D->nranks = R;
        TimedEvents te;
        BCMGX_CUDA(cudaEventRecord(te.e0, D->stream));
        D->parts.push_back(new_part(D.get(), me));
        // the ranks' blocks: every rank's row count, in rank order
        const std::vector<long long> cnt = gather_counts(D.get(), { (long long)A_rows->n });
        D->offs.push_back(offsets_of(cnt));
        BCMGX_REQUIRE(D->offs[0][me] == row_offset && D->offs[0][R] == n_global, BCMGX_ERR_INVALID_INPUT,
            "the ranks' row blocks must be consecutive in rank order and cover the matrix");
        bcmgx_csr rows = *A_rows;
        load_rows(&rows, 0, rows.n, (int)n_global, D->parts[0].H->lv[0].A, D->stream);
        dist_build(D.get(), n_global);
        dist_workspace(D.get());
        BCMGX_CUDA(cudaEventRecord(te.e1, D->stream));
        D->setup_ms = te.ms();
        *out = D.release();
    });
}

int bcmgx_dist_solve(bcmgx_dist* D, const double* b, double* x, int on_device, bcmgx_solve_info* info)
{
    int status = BCMGX_OK;
    int rc = dist_guarded([&] {
        BCMGX_REQUIRE(D && b && x, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        DevGuard g(D->device);
        int64_t n = 0;
        for (Part& P : D->parts) n += P.H->lv[0].A.n;
        cudaStream_t s = D->stream;
        if (on_device) {
            if (D->own_stream) {
                cudaEvent_t ev;
                BCMGX_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
                BCMGX_CUDA(cudaEventRecord(ev, cudaStreamLegacy));
                BCMGX_CUDA(cudaStreamWaitEvent(s, ev, 0));
                cudaEventDestroy(ev);
            }
            status = dist_fcg(D, b, x, info);
        } else {
            DBuf<double> bd, xd;
            bd.alloc(n, s);
            xd.alloc(n, s);
            BCMGX_CUDA(cudaMemcpyAsync(bd.p, b, sizeof(double) * n, cudaMemcpyHostToDevice, s));
            BCMGX_CUDA(cudaMemcpyAsync(xd.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, s));
            status = dist_fcg(D, bd.p, xd.p, info);
            BCMGX_CUDA(cudaMemcpyAsync(x, xd.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
            BCMGX_CUDA(cudaStreamSynchronize(s));
        }
        if (status == BCMGX_ERR_NO_CONVERGENCE) set_last_error("itnlim reached before the tolerance");
        if (status == BCMGX_ERR_NOT_SPD) set_last_error("FCG breakdown: non-positive or non-finite curvature");
    });
    return rc != BCMGX_OK ? rc : status;
}

int bcmgx_dist_get_info(const bcmgx_dist* D, bcmgx_hierarchy_info* info)
{
    return dist_guarded([&] {
        BCMGX_REQUIRE(D && info, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        std::memset(info, 0, sizeof(*info));
        const int L = (int)D->offs.size();
        info->num_levels = L;
        for (int l = 0; l < L && l < BCMGX_MAX_LEVELS; l++) {
            info->n[l] = (int)D->offs[l].back();
            info->nnz[l] = D->level_nnz[l];
            info->tpr[l] = D->parts[0].H->lv[l].A.tpr;
            info->index_bytes[l] = D->parts[0].H->lv[l].A.dcol.p ? 2 : 4;
            info->value_codes[l] = D->parts[0].H->lv[l].A.vcode.p ? D->parts[0].H->lv[l].A.nvalues : 0;
        }
        info->op_cmplx = D->op_cmplx;
        info->op_wcmplx = D->op_wcmplx;
        info->avg_cratio = D->avg_cratio;
        info->maxcoarsesize = D->maxcoarsesize;
        info->ftcoarse = D->ftcoarse;
        info->setup_ms = D->setup_ms;
    });
}

int bcmgx_dist_get_level(const bcmgx_dist* D, int l, int* rows, int64_t* nnz, int* row, int* col, double* val,
    int64_t* offs)
{
    return dist_guarded([&] {
        BCMGX_REQUIRE(D && l >= 0 && l < (int)D->offs.size() && rows && nnz, BCMGX_ERR_INVALID_INPUT, "bad argument");
        DevGuard g(D->device);
        cudaStream_t s = D->stream;
        int nr = 0;
        int64_t nz = 0;
        for (const Part& P : D->parts) {
            nr += P.H->lv[l].A.n;
            nz += P.H->lv[l].A.nnz;
        }
        *rows = nr;
        *nnz = nz;
        if (offs) std::copy(D->offs[l].begin(), D->offs[l].end(), offs);
        int ro = 0;
        int64_t eo = 0;
        if (row) row[0] = 0;
        for (const Part& P : D->parts) {
            const DevCsr& A = P.H->lv[l].A;
            const Halo& h = P.halo[l];
            const int r0 = (int)D->offs[l][P.rank];
            std::vector<int> rr((size_t)A.n + 1), cc(A.nnz);
            BCMGX_CUDA(cudaMemcpyAsync(rr.data(), A.row.p, sizeof(int) * rr.size(), cudaMemcpyDeviceToHost, s));
            BCMGX_CUDA(cudaMemcpyAsync(cc.data(), A.col.p, sizeof(int) * cc.size(), cudaMemcpyDeviceToHost, s));
            if (val) BCMGX_CUDA(cudaMemcpyAsync(val + eo, A.val.p, sizeof(double) * A.nnz, cudaMemcpyDeviceToHost, s));
            BCMGX_CUDA(cudaStreamSynchronize(s));
            if (row)
                for (int i = 1; i <= A.n; i++) row[ro + i] = (int)(eo + rr[i]);
            if (col)
                for (int64_t j = 0; j < A.nnz; j++) col[eo + j] = cc[j] < A.n ? cc[j] + r0 : h.gid[cc[j] - A.n];
            ro += A.n;
            eo += A.nnz;
        }
    });
}

int bcmgx_dist_get_prolongator(const bcmgx_dist* D, int l, int* agg, double* p, double* M)
{
    return dist_guarded([&] {
        BCMGX_REQUIRE(D && l >= 0 && l < (int)D->offs.size(), BCMGX_ERR_INVALID_INPUT, "bad level");
        if (agg || p) BCMGX_REQUIRE(l + 1 < (int)D->offs.size(), BCMGX_ERR_INVALID_INPUT, "coarsest level has no prolongator");
        DevGuard g(D->device);
        cudaStream_t s = D->stream;
        int64_t o = 0;
        for (const Part& P : D->parts) {
            const Level& V = P.H->lv[l];
            const int n = V.A.n;
            if (agg) {
                BCMGX_CUDA(cudaMemcpyAsync(agg + o, V.agg.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
                BCMGX_CUDA(cudaStreamSynchronize(s));
                const int shift = (int)D->offs[l + 1][P.rank];
                for (int i = 0; i < n; i++) agg[o + i] += shift;
            }
            if (p) BCMGX_CUDA(cudaMemcpyAsync(p + o, V.p.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
            if (M) BCMGX_CUDA(cudaMemcpyAsync(M + o, V.M.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
            o += n;
        }
        BCMGX_CUDA(cudaStreamSynchronize(s));
    });
}

int bcmgx_dist_free(bcmgx_dist* D)
{
    return dist_guarded([&] {
        if (!D) return;
        DevGuard g(D->device);
        delete D;
    });
}

int bcmgx_nccl_unique_id(unsigned char* id128)
{
    return dist_guarded([&] {
        BCMGX_REQUIRE(id128, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        static_assert(sizeof(ncclUniqueId) == 128, "NCCL unique ids are 128 bytes");
        ncclUniqueId id;
        BCMGX_NCCL(nccl().GetUniqueId(&id));
        std::memcpy(id128, &id, sizeof(id));
    });
}

int bcmgx_nccl_comm_init(int nranks, int rank, const unsigned char* id128, void** comm)
{
    return dist_guarded([&] {
        BCMGX_REQUIRE(id128 && comm && nranks >= 1 && rank >= 0 && rank < nranks, BCMGX_ERR_INVALID_INPUT, "bad argument");
        ncclUniqueId id;
        std::memcpy(&id, id128, sizeof(id));
        ncclComm_t c = nullptr;
        BCMGX_NCCL(nccl().CommInitRank(&c, nranks, id, rank));
        *comm = c;
    });
}

int bcmgx_nccl_comm_destroy(void* comm)
{
    return dist_guarded([&] {
        if (!comm) return;
        BCMGX_NCCL(nccl().CommDestroy((ncclComm_t)comm));
    });
}

}  // extern "C"
