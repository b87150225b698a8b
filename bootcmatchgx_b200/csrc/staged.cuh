// staged.cuh -- CSR row kernels whose matrix stream is staged in shared memory by bulk async
// copies (sm_100a).
//
// The plain row kernels (rowops.cuh) load each entry's column and value into registers and then
// gather x through them, so every row pays two dependent rounds of memory latency, and the
// entries in flight are bounded by the registers of the resident warps. Here one producer warp
// per block streams fixed tiles of R consecutive rows -- their row offsets, column indices and
// values -- into a ring of shared-memory stages with cp.async.bulk (completion counted on an
// mbarrier, no multicast), several tiles ahead of the consumers. The consumer warps read a
// row's entries from shared memory and gather x, with the lane-to-entry mapping and the
// summation order of k_rowop<S>, so the results are bit-identical to it.
//
// Bulk copies move 16-byte granules: a tile's entry range is widened to multiples of 8 entries
// and its row offsets to multiples of 4, so the copies may read up to 7 entries and 3 row offsets
// past the end of the arrays (every device buffer of the library carries 64 bytes of padding).
// A tile whose widened range does not fit a stage is read from global memory instead. Every
// wait on an mbarrier gives up after a time limit and stores a nonzero code in *fault (1: the
// producer waited for a free stage, 2: a consumer for a full one, 4: the final drain). The limit
// is wait_ns (one second in production) for the first two; the drain, which must not let the
// block exit while bulk copies into its shared memory are in flight, always waits up to one
// second. A consumer warp decides to give up as a whole (every lane leaves the tile loop
// together), so no shuffle runs with lanes that have left.
#pragma once

#include <algorithm>

#include "rowops.cuh"

namespace bcmgx {

constexpr int kStageWarps = 12;                  // consumer warps per block (+1 producer warp)
constexpr int kStageThreads = (kStageWarps + 1) * 32;
constexpr int kStageMaxRows = kStageWarps * 32;  // rows per tile at most: one per lane (S = 1)
constexpr int kStageRowSlots = kStageMaxRows + 8;

// Shared-memory budget per value source / index type: 4 stages of 18 KB for entries of at most 6
// bytes (3 blocks per SM), 3 stages of 30 KB for wider entries (2 blocks per SM). A coded matrix
// (ValSrc: one byte per entry) also keeps its value table after the stages. (Stages of 10 KB for
// coded entries cut the tiles from 192 to 100 rows and made the sweep slower, 0.133 -> 0.163 ms.)
template <typename VS, typename IT>
struct StageCfg {
    using VT = typename ValSrc<VS>::type;
    static constexpr bool kCoded = ValSrc<VS>::coded;
    static constexpr int kVal = ValSrc<VS>::bytes;                 // value bytes streamed per entry
    static constexpr int kEntry = (int)sizeof(IT) + kVal;
    // entries per copy granule: both streams of a tile move whole 16-byte granules
    static constexpr int G = std::max(8, 16 / std::min((int)sizeof(IT), kVal));
    static constexpr int kBytes = kEntry <= 6 ? 18432 : 30720;
    static constexpr int NS = kEntry <= 6 ? 4 : 3;
    static constexpr int CAP = ((kBytes - kStageRowSlots * 4) / kEntry) & ~(G - 1);   // entries per stage
    static constexpr int COLS = kStageRowSlots * 4;                                  // byte offsets in a stage
    static constexpr int VALS = COLS + CAP * (int)sizeof(IT);
    static constexpr int STAGE = VALS + CAP * kVal;
    static constexpr int TAB = NS * STAGE;                                          // the value table (coded)
    static constexpr int SMEM = TAB + (kCoded ? kValueCodes * (int)sizeof(VT) : 0);
    static_assert(COLS % 16 == 0 && VALS % 16 == 0 && STAGE % 16 == 0, "stage layout must keep 16-byte granules");
    static_assert((G * (int)sizeof(IT)) % 16 == 0 && (G * kVal) % 16 == 0, "a granule must be whole 16-byte units");
    static_assert(SMEM <= 227 * 1024, "the stage ring must fit a block's shared memory");
    static_assert(CAP >= 64 * 8, "a stage must hold a useful tile");
    static_assert((kStageMaxRows + 4) <= kStageRowSlots, "a tile's widened row offsets must fit their slots");
};

// Rows per tile for a matrix of n rows and nnz entries and S threads per row: the largest multiple
// of 4 whose entries (average row length plus 4 %, plus the widening to whole granules) fit a
// stage, at most one row per consumer sub-warp (kStageWarps * 32 / S), so that every sub-warp owns
// at most one row of a tile.
template <typename VS, typename IT>
inline int stage_tile_rows(int n, int64_t nnz, int S)
{
    using C = StageCfg<VS, IT>;
    const double avg = n > 0 ? std::max(1.0, (double)nnz / n) : 1.0;
    int r = (int)((C::CAP - 2 * C::G) / (avg * 1.04));
    r = std::min(r, kStageWarps * 32 / S) & ~3;
    return std::max(r, 4);
}

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
constexpr unsigned long long kStageWaitNs = 1000000000ull;   // one second

// Waits for the phase of parity `parity` to complete; false after about limit_ns nanoseconds.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity,
    unsigned long long limit_ns = kStageWaitNs)
{
    if (mbar_try_wait(b, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        for (int i = 0; i < 64; i++)
            if (mbar_try_wait(b, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}
// L2 policy for data read once per pass: evict first, so that the gathered vectors stay in L2.
__device__ __forceinline__ unsigned long long l2_evict_first()
{
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
// Global -> shared bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned),
// completing as transaction bytes on mbarrier `bar`, with L2 policy `pol`.
__device__ __forceinline__ void bulk_to_smem(void* dst, const void* src, unsigned bytes, unsigned long long* bar,
    unsigned long long pol)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;"
        ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
        : "memory");
}

__device__ __forceinline__ int col_of(short v, int r) { return r + (int)v; }
__device__ __forceinline__ int col_of(int v, int) { return v; }

extern __shared__ __align__(128) unsigned char stage_smem[];

// Epilogue operands of one row (those the operation reads), loaded ahead of its entries; f and M
// are read once per pass and streamed (evict-first).
template <int OP, typename AT, typename XT, typename FT, typename MT, typename YT>
__device__ __forceinline__ void row_operands(int r, const XT* __restrict__ x, const FT* __restrict__ f,
    const MT* __restrict__ M, const YT* __restrict__ y, double beta, AT& o1, AT& o2, AT& o3)
{
    if (OP == OP_AXPBY) {
        if (beta != 0.0) o1 = (AT)y[r];
    } else if (OP == OP_RESID) {
        o1 = (AT)ld_stream(f + r);
    } else {
        o1 = (AT)ld_stream(f + r);
        o2 = (AT)ld_stream(M + r);
        o3 = (AT)ld_ro(x + r);
    }
}

// The operations of k_rowop (y = alpha A x + beta y, y = f - A x, or one l1-Jacobi sweep) over
// tiles of R rows, tile t on block t mod gridDim.x, row i of a tile on consumer sub-warp i.
// Launch with kStageThreads threads and StageCfg<VS, IT>::SMEM bytes of dynamic shared memory;
// R = stage_tile_rows<VS, IT>(n, nnz, S): a multiple of 4, at most kStageWarps * 32 / S. VS: the
// values, stored or coded (the codes are staged, the table sits in shared memory).
// wait_ns: limit of the producer's and the consumers' stage waits (kStageWaitNs in production).
// drop_first: a fault-path test hook; when set, block 0's producer issues no copy for its first
// tile, so that the consumers' wait for that stage runs out (the drain skips that stage, which
// has no copy in flight).
template <int S, int OP, typename VS, typename XT, typename FT, typename MT, typename YT, typename IT>
__global__ void __launch_bounds__(kStageThreads) k_rowop_staged(int n, int R, const int* __restrict__ row,
    const IT* __restrict__ col, VS val, const XT* __restrict__ x, const FT* __restrict__ f,
    const MT* __restrict__ M, YT* __restrict__ y, double alpha, double beta, const int* __restrict__ skip,
    int* __restrict__ fault, unsigned long long wait_ns, int drop_first)
{
    dep_wait();
    dep_release();
    if (skip && *skip) return;
    using C = StageCfg<VS, IT>;
    using VT = typename C::VT;
    using AT = typename Acc<VT>::type;
    constexpr int NS = C::NS, CAP = C::CAP, K = 8, SPW = 32 / S, G = C::G;
    __shared__ unsigned long long full[NS], empty[NS];
    __shared__ int meta[NS][2];   // widened first entry of the stage; 1 when its entries are staged
    const int warp = threadIdx.x >> 5, l32 = threadIdx.x & 31;
    const int ntiles = (int)(((long)n + R - 1) / R);
    VT* tab_s = (VT*)(stage_smem + C::TAB);
    if constexpr (C::kCoded) {
        for (int i = threadIdx.x; i < kValueCodes; i += blockDim.x) tab_s[i] = __ldg(val.tab + i);
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < NS; k++) {
            mbar_init(&full[k], 1);
            mbar_init(&empty[k], kStageWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (warp == kStageWarps) {
        // producer: one thread issues the copies of every tile of this block, NS tiles ahead
        if (l32 != 0) return;
        const unsigned long long pol = l2_evict_first();
        const int dropped = (drop_first && blockIdx.x == 0) ? 0 : -1;   // tile index with no copy
        int it = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
            const int st = it % NS;
            if (it >= NS && !mbar_wait(&empty[st], ((unsigned)(it / NS) & 1u) ^ 1u, wait_ns)) {
                *(volatile int*)fault = 1;
                break;
            }
            if (it == dropped) continue;
            const int t0 = t * R, t1 = min(t0 + R, n);
            const int a0 = __ldg(row + t0) & ~(G - 1), a1 = (__ldg(row + t1) + G - 1) & ~(G - 1);
            const int cnt = a1 - a0, nrp = (t1 - t0 + 4) & ~3;
            const bool fits = cnt <= CAP;
            unsigned char* base = stage_smem + st * C::STAGE;
            meta[st][0] = a0;
            meta[st][1] = fits ? 1 : 0;
            const unsigned bytes = (unsigned)nrp * 4u + (fits ? (unsigned)cnt * (unsigned)C::kEntry : 0u);
            mbar_expect_tx(&full[st], bytes);
            bulk_to_smem(base, row + t0, (unsigned)nrp * 4u, &full[st], pol);
            if (fits && cnt > 0) {
                bulk_to_smem(base + C::COLS, col + a0, (unsigned)cnt * (unsigned)sizeof(IT), &full[st], pol);
                if constexpr (C::kCoded)
                    bulk_to_smem(base + C::VALS, val.code + a0, (unsigned)cnt, &full[st], pol);
                else
                    bulk_to_smem(base + C::VALS, val + a0, (unsigned)cnt * (unsigned)sizeof(VT), &full[st], pol);
            }
        }
        // the copies still in flight land before the block's shared memory is released
        for (int k = max(0, it - NS); k < it; k++)
            if (k != dropped && !mbar_wait(&full[k % NS], (unsigned)(k / NS) & 1u)) *(volatile int*)fault = 4;
        return;
    }
    const int lane = l32 & (S - 1), wsub = l32 / S;
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
        const int st = it % NS;
        const int t0 = t * R, nr = min(R, n - t0);
        // this sub-warp's row: its epilogue operands are requested before the wait for the stage
        // and used only after the row's gathers, so their latency overlaps the wait and the gathers
        const int i1 = warp * SPW + wsub;
        AT p1 = 0, p2 = 0, p3 = 0;
        if (i1 < nr && lane == 0) row_operands<OP>(t0 + i1, x, f, M, y, beta, p1, p2, p3);
        // every lane waits (each needs the barrier's acquire for its reads of the stage), and the
        // warp gives up only as a whole
        if (!__all_sync(0xffffffffu, mbar_wait(&full[st], (unsigned)(it / NS) & 1u, wait_ns))) {
            if (l32 == 0) *(volatile int*)fault = 2;
            break;
        }
        const unsigned char* base = stage_smem + st * C::STAGE;
        const int a0 = meta[st][0];
        const bool fits = meta[st][1] != 0;
        const int* rp = (const int*)base;
        const IT* cs = (const IT*)(base + C::COLS) - a0;
        const VT* vs = (const VT*)(base + C::VALS) - a0;
        const unsigned char* vc = (const unsigned char*)(base + C::VALS) - a0;   // codes (coded values)
        // partial sum of row i of the tile over this lane's entries (reads the stage)
        auto row_sum = [&](int i) {
            AT s = 0;
            if (i < nr) {
                const int r = t0 + i;
                const int b = rp[i], e = rp[i + 1];
                if (fits) {
                    for (int j0 = b + lane; j0 < e; j0 += K * S) {
                        int c[K];
                        VT v[K];
                        XT xv[K];
#pragma unroll
                        for (int k = 0; k < K; k++) {
                            const int j = j0 + k * S;
                            c[k] = j < e ? col_of(cs[j], r) : -1;
                            if constexpr (C::kCoded) v[k] = j < e ? tab_s[vc[j]] : VT(0);
                            else v[k] = j < e ? vs[j] : VT(0);
                        }
#pragma unroll
                        for (int k = 0; k < K; k++) xv[k] = c[k] >= 0 ? ld_ro(x + c[k]) : XT(0);
#pragma unroll
                        for (int k = 0; k < K; k++) s += (AT)v[k] * (AT)xv[k];
                    }
                } else {
                    s = row_partial<S, AT>(b, e, lane, r, col, val, x);
                }
            }
            return s;
        };
        // sub-warp reduction and the row's result (all lanes of the warp together, for the shuffles)
        auto row_store = [&](int i, AT s, AT o1, AT o2, AT o3) {
            s = subwarp_sum<S>(s);
            if (i < nr && lane == 0) {
                const int r = t0 + i;
                if (OP == OP_AXPBY) {
                    AT o = (AT)alpha * s;
                    if (beta != 0.0) o += (AT)beta * o1;
                    y[r] = (YT)o;
                } else if (OP == OP_RESID) {
                    y[r] = (YT)(o1 - s);
                } else {
                    y[r] = (YT)(((-s + o1) / o2) + o3);
                }
            }
        };
        const AT s1 = row_sum(i1);
        // the stage is released as soon as the warp has read its entries
        __syncwarp();
        if (l32 == 0) mbar_arrive(&empty[st]);
        row_store(i1, s1, p1, p2, p3);
    }
}

}  // namespace bcmgx
