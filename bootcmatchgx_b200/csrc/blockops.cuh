// blockops.cuh -- kernels on blocks of K <= 32 vectors (many right-hand sides of one system).
//
// A block is stored row-major with leading dimension ld >= K: entry (i, k) at i*ld + k. Inside
// the multi-right-hand-side solve ld = KP, the next power of two >= K, and the padding columns
// are zero.
//
// CSR products (SpMM): a warp is split into slots of LPE lanes and each slot owns one row, so a
// warp works on 32 / LPE consecutive rows at once. Each lane of a slot owns W consecutive columns
// (one 8- or 16-byte vector load per neighbour: W = 2 for FP64, 4 for FP32 blocks), so the
// per-entry index, value and address arithmetic is shared by W columns and no cross-lane
// reduction is needed; a lane stores its W results as one vector. A warp stages the matrix
// entries of its rows in shared memory with coalesced evict-first loads (blk_rows), and the
// gathers go through L1 / L2, where neighbouring rows reuse them.
#pragma once

#include "common.cuh"

namespace bcmgx {

constexpr int kMaxRhs = 32;

// W consecutive elements as one vector load (16-byte aligned when W * sizeof(T) == 16)
template <int W, typename T>
__device__ __forceinline__ void ldv(const T* p, T (&o)[W]);
template <>
__device__ __forceinline__ void ldv<1, double>(const double* p, double (&o)[1]) { o[0] = __ldg(p); }
template <>
__device__ __forceinline__ void ldv<2, double>(const double* p, double (&o)[2])
{
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    o[0] = v.x;
    o[1] = v.y;
}
template <>
__device__ __forceinline__ void ldv<1, float>(const float* p, float (&o)[1]) { o[0] = __ldg(p); }
template <>
__device__ __forceinline__ void ldv<2, float>(const float* p, float (&o)[2])
{
    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
    o[0] = v.x;
    o[1] = v.y;
}
template <>
__device__ __forceinline__ void ldv<4, float>(const float* p, float (&o)[4])
{
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
}

// W consecutive elements as one vector store (same alignment rule as ldv)
template <int W, typename T>
__device__ __forceinline__ void stv(T* p, const T (&v)[W])
{
    if constexpr (W == 4 && sizeof(T) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else if constexpr (W == 2 && sizeof(T) == 4) {
        *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    } else if constexpr (W == 2 && sizeof(T) == 8) {
        *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
    } else if constexpr (W == 4 && sizeof(T) == 8) {
        reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
    } else {
#pragma unroll
        for (int w = 0; w < W; w++) p[w] = v[w];
    }
}

// W elements of any type (vector loads where ldv has them, else element by element)
template <int W, typename T>
__device__ __forceinline__ void ldw(const T* p, T (&o)[W])
{
    if constexpr ((sizeof(T) == 4 && (W == 1 || W == 2 || W == 4)) || (sizeof(T) == 8 && (W == 1 || W == 2))) {
        ldv<W>(p, o);
    } else if constexpr (sizeof(T) == 8 && W == 4) {
        double a[2], b[2];
        ldv<2>(p, a);
        ldv<2>(p + 2, b);
        o[0] = a[0];
        o[1] = a[1];
        o[2] = b[0];
        o[3] = b[1];
    } else {
#pragma unroll
        for (int w = 0; w < W; w++) o[w] = p[w];
    }
}

// Lanes per slot and columns per lane for K columns gathered from elements of `bytes` bytes:
// power-of-two K uses vector loads (W = min(K, 16 / bytes)); any other K one column per lane.
struct BlkShape {
    int W, lpe_log2;
};
inline BlkShape blk_shape(int K, int bytes)
{
    int kp = 1;
    while (kp < K) kp <<= 1;
    int W = 1;
    if (kp == K) W = K < 16 / bytes ? K : 16 / bytes;
    int lpe = kp / W, lg = 0;
    while ((1 << lg) < lpe) lg++;
    return BlkShape { W, lg };
}

// Element loop of the element-wise kernels over n rows of a block with 2^lk columns.
#define BCMGX_BLOCK_ELEMS(i, n, lk)                                                             \
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < ((long)(n) << (lk));          \
         i += (long)gridDim.x * blockDim.x)

// Matrix entries of one warp step staged in shared memory: the column as an element offset
// into the block (col * ld, so the gather address is one multiply-add) and the value.
template <typename VT>
struct BlkEnt;
template <>
struct BlkEnt<float> {
    int off;
    float v;
};
template <>
struct __align__(16) BlkEnt<double> {
    double v;
    int off;
    int pad;
};

// Rows a warp stages per step (at least one row group) and the staging capacity per warp:
// 32 entries per row on average; a step over longer rows reads its entries from global memory.
template <typename VT>
struct BlkStage {
    static constexpr int rows = sizeof(VT) == 4 ? 8 : 4;
    static constexpr int cap = 32 * rows;
};
// resident blocks per SM the kernel is compiled for: 5 (48 registers) for four columns per
// lane, else 6 (40 registers)
template <typename VT, int W>
constexpr int blk_min_blocks() { return W == 4 ? 5 : 6; }
constexpr int kBlkRowopThreads = 256;

// acc[w] = sum over staged entries [b, e) of v * Xc[off + w], entries in order; U entries per
// batch without predicates (all loads of the batch issue before its multiply-adds), then the
// remainder one entry at a time.
// Entries per batch: 3 keeps the batch's loads in registers at the 40-48 register budget (4
// spills; on 32-column blocks of the 27-point 100^3 matrix, 3 was 4-8 % faster than 4 and 2)
#ifndef BCMGX_BLK_BATCH
#define BCMGX_BLK_BATCH 3
#endif
template <int W, typename AT, typename VT, typename XT>
__device__ __forceinline__ void blk_row_staged(int b, int e, const BlkEnt<VT>* s, const XT* __restrict__ Xc, AT (&acc)[W])
{
    constexpr int U = BCMGX_BLK_BATCH;
#pragma unroll
    for (int w = 0; w < W; w++) acc[w] = 0;
    int j = b;
    for (; j + U <= e; j += U) {
        BlkEnt<VT> q[U];
        XT x[U][W];
#pragma unroll
        for (int k = 0; k < U; k++) q[k] = s[j + k];
#pragma unroll
        for (int k = 0; k < U; k++) ldv<W>(Xc + q[k].off, x[k]);
#pragma unroll
        for (int k = 0; k < U; k++)
#pragma unroll
            for (int w = 0; w < W; w++) acc[w] += (AT)q[k].v * (AT)x[k][w];
    }
    for (; j < e; j++) {
        const BlkEnt<VT> q = s[j];
        XT x[W];
        ldv<W>(Xc + q.off, x);
#pragma unroll
        for (int w = 0; w < W; w++) acc[w] += (AT)q.v * (AT)x[w];
    }
}

// The row loop of the block SpMM kernels. Each warp takes steps of rw consecutive rows (whole
// row groups of 32 / LPE rows, at least BlkStage::rows): lanes 0..rw-1 load the row offsets,
// the warp copies the step's entries into its shared-memory stage `st` (BlkStage::cap entries)
// with coalesced loads, and then each slot reads its row's entries from there as broadcasts.
// Per entry a slot issues one shared load, one address multiply-add, one vector gather and W
// multiply-adds; per-lane index and value loads from global memory hit a different cache line
// for every slot and cost more L1 throughput than the gathers. A step whose entries do not fit
// (or stage_ok = 0: X has 2^31 or more elements, past the 32-bit staged offsets) reads them from
// global memory. For every row r this lane computes, epi(r, o, s) receives o = r * ld + c0 and
// the sums s[w] of column c0 + w, entries added in row order. All lanes of a warp run the loop
// (it has warp-synchronous steps); lanes without a column (c0 >= K) skip the epilogue.
template <int W, typename VT, typename XT, typename Epi>
__device__ __forceinline__ void blk_rows(int n, int lpe_log2, int ld, int K, const int* __restrict__ row,
    const int* __restrict__ col, const VT* __restrict__ val, const XT* __restrict__ X, int stage_ok, BlkEnt<VT>* st,
    Epi&& epi)
{
    using AT = typename Acc<VT>::type;
    using ST = BlkStage<VT>;
    const int warps = blockDim.x >> 5;
    const int lane = threadIdx.x & 31;
    const int slot = lane >> lpe_log2;
    const int c0 = (lane & ((1 << lpe_log2) - 1)) * W;
    const int rpg = 32 >> lpe_log2;
    const int rw = rpg > ST::rows ? rpg : ST::rows;
    const bool active = c0 < K;
    const XT* Xc = X + c0;
    const long wstride = (long)gridDim.x * warps * rw;
    for (long w0 = ((long)blockIdx.x * warps + (threadIdx.x >> 5)) * rw; w0 < n; w0 += wstride) {
        const int nr = (int)(w0 + rw < n ? rw : n - w0);
        const int rp = lane < nr ? __ldg(row + w0 + lane) : 0;
        const int e0 = __ldg(row + w0 + nr);
        const int b0 = __shfl_sync(0xffffffffu, rp, 0);
        const bool staged = stage_ok && e0 - b0 <= ST::cap;
        if (staged) {
            for (int t = lane; t < e0 - b0; t += 32) {
                BlkEnt<VT> q;
                q.v = ld_stream(val + b0 + t);
                q.off = ld_stream(col + b0 + t) * ld;
                st[t] = q;
            }
        }
        __syncwarp();
        for (int g = 0; g < rw; g += rpg) {
            const int lr = g + slot;
            const int rb = __shfl_sync(0xffffffffu, rp, lr & 31);
            const int rn = __shfl_sync(0xffffffffu, rp, (lr + 1) & 31);
            if (lr >= nr || !active) continue;
            const int re = lr + 1 < nr ? rn : e0;
            AT s[W];
            if (staged) {
                blk_row_staged<W>(rb - b0, re - b0, st, Xc, s);
            } else {
#pragma unroll
                for (int w = 0; w < W; w++) s[w] = 0;
                for (int j = rb; j < re; j++) {
                    const AT v = (AT)ld_stream(val + j);
                    XT x[W];
                    ldv<W>(Xc + (long)ld_stream(col + j) * ld, x);
#pragma unroll
                    for (int w = 0; w < W; w++) s[w] += v * (AT)x[w];
                }
            }
            const long r = w0 + lr;
            epi(r, r * ld + c0, s);
        }
        __syncwarp();
    }
}

// rows one block of a blk_rows kernel covers per step, for the grid size
template <typename VT>
inline long blk_rows_per_block(int lpe_log2, int threads)
{
    const int rpg = 32 >> lpe_log2;
    return (long)(threads / 32) * (rpg > BlkStage<VT>::rows ? rpg : BlkStage<VT>::rows);
}

// Y = alpha A X + beta Y (OP 0), Y = F - A X (OP 1), or one l1-Jacobi sweep
// Y = ((F - A X) / M) + X (OP 2), the same updates as k_rowop, column by column. With W > 1,
// ld is a multiple of W, K = LPE * W and all blocks are 16-byte aligned.
template <int OP, int W, typename VT, typename XT, typename FT, typename MT, typename YT>
__global__ void __launch_bounds__(kBlkRowopThreads, blk_min_blocks<VT, W>()) k_blk_rowop(int n, int lpe_log2, int ld,
    int K, const int* __restrict__ row, const int* __restrict__ col, const VT* __restrict__ val,
    const XT* __restrict__ X, const FT* __restrict__ F, const MT* __restrict__ M, YT* __restrict__ Y, double alpha,
    double beta, int stage_ok, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    using AT = typename Acc<VT>::type;
    __shared__ BlkEnt<VT> stage[kBlkRowopThreads / 32][BlkStage<VT>::cap];
    blk_rows<W>(n, lpe_log2, ld, K, row, col, val, X, stage_ok, stage[threadIdx.x >> 5],
        [&](long r, long o, const AT (&s)[W]) {
            YT y[W];
            if (OP == 0) {
                YT y0[W];
                if (beta != 0.0) ldw<W>(Y + o, y0);
#pragma unroll
                for (int w = 0; w < W; w++) {
                    AT t = (AT)alpha * s[w];
                    if (beta != 0.0) t += (AT)beta * (AT)y0[w];
                    y[w] = (YT)t;
                }
            } else if (OP == 1) {
                FT f[W];
                ldw<W>(F + o, f);
#pragma unroll
                for (int w = 0; w < W; w++) y[w] = (YT)((AT)f[w] - s[w]);
            } else {
                FT f[W];
                XT x[W];
                ldw<W>(F + o, f);
                ldw<W>(X + o, x);
                const AT m = (AT)M[r];
#pragma unroll
                for (int w = 0; w < W; w++) y[w] = (YT)(((-s[w] + (AT)f[w]) / m) + (AT)x[w]);
            }
            stv<W>(Y + o, y);
        });
}

// sweep from a zero iterate: U = F / M, optionally keeping a converted copy of F
template <typename FT, typename MT, typename YT, typename CT>
__global__ void k_blk_first_sweep(int n, int lk, const FT* __restrict__ F, const MT* __restrict__ M, YT* __restrict__ U,
    CT* __restrict__ Fcopy, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    using AT = typename Wider<MT>::type;
    BCMGX_BLOCK_ELEMS(i, n, lk)
    {
        const AT f = (AT)F[i];
        if (Fcopy) Fcopy[i] = (CT)f;
        U[i] = (YT)(f / (AT)M[i >> lk]);
    }
}

template <typename ST, typename DT>
__global__ void k_blk_convert(int n, int lk, const ST* __restrict__ a, DT* __restrict__ b, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    BCMGX_BLOCK_ELEMS(i, n, lk) b[i] = (DT)a[i];
}

template <typename T>
__global__ void k_blk_zero(int n, int lk, T* __restrict__ a, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    BCMGX_BLOCK_ELEMS(i, n, lk) a[i] = T(0);
}

// Y = p .* XC[agg] + X row by row (P has one entry per row; Y may alias X)
template <typename PT, typename CT, typename XT, typename YT>
__global__ void k_blk_prolong(int n, int lk, const int* __restrict__ agg, const PT* __restrict__ p, const CT* __restrict__ XC,
    const XT* X, YT* Y, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    using AT = typename Wider<YT>::type;
    const long mask = (1L << lk) - 1;
    BCMGX_BLOCK_ELEMS(i, n, lk)
    {
        const long r = i >> lk;
        Y[i] = (YT)((AT)p[r] * (AT)XC[((long)agg[r] << lk) + (i & mask)] + (AT)X[i]);
    }
}

}  // namespace bcmgx
