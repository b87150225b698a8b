// blockops.cuh -- kernels on blocks of K <= 32 vectors (many right-hand sides of one system).
//
// A block is stored row-major with leading dimension ld >= K: entry (i, k) at i*ld + k. Inside
// the multi-right-hand-side solve ld = KP, the next power of two >= K, and the padding columns
// are zero.
//
// CSR products (SpMM): one warp per row. The warp is split into slots of LPE lanes; each lane of
// a slot owns W consecutive columns (one 8- or 16-byte vector load per neighbour), so one warp
// instruction gathers EPI = 32 / LPE matrix entries at once: the per-entry index, value and
// address arithmetic is shared by W columns and the instruction count per row drops by W x EPI
// / 32 against a lane-per-column layout. The slots' partial sums meet in a butterfly, then the
// result is redistributed so that lane k holds column k (coalesced stores, per-column dots).
// Matrix entries are streamed with evict-first loads and the gathers go through L1 / L2, where
// neighbouring rows reuse them.
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

// Entries per batch and slot: enough independent gathers in flight per lane.
template <int W> struct BlkUnroll { static constexpr int U = 4; };
template <> struct BlkUnroll<2> { static constexpr int U = 2; };

// sum over the entries of row [b, e) of a_ij * X[j*ld + k], returned in lane k (k < K); lanes of
// column group g load columns [g*W, g*W + W) when g*W < K. Entries of a slot are summed in
// order, slots are combined by a butterfly. The warp stays converged (the row is warp-uniform).
template <int W, typename AT, typename VT, typename XT>
__device__ __forceinline__ AT blk_row(int b, int e, int lane, int lpe_log2, int ld, int K, const int* __restrict__ col,
    const VT* __restrict__ val, const XT* __restrict__ X)
{
    constexpr int U = BlkUnroll<W>::U;
    const int lpe = 1 << lpe_log2;
    const int epi = 32 >> lpe_log2;
    const int slot = lane >> lpe_log2;
    const int c0 = (lane & (lpe - 1)) * W;
    const bool on = c0 < K;
    AT s[W];
#pragma unroll
    for (int w = 0; w < W; w++) s[w] = 0;
    for (int j0 = b + slot; j0 - slot < e; j0 += epi * U) {
        int c[U];
        VT v[U];
        XT x[U][W];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const int j = j0 + k * epi;
            c[k] = j < e ? ld_stream(col + j) : -1;
            v[k] = j < e ? ld_stream(val + j) : VT(0);
        }
#pragma unroll
        for (int k = 0; k < U; k++) {
            if (c[k] >= 0 && on) {
                ldv<W>(X + (long)c[k] * ld + c0, x[k]);
            } else {
#pragma unroll
                for (int w = 0; w < W; w++) x[k][w] = XT(0);
            }
        }
#pragma unroll
        for (int k = 0; k < U; k++)
#pragma unroll
            for (int w = 0; w < W; w++) s[w] += (AT)v[k] * (AT)x[k][w];
    }
    for (int o = lpe; o < 32; o <<= 1)
#pragma unroll
        for (int w = 0; w < W; w++) s[w] += __shfl_xor_sync(0xffffffffu, s[w], o);
    // column `lane` sits in element lane % W of group lane / W
    AT out = 0;
#pragma unroll
    for (int w = 0; w < W; w++) {
        const AT t = __shfl_sync(0xffffffffu, s[w], (lane / W) & 31);
        if (lane % W == w) out = t;
    }
    return out;
}

// Row loop of the SpMM kernels: warp w of the grid takes rows w, w + warps, ...
#define BCMGX_BLOCK_ROWS(r, n)                                                                  \
    for (long r = ((long)blockIdx.x * blockDim.x + threadIdx.x) / 32; r < (n);                  \
         r += (long)gridDim.x * blockDim.x / 32)

// Element loop of the element-wise kernels over n rows of a block with 2^lk columns.
#define BCMGX_BLOCK_ELEMS(i, n, lk)                                                             \
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < ((long)(n) << (lk));          \
         i += (long)gridDim.x * blockDim.x)

// Y = alpha A X + beta Y (OP 0), Y = F - A X (OP 1), or one l1-Jacobi sweep
// Y = ((F - A X) / M) + X (OP 2), the same updates as k_rowop, column by column.
template <int OP, int W, typename VT, typename XT, typename FT, typename MT, typename YT>
__global__ void __launch_bounds__(256) k_blk_rowop(int n, int lpe_log2, int ld, int K, const int* __restrict__ row,
    const int* __restrict__ col, const VT* __restrict__ val, const XT* __restrict__ X, const FT* __restrict__ F,
    const MT* __restrict__ M, YT* __restrict__ Y, double alpha, double beta, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    using AT = typename Acc<VT>::type;
    const int lane = threadIdx.x & 31;
    BCMGX_BLOCK_ROWS(r, n)
    {
        const AT s = blk_row<W, AT>(__ldg(row + r), __ldg(row + r + 1), lane, lpe_log2, ld, K, col, val, X);
        if (lane < K) {
            const long o = r * ld + lane;
            if (OP == 0) {
                AT y = (AT)alpha * s;
                if (beta != 0.0) y += (AT)beta * (AT)Y[o];
                Y[o] = (YT)y;
            } else if (OP == 1) {
                Y[o] = (YT)((AT)F[o] - s);
            } else {
                Y[o] = (YT)(((-s + (AT)F[o]) / (AT)M[r]) + (AT)X[o]);
            }
        }
    }
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
