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
// reduction is needed; a lane stores its W results as one vector. Matrix entries are streamed
// with evict-first loads (broadcast within a slot) and the gathers go through L1 / L2, where
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

// s[w] = sum over the entries of row [b, e) of a_ij * X[j*ld + c0 + w] (w < W), entries in
// order, U entries per batch: all index / value loads, then all gathers, then the FMAs.
template <int W, typename AT, typename VT, typename XT>
__device__ __forceinline__ void blk_row(int b, int e, int c0, int ld, const int* __restrict__ col,
    const VT* __restrict__ val, const XT* __restrict__ X, AT (&s)[W])
{
    constexpr int U = 4;
#pragma unroll
    for (int w = 0; w < W; w++) s[w] = 0;
    for (int j0 = b; j0 < e; j0 += U) {
        int c[U];
        VT v[U];
        XT x[U][W];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const int j = j0 + k;
            c[k] = j < e ? ld_stream(col + j) : -1;
            v[k] = j < e ? ld_stream(val + j) : VT(0);
        }
#pragma unroll
        for (int k = 0; k < U; k++) {
            if (c[k] >= 0) {
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
}

// Row loop of the SpMM kernels: warp w of the grid takes the row group starting at w * rpw
// (rpw = 32 / LPE rows), then every warps * rpw rows; slot s of the warp owns row r0 + s.
#define BCMGX_BLOCK_ROWGROUPS(r0, n, rpw)                                                         \
    for (long r0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) / 32 * (rpw); r0 < (n);          \
         r0 += (long)gridDim.x * blockDim.x / 32 * (rpw))

// Element loop of the element-wise kernels over n rows of a block with 2^lk columns.
#define BCMGX_BLOCK_ELEMS(i, n, lk)                                                             \
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < ((long)(n) << (lk));          \
         i += (long)gridDim.x * blockDim.x)

// Y = alpha A X + beta Y (OP 0), Y = F - A X (OP 1), or one l1-Jacobi sweep
// Y = ((F - A X) / M) + X (OP 2), the same updates as k_rowop, column by column. With W > 1,
// ld is a multiple of W, K = LPE * W and all blocks are 16-byte aligned.
template <int OP, int W, typename VT, typename XT, typename FT, typename MT, typename YT>
__global__ void __launch_bounds__(256) k_blk_rowop(int n, int lpe_log2, int ld, int K, const int* __restrict__ row,
    const int* __restrict__ col, const VT* __restrict__ val, const XT* __restrict__ X, const FT* __restrict__ F,
    const MT* __restrict__ M, YT* __restrict__ Y, double alpha, double beta, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    using AT = typename Acc<VT>::type;
    const int lane = threadIdx.x & 31;
    const int slot = lane >> lpe_log2;
    const int c0 = (lane & ((1 << lpe_log2) - 1)) * W;
    if (c0 >= K) return;   // one-column-per-lane shapes: lanes past the last column
    BCMGX_BLOCK_ROWGROUPS(r0, n, 32 >> lpe_log2)
    {
        const long r = r0 + slot;
        if (r >= n) continue;
        AT s[W];
        blk_row<W>(__ldg(row + r), __ldg(row + r + 1), c0, ld, col, val, X, s);
        const long o = r * ld + c0;
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
