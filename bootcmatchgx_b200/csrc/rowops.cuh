// rowops.cuh -- CSR row kernels of the solve phase: SpMV, residual, l1-Jacobi sweep.
//
// One sub-warp of S lanes owns a row (S = 1..32, chosen per matrix by the autotuner); the lanes
// stride over the row's entries, matrix data is streamed with evict-first loads and the vector
// gathers go through the read-only path, so x stays resident in L2 while A streams from HBM.
#pragma once

#include "common.cuh"

namespace bcmgx {

enum RowOp { OP_AXPBY = 0, OP_RESID = 1, OP_JACOBI = 2 };

// Matrix values as the row kernels read them: stored (a `const T*`, one value per entry), or
// coded (value-indexed CSR, Kourtis, Goumas and Koziris, "Optimizing sparse matrix-vector
// multiplication using index and value compression", CF 2008): one byte per entry indexing a
// table of the matrix's distinct values (at most 256). The table holds the very values the stored
// form holds, so both forms give the same results bit for bit; the coded one streams 1 byte per
// entry instead of 4 or 8.
template <typename T>
struct Coded {
    const unsigned char* code;   // nnz codes
    const T* tab;                // kValueCodes values (unused slots zero)
};
template <typename VS> struct ValSrc;
template <typename T> struct ValSrc<const T*> {
    using type = T;
    static constexpr int bytes = (int)sizeof(T);   // bytes streamed per entry
    static constexpr bool coded = false;
};
template <typename T> struct ValSrc<T*> : ValSrc<const T*> {};
template <typename T> struct ValSrc<Coded<T>> {
    using type = T;
    static constexpr int bytes = 1;
    static constexpr bool coded = true;
};
template <typename T>
__device__ __forceinline__ T val_at(const T* __restrict__ v, int j) { return ld_stream(v + j); }
template <typename T>
__device__ __forceinline__ T val_at(const Coded<T>& v, int j) { return __ldg(v.tab + __ldcs(v.code + j)); }

// Column index of entry j: int32 columns as stored, or int16 offsets from the row (a level whose
// entries all lie within 32767 of the diagonal keeps this compact copy of its columns, which
// cuts the index stream of every row kernel in half).
__device__ __forceinline__ int col_at(const int* __restrict__ col, int j, int) { return ld_stream(col + j); }
__device__ __forceinline__ int col_at(const short* __restrict__ dcol, int j, int r) { return r + (int)__ldcs(dcol + j); }

// Partial dot product of one row over the lanes of a sub-warp. Entries are taken in batches of
// K per lane: all K column and value loads are issued, then all K gathers of x, then the K
// multiply-adds, so a row of up to K*S entries costs one round of memory latency per lane. The
// gathers use the read-only path unless RO is false (x written earlier by the same kernel).
constexpr int kRowBatch = 8;   // entries per lane and batch in row_partial

// one batch of row_partial's loads: the indices and values of entries j0, j0 + S, ... (K of them)
template <int S, typename VS, typename IT, typename VT>
__device__ __forceinline__ void row_batch(int j0, int e, int r, const IT* __restrict__ col, VS val, int (&c)[kRowBatch],
    VT (&v)[kRowBatch])
{
#pragma unroll
    for (int k = 0; k < kRowBatch; k++) {
        const int j = j0 + k * S;
        c[k] = j < e ? col_at(col, j, r) : -1;
        v[k] = j < e ? val_at(val, j) : VT(0);
    }
}

template <int S, typename AT, bool RO = true, typename VS, typename XT, typename IT>
__device__ __forceinline__ AT row_partial(int b, int e, int lane, int r, const IT* __restrict__ col, VS val,
    const XT* x)
{
    using VT = typename ValSrc<VS>::type;
    constexpr int K = kRowBatch;
    AT s = 0;
    for (int j0 = b + lane; j0 < e; j0 += K * S) {
        int c[K];
        VT v[K];
        XT xv[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int j = j0 + k * S;
            c[k] = j < e ? col_at(col, j, r) : -1;
            v[k] = j < e ? val_at(val, j) : VT(0);
        }
#pragma unroll
        for (int k = 0; k < K; k++) xv[k] = c[k] >= 0 ? (RO ? ld_ro(x + c[k]) : x[c[k]]) : XT(0);
#pragma unroll
        for (int k = 0; k < K; k++) s += (AT)v[k] * (AT)xv[k];
    }
    return s;
}

// row_partial whose first batch (c0, v0, for entries b + lane, b + lane + S, ...) was loaded
// already: the same batches, gathers and order
template <int S, typename AT, typename VS, typename XT, typename IT, typename VT>
__device__ __forceinline__ AT row_partial_from(int b, int e, int lane, const XT* x, const int (&c0)[kRowBatch],
    const VT (&v0)[kRowBatch], const IT* __restrict__ col, VS val, int r)
{
    constexpr int K = kRowBatch;
    AT s = 0;
    int j0 = b + lane;
    if (j0 < e) {
        XT xv[K];
#pragma unroll
        for (int k = 0; k < K; k++) xv[k] = c0[k] >= 0 ? ld_ro(x + c0[k]) : XT(0);
#pragma unroll
        for (int k = 0; k < K; k++) s += (AT)v0[k] * (AT)xv[k];
    }
    for (j0 += K * S; j0 < e; j0 += K * S) {
        int c[K];
        VT v[K];
        XT xv[K];
        row_batch<S>(j0, e, r, col, val, c, v);
#pragma unroll
        for (int k = 0; k < K; k++) xv[k] = c[k] >= 0 ? ld_ro(x + c[k]) : XT(0);
#pragma unroll
        for (int k = 0; k < K; k++) s += (AT)v[k] * (AT)xv[k];
    }
    return s;
}

// y = alpha*A*x + beta*y (OP_AXPBY), y = f - A*x (OP_RESID) or one l1-Jacobi sweep
// y = ((f - A*x) / M) + x (OP_JACOBI, the update of _jacobi_it_full<0>, l1jacobi.cu:345-379).
// Grid-stride over rows; all lanes of a sub-warp stay converged for the shuffles. VS: the values
// (ValSrc: stored or coded).
// pre: the matrix was complete before the launch (no kernel still running may write it), so each
// thread's first row bounds and first batch of indices and values are read before the dependency
// wait, overlapping the previous kernel's tail; the sums are row_partial's.
template <int S, int OP, typename VS, typename XT, typename FT, typename MT, typename YT, typename IT>
__global__ void __launch_bounds__(256) k_rowop(int n, const int* __restrict__ row, const IT* __restrict__ col,
    VS val, const XT* __restrict__ x, const FT* __restrict__ f, const MT* __restrict__ M,
    YT* __restrict__ y, double alpha, double beta, const int* __restrict__ skip, int pre)
{
    using VT = typename ValSrc<VS>::type;
    using AT = typename Acc<VT>::type;
    constexpr int K = kRowBatch;
    const int lane = threadIdx.x & (S - 1);
    const int sub = (threadIdx.x & 31) / S;
    const long stride = (long)gridDim.x * blockDim.x / S;
    const long base0 = ((long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / S;
    int pb = 0, pe = 0;
    int pc[K];
    VT pv[K];
    const bool have = pre && base0 + sub < n;
    if (have) {
        const int r = (int)(base0 + sub);
        pb = __ldg(row + r);
        pe = __ldg(row + r + 1);
        row_batch<S>(pb + lane, pe, r, col, val, pc, pv);
    }
    dep_wait();
    dep_release();
    if (skip && *skip) return;
    // base is uniform across the warp, so every lane reaches the shuffles together
    for (long base = base0; base < n; base += stride) {
        const long r0 = base + sub;
        const int r = (int)r0;
        AT s = 0;
        if (r0 < n) {
            if (have && base == base0) s = row_partial_from<S, AT>(pb, pe, lane, x, pc, pv, col, val, r);
            else s = row_partial<S, AT>(__ldg(row + r), __ldg(row + r + 1), lane, r, col, val, x);
        }
        s = subwarp_sum<S>(s);
        if (r0 < n && lane == 0) {
            if (OP == OP_AXPBY) {
                AT o = (AT)alpha * s;
                if (beta != 0.0) o += (AT)beta * (AT)y[r];
                y[r] = (YT)o;
            } else if (OP == OP_RESID) {
                y[r] = (YT)((AT)f[r] - s);
            } else {
                y[r] = (YT)(((-s + (AT)f[r]) / (AT)M[r]) + (AT)x[r]);
            }
        }
    }
}

}  // namespace bcmgx
