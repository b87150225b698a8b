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
template <int S, typename AT, bool RO = true, typename VS, typename XT, typename IT>
__device__ __forceinline__ AT row_partial(int b, int e, int lane, int r, const IT* __restrict__ col, VS val,
    const XT* x)
{
    using VT = typename ValSrc<VS>::type;
    constexpr int K = 8;
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

// y = alpha*A*x + beta*y (OP_AXPBY), y = f - A*x (OP_RESID) or one l1-Jacobi sweep
// y = ((f - A*x) / M) + x (OP_JACOBI, the update of _jacobi_it_full<0>, l1jacobi.cu:345-379).
// Grid-stride over rows; all lanes of a sub-warp stay converged for the shuffles. VS: the values
// (ValSrc: stored or coded).
template <int S, int OP, typename VS, typename XT, typename FT, typename MT, typename YT, typename IT>
__global__ void __launch_bounds__(256) k_rowop(int n, const int* __restrict__ row, const IT* __restrict__ col,
    VS val, const XT* __restrict__ x, const FT* __restrict__ f, const MT* __restrict__ M,
    YT* __restrict__ y, double alpha, double beta, const int* __restrict__ skip)
{
    dep_wait();
    dep_release();
    if (skip && *skip) return;
    using VT = typename ValSrc<VS>::type;
    using AT = typename Acc<VT>::type;
    const int lane = threadIdx.x & (S - 1);
    const int sub = (threadIdx.x & 31) / S;
    const long stride = (long)gridDim.x * blockDim.x / S;
    // base is uniform across the warp, so every lane reaches the shuffles together
    for (long base = ((long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / S; base < n; base += stride) {
        const long r0 = base + sub;
        const int r = (int)r0;
        AT s = 0;
        if (r0 < n) s = row_partial<S, AT>(__ldg(row + r), __ldg(row + r + 1), lane, r, col, val, x);
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
