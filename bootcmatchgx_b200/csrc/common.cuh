// common.cuh -- device helpers shared by the bcmgx kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace bcmgx {

constexpr int kWarp = 32;
// largest value table of a value-indexed (coded) matrix: one-byte codes
constexpr int kValueCodes = 256;

// Streaming loads for matrix data (read once per pass; evict-first so the vectors stay in L2).
__device__ __forceinline__ int ld_stream(const int* p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
// Vector gathers through the read-only path.
template <typename T>
__device__ __forceinline__ T ld_ro(const T* p) { return __ldg(p); }

// Programmatic dependent launch (launch_dep): dep_wait() returns once the kernel before this one in
// the stream has completed and its writes are visible (at once for an ordinary launch);
// dep_release() lets the next kernel of the stream be scheduled while this one runs. A kernel that
// launch_dep launches calls dep_wait() before it touches a vector an earlier kernel writes and
// before it returns, so that its own completion implies its predecessors'.
__device__ __forceinline__ void dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void dep_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Loads / stores that bypass L1 (values written by other SMs during the same kernel).
__device__ __forceinline__ int ld_cg(const int* p) { return __ldcg(p); }
__device__ __forceinline__ unsigned ld_cg(const unsigned* p) { return __ldcg(p); }
__device__ __forceinline__ void st_cg(int* p, int v) { __stcg(p, v); }

template <typename T> struct Acc { using type = T; };
template <> struct Acc<double> { using type = double; };
template <> struct Acc<float> { using type = float; };
// arithmetic type of an element-wise step that writes T: float only for float results
template <typename T> struct Wider { using type = double; };
template <> struct Wider<float> { using type = float; };

// a * b + c with one rounding (an explicit fused multiply-add, so that kernels which must agree
// bit for bit do not depend on the compiler's contraction choices)
__device__ __forceinline__ double mad_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mad_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

template <int S, typename T>
__device__ __forceinline__ T subwarp_sum(T v)
{
#pragma unroll
    for (int o = S / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, S);
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum of K per-thread values over the block; valid in thread 0. blockDim.x <= 1024.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K])
{
    __shared__ double sh[K][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; k++) sh[k][wid] = v[k];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            double t = lane < nw ? sh[k][lane] : 0.0;
            v[k] = warp_sum(t);
        }
    }
    __syncthreads();
}

// Deterministic two-stage grid reduction: every block stores its K partial sums, the last block
// to finish (ticket) adds all partials in block order and returns true in all of its threads
// with the totals in out[] (valid in thread 0). The ticket is reset for the next use.
template <int K>
__device__ __forceinline__ bool grid_sum(double (&v)[K], double* partials, int* ticket, double (&out)[K])
{
    block_sum<K>(v);
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) partials[(size_t)blockIdx.x * K + k] = v[k];
        __threadfence();
        int t = atomicAdd(ticket, 1);
        last = (t == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] += __ldcg(partials + (size_t)b * K + k);
    block_sum<K>(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) out[k] = acc[k];
        *ticket = 0;
    }
    return true;
}

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace bcmgx
