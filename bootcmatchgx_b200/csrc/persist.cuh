// persist.cuh -- the coarse part of a V-cycle as one persistent kernel.
//
// Below some size every level of the cycle is bound by kernel-launch latency, not by memory: a
// sweep of a 100k-entry level takes a microsecond of work and several of launch. The steps that
// the multi-launch cycle would run on those levels (the same steps, in the same order, recorded
// from Cycle::run) form a program of PStep records; one cooperative kernel runs them all, with a
// grid-wide barrier between consecutive steps. Each step's arithmetic is that of the kernel it
// stands for (k_rowop<S>, k_first_sweep, k_convert, k_zero, k_restrict, k_prolong: the same types,
// operations and summation order), so the results equal the multi-launch cycle's bit for bit.
// Vectors written by the program are read back with L1-bypassing loads (.cg): other SMs wrote
// them. Every barrier wait is bounded (about one second on %globaltimer): a block that gives up
// stores code 8 in the fault word and marks the program's barrier state as poisoned, after which
// the remaining steps and launches of the solve return at once; the entry point then reports
// BCMGX_ERR_TIMEOUT.
#pragma once

#include "rowops.cuh"

namespace bcmgx {

enum PersistOp { P_JACOBI = 0, P_RESID = 1, P_FIRST = 2, P_CONVERT = 3, P_ZERO = 4, P_RESTRICT = 5, P_PROLONG = 6 };

// One step of a program. Types: 0 = FP64, 1 = FP32 (of the matrix values, of each vector).
struct PStep {
    int op, n, S;                       // operation, rows / elements, lanes per row (row steps)
    int vt, coded, col16;               // matrix value type, one-byte value codes, int16 column offsets
    int xt, ft, mt, yt, ct;             // types of x, f (or the restricted / prolonged source), M, y, the extra vector
    const int* row;
    const void* col;
    const void* val;                    // stored values, or the value table when coded
    const unsigned char* code;
    const void* x;                      // row steps: x; convert: source; prolong: the fine iterate
    const void* f;                      // row / first steps: right-hand side; restrict: residual
    const void* M;                      // divisor; restrict: R's values; prolong: P's values
    void* y;                            // output
    void* extra;                        // first: the converted copy of f (or null)
    const int* idx;                     // restrict: R's row offsets; prolong: the aggregates
    const int* idx2;                    // restrict: R's column indices
    const void* xc;                     // prolong: the coarse correction
    // argument slots: 0 = the pointer above; 1, 2, 3 = the launch's f, x0, dst vectors (a program
    // of the whole cycle takes FCG's vectors, which change between iterations)
    unsigned char sx, sf, sy, se, sc;
};

constexpr int kPersistThreads = 512;
constexpr unsigned long long kPersistWaitNs = 1000000000ull;

template <typename T>
__device__ __forceinline__ T ldv(const void* p, int t, long i)   // a written vector, converted to T
{
    return t ? (T)__ldcg((const float*)p + i) : (T)__ldcg((const double*)p + i);
}
template <typename T>
__device__ __forceinline__ void stv(void* p, int t, long i, T v)
{
    if (t) ((float*)p)[i] = (float)v;
    else ((double*)p)[i] = (double)v;
}

// The row partial of row_partial<S> (same lane-to-entry mapping, batches and order) with x read
// through L2.
template <int S, typename AT, typename VT, typename XT>
__device__ __forceinline__ AT prow_partial(const PStep& p, int b, int e, int lane, int r)
{
    constexpr int K = 8;
    AT s = 0;
    const XT* x = (const XT*)p.x;
    for (int j0 = b + lane; j0 < e; j0 += K * S) {
        int c[K];
        VT v[K];
        XT xv[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int j = j0 + k * S;
            c[k] = j < e ? (p.col16 ? r + (int)__ldcs((const short*)p.col + j) : __ldcs((const int*)p.col + j)) : -1;
            v[k] = j < e ? (p.coded ? __ldg((const VT*)p.val + __ldcs(p.code + j)) : __ldcs((const VT*)p.val + j)) : VT(0);
        }
#pragma unroll
        for (int k = 0; k < K; k++) xv[k] = c[k] >= 0 ? __ldcg(x + c[k]) : XT(0);
#pragma unroll
        for (int k = 0; k < K; k++) s += (AT)v[k] * (AT)xv[k];
    }
    return s;
}

// a row step with S lanes per row over the whole grid (k_rowop<S>'s row loop)
template <int S, typename VT>
__device__ void prow_step(const PStep& p)
{
    using AT = typename Acc<VT>::type;
    const int lane = threadIdx.x & (S - 1);
    const int sub = (threadIdx.x & 31) / S;
    const long stride = (long)gridDim.x * blockDim.x / S;
    const int n = p.n;
    for (long base = ((long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / S; base < n; base += stride) {
        const long r0 = base + sub;
        const int r = (int)r0;
        AT s = 0;
        if (r0 < n) s = prow_partial<S, AT, VT, VT>(p, __ldg(p.row + r), __ldg(p.row + r + 1), lane, r);
        s = subwarp_sum<S>(s);
        if (r0 < n && lane == 0) {
            if (p.op == P_RESID) {
                stv(p.y, p.yt, r, (AT)(ldv<AT>(p.f, p.ft, r) - s));
            } else {
                const AT fr = ldv<AT>(p.f, p.ft, r);
                const AT Mr = p.mt ? (AT)__ldg((const float*)p.M + r) : (AT)__ldg((const double*)p.M + r);
                const AT xr = ldv<AT>(p.x, p.xt, r);
                stv(p.y, p.yt, r, (AT)(((-s + fr) / Mr) + xr));
            }
        }
    }
}

template <typename VT>
__device__ void prow_dispatch(const PStep& p)
{
    switch (p.S) {
    case 1: prow_step<1, VT>(p); break;
    case 2: prow_step<2, VT>(p); break;
    case 4: prow_step<4, VT>(p); break;
    case 8: prow_step<8, VT>(p); break;
    case 16: prow_step<16, VT>(p); break;
    default: prow_step<32, VT>(p); break;
    }
}

// element-wise steps: the arithmetic type is float only for an FP32 result (Wider), except the
// first sweep, whose type follows M (k_first_sweep)
template <typename AT>
__device__ void pelem_step(const PStep& p)
{
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += stride) {
        if (p.op == P_FIRST) {
            const AT fi = ldv<AT>(p.f, p.ft, i);
            if (p.extra) stv(p.extra, p.ct, i, fi);
            const AT Mi = p.mt ? (AT)__ldg((const float*)p.M + i) : (AT)__ldg((const double*)p.M + i);
            stv(p.y, p.yt, i, (AT)(fi / Mi));
        } else if (p.op == P_CONVERT) {
            if (p.xt) stv(p.y, p.yt, i, __ldcg((const float*)p.x + i));
            else stv(p.y, p.yt, i, __ldcg((const double*)p.x + i));
        } else if (p.op == P_ZERO) {
            stv(p.y, p.yt, i, AT(0));
        } else if (p.op == P_RESTRICT) {
            AT s = 0;
            const int t1 = __ldg(p.idx + i + 1);
            for (int t = __ldg(p.idx + i); t < t1; t++) {
                const int k = __ldg(p.idx2 + t);
                const AT rv = p.mt ? (AT)__ldg((const float*)p.M + t) : (AT)__ldg((const double*)p.M + t);
                s = mad_rn(rv, ldv<AT>(p.f, p.ft, k), s);
            }
            stv(p.y, p.yt, i, s);
        } else {   // P_PROLONG
            const int c = __ldg(p.idx + i);
            const AT pv = p.mt ? (AT)__ldg((const float*)p.M + i) : (AT)__ldg((const double*)p.M + i);
            stv(p.y, p.yt, i, mad_rn(pv, ldv<AT>(p.xc, p.ct, c), ldv<AT>(p.x, p.xt, i)));
        }
    }
}

__device__ __forceinline__ unsigned long long pglobal_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned* p, unsigned v)
{
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier on bar[0] (arrivals) and bar[1] (generation); bar[2] != 0: poisoned by an
// earlier timeout. The block's writes are ordered before its arrival by the block barrier and the
// arrival's release; the waiters' acquire of the new generation orders the next step's loads
// after every block's writes. Returns false after a bounded wait of wait_ns (fault code 8).
__device__ __forceinline__ bool pgrid_sync(unsigned* bar, int* fault, unsigned long long wait_ns)
{
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned g = ld_acquire_gpu(bar + 1);
        if (atom_add_acq_rel_gpu(bar, 1u) == gridDim.x - 1) {
            bar[0] = 0u;
            st_release_gpu(bar + 1, g + 1u);
        } else {
            const unsigned long long t0 = pglobal_ns();
            while (ld_acquire_gpu(bar + 1) == g) {
                if (*(volatile unsigned*)(bar + 2) != 0u || pglobal_ns() - t0 > wait_ns) {
                    ok = 0;
                    *(volatile unsigned*)(bar + 2) = 1u;
                    *(volatile int*)fault = 8;
                    break;
                }
            }
        }
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

__device__ __forceinline__ const void* pslot(const void* p, unsigned char slot, const void* a0, const void* a1,
    const void* a2)
{
    return slot == 0 ? p : slot == 1 ? a0 : slot == 2 ? a1 : a2;
}

// Runs steps[0 .. nsteps) with a barrier between consecutive steps. Launched cooperatively (every
// block resident), kPersistThreads threads per block; skip: the solve has converged. af, ax, ay:
// the vectors of argument slots 1, 2, 3. wait_ns: the barrier's wait limit (kPersistWaitNs in
// production); drop_block0: a fault-path test hook, block 0 leaves before the first barrier so
// that the other blocks' wait there runs out.
__global__ void __launch_bounds__(kPersistThreads) k_persist(const PStep* __restrict__ steps, int nsteps, unsigned* bar,
    int* fault, const int* __restrict__ skip, const void* af, const void* ax, void* ay, unsigned long long wait_ns,
    int drop_block0)
{
    if (skip && *skip) return;
    if (*(volatile unsigned*)(bar + 2) != 0u) return;
    if (drop_block0 && blockIdx.x == 0) return;
    __shared__ PStep ps;
    for (int k = 0; k < nsteps; k++) {
        if (threadIdx.x == 0) {
            PStep q = steps[k];
            q.x = pslot(q.x, q.sx, af, ax, ay);
            q.f = pslot(q.f, q.sf, af, ax, ay);
            q.y = (void*)pslot(q.y, q.sy, af, ax, ay);
            q.extra = (void*)pslot(q.extra, q.se, af, ax, ay);
            q.xc = pslot(q.xc, q.sc, af, ax, ay);
            ps = q;
        }
        __syncthreads();
        const PStep p = ps;
        if (p.op == P_JACOBI || p.op == P_RESID) {
            if (p.vt) prow_dispatch<float>(p);
            else prow_dispatch<double>(p);
        } else if (p.op == P_FIRST) {
            if (p.mt) pelem_step<float>(p);
            else pelem_step<double>(p);
        } else {
            if (p.yt) pelem_step<float>(p);
            else pelem_step<double>(p);
        }
        if (k + 1 < nsteps && !pgrid_sync(bar, fault, wait_ns)) return;
    }
}

}  // namespace bcmgx
