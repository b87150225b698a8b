// sliced.cuh -- row kernels over a sliced copy of a level matrix (sm_100a).
//
// The CSR row kernels (rowops.cuh, staged.cuh) hand each row to a sub-warp whose lanes stride
// over the row: every entry costs a bounds test, a select and scalar loads of its index and value,
// and a level matrix streamed as one-byte value codes and int16 column offsets (3 bytes an entry)
// leaves those kernels bound by instruction issue, not by HBM. The sliced form stores the rows of
// each group of 32 consecutive rows (a slice, one warp) interleaved: the slice's entries are
// blocks of 4 entries per lane, lane l of block q holding entries 4q .. 4q+3 of row 32s + l, so a
// warp loads a block with one coalesced vector load per lane (8 bytes of int16 offsets, 4 bytes
// of codes). A slice is as wide as its longest row, rounded up to whole blocks; the padding
// entries point at the row itself (offset 0, or the row's own column) with value 0, and lanes past
// the last row repeat the last row's padding. One lane owns one row and adds its entries in
// their CSR order with the same multiply-adds as k_rowop<1>, so the sliced kernels' results equal
// k_rowop<1>'s bit for bit (a padding term adds a zero product to a sum that is never -0).
//
// Format (DevCsr): sl_ptr[s] = first entry of slice s (a multiple of 128), sl_ptr[nslices] = the
// total; sl_off (int16 offsets) or sl_col (int32 columns); sl_code (one-byte value codes into the
// level's tables) or sl_val32 / sl_val64 (stored values).
#pragma once

#include "rowops.cuh"

namespace bcmgx {

constexpr int kSliceRows = 32;                       // rows per slice (one warp)
constexpr int kSliceG = 4;                           // entries per lane per block
constexpr int kSliceBlock = kSliceRows * kSliceG;    // entries per block of a slice

// loads from a shared-memory stage by 32-bit shared addresses
__device__ __forceinline__ uint2 lds_v2(unsigned a)
{
    uint2 v;
    asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(a));
    return v;
}
__device__ __forceinline__ unsigned lds_v1(unsigned a)
{
    unsigned v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ uint4 lds_v4(unsigned a)
{
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
    return v;
}

// raw index words of a block (decoded into columns only when the gathers are issued); load:
// from the sliced arrays in global memory (streamed), lds: from a shared-memory stage
template <typename IT> struct SlIdxRaw;
template <> struct SlIdxRaw<short> {
    uint2 u;
    __device__ __forceinline__ void load(const short* p) { u = __ldcs((const uint2*)p); }
    __device__ __forceinline__ void lds(const unsigned char* p) { u = *(const uint2*)p; }
    __device__ __forceinline__ void ldsa(unsigned a) { u = lds_v2(a); }
    __device__ __forceinline__ int col(int i, int rr) const
    {
        const unsigned w = i < 2 ? u.x : u.y;
        return rr + ((i & 1) ? ((int)w >> 16) : (int)(short)(w & 0xffffu));
    }
};
template <> struct SlIdxRaw<int> {
    int4 u;
    __device__ __forceinline__ void load(const int* p) { u = __ldcs((const int4*)p); }
    __device__ __forceinline__ void lds(const unsigned char* p) { u = *(const int4*)p; }
    __device__ __forceinline__ void ldsa(unsigned a)
    {
        const uint4 v = lds_v4(a);
        u = make_int4((int)v.x, (int)v.y, (int)v.z, (int)v.w);
    }
    __device__ __forceinline__ int col(int i, int) const { return i == 0 ? u.x : i == 1 ? u.y : i == 2 ? u.z : u.w; }
};

// Values of a block: coded (4 one-byte codes into the table in shared memory) or stored.
template <typename VS> struct SlVal;
template <typename T> struct SlVal<Coded<T>> {
    using VT = T;
    static constexpr int kRegs = 1;
    static constexpr int kBytes = 1;   // per entry
    unsigned u;
    __device__ __forceinline__ void load(const void* p) { u = __ldcs((const unsigned*)p); }
    __device__ __forceinline__ void lds(const unsigned char* p) { u = *(const unsigned*)p; }
    __device__ __forceinline__ void ldsa(unsigned a) { u = lds_v1(a); }
    __device__ __forceinline__ T get(int i, const T* tab) const { return tab[__byte_perm(u, 0u, 0x4440u + i)]; }
};
template <> struct SlVal<const float*> {
    using VT = float;
    static constexpr int kRegs = 4;
    static constexpr int kBytes = 4;
    float4 u;
    __device__ __forceinline__ void load(const void* p) { u = __ldcs((const float4*)p); }
    __device__ __forceinline__ void lds(const unsigned char* p) { u = *(const float4*)p; }
    __device__ __forceinline__ void ldsa(unsigned a)
    {
        const uint4 v = lds_v4(a);
        u = make_float4(__uint_as_float(v.x), __uint_as_float(v.y), __uint_as_float(v.z), __uint_as_float(v.w));
    }
    __device__ __forceinline__ float get(int i, const float*) const { return i == 0 ? u.x : i == 1 ? u.y : i == 2 ? u.z : u.w; }
};
template <> struct SlVal<const double*> {
    using VT = double;
    static constexpr int kRegs = 8;
    static constexpr int kBytes = 8;
    double2 a, b;
    __device__ __forceinline__ void load(const void* p)
    {
        a = __ldcs((const double2*)p);
        b = __ldcs((const double2*)p + 1);
    }
    __device__ __forceinline__ void lds(const unsigned char* p)
    {
        a = *(const double2*)p;
        b = *((const double2*)p + 1);
    }
    __device__ __forceinline__ void ldsa(unsigned addr)
    {
        const uint4 v = lds_v4(addr), w = lds_v4(addr + 16);
        a = make_double2(__hiloint2double((int)v.y, (int)v.x), __hiloint2double((int)v.w, (int)v.z));
        b = make_double2(__hiloint2double((int)w.y, (int)w.x), __hiloint2double((int)w.w, (int)w.z));
    }
    __device__ __forceinline__ double get(int i, const double*) const { return i == 0 ? a.x : i == 1 ? a.y : i == 2 ? b.x : b.y; }
};

// The sliced arrays a launch reads: indices (int16 offsets or int32 columns) and the value source
// (codes + table, or stored values), base pointers of the slice layout.
template <typename VS> struct SlSrc;
template <typename T> struct SlSrc<Coded<T>> {
    const unsigned char* code;
    const T* tab;
    __device__ __forceinline__ const void* at(long j) const { return code + j; }
};
template <typename T> struct SlSrc<const T*> {
    const T* val;
    __device__ __forceinline__ const void* at(long j) const { return val + j; }
};

// Shared-memory stages of the sliced kernel: every warp keeps kSlStages stages of kSlStageBytes,
// each holding one slice's index words (first) and value words (after NBMAX blocks of indices),
// filled by the warp's own cp.async copies kSlStages - 1 slices ahead of the one it works on. A
// slice wider than NBMAX blocks is read from global memory instead. The depth of the ring, not
// the number of resident warps, sets the rate (at 27-point 160^3, level 0: 2 stages with 32
// resident warps 0.131 ms a sweep, 3 with 24 warps 0.090 ms, 4 with 16 warps 0.085 ms; 5 with 12
// warps in 6-warp blocks 0.100 ms, 5 with 8 warps 0.134 ms).
constexpr int kSlWarps = 8;            // warps per block (256 threads)
constexpr int kSlStages = 4;
constexpr int kSlMinBlocks = 2;        // blocks per SM that the stages (96 KB a block) leave room for
constexpr int kSlStageBytes = 3072;
template <typename IT, typename VS>
struct SlStage {
    static constexpr int kIdxB = kSliceBlock * (int)sizeof(IT);            // index bytes of a block
    static constexpr int kValB = kSliceBlock * SlVal<VS>::kBytes;         // value bytes of a block
    static constexpr int NBMAX = kSlStageBytes / (kIdxB + kValB);
    static constexpr int VAL = NBMAX * kIdxB;                              // offset of the values in a stage
    static constexpr int SMEM = kSlWarps * kSlStages * kSlStageBytes;
    static_assert(NBMAX >= 1, "a stage must hold one block");
    static_assert(kIdxB % 16 == 0 && kValB % 16 == 0 && VAL % 16 == 0, "stages copy whole 16-byte chunks");
};

__device__ __forceinline__ void cp_async16(unsigned dst, const void* src, unsigned long long pol)
{
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "l"(pol) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

extern __shared__ __align__(128) unsigned char sl_smem[];

// The row sum of a lane over a staged slice of exactly NBC blocks (known at compile time: every
// loop unrolled, no per-block test), in the order of the general path: block by block, entry by
// entry. sb: the stage's 32-bit shared address.
template <int NBC, typename VS, typename XT, typename IT, typename AT, typename VT>
__device__ __forceinline__ AT slice_sum_fixed(unsigned sb, int lane, int rr, const XT* __restrict__ x, const VT* tab_s)
{
    using V = SlVal<VS>;
    using ST = SlStage<IT, VS>;
    constexpr int GB = sizeof(XT) == 4 ? 4 : 2;
    SlIdxRaw<IT> ix[NBC];
    V vv[NBC];
#pragma unroll
    for (int u = 0; u < NBC; u++) {
        ix[u].ldsa(sb + (unsigned)(u * ST::kIdxB + lane * kSliceG * (int)sizeof(IT)));
        vv[u].ldsa(sb + (unsigned)(ST::VAL + u * ST::kValB + lane * kSliceG * V::kBytes));
    }
    AT s = 0;
#pragma unroll
    for (int g = 0; g < NBC; g += GB) {
        XT xv[GB][kSliceG];
#pragma unroll
        for (int u = 0; u < GB; u++)
            if (g + u < NBC)
#pragma unroll
                for (int i = 0; i < kSliceG; i++) xv[u][i] = ld_ro(x + ix[g + u].col(i, rr));
#pragma unroll
        for (int u = 0; u < GB; u++)
            if (g + u < NBC)
#pragma unroll
                for (int i = 0; i < kSliceG; i++) s += (AT)vv[g + u].get(i, tab_s) * (AT)xv[u][i];
    }
    return s;
}

// y = alpha A x + beta y, y = f - A x, or one l1-Jacobi sweep (the operations of k_rowop) over the
// sliced form: one warp per slice (grid-stride over slices), one lane per row. Each warp copies the
// index and value words of its next slices into its shared-memory stages (cp.async, 16 bytes per
// lane and copy, completion awaited per warp with cp.async.wait_group: no wait on another warp),
// so that a slice's gathers start without a round trip to memory for its indices. Blocks are taken
// in chunks of up to 8 (their words read first), then gathered GB blocks at a time. Launch with
// kSlWarps * 32 threads and SlStage<IT, VS>::SMEM bytes of dynamic shared memory.
// FIT: every slice fits a stage (the matrix's longest row has at most NBMAX blocks), so no slice
// takes the global-memory path.
template <int OP, typename VS, typename XT, typename FT, typename MT, typename YT, typename IT, bool FIT>
__global__ void __launch_bounds__(kSlWarps * 32, kSlMinBlocks) k_rowop_sliced(int n, const int* __restrict__ sptr,
    const IT* __restrict__ sidx, SlSrc<VS> sv, const XT* __restrict__ x, const FT* __restrict__ f,
    const MT* __restrict__ M, YT* __restrict__ y, double alpha, double beta, const int* __restrict__ skip)
{
    using V = SlVal<VS>;
    using VT = typename V::VT;
    using AT = typename Acc<VT>::type;
    using ST = SlStage<IT, VS>;
    constexpr int kIdxRegs = sizeof(IT) == 2 ? 2 : 4;
    constexpr int kMeta = kIdxRegs + V::kRegs;
    constexpr int CB = kMeta <= 3 ? 8 : kMeta <= 6 ? 4 : 2;            // blocks per chunk
    constexpr int GB = sizeof(XT) == 4 ? 4 : 2;                          // blocks per gather group
    constexpr int GBc = GB < CB ? GB : CB;
    __shared__ VT tab_s[kValueCodes];   // the value table of a coded matrix
    if constexpr (ValSrc<VS>::coded) {
        for (int i = threadIdx.x; i < kValueCodes; i += blockDim.x) tab_s[i] = __ldg(sv.tab + i);
        __syncthreads();
    }
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long nsl = ((long)n + kSliceRows - 1) / kSliceRows;
    const long nw = (long)gridDim.x * (blockDim.x / 32);
    const long gw = (long)blockIdx.x * (blockDim.x / 32) + wib;
    unsigned char* stage0 = sl_smem + (size_t)wib * kSlStages * kSlStageBytes;
    const unsigned stage0_s = (unsigned)__cvta_generic_to_shared(stage0);
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));

    // the slice's first entry and entry count (0 past the last slice)
    auto ptrs = [&](long sl, int& b, int& e) {
        if (sl < nsl) {
            b = __ldg(sptr + sl);
            e = __ldg(sptr + sl + 1);
        } else {
            b = e = 0;
        }
    };
    // copies of a slice's words into stage st (nothing when it is empty or wider than a stage)
    auto issue = [&](int st, int b, int e) {
        const int nb = (e - b) / kSliceBlock;
        if (nb > 0 && (FIT || nb <= ST::NBMAX)) {
            const unsigned dst = stage0_s + (unsigned)(st * kSlStageBytes);
            const unsigned char* gi = (const unsigned char*)(sidx + b);
            const unsigned char* gv = (const unsigned char*)sv.at(b);
            const int ci = nb * ST::kIdxB / 16, cv = nb * ST::kValB / 16;
            for (int c = lane; c < ci; c += 32) cp_async16(dst + c * 16, gi + c * 16, pol);
            for (int c = lane; c < cv; c += 32) cp_async16(dst + ST::VAL + c * 16, gv + c * 16, pol);
        }
        cp_async_commit();
    };

    int pb[kSlStages], pe[kSlStages];
#pragma unroll
    for (int k = 0; k < kSlStages; k++) ptrs(gw + k * nw, pb[k], pe[k]);
#pragma unroll
    for (int k = 0; k + 1 < kSlStages; k++) issue(k, pb[k], pe[k]);
    // the prologue above reads only the sliced copy and its table, which no kernel of a solve
    // writes (build_sliced returns after they are complete); vectors are read after the wait
    dep_wait();
    dep_release();
    if (skip && *skip) {
        cp_async_wait<0>();   // no copy into this block's shared memory outlives the block
        return;
    }
    int st = 0;
    for (long sl = gw; sl < nsl; sl += nw) {
        // the stage that the slice kSlStages - 1 ahead goes to was read by this warp one slice ago
        __syncwarp();
        issue(st == 0 ? kSlStages - 1 : st - 1, pb[kSlStages - 1], pe[kSlStages - 1]);
        int bn, en;
        ptrs(sl + kSlStages * nw, bn, en);
        cp_async_wait<kSlStages - 1>();   // this slice's copies (the group before the last ones) have landed
        const int b0 = pb[0], e0 = pe[0];
        __syncwarp();         // ... including those of the other lanes
        const int r = (int)(sl * kSliceRows) + lane;
        const bool live = r < n;
        const int rr = live ? r : n - 1;
        const int nb = (e0 - b0) / kSliceBlock;
        const bool staged = FIT || nb <= ST::NBMAX;
        const unsigned char* sbase = stage0 + st * kSlStageBytes;
        // epilogue operands first: their latency overlaps the row's gathers
        AT o1 = 0, o2 = 0, o3 = 0;
        if (live) {
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
        AT s = 0;
        const long base = (long)b0 + lane * kSliceG;
        bool fixed = false;
        if (staged) {
            // the width of a staged slice as a compile-time count
            const unsigned sb = stage0_s + (unsigned)(st * kSlStageBytes);
            fixed = true;
            switch (nb) {
            case 1: s = slice_sum_fixed<1, VS, XT, IT, AT>(sb, lane, rr, x, tab_s); break;
            case 2: s = slice_sum_fixed<2, VS, XT, IT, AT>(sb, lane, rr, x, tab_s); break;
            case 3: if constexpr (ST::NBMAX >= 3) { s = slice_sum_fixed<3, VS, XT, IT, AT>(sb, lane, rr, x, tab_s); break; } [[fallthrough]];
            case 4: if constexpr (ST::NBMAX >= 4) { s = slice_sum_fixed<4, VS, XT, IT, AT>(sb, lane, rr, x, tab_s); break; } [[fallthrough]];
            case 5: if constexpr (ST::NBMAX >= 5) { s = slice_sum_fixed<5, VS, XT, IT, AT>(sb, lane, rr, x, tab_s); break; } [[fallthrough]];
            case 6: if constexpr (ST::NBMAX >= 6) { s = slice_sum_fixed<6, VS, XT, IT, AT>(sb, lane, rr, x, tab_s); break; } [[fallthrough]];
            case 7: if constexpr (ST::NBMAX >= 7) { s = slice_sum_fixed<7, VS, XT, IT, AT>(sb, lane, rr, x, tab_s); break; } [[fallthrough]];
            case 8: if constexpr (ST::NBMAX >= 8) { s = slice_sum_fixed<8, VS, XT, IT, AT>(sb, lane, rr, x, tab_s); break; } [[fallthrough]];
            default: fixed = nb == 0;
            }
        }
        for (int q0 = 0; !fixed && q0 < nb; q0 += CB) {
            SlIdxRaw<IT> ix[CB];
            V vv[CB];
#pragma unroll
            for (int u = 0; u < CB; u++)
                if (q0 + u < nb) {
                    if (staged) {
                        ix[u].lds(sbase + (q0 + u) * ST::kIdxB + lane * kSliceG * (int)sizeof(IT));
                        vv[u].lds(sbase + ST::VAL + (q0 + u) * ST::kValB + lane * kSliceG * V::kBytes);
                    } else {
                        const long j = base + (long)(q0 + u) * kSliceBlock;
                        ix[u].load(sidx + j);
                        vv[u].load(sv.at(j));
                    }
                }
#pragma unroll
            for (int g = 0; g < CB; g += GBc) {
                XT xv[GBc][kSliceG];
#pragma unroll
                for (int u = 0; u < GBc; u++)
                    if (q0 + g + u < nb)
#pragma unroll
                        for (int i = 0; i < kSliceG; i++) xv[u][i] = ld_ro(x + ix[g + u].col(i, rr));
#pragma unroll
                for (int u = 0; u < GBc; u++)
                    if (q0 + g + u < nb)
#pragma unroll
                        for (int i = 0; i < kSliceG; i++) s += (AT)vv[g + u].get(i, tab_s) * (AT)xv[u][i];
            }
        }
        if (live) {
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
#pragma unroll
        for (int k = 0; k + 1 < kSlStages; k++) {
            pb[k] = pb[k + 1];
            pe[k] = pe[k + 1];
        }
        pb[kSlStages - 1] = bn;
        pe[kSlStages - 1] = en;
        st = st == kSlStages - 1 ? 0 : st + 1;
    }
    cp_async_wait<0>();
}

// ---- pattern-indexed rows ----
// A coded level whose rows' column-offset sequences take at most 255 forms (build_patterns) keeps,
// besides its sliced codes, one byte per row naming its form and a table of the forms' int16
// offsets (zero past a form's length). k_rowop_slpat streams the codes and the form bytes only (about
// 1 byte per entry and 1 per row instead of 3 per entry) and reads the offsets from the table in
// shared memory; it adds a row's entries in the order of k_rowop_sliced, so the results are the same
// bit for bit. Stages hold a slice's 32 form bytes, then its code blocks.
constexpr int kSpStages = 6;
constexpr int kSpStageBytes = 32 + 8 * kSliceBlock;   // the form bytes and up to 8 blocks of codes

// the row sum of a lane over a slice of exactly NBC blocks: offsets from the form's table row (pr, a
// 32-bit shared address, 8-byte aligned), codes from the stage (sb)
template <int NBC, typename T, typename XT, typename AT>
__device__ __forceinline__ AT slpat_sum_fixed(unsigned sb, unsigned pr, int lane, int rr, const XT* __restrict__ x,
    const T* tab_s)
{
    constexpr int GB = sizeof(XT) == 4 ? 4 : 2;
    SlIdxRaw<short> ix[NBC];
    SlVal<Coded<T>> vv[NBC];
#pragma unroll
    for (int u = 0; u < NBC; u++) {
        ix[u].ldsa(pr + (unsigned)(u * kSliceG * (int)sizeof(short)));
        vv[u].ldsa(sb + (unsigned)(32 + u * kSliceBlock + lane * kSliceG));
    }
    AT s = 0;
#pragma unroll
    for (int g = 0; g < NBC; g += GB) {
        XT xv[GB][kSliceG];
#pragma unroll
        for (int u = 0; u < GB; u++)
            if (g + u < NBC)
#pragma unroll
                for (int i = 0; i < kSliceG; i++) xv[u][i] = ld_ro(x + ix[g + u].col(i, rr));
#pragma unroll
        for (int u = 0; u < GB; u++)
            if (g + u < NBC)
#pragma unroll
                for (int i = 0; i < kSliceG; i++) s += (AT)vv[g + u].get(i, tab_s) * (AT)xv[u][i];
    }
    return s;
}

// The operations of k_rowop_sliced (OP_AXPBY, OP_RESID, OP_JACOBI) on a pattern-indexed coded level
// whose slices are all at most 8 blocks wide. Dynamic shared memory: the form table (npat * W int16,
// rounded up to 16 bytes) and kSlWarps * kSpStages * kSpStageBytes of stages.
template <int OP, typename T, typename XT, typename FT, typename MT, typename YT>
__global__ void __launch_bounds__(kSlWarps * 32, 3) k_rowop_slpat(int n, const int* __restrict__ sptr,
    const unsigned char* __restrict__ pid, const unsigned char* __restrict__ code, const T* __restrict__ tab,
    const short* __restrict__ pat, int npat, int W, const XT* __restrict__ x, const FT* __restrict__ f,
    const MT* __restrict__ M, YT* __restrict__ y, double alpha, double beta, const int* __restrict__ skip)
{
    using AT = typename Acc<T>::type;
    __shared__ T tab_s[kValueCodes];
    short* pat_s = (short*)sl_smem;
    const int patb = ((npat * W * (int)sizeof(short)) + 15) & ~15;
    for (int i = threadIdx.x; i < kValueCodes; i += blockDim.x) tab_s[i] = __ldg(tab + i);
    for (int i = threadIdx.x; i < npat * W; i += blockDim.x) pat_s[i] = __ldg(pat + i);
    __syncthreads();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long nsl = ((long)n + kSliceRows - 1) / kSliceRows;
    const long nw = (long)gridDim.x * (blockDim.x / 32);
    const long gw = (long)blockIdx.x * (blockDim.x / 32) + wib;
    unsigned char* stage0 = sl_smem + patb + (size_t)wib * kSpStages * kSpStageBytes;
    const unsigned stage0_s = (unsigned)__cvta_generic_to_shared(stage0);
    const unsigned pat_sa = (unsigned)__cvta_generic_to_shared(pat_s);
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    auto ptrs = [&](long sl, int& b, int& e) {
        if (sl < nsl) {
            b = __ldg(sptr + sl);
            e = __ldg(sptr + sl + 1);
        } else {
            b = e = 0;
        }
    };
    // a slice's 32 form bytes (two 16-byte copies) and its code blocks into stage st
    auto issue = [&](int st, long sl, int b, int e) {
        const int nb = (e - b) / kSliceBlock;
        if (sl < nsl && nb > 0) {
            const unsigned dst = stage0_s + (unsigned)(st * kSpStageBytes);
            if (lane < 2) cp_async16(dst + lane * 16, pid + sl * kSliceRows + lane * 16, pol);
            const int cv = nb * kSliceBlock / 16;
            for (int c = lane; c < cv; c += 32) cp_async16(dst + 32 + c * 16, code + b + c * 16, pol);
        }
        cp_async_commit();
    };
    int pb[kSpStages], pe[kSpStages];
#pragma unroll
    for (int k = 0; k < kSpStages; k++) ptrs(gw + k * nw, pb[k], pe[k]);
#pragma unroll
    for (int k = 0; k + 1 < kSpStages; k++) issue(k, gw + k * nw, pb[k], pe[k]);
    // the prologue reads only the sliced codes, the form bytes and the tables, which no kernel of a
    // solve writes (build_sliced returns after they are complete); vectors are read after the wait
    dep_wait();
    dep_release();
    if (skip && *skip) {
        cp_async_wait<0>();
        return;
    }
    int st = 0;
    for (long sl = gw; sl < nsl; sl += nw) {
        __syncwarp();
        issue(st == 0 ? kSpStages - 1 : st - 1, sl + (kSpStages - 1) * nw, pb[kSpStages - 1], pe[kSpStages - 1]);
        int bn, en;
        ptrs(sl + kSpStages * nw, bn, en);
        cp_async_wait<kSpStages - 1>();
        const int b0 = pb[0], e0 = pe[0];
        __syncwarp();
        const int r = (int)(sl * kSliceRows) + lane;
        const bool live = r < n;
        const int rr = live ? r : n - 1;
        const int nb = (e0 - b0) / kSliceBlock;
        const unsigned char* sbase = stage0 + st * kSpStageBytes;
        const unsigned sb = stage0_s + (unsigned)(st * kSpStageBytes);
        AT o1 = 0, o2 = 0, o3 = 0;
        if (live) {
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
        const unsigned pr = pat_sa + (unsigned)((int)sbase[lane] * W * (int)sizeof(short));
        AT s = 0;
        switch (nb) {
        case 1: s = slpat_sum_fixed<1, T, XT, AT>(sb, pr, lane, rr, x, tab_s); break;
        case 2: s = slpat_sum_fixed<2, T, XT, AT>(sb, pr, lane, rr, x, tab_s); break;
        case 3: s = slpat_sum_fixed<3, T, XT, AT>(sb, pr, lane, rr, x, tab_s); break;
        case 4: s = slpat_sum_fixed<4, T, XT, AT>(sb, pr, lane, rr, x, tab_s); break;
        case 5: s = slpat_sum_fixed<5, T, XT, AT>(sb, pr, lane, rr, x, tab_s); break;
        case 6: s = slpat_sum_fixed<6, T, XT, AT>(sb, pr, lane, rr, x, tab_s); break;
        case 7: s = slpat_sum_fixed<7, T, XT, AT>(sb, pr, lane, rr, x, tab_s); break;
        case 8: s = slpat_sum_fixed<8, T, XT, AT>(sb, pr, lane, rr, x, tab_s); break;
        default: break;
        }
        if (live) {
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
#pragma unroll
        for (int k = 0; k + 1 < kSpStages; k++) {
            pb[k] = pb[k + 1];
            pe[k] = pe[k + 1];
        }
        pb[kSpStages - 1] = bn;
        pe[kSpStages - 1] = en;
        st = st == kSpStages - 1 ? 0 : st + 1;
    }
    cp_async_wait<0>();
}

// ---- building the sliced form from the CSR arrays ----

// entries of slice s: 128 x the blocks of its longest row
__global__ void k_sl_width(int n, const int* __restrict__ row, int* __restrict__ cnt)
{
    const int lane = threadIdx.x & 31;
    const long nsl = ((long)n + kSliceRows - 1) / kSliceRows;
    for (long sl = ((long)blockIdx.x * blockDim.x + threadIdx.x) / 32; sl < nsl;
         sl += (long)gridDim.x * blockDim.x / 32) {
        const long r = sl * kSliceRows + lane;
        int len = r < n ? __ldg(row + r + 1) - __ldg(row + r) : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) len = max(len, __shfl_xor_sync(0xffffffffu, len, o));
        if (lane == 0) cnt[sl] = ((len + kSliceG - 1) / kSliceG) * kSliceBlock;
    }
}

// Fills the slice layout: entry k of row r (slice s, lane l) at sptr[s] + (k / 4) * 128 + 4 l + k % 4.
// Index: int16 offsets (from dcol) or int32 columns; values: codes (pad = zero_code), FP32 or
// FP64 values (pad = 0), each written only when its output pointer is given.
template <typename IT>
__global__ void k_sl_fill(int n, const int* __restrict__ row, const IT* __restrict__ cidx, const int* __restrict__ sptr,
    IT* __restrict__ sidx, const unsigned char* __restrict__ code, unsigned char* __restrict__ scode, int zero_code,
    const float* __restrict__ v32, float* __restrict__ sv32, const double* __restrict__ v64, double* __restrict__ sv64)
{
    const int lane = threadIdx.x & 31;
    const long nsl = ((long)n + kSliceRows - 1) / kSliceRows;
    for (long sl = ((long)blockIdx.x * blockDim.x + threadIdx.x) / 32; sl < nsl;
         sl += (long)gridDim.x * blockDim.x / 32) {
        const int r = (int)(sl * kSliceRows) + lane;
        const int rr = r < n ? r : n - 1;
        const int b = r < n ? __ldg(row + r) : 0, e = r < n ? __ldg(row + r + 1) : 0;
        const int s0 = __ldg(sptr + sl), width = (__ldg(sptr + sl + 1) - s0) / kSliceRows;
        for (int k = 0; k < width; k++) {
            const long j = (long)s0 + (long)(k / kSliceG) * kSliceBlock + lane * kSliceG + (k % kSliceG);
            const bool in = b + k < e;
            const int t = b + k;
            if constexpr (sizeof(IT) == 2) sidx[j] = in ? cidx[t] : (IT)0;
            else sidx[j] = in ? cidx[t] : (IT)rr;
            if (scode) scode[j] = in ? code[t] : (unsigned char)zero_code;
            if (sv32) sv32[j] = in ? v32[t] : 0.0f;
            if (sv64) sv64[j] = in ? v64[t] : 0.0;
        }
    }
}

}  // namespace bcmgx
