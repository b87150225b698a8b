// setup.cu -- hierarchy construction on the device (BCMG: suitor matching + pairwise aggregation).
//
// Restates, at np = 1: adaptiveCoarsening / matchingAggregation
// (BCMGX/src/preconditioner/bcmg/matchingAggregation.cu:106-466), matchingPairAggregation /
// makeP_GPU (matchingPairAggregation.cu:24-237), the edge weights (matching.cu:13-288), the suitor
// matching (suitor.cu:51-329) and the two nsparse products of the Galerkin step.
//
// Every floating-point operation of this file is an explicit round-to-nearest intrinsic
// (__dmul_rn, __dadd_rn, ...) so nothing is contracted into an FMA: the hierarchy is
// bit-identical to the CPU restatement. Integer results (matching, aggregates, sizes) do not
// depend on thread scheduling:
//  * the suitor matching is lock-free: every vertex ranks its neighbours once, offers are
//    ranks combined with atomicMax (64-bit words that also name the proposer), and each
//    vertex's search pointer only moves forward, so the work is bounded by nnz and the result
//    is the greedy matching of the edge order;
//  * aggregates are numbered by prefix sums (pairs by master id, then singletons by id);
//  * every Galerkin entry is a sum of at most two rounded products, formed in a fixed order.
#include "internal.h"
#include "common.cuh"

#include <cub/device/device_segmented_sort.cuh>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <mutex>

namespace bcmgx {

int num_sms();

constexpr double kSuitorEps = 3.885780586188048e-10;   // suitor.h:8
constexpr int kFtcoarseInc = 100;                       // matchingAggregation.cu:8
constexpr double kCoarseRatioThreshold = 1.2;           // matchingAggregation.cu:9

enum : int {
    ERR_ROW0 = 1, ERR_ROWN = 2, ERR_ROWORDER = 4, ERR_COLRANGE = 8, ERR_COLSORT = 16, ERR_NODIAG = 32,
    ERR_SUITOR_BUDGET = 64, ERR_ASYM_MATCH = 128, ERR_BADW = 256, ERR_GALERKIN_CAP = 512, ERR_GALERKIN_OFS = 1024,
};

// Optional phase timing of the set-up (environment BCMGX_PROFILE=1): the stream is synchronised
// at phase boundaries and host wall time is accumulated per phase, printed to stderr.
static bool prof_on()
{
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("BCMGX_PROFILE");
        v = (e && std::atoi(e) > 0) ? 1 : 0;
    }
    return v == 1;
}

struct PhaseTimer {
    bcmgx_hierarchy* H;
    const char* name;
    std::chrono::steady_clock::time_point t0;
    PhaseTimer(bcmgx_hierarchy* h, const char* nm) : H(h), name(nm)
    {
        if (prof_on()) {
            cudaStreamSynchronize(H->stream);
            t0 = std::chrono::steady_clock::now();
        }
    }
    ~PhaseTimer()
    {
        if (!prof_on()) return;
        cudaStreamSynchronize(H->stream);
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        for (auto& pr : H->prof)
            if (pr.first == name) {
                pr.second += ms;
                return;
            }
        H->prof.push_back({ name, ms });
    }
};

static int gs_grid(long n, int threads = 256)
{
    return (int)std::max<long>(1, std::min<long>((n + threads - 1) / threads, (long)num_sms() * 16));
}
static int warp_grid(long rows, int threads = 256)
{
    return gs_grid(rows * 32, threads);
}

// ------------------------------------------------------------------------------------------
// prefix sums (three phases: tile sums, scan of tile sums, tile scans)
// ------------------------------------------------------------------------------------------
constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ long long block_excl_scan(long long v, long long* total)
{
    __shared__ long long ws[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[wid] = x;
    __syncthreads();
    if (wid == 0) {
        long long t = lane < nw ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        ws[lane] = t;
    }
    __syncthreads();
    const long long off = wid > 0 ? ws[wid - 1] : 0;
    *total = ws[nw - 1];
    __syncthreads();
    return off + x - v;
}

__global__ void k_scan_tiles(const int* __restrict__ in, long n, long long* tile_sums)
{
    const long base = (long)blockIdx.x * kScanTile + (long)threadIdx.x * kScanItems;
    long long s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (base + k < n) s += in[base + k];
    long long tot;
    block_excl_scan(s, &tot);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// total: the sum (64-bit); out_total, when given: the sum as the int32 entry after the scan
__global__ void k_scan_top(long long* tile_sums, int ntiles, long long* total, int* out_total)
{
    long long carry = 0;
    for (int b0 = 0; b0 < ntiles; b0 += blockDim.x) {
        const int i = b0 + threadIdx.x;
        long long v = i < ntiles ? tile_sums[i] : 0;
        long long tot;
        long long ex = block_excl_scan(v, &tot);
        if (i < ntiles) tile_sums[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) {
        *total = carry;
        if (out_total) *out_total = carry <= 0x7fffffffLL ? (int)carry : -1;
    }
}

__global__ void k_scan_down(const int* __restrict__ in, int* __restrict__ out, long n, const long long* tile_offs)
{
    const long base = (long)blockIdx.x * kScanTile + (long)threadIdx.x * kScanItems;
    int v[kScanItems];
    long long s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    long long tot;
    long long ex = block_excl_scan(s, &tot) + tile_offs[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) out[base + k] = (int)ex;
        ex += v[k];
    }
}

// Exclusive prefix sum of in[0..n) into out[0..n); when with_total, out[n] = total.
// Returns the total (synchronises the stream).
// Exclusive scan of n ints into out (and the total into out[n] when with_total), on the device;
// tot receives the 64-bit total.
static void scan_launch(const int* in, int* out, long n, bool with_total, long long* tot, cudaStream_t s)
{
    const int ntiles = std::max(1, (int)((n + kScanTile - 1) / kScanTile));
    DBuf<long long> tiles;
    tiles.alloc(ntiles, s);
    if (n > 0) { note_launch(); k_scan_tiles<<<ntiles, kScanThreads, 0, s>>>(in, n, tiles.p); }
    else BCMGX_CUDA(cudaMemsetAsync(tiles.p, 0, sizeof(long long), s));
    note_launch(); k_scan_top<<<1, 1024, 0, s>>>(tiles.p, ntiles, tot, with_total ? out + n : nullptr);
    if (n > 0) { note_launch(); k_scan_down<<<ntiles, kScanThreads, 0, s>>>(in, out, n, tiles.p); }
    BCMGX_CHECK_LAUNCH();
}

long long scan_exclusive(const int* in, int* out, long n, bool with_total, cudaStream_t s)
{
    DBuf<long long> tot;
    tot.alloc(1, s);
    scan_launch(in, out, n, with_total, tot.p, s);
    long long total = 0;
    BCMGX_CUDA(cudaMemcpyAsync(&total, tot.p, sizeof(long long), cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaStreamSynchronize(s));
    BCMGX_REQUIRE(total <= 0x7fffffffLL, BCMGX_ERR_UNSUPPORTED, "more than 2^31-1 entries (int32 offsets)");
    return total;
}

// The same scan with the total only on the device (out[n]), for callers that know it already or
// do not need it: no host synchronisation. The total must fit int32 (out[n] = -1 otherwise).
void scan_exclusive_dev(const int* in, int* out, long n, cudaStream_t s)
{
    DBuf<long long> tot;
    tot.alloc(1, s);
    scan_launch(in, out, n, true, tot.p, s);
}

// ------------------------------------------------------------------------------------------
// matrix checks and small per-row kernels
// ------------------------------------------------------------------------------------------
__global__ void k_validate(int n, int m, long long nnz, const int* __restrict__ row, const int* __restrict__ col,
    int* err, int* max_row, int need_diag)
{
    const int lane = threadIdx.x & 31;
    int mx = 0;
    for (long r = ((long)blockIdx.x * blockDim.x + threadIdx.x) / 32; r < n; r += (long)gridDim.x * blockDim.x / 32) {
        const int b = row[r], e = row[r + 1];
        int bad = 0;
        if (r == 0 && b != 0) bad |= ERR_ROW0;
        if (r == n - 1 && (long long)e != nnz) bad |= ERR_ROWN;
        if (e < b || b < 0 || (long long)e > nnz) {
            bad |= ERR_ROWORDER;
        } else {
            bool diag = false;
            for (int j = b + lane; j < e; j += 32) {
                const int c = col[j];
                if (c < 0 || c >= m) bad |= ERR_COLRANGE;
                if (j > b && col[j - 1] >= c) bad |= ERR_COLSORT;
                if (c == r) diag = true;
            }
            diag = __any_sync(0xffffffffu, diag);
            if (need_diag && !diag) bad |= ERR_NODIAG;
            mx = max(mx, e - b);
        }
        bad = __reduce_or_sync(0xffffffffu, bad);
        if (lane == 0 && bad) atomicOr(err, bad);
    }
    if (lane == 0 && mx > 0) atomicMax(max_row, mx);
}

// The input checks of k_validate with 8 lanes per row (4 rows of a warp in flight, the previous
// column passed by shuffles), plus the largest |col - row| and, when dcol is given, every column
// as an int16 offset from its row (clamped; the caller keeps them only when the largest offset
// fits): one pass over the input instead of three.
__global__ void k_validate_offsets(int n, int m, long long nnz, const int* __restrict__ row, const int* __restrict__ col,
    int* err, int* max_row, int* max_off, short* __restrict__ dcol, int need_diag, int* __restrict__ dpos)
{
    constexpr int S = 8;
    const int lane = threadIdx.x & (S - 1);
    const int sub = (threadIdx.x & 31) / S;
    const unsigned mask = 0xffu << (sub * S);
    const long stride = (long)gridDim.x * blockDim.x / S;
    int mx = 0, mo = 0;
    for (long base = ((long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / S; base < n; base += stride) {
        const long r = base + sub;
        int bad = 0;
        if (r < n) {
            const int b = row[r], e = row[r + 1];
            if (r == 0 && b != 0) bad |= ERR_ROW0;
            if (r == n - 1 && (long long)e != nnz) bad |= ERR_ROWN;
            if (e < b || b < 0 || (long long)e > nnz) {
                bad |= ERR_ROWORDER;
            } else {
                bool diag = false;
                int carry = 0;
                constexpr int U = 4;   // chunks of S entries whose columns are requested together
                for (int j00 = b; j00 < e; j00 += U * S) {
                    int cv[U];
#pragma unroll
                    for (int u = 0; u < U; u++) {
                        const int j = j00 + u * S + lane;
                        cv[u] = j < e ? __ldcs(col + j) : 0x7fffffff;
                    }
#pragma unroll
                    for (int u = 0; u < U; u++) {
                        const int j0 = j00 + u * S;
                        if (j0 >= e) break;   // uniform across the row's lanes
                        const int j = j0 + lane;
                        const int c = cv[u];
                        int prev = __shfl_up_sync(mask, c, 1, S);
                        if (lane == 0) prev = carry;
                        if (j < e) {
                            if (c < 0 || c >= m) bad |= ERR_COLRANGE;
                            if (j > b && prev >= c) bad |= ERR_COLSORT;
                            if (c == (int)r) {
                                diag = true;
                                if (dpos) dpos[r] = j;
                            }
                            const int off = c - (int)r;
                            mo = max(mo, off < 0 ? -off : off);
                            if (dcol) dcol[j] = (short)max(-32768, min(32767, off));
                        }
                        carry = __shfl_sync(mask, c, S - 1, S);
                    }
                }
                diag = (__ballot_sync(mask, diag) & mask) != 0;
                if (need_diag && !diag) bad |= ERR_NODIAG;
                if (dpos && !diag && lane == 0) dpos[r] = -1;
                mx = max(mx, e - b);
            }
        }
        bad = __reduce_or_sync(0xffffffffu, bad);
        if ((threadIdx.x & 31) == 0 && bad) atomicOr(err, bad);
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    mo = __reduce_max_sync(0xffffffffu, mo);
    if ((threadIdx.x & 31) == 0) {
        if (mx > 0) atomicMax(max_row, mx);
        if (mo > 0) atomicMax(max_off, mo);
    }
}

__global__ void k_row_max(int n, const int* __restrict__ row, int* max_row)
{
    int mx = 0;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long)gridDim.x * blockDim.x)
        mx = max(mx, row[r + 1] - row[r]);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((threadIdx.x & 31) == 0) atomicMax(max_row, mx);
}

// M_i = sum_j |a_ij| in column order (_row_sum_2, CSR.cu:1362-1379).
__global__ void k_abs_row_sum(int n, const int* __restrict__ row, const double* __restrict__ val, double* __restrict__ M,
    float* __restrict__ M32)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        // the row's values are loaded 8 at a time (independent loads), then added in column order
        double s = 0.0;
        const int b = row[i], e = row[i + 1];
        for (int j0 = b; j0 < e; j0 += 8) {
            double v[8];
#pragma unroll
            for (int k = 0; k < 8; k++) v[k] = j0 + k < e ? __ldcs(val + j0 + k) : 0.0;
#pragma unroll
            for (int k = 0; k < 8; k++)
                if (j0 + k < e) s = __dadd_rn(s, fabs(v[k]));
        }
        M[i] = s;
        if (M32) M32[i] = (float)s;
    }
}

// Standalone l1-Jacobi divisor D_i = a_ii + sum_{j != i} |a_ij|: the diagonal (mydiag) plus the
// off-diagonal absolute sum in column order (add_absrowsum_nodiag, op/addAbsoluteRowSumNoDiag.cu).
__global__ void k_l1_divisor(int n, const int* __restrict__ row, const int* __restrict__ col, const double* __restrict__ val,
    double* __restrict__ D)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double d = 0.0, off = 0.0;
        for (int j = row[i]; j < row[i + 1]; j++) {
            if (col[j] == i) d = val[j];
            else off = __dadd_rn(off, fabs(val[j]));
        }
        D[i] = __dadd_rn(d, off);
    }
}

__global__ void k_to_f32(long n, const double* __restrict__ a, float* __restrict__ b)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) b[i] = (float)a[i];
}

__global__ void k_fill(long n, double* a, double v)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) a[i] = v;
}

// ------------------------------------------------------------------------------------------
// edge weights (makeAH, toMaximumProductMatrix, _write_T_warp)
// ------------------------------------------------------------------------------------------

// C_r = (a_rr * w_r) * w_r from the first diagonal entry (_makeC, matching.cu:113-135).
__global__ void k_diag_c(int n, const int* __restrict__ row, const int* __restrict__ col, const double* __restrict__ val,
    const double* __restrict__ w, double* __restrict__ C, int* err)
{
    // 8 lanes per row look for the row's first diagonal entry together (4 rows of a warp in flight)
    constexpr int S = 8;
    const int lane = threadIdx.x & (S - 1);
    const int sub = (threadIdx.x & 31) / S;
    const unsigned mask = 0xffu << (sub * S);
    const long stride = (long)gridDim.x * blockDim.x / S;
    for (long base = ((long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / S; base < n; base += stride) {
        const long r = base + sub;
        if (r >= n) continue;
        const int b = row[r], e = row[r + 1];
        int found = -1;
        for (int j0 = b; j0 < e && found < 0; j0 += S) {
            const int j = j0 + lane;
            const unsigned hit = __ballot_sync(mask, j < e && col[j] == (int)r) & mask;
            if (hit) found = j0 + (__ffs(hit >> (sub * S)) - 1);
        }
        if (lane == 0) {
            double c = 0.0;
            if (found >= 0) c = __dmul_rn(__dmul_rn(val[found], w[r]), w[r]);
            else atomicOr(err, ERR_NODIAG);
            C[r] = c;
        }
    }
}

// k_diag_c for a matrix whose diagonal positions were recorded by the kernel that produced it
// (k_validate_offsets, k_compact_rows): one gather per row, the same product.
__global__ void k_diag_c_pos(int n, const int* __restrict__ dpos, const double* __restrict__ val,
    const double* __restrict__ w, double* __restrict__ C, int* err)
{
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long)gridDim.x * blockDim.x) {
        const int j = dpos[r];
        double c = 0.0;
        if (j >= 0) {
            const double wr = w[r];
            c = __dmul_rn(__dmul_rn(__ldg(val + j), wr), wr);
        } else {
            atomicOr(err, ERR_NODIAG);
        }
        C[r] = c;
    }
}

// Row loop of the matching kernels: a sub-warp of S lanes (a power of two, 4..32, from the
// average row length) owns a row and its lanes stride over the row's entries, so a warp keeps
// 32 / S rows in flight; each lane takes its entries in batches of kSetupBatch, issuing all loads
// of a batch before the loads that depend on them.
constexpr int kSetupBatch = 4;
#define BCMGX_SUBWARP_ROWS(r, n, S)                                                                  \
    for (long r = ((long)blockIdx.x * blockDim.x + threadIdx.x) / (S); r < (n);                      \
         r += (long)gridDim.x * blockDim.x / (S))

// lanes per row for the matching kernels: about 4 entries per lane
static int setup_subwarp(long n, int64_t nnz)
{
    const double avg = n > 0 ? (double)nnz / (double)n : 1.0;
    return avg <= 12 ? 4 : avg <= 40 ? 8 : avg <= 96 ? 16 : 32;
}

// launch of a matching kernel K<S> for the lanes-per-row choice S of setup_subwarp
#define BCMGX_SUBWARP_LAUNCH(K, S, n, s, ...)                                                      \
    do {                                                                                           \
        note_launch();                                                                             \
        switch (S) {                                                                               \
        case 4: K<4><<<gs_grid((long)(n) * 4), 256, 0, s>>>(__VA_ARGS__); break;                   \
        case 8: K<8><<<gs_grid((long)(n) * 8), 256, 0, s>>>(__VA_ARGS__); break;                   \
        case 16: K<16><<<gs_grid((long)(n) * 16), 256, 0, s>>>(__VA_ARGS__); break;                \
        default: K<32><<<gs_grid((long)(n) * 32), 256, 0, s>>>(__VA_ARGS__); break;                \
        }                                                                                          \
    } while (0)
// the same for a kernel K<S, X> with a second template argument X
#define BCMGX_SUBWARP_LAUNCH2(K, X, S, n, s, ...)                                                  \
    do {                                                                                           \
        note_launch();                                                                             \
        switch (S) {                                                                               \
        case 4: K<4, X><<<gs_grid((long)(n) * 4), 256, 0, s>>>(__VA_ARGS__); break;                \
        case 8: K<8, X><<<gs_grid((long)(n) * 8), 256, 0, s>>>(__VA_ARGS__); break;                \
        case 16: K<16, X><<<gs_grid((long)(n) * 16), 256, 0, s>>>(__VA_ARGS__); break;             \
        default: K<32, X><<<gs_grid((long)(n) * 32), 256, 0, s>>>(__VA_ARGS__); break;             \
        }                                                                                          \
    } while (0)

// a_hat = 1 - (2 a w_r w_c) / (C_r + C_c), or DBL_EPSILON if C_r + C_c <= DBL_EPSILON
// (_makeAH_warp, matching.cu:66-111). Symmetric in (r, c) apart from a.
__device__ __forceinline__ double ahat(double a, double Cr, double Cc, double wr, double wc)
{
    const double norm = __dadd_rn(Cr, Cc);
    if (norm > DBL_EPSILON) {
        const double wt = __dmul_rn(wr, wc);
        return __dsub_rn(1.0, __ddiv_rn(__dmul_rn(__dmul_rn(2.0, a), wt), norm));
    }
    return DBL_EPSILON;
}

// Position of the transposed entry: tpos[j] for a_rc is the index of a_cr in row c (-1 if the
// pattern has no a_cr); the diagonal maps to itself. The first probe is the mirror position:
// entry k of row r (of d_r entries) is looked for at entry d_c - 1 - k of row c, where a
// symmetric stencil puts it when both rows are full; a miss narrows the range and the binary
// search goes on from there. The searches of a lane's batch run in lock step, one round of
// independent loads per halving. MODE 0: the positions; 1: also the minimum over the off-diagonal
// |a_hat| (find_Max_Min with AbsMin, matching.cu:188-217) into *min_bits (the bit pattern of a
// non-negative double orders like its value, so atomicMin on it is exact), its loads going out
// with the search's first round; 2: the minimum alone.
template <int S, int MODE>
__global__ void __launch_bounds__(256, 4) k_tpos(int n, const int* __restrict__ row, const int* __restrict__ col, int* __restrict__ tpos,
    const double* __restrict__ val, const double* __restrict__ w, const double* __restrict__ C,
    unsigned long long* min_bits)
{
    constexpr bool TP = MODE != 2, MIN = MODE != 0;
    constexpr int U = kSetupBatch;
    const int lane = threadIdx.x & (S - 1);
    double mn = DBL_MAX;
    BCMGX_SUBWARP_ROWS(r, n, S)
    {
        const int b = __ldg(row + r), e = __ldg(row + r + 1);
        double Cr = 0.0, wr = 0.0;
        if (MIN) {
            Cr = __ldg(C + r);
            wr = __ldg(w + r);
        }
        for (int j0 = b + lane; j0 < e; j0 += U * S) {
            int c[U], lo[U], hi[U], end[U], fnd[U];
            double a[U], Cc[U], wc[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                c[u] = j0 + u * S < e ? __ldg(col + j0 + u * S) : -1;
                if (MIN) a[u] = j0 + u * S < e ? __ldg(val + j0 + u * S) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const bool srch = c[u] >= 0 && c[u] != (int)r;
                lo[u] = TP && srch ? __ldg(row + c[u]) : 0;
                end[u] = TP && srch ? __ldg(row + c[u] + 1) : 0;
                if (MIN) {
                    Cc[u] = srch ? __ldg(C + c[u]) : 0.0;
                    wc[u] = srch ? __ldg(w + c[u]) : 0.0;
                }
                hi[u] = end[u];
                fnd[u] = -1;
            }
            if (MIN) {
#pragma unroll
                for (int u = 0; u < U; u++)
                    if (c[u] >= 0 && c[u] != (int)r) mn = fmin(mn, fabs(ahat(a[u], Cr, Cc[u], wr, wc[u])));
            }
            if (!TP) continue;
            {
                int g[U], cm[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    g[u] = -1;
                    if (lo[u] < hi[u]) {
                        const int k = j0 + u * S - b;
                        g[u] = min(max(hi[u] - 1 - k, lo[u]), hi[u] - 1);
                        cm[u] = __ldg(col + g[u]);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; u++)
                    if (g[u] >= 0) {
                        if (cm[u] == (int)r) {
                            fnd[u] = g[u];
                            hi[u] = lo[u];
                        } else if (cm[u] < (int)r) {
                            lo[u] = g[u] + 1;
                        } else {
                            hi[u] = g[u];
                        }
                    }
            }
            for (int step = 0; step < 32; step++) {
                int cm[U];
                bool any = false;
#pragma unroll
                for (int u = 0; u < U; u++)
                    if (lo[u] < hi[u]) {
                        any = true;
                        cm[u] = __ldg(col + ((lo[u] + hi[u]) >> 1));
                    }
                if (!any) break;
#pragma unroll
                for (int u = 0; u < U; u++)
                    if (lo[u] < hi[u]) {
                        const int mid = (lo[u] + hi[u]) >> 1;
                        if (cm[u] < (int)r) lo[u] = mid + 1;
                        else hi[u] = mid;
                    }
            }
            int hit[U];
#pragma unroll
            for (int u = 0; u < U; u++)
                hit[u] = fnd[u] >= 0 ? (int)r : (c[u] >= 0 && c[u] != (int)r && lo[u] < end[u] ? __ldg(col + lo[u]) : -1);
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int j = j0 + u * S;
                if (c[u] < 0) continue;
                tpos[j] = c[u] == (int)r ? j : (fnd[u] >= 0 ? fnd[u] : (hit[u] == (int)r ? lo[u] : -1));
            }
        }
    }
    if (MIN) {
        unsigned long long bits = (unsigned long long)__double_as_longlong(mn);
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(0xffffffffu, bits, o);
            bits = other < bits ? other : bits;
        }
        if ((threadIdx.x & 31) == 0) atomicMin(min_bits, bits);
    }
}

// The transposed positions and the |a_hat| minimum: one fused pass (k_tpos<S, 1>) or two
// (BCMGX_TPOS_FUSE=0).
static void tpos_min_launch(int S, int n, const int* row, const int* col, int* tpos, const double* val, const double* w,
    const double* C, unsigned long long* min_bits, cudaStream_t s)
{
    static const bool fuse = [] {
        const char* e = std::getenv("BCMGX_TPOS_FUSE");
        return !(e && e[0] == '0');
    }();
    if (fuse) {
        BCMGX_SUBWARP_LAUNCH2(k_tpos, 1, S, n, s, n, row, col, tpos, val, w, C, min_bits);
    } else {
        BCMGX_SUBWARP_LAUNCH2(k_tpos, 0, S, n, s, n, row, col, tpos, val, w, C, min_bits);
        BCMGX_SUBWARP_LAUNCH2(k_tpos, 2, S, n, s, n, row, col, tpos, val, w, C, min_bits);
    }
}

// W = log(|a_hat|), or log(SUITOR_EPS / (0.999 min)) where a_hat == 0 (_make_w,
// matching.cu:219-229); a lower entry takes the value of its upper counterpart
// (_write_T_warp, matching.cu:29-64), i.e. is computed from a_cr. Diagonal slots are 0.
template <int S>
__global__ void k_logw(int n, const int* __restrict__ row, const int* __restrict__ col, const double* __restrict__ val,
    const double* __restrict__ w, const double* __restrict__ C, const int* __restrict__ tpos, double zero_sub,
    double* __restrict__ W, const double* __restrict__ zero_sub_dev = nullptr)
{
    if (zero_sub_dev) zero_sub = *zero_sub_dev;
    constexpr int U = kSetupBatch;
    const int lane = threadIdx.x & (S - 1);
    BCMGX_SUBWARP_ROWS(r, n, S)
    {
        const int b = __ldg(row + r), e = __ldg(row + r + 1);
        const double Cr = __ldg(C + r), wr = __ldg(w + r);
        for (int j0 = b + lane; j0 < e; j0 += U * S) {
            int c[U], src[U];
            double a[U], Cc[U], wc[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int j = j0 + u * S;
                c[u] = j < e ? __ldg(col + j) : -1;
                src[u] = j < e ? __ldg(tpos + j) : -1;
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const bool off = c[u] >= 0 && c[u] != (int)r;
                src[u] = (c[u] < (int)r && src[u] >= 0) ? src[u] : j0 + u * S;
                a[u] = off ? __ldg(val + src[u]) : 0.0;
                Cc[u] = off ? __ldg(C + c[u]) : 0.0;
                wc[u] = off ? __ldg(w + c[u]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int j = j0 + u * S;
                if (c[u] < 0) continue;
                if (c[u] == (int)r) {
                    W[j] = 0.0;
                    continue;
                }
                const double sa = fabs(ahat(a[u], Cr, Cc[u], wr, wc[u]));
                W[j] = log(sa != 0.0 ? sa : zero_sub);
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// suitor matching
// ------------------------------------------------------------------------------------------

// Per row: rank of every candidate (off-diagonal, W > 0) in the row's preference order,
// (W, column) descending (find_Candidate, suitor.cu:80-147).
// Ranks of a row of at most 32 entries held in registers (lane = entry t = b + lane, column ct
// and weight wt; ct = -1 past the row). When the weights differ, every lane compares its entry
// with all of the row's: the row's (weight, column) keys go to the warp's slots in shared memory
// (`keys`, 32 per warp) and are read back as broadcasts, one 16-byte load per compared entry
// (three shuffles per entry made shuffle throughput the bound).
struct alignas(16) RankKey {
    double w;
    int c;     // column, -1 for an entry that is not a candidate
    int pad;
};
__device__ __forceinline__ void rank_row32(long r, int b, int e, int ct, double wt, int* __restrict__ rank,
    int* __restrict__ degE, RankKey* keys)
{
    const int lane = threadIdx.x & 31;
    const int t = b + lane;
    const bool in = t < e;
    const bool el = in && ct != r && wt > 0.0;
    const unsigned elig = __ballot_sync(0xffffffffu, el);
    int rk = 0;
    const double w0 = __shfl_sync(0xffffffffu, wt, elig ? __ffs(elig) - 1 : 0);
    if (__ballot_sync(0xffffffffu, el && wt != w0) == 0u) {
        // all candidates weigh the same: the order is by column alone (columns ascend with the
        // lane), so the rank is the number of candidates in higher lanes
        rk = __popc(lane == 31 ? 0u : (elig >> (lane + 1)));
    } else {
        __syncwarp();   // the warp's previous row has been read
        keys[lane].w = wt;
        keys[lane].c = el ? ct : -1;
        __syncwarp();
        const int d = e - b;
        for (int k = 0; k < d; k++) {
            const RankKey q = keys[k];
            rk += (q.c >= 0 && (q.w > wt || (q.w == wt && q.c > ct))) ? 1 : 0;
        }
    }
    if (in) rank[t] = el ? rk : -1;
    if (lane == 0) degE[r] = __popc(elig);
}

// k_rank for a matrix whose rows all have at most 32 entries, with every entry's weight formed
// in registers by k_logw's expression (same operations, same rounding) instead of read from W:
// the weights are never stored. A warp's rows are pipelined two deep: while it ranks row r, the
// columns and transposed positions of its next row and the bounds of the row after are in
// flight, so a row costs one memory round trip instead of three dependent ones.
__global__ void __launch_bounds__(256, 8) k_rank_w(int n, const int* __restrict__ row, const int* __restrict__ col, const double* __restrict__ val,
    const double* __restrict__ w, const double* __restrict__ C, const int* __restrict__ tpos, double zero_sub,
    int* __restrict__ rank, int* __restrict__ degE, const double* __restrict__ zero_sub_dev)
{
    if (zero_sub_dev) zero_sub = *zero_sub_dev;
    const int lane = threadIdx.x & 31;
    __shared__ RankKey keys[8][32];   // 256-thread blocks
    RankKey* wkeys = keys[(threadIdx.x >> 5) & 7];
    const long step = (long)gridDim.x * blockDim.x / 32;
    long r = ((long)blockIdx.x * blockDim.x + threadIdx.x) / 32;   // uniform across the warp
    if (r >= n) return;
    int b = __ldg(row + r), e = __ldg(row + r + 1);
    int ct = b + lane < e ? __ldg(col + b + lane) : -1;
    int tp = b + lane < e ? __ldg(tpos + b + lane) : -1;
    long r1 = r + step;
    int b1 = 0, e1 = 0;
    if (r1 < n) {
        b1 = __ldg(row + r1);
        e1 = __ldg(row + r1 + 1);
    }
    while (true) {
        const long r2 = r1 + step;
        int b2 = 0, e2 = 0;
        if (r2 < n) {
            b2 = __ldg(row + r2);
            e2 = __ldg(row + r2 + 1);
        }
        int ct1 = -1, tp1 = -1;
        if (b1 + lane < e1) {
            ct1 = __ldg(col + b1 + lane);
            tp1 = __ldg(tpos + b1 + lane);
        }
        const int t = b + lane;
        double wt = 0.0;
        if (ct >= 0 && ct != (int)r) {
            const int src = (ct < (int)r && tp >= 0) ? tp : t;
            const double sa = fabs(ahat(__ldg(val + src), __ldg(C + r), __ldg(C + ct), __ldg(w + r), __ldg(w + ct)));
            wt = log(sa != 0.0 ? sa : zero_sub);
        }
        rank_row32(r, b, e, ct, wt, rank, degE, wkeys);
        if (r1 >= n) break;
        r = r1;
        b = b1;
        e = e1;
        ct = ct1;
        tp = tp1;
        r1 = r2;
        b1 = b2;
        e1 = e2;
    }
}

__global__ void k_rank(int n, const int* __restrict__ row, const int* __restrict__ col, const double* __restrict__ W,
    int* __restrict__ rank, int* __restrict__ degE)
{
    const int lane = threadIdx.x & 31;
    __shared__ RankKey keys[8][32];   // 256-thread blocks
    RankKey* wkeys = keys[(threadIdx.x >> 5) & 7];
    for (long r = ((long)blockIdx.x * blockDim.x + threadIdx.x) / 32; r < n; r += (long)gridDim.x * blockDim.x / 32) {
        const int b = row[r], e = row[r + 1];
        if (e - b <= 32) {
            const int t = b + lane;
            const bool in = t < e;
            rank_row32(r, b, e, in ? col[t] : -1, in ? W[t] : 0.0, rank, degE, wkeys);
            continue;
        }
        int cnt = 0;
        for (int t0 = b; t0 < e; t0 += 32) {
            const int t = t0 + lane;
            bool el = false;
            if (t < e) {
                const int ct = col[t];
                const double wt = W[t];
                el = (ct != r) && (wt > 0.0);
                if (el) {
                    int rk = 0;
                    for (int k = b; k < e; k++) {
                        const int ck = col[k];
                        const double wk = W[k];
                        rk += (ck != r && wk > 0.0 && (wk > wt || (wk == wt && ck > ct))) ? 1 : 0;
                    }
                    rank[t] = rk;
                } else {
                    rank[t] = -1;
                }
            }
            cnt += __popc(__ballot_sync(0xffffffffu, el));
        }
        if (lane == 0) degE[r] = cnt;
    }
}

// Preference records: pref[row[v] + k] = {k-th candidate y of v, v's offer value at y}, where
// the offer value is degE[y] - (rank of v in y's list), or 0 when y does not rank v (no
// transposed entry: the pair is never proposed). rinfo[v] = {row[v], degE[v]}. With mark_last
// (the wide suitor's form) the last record of each list also carries kPrefLast. The row's
// entries are taken in CSR order (their column, transposed position and rank read together) and
// each record is stored at its rank.
constexpr int kPrefLast = 1 << 30;
template <int S>
__global__ void k_pref(int n, const int* __restrict__ row, const int* __restrict__ col, const int* __restrict__ rank,
    const int* __restrict__ tpos, const int* __restrict__ degE, int2* __restrict__ pref, int2* __restrict__ rinfo,
    int mark_last)
{
    constexpr int U = kSetupBatch;
    const int lane = threadIdx.x & (S - 1);
    BCMGX_SUBWARP_ROWS(r, n, S)
    {
        const int b = __ldg(row + r), e = __ldg(row + r + 1), dE = __ldg(degE + r);
        for (int j0 = b + lane; j0 < e; j0 += U * S) {
            int rk[U], y[U], tj[U], ry[U], dy[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int j = j0 + u * S;
                rk[u] = j < e ? __ldg(rank + j) : -1;
                y[u] = j < e ? __ldg(col + j) : 0;
                tj[u] = j < e ? __ldg(tpos + j) : -1;
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                ry[u] = (rk[u] >= 0 && tj[u] >= 0) ? __ldg(rank + tj[u]) : -1;
                dy[u] = rk[u] >= 0 ? __ldg(degE + y[u]) : 0;
            }
#pragma unroll
            for (int u = 0; u < U; u++)
                if (rk[u] >= 0) {
                    const int last = (mark_last && rk[u] == dE - 1) ? kPrefLast : 0;
                    pref[b + rk[u]] = make_int2(y[u], (ry[u] >= 0 ? dy[u] - ry[u] : 0) | last);
                }
        }
        if (lane == 0) rinfo[r] = make_int2(b, dE);
    }
}


// Lock-free suitor. A vertex proposes to its candidates in preference order; y keeps the best
// suitor by atomicMax on its offer word (set_suitor/find_Candidate, suitor.cu:51-147, with the
// same order: weight, then the higher id). A successful proposal that displaces a previous
// suitor d hands d to the same thread (as set_suitor does), which resumes d right after y in
// d's list: that position follows from y's own record of d (no shared pointer, no fence).
// Vertices start top-down (highest id first): under the id tie rule the higher vertices settle
// first, and lower vertices then skip candidates whose current offer already beats theirs.
// Every vertex's position only moves forward, so the work is bounded by nnz; `budget` guards
// the loop.
__global__ void k_suitor(int n, const int2* __restrict__ rinfo, const int2* __restrict__ pref, unsigned* offer,
    long long budget, int* err, int descending)
{
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        int cur = descending ? (int)(n - 1 - t) : (int)t;
        int k = 0;
        long long steps = 0;
        while (cur >= 0) {
            const int2 ci = rinfo[cur];
            int next = -1, nextk = 0;
            for (; k < ci.y; k++) {
                if (++steps > budget) {
                    atomicOr(err, ERR_SUITOR_BUDGET);
                    return;
                }
                const int2 pr = pref[ci.x + k];
                const unsigned mine = (unsigned)pr.y;
                if (mine == 0u || ld_cg(offer + pr.x) >= mine) continue;
                const unsigned old = atomicMax(offer + pr.x, mine);
                if (old < mine) {
                    if (old != 0u) {
                        const int2 yi = rinfo[pr.x];
                        const int2 dr = pref[yi.x + yi.y - (int)old];
                        next = dr.x;
                        nextk = rinfo[dr.x].y - dr.y + 1;
                    }
                    break;
                }
            }
            cur = next;
            k = nextk;
        }
    }
}

// The same suitor with 64-bit offer words [offer value (16 bits) | last (1) | position p (47)],
// for rows of fewer than 65536 entries: p is the proposer's record in pref (row[v] + its list
// index) and `last` marks the proposer's last candidate. Offer values at y differ between
// proposers, so atomicMax orders the words as it orders the offer values and the matching is the
// same; but the word a proposal displaces holds the old suitor's position, so the displaced
// vertex resumes at record p + 1 with one load (no lookup of its row), and the proposal needs no
// load of the current offer first. Each step of a displacement chain is then two dependent memory
// operations (preference record, atomic); the record after the current one is requested before
// the atomic, so a refused proposal costs the atomic's round trip alone.
__global__ void k_suitor_w(int n, const int2* __restrict__ rinfo, const int2* __restrict__ pref,
    unsigned long long* offer, long long budget, int* err, int descending)
{
    constexpr unsigned long long kPosMask = (1ull << 47) - 1;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const int v = descending ? (int)(n - 1 - t) : (int)t;
        const int2 vi = __ldg(rinfo + v);
        if (vi.y <= 0) continue;
        long long p = vi.x;
        long long steps = 0;
        int2 nxt = __ldg(pref + p);
        while (true) {
            if (++steps > budget) {
                atomicOr(err, ERR_SUITOR_BUDGET);
                return;
            }
            const int2 pr = nxt;
            const bool last = (pr.y & kPrefLast) != 0;
            if (!last) nxt = __ldg(pref + p + 1);
            const unsigned ov = (unsigned)pr.y & 0xffffu;
            if (ov != 0u) {
                const unsigned long long mine = ((unsigned long long)ov << 48) |
                    (last ? (1ull << 47) : 0ull) | (unsigned long long)p;
                const unsigned long long old = atomicMax(offer + pr.x, mine);
                if (old < mine) {
                    // accepted: the displaced suitor (if any, and if it has candidates left) walks on
                    if (old == 0ull || ((old >> 47) & 1ull)) break;
                    p = (long long)(old & kPosMask) + 1;
                    nxt = __ldg(pref + p);
                    continue;
                }
            }
            if (last) break;
            p++;
        }
    }
}

// M[y] = the suitor v of y: its offer value degE[y] - (rank of v in y's list) names v's place in
// y's own list, whose record holds v.
__global__ void k_suitor_result_w(int n, const int2* __restrict__ rinfo, const int2* __restrict__ pref,
    const unsigned long long* __restrict__ offer, int* __restrict__ M)
{
    for (long y = (long)blockIdx.x * blockDim.x + threadIdx.x; y < n; y += (long)gridDim.x * blockDim.x) {
        const unsigned long long o = offer[y];
        const int2 yi = rinfo[y];
        M[y] = o ? __ldg(pref + yi.x + yi.y - (int)(o >> 48)).x : -1;
    }
}

// M[y] = suitor of y, or -1 (the suitors array the reference returns, suitor.cu:303-329).
__global__ void k_suitor_result(int n, const int2* __restrict__ rinfo, const int2* __restrict__ pref,
    const unsigned* __restrict__ offer, int* __restrict__ M)
{
    for (long y = (long)blockIdx.x * blockDim.x + threadIdx.x; y < n; y += (long)gridDim.x * blockDim.x) {
        const unsigned o = offer[y];
        const int2 yi = rinfo[y];
        M[y] = o ? pref[yi.x + yi.y - (int)o].x : -1;
    }
}

__global__ void k_check_symmetric(int n, const int* __restrict__ M, int* err)
{
    for (long v = (long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long)gridDim.x * blockDim.x) {
        const int u = M[v];
        if (u >= 0 && (u >= n || M[u] != (int)v)) atomicOr(err, ERR_ASYM_MATCH);
    }
}

// ------------------------------------------------------------------------------------------
// pairwise prolongator (makeP_GPU) and coarse weights
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double pair_norm(double a, double b)
{
    return __dsqrt_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)));
}

// A matched pair whose ||(w_v, w_u)|| > DBL_EPSILON is an aggregate with master min(v,u)
// (_aggregate_symmetric_unsorted, matchingPairAggregation.cu:47-79); every other vertex with
// |w| > DBL_EPSILON is a singleton (_aggregate_symmetric_step_two, :24-45).
__global__ void k_pair_flags(int n, const int* __restrict__ M, const double* __restrict__ w, int* __restrict__ fm,
    int* __restrict__ fs, int* err)
{
    for (long v = (long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long)gridDim.x * blockDim.x) {
        const int u = M[v];
        bool inpair = false;
        if (u >= 0) inpair = pair_norm(w[v], w[u]) > DBL_EPSILON;
        fm[v] = (inpair && v < u) ? 1 : 0;
        const bool good_single = !inpair && fabs(w[v]) > DBL_EPSILON;
        fs[v] = good_single ? 1 : 0;
        if (!inpair && !good_single) atomicOr(err, ERR_BADW);
    }
}

// Column/value of every row of P, the fine rows of every aggregate and the coarse weights
// w_c = R w (shifted_CSRVector_product_adaptive_miniwarp2, CSR.cu:1195-1255). Pairs take ids
// 0..npairs-1 in master order (cub::DeviceSelect, matchingPairAggregation.cu:127-148);
// singletons follow in vertex order (the makePCol_CPU order, matchingAggregation.cu:62-87).
__global__ void k_make_p(int n, const int* __restrict__ M, const double* __restrict__ w, const int* __restrict__ fm,
    const int* __restrict__ pofs, const int* __restrict__ sofs, int npairs, int* __restrict__ agg, double* __restrict__ p,
    int* __restrict__ fine0, int* __restrict__ fine1, double* __restrict__ wc)
{
    for (long v = (long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long)gridDim.x * blockDim.x) {
        const int u = M[v];
        const double wv = w[v];
        if (fm[v]) {
            const int id = pofs[v];
            const double wu = w[u];
            const double nrm = pair_norm(wv, wu);
            const double pv = __ddiv_rn(wv, nrm), pu = __ddiv_rn(wu, nrm);
            agg[v] = id;
            agg[u] = id;
            p[v] = pv;
            p[u] = pu;
            fine0[id] = (int)v;
            fine1[id] = u;
            wc[id] = __dadd_rn(__dmul_rn(pv, wv), __dmul_rn(pu, wu));
        } else {
            bool inpair = (u >= 0) && pair_norm(wv, w[u]) > DBL_EPSILON;
            if (!inpair) {
                const int id = npairs + sofs[v];
                const double pv = __ddiv_rn(wv, fabs(wv));
                agg[v] = id;
                p[v] = pv;
                fine0[id] = (int)v;
                fine1[id] = -1;
                wc[id] = __dmul_rn(pv, wv);
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// Galerkin product C = P^T A P for a pairwise P
// ------------------------------------------------------------------------------------------
// One warp per coarse row I with fine rows f0 (< f1). Every entry a_ij of the fine rows gives
// the rounded product t = a_ij p_j under key (J = agg(j), source row, position). After a rank
// sort by key, each group of equal J is (AP)_{f0,J} = sum of its f0 terms and (AP)_{f1,J}
// likewise (<= 2 terms each), and C_IJ = p_f0 (AP)_{f0,J} + p_f1 (AP)_{f1,J}: the values
// nsparse forms for A*P and then R*(AP) (kernel_spgemm_hash_d.cu:792-799), since a sum of at most
// two rounded terms does not depend on their order. Row I is written from off[I] (the prefix sum
// of the rows' candidate counts, which bound their lengths) and its length at Crow[I]; a
// compaction then forms the CSR matrix. cap is the candidates a warp's shared memory holds: a
// row with more is appended to long_rows (for a second launch with room for it, over that list:
// rows = long_rows, nc its length), or flagged as an error when long_rows is NULL.
// Rank sort of a coarse row's distinct 32-bit keys (k_galerkin's narrow form): lane l ranks keys
// l, l + 32, ... (NS of them) against all cnt keys in one pass of broadcast reads, and writes each
// key and its product to its sorted slot.
template <int NS>
__device__ __forceinline__ void gal_rank_pass(const unsigned* key32, const double* tv, int cnt, int lane,
    unsigned* skey32, double* sval)
{
    unsigned kt[NS];
    int pos[NS];
#pragma unroll
    for (int i = 0; i < NS; i++) {
        kt[i] = lane + 32 * i < cnt ? key32[lane + 32 * i] : 0xffffffffu;
        pos[i] = 0;
    }
#pragma unroll 4
    for (int u = 0; u < cnt; u++) {
        const unsigned ku = key32[u];
#pragma unroll
        for (int i = 0; i < NS; i++) pos[i] += ku < kt[i] ? 1 : 0;
    }
#pragma unroll
    for (int i = 0; i < NS; i++)
        if (lane + 32 * i < cnt) {
            skey32[pos[i]] = kt[i];
            sval[pos[i]] = tv[lane + 32 * i];
        }
}

__global__ void k_galerkin(int nc, const int* __restrict__ rows, const int* __restrict__ fine0, const int* __restrict__ fine1,
    const int* __restrict__ agg, const double* __restrict__ p, const int4* __restrict__ span, const int* __restrict__ Acol,
    const double* __restrict__ Aval, const int* __restrict__ off, long long out_cap, int* __restrict__ Crow,
    int* __restrict__ Ccol, double* __restrict__ Cval, int cap, int* __restrict__ long_rows, int* __restrict__ nlong,
    int* __restrict__ long_max, int* err, int ncols)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int wpb = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long* key = (unsigned long long*)smem + (size_t)wid * cap;
    double* tv = (double*)(smem + (size_t)wpb * cap * 8) + (size_t)wid * cap;
    int* sidx = (int*)(smem + (size_t)wpb * cap * 16) + (size_t)wid * cap;
    // the 32-bit-key form keeps its keys and sorted keys in the warp's key[] bytes, its products in
    // tv and the sorted products in a region of its own after sidx (warps of a block may take
    // different forms at the same time)
    unsigned* key32 = (unsigned*)key;
    unsigned* skey32 = key32 + cap;
    double* sval = (double*)(smem + (size_t)wpb * cap * 20) + (size_t)wid * cap;
    const bool narrow = ncols < (1 << 25);   // every J = agg(c) < ncols fits the 32-bit key
    for (long k = (long)blockIdx.x * wpb + wid; k < nc; k += (long)gridDim.x * wpb) {
        const int I = rows ? rows[k] : (int)k;
        const int f0 = fine0[I], f1 = fine1[I];
        const int4 sp = __ldg(span + I);
        const int b0 = sp.x, d0 = sp.y, b1 = sp.z, d1 = sp.w;
        const int cnt = d0 + d1;
        // the fine rows' prolongator values, requested before the row's entries and used last
        const double p0 = p[f0], p1 = f1 >= 0 ? p[f1] : 0.0;
        if (off[I] < 0 || (long long)off[I] + cnt > out_cap) {
            if (lane == 0) {
                atomicOr(err, ERR_GALERKIN_OFS);
                Crow[I] = 0;
            }
            continue;
        }
        if (cnt > cap) {
            if (lane == 0) {
                if (long_rows) {
                    long_rows[atomicAdd(nlong, 1)] = I;
                    atomicMax(long_max, cnt);
                } else {
                    atomicOr(err, ERR_GALERKIN_CAP);
                }
            }
            continue;
        }
        if (narrow && cnt <= 128) {
            // keys (J << 7) | t are distinct and order like (J, source row, position): a 32-bit
            // rank sort that writes each key and its product straight to its sorted slot
            for (int t = lane; t < cnt; t += 32) {
                const int j = t < d0 ? b0 + t : b1 + (t - d0);
                const int c = Acol[j];
                key32[t] = ((unsigned)agg[c] << 7) | (unsigned)t;
                tv[t] = __dmul_rn(Aval[j], p[c]);
            }
            __syncwarp();
            // when both fine rows' aggregate ids ascend along the row (the first sweep of a level
            // numbers pairs by master id), their key lists are sorted: a merge places every key
            bool asc = true;
            for (int t = lane; t + 1 < cnt; t += 32)
                if (t + 1 != d0 && (key32[t] >> 7) > (key32[t + 1] >> 7)) asc = false;
            if (__all_sync(0xffffffffu, asc)) {
                for (int t = lane; t < cnt; t += 32) {
                    const unsigned kt = key32[t];
                    const unsigned* other = t < d0 ? key32 + d0 : key32;
                    int lo = 0, hi = t < d0 ? cnt - d0 : d0;
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (other[mid] < kt) lo = mid + 1;
                        else hi = mid;
                    }
                    const int pos = (t < d0 ? t : t - d0) + lo;
                    skey32[pos] = kt;
                    sval[pos] = tv[t];
                }
            } else {
            // rank sort: each lane ranks its (up to 4) keys in one pass over the row's keys
            switch ((cnt + 31) >> 5) {
            case 1: gal_rank_pass<1>(key32, tv, cnt, lane, skey32, sval); break;
            case 2: gal_rank_pass<2>(key32, tv, cnt, lane, skey32, sval); break;
            case 3: gal_rank_pass<3>(key32, tv, cnt, lane, skey32, sval); break;
            default: gal_rank_pass<4>(key32, tv, cnt, lane, skey32, sval); break;
            }
            }
            __syncwarp();
            const long outbase = off[I];
            int nheads = 0;
            for (int base = 0; base < cnt; base += 32) {
                const int sidx0 = base + lane;
                bool head = false;
                int J = -1;
                if (sidx0 < cnt) {
                    J = (int)(skey32[sidx0] >> 7);
                    head = (sidx0 == 0) || ((int)(skey32[sidx0 - 1] >> 7) != J);
                }
                const unsigned hm = __ballot_sync(0xffffffffu, head);
                if (head) {
                    double ap0 = 0.0, ap1 = 0.0;
                    int n0 = 0, n1 = 0;
                    for (int g = sidx0; g < cnt; g++) {
                        const unsigned kk = skey32[g];
                        if ((int)(kk >> 7) != J) break;
                        const double tt = sval[g];
                        if ((int)(kk & 127u) < d0) {
                            ap0 = n0 == 0 ? tt : __dadd_rn(ap0, tt);
                            n0++;
                        } else {
                            ap1 = n1 == 0 ? tt : __dadd_rn(ap1, tt);
                            n1++;
                        }
                    }
                    double cv;
                    if (n0 && n1) cv = __dadd_rn(__dmul_rn(p0, ap0), __dmul_rn(p1, ap1));
                    else if (n0) cv = __dmul_rn(p0, ap0);
                    else cv = __dmul_rn(p1, ap1);
                    const long o = outbase + nheads + __popc(hm & ((1u << lane) - 1u));
                    Ccol[o] = J;
                    Cval[o] = cv;
                }
                nheads += __popc(hm);
            }
            if (lane == 0) Crow[I] = nheads;
            __syncwarp();
            continue;
        }
        for (int t = lane; t < cnt; t += 32) {
            const int j = t < d0 ? b0 + t : b1 + (t - d0);
            const int c = Acol[j];
            const unsigned src = t < d0 ? 0u : 1u;
            key[t] = ((unsigned long long)(unsigned)agg[c] << 32) | ((unsigned long long)src << 31) | (unsigned)t;
            tv[t] = __dmul_rn(Aval[j], p[c]);
        }
        __syncwarp();
        for (int t = lane; t < cnt; t += 32) {
            const unsigned long long kt = key[t];
            int pos = 0;
            for (int u = 0; u < cnt; u++) pos += key[u] < kt ? 1 : 0;
            sidx[pos] = t;
        }
        __syncwarp();
        const long outbase = off[I];
        int nheads = 0;
        for (int base = 0; base < cnt; base += 32) {
            const int s = base + lane;
            bool head = false;
            int J = -1;
            if (s < cnt) {
                J = (int)(key[sidx[s]] >> 32);
                head = (s == 0) || ((int)(key[sidx[s - 1]] >> 32) != J);
            }
            const unsigned hm = __ballot_sync(0xffffffffu, head);
            if (head) {
                double ap0 = 0.0, ap1 = 0.0;
                int n0 = 0, n1 = 0;
                for (int g = s; g < cnt; g++) {
                    const unsigned long long kk = key[sidx[g]];
                    if ((int)(kk >> 32) != J) break;
                    const double tt = tv[sidx[g]];
                    if (((kk >> 31) & 1ull) == 0) {
                        ap0 = n0 == 0 ? tt : __dadd_rn(ap0, tt);
                        n0++;
                    } else {
                        ap1 = n1 == 0 ? tt : __dadd_rn(ap1, tt);
                        n1++;
                    }
                }
                double cv;
                if (n0 && n1) cv = __dadd_rn(__dmul_rn(p0, ap0), __dmul_rn(p1, ap1));
                else if (n0) cv = __dmul_rn(p0, ap0);
                else cv = __dmul_rn(p1, ap1);
                const long o = outbase + nheads + __popc(hm & ((1u << lane) - 1u));
                Ccol[o] = J;
                Cval[o] = cv;
            }
            nheads += __popc(hm);
        }
        if (lane == 0) Crow[I] = nheads;
        __syncwarp();
    }
}

// Coarse rows longer than a warp's shared memory holds: their candidates in global memory, one
// block per row, the (J, source row, position) keys of k_galerkin at seg[k] onwards.
__global__ void k_galerkin_long_fill(int nrows, const int* __restrict__ rows, const int* __restrict__ fine0,
    const int* __restrict__ fine1, const int* __restrict__ agg, const double* __restrict__ p, const int* __restrict__ Arow,
    const int* __restrict__ Acol, const double* __restrict__ Aval, const int* __restrict__ seg,
    unsigned long long* __restrict__ key, double* __restrict__ tv)
{
    for (int k = blockIdx.x; k < nrows; k += gridDim.x) {
        const int I = rows[k];
        const int f0 = fine0[I], f1 = fine1[I];
        const int b0 = Arow[f0], d0 = Arow[f0 + 1] - b0;
        const int b1 = f1 >= 0 ? Arow[f1] : 0, d1 = f1 >= 0 ? Arow[f1 + 1] - b1 : 0;
        const long o = seg[k];
        for (int t = threadIdx.x; t < d0 + d1; t += blockDim.x) {
            const int j = t < d0 ? b0 + t : b1 + (t - d0);
            const int c = Acol[j];
            const unsigned src = t < d0 ? 0u : 1u;
            key[o + t] = ((unsigned long long)(unsigned)agg[c] << 32) | ((unsigned long long)src << 31) | (unsigned)t;
            tv[o + t] = __dmul_rn(Aval[j], p[c]);
        }
    }
}

// The long rows' sorted candidates -> their entries of C, with k_galerkin's sums: one block per
// row walks its candidates in chunks of blockDim, marks the first of every J, and numbers the
// marks by a block-wide scan of the warps' ballots.
__global__ void __launch_bounds__(1024) k_galerkin_long_rows(int nrows, const int* __restrict__ rows,
    const int* __restrict__ fine0, const int* __restrict__ fine1, const double* __restrict__ p, const int* __restrict__ seg,
    const unsigned long long* __restrict__ key, const double* __restrict__ tv, const int* __restrict__ off,
    int* __restrict__ Crow, int* __restrict__ Ccol, double* __restrict__ Cval)
{
    __shared__ int wsum[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = blockIdx.x; k < nrows; k += gridDim.x) {
        const int I = rows[k];
        const int f0 = fine0[I], f1 = fine1[I];
        const long o = seg[k];
        const int cnt = seg[k + 1] - seg[k];
        const double p0 = p[f0], p1 = f1 >= 0 ? p[f1] : 0.0;
        int nheads = 0;
        for (int base = 0; base < cnt; base += blockDim.x) {
            const int g = base + threadIdx.x;
            bool head = false;
            int J = -1;
            if (g < cnt) {
                J = (int)(key[o + g] >> 32);
                head = g == 0 || (int)(key[o + g - 1] >> 32) != J;
            }
            const unsigned hm = __ballot_sync(0xffffffffu, head);
            if (lane == 0) wsum[wid] = __popc(hm);
            __syncthreads();
            int before = 0, chunk = 0;
            for (int w = 0; w < nw; w++) {
                before += w < wid ? wsum[w] : 0;
                chunk += wsum[w];
            }
            if (head) {
                double ap0 = 0.0, ap1 = 0.0;
                int n0 = 0, n1 = 0;
                for (int h = g; h < cnt; h++) {
                    const unsigned long long kk = key[o + h];
                    if ((int)(kk >> 32) != J) break;
                    const double tt = tv[o + h];
                    if (((kk >> 31) & 1ull) == 0) {
                        ap0 = n0 == 0 ? tt : __dadd_rn(ap0, tt);
                        n0++;
                    } else {
                        ap1 = n1 == 0 ? tt : __dadd_rn(ap1, tt);
                        n1++;
                    }
                }
                double cv;
                if (n0 && n1) cv = __dadd_rn(__dmul_rn(p0, ap0), __dmul_rn(p1, ap1));
                else if (n0) cv = __dmul_rn(p0, ap0);
                else cv = __dmul_rn(p1, ap1);
                const long d = (long)off[I] + nheads + before + __popc(hm & ((1u << lane) - 1u));
                Ccol[d] = J;
                Cval[d] = cv;
            }
            nheads += chunk;
            __syncthreads();
        }
        if (threadIdx.x == 0) Crow[I] = nheads;
    }
}

// Candidate count of each listed row (as k_galerkin_counts, over a list).
__global__ void k_galerkin_list_counts(int nrows, const int* __restrict__ rows, const int* __restrict__ fine0,
    const int* __restrict__ fine1, const int* __restrict__ Arow, int* __restrict__ cnt)
{
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < nrows; k += (long)gridDim.x * blockDim.x) {
        const int I = rows[k];
        const int f0 = fine0[I], f1 = fine1[I];
        cnt[k] = (Arow[f0 + 1] - Arow[f0]) + (f1 >= 0 ? Arow[f1 + 1] - Arow[f1] : 0);
    }
}

// Number of candidate entries of every coarse row: the entries of its fine rows.
// cnt[I]: the candidate entries of coarse row I (its fine rows' entries); span[I]: the first entry
// and the length of each fine row (b0, d0, b1, d1), so that the product kernel finds them with one
// load instead of two dependent ones
__global__ void k_galerkin_counts(int nc, const int* __restrict__ fine0, const int* __restrict__ fine1,
    const int* __restrict__ Arow, int* __restrict__ cnt, int4* __restrict__ span)
{
    for (long I = (long)blockIdx.x * blockDim.x + threadIdx.x; I < nc; I += (long)gridDim.x * blockDim.x) {
        const int f0 = fine0[I], f1 = fine1[I];
        const int b0 = Arow[f0], d0 = Arow[f0 + 1] - b0;
        const int b1 = f1 >= 0 ? Arow[f1] : 0, d1 = f1 >= 0 ? Arow[f1 + 1] - b1 : 0;
        cnt[I] = d0 + d1;
        span[I] = make_int4(b0, d0, b1, d1);
    }
}

// rows written from off[I] -> CSR; 8 lanes per row (4 rows of a warp in flight), each lane
// moving up to 4 entries per round with all of their loads issued first
__global__ void k_compact_rows(int nc, const int* __restrict__ off, const int* __restrict__ rowptr, const int* __restrict__ pcol,
    const double* __restrict__ pval, int* __restrict__ col, double* __restrict__ val, int* __restrict__ dpos)
{
    constexpr int S = 8, U = 4;
    const int lane = threadIdx.x & (S - 1);
    for (long I = ((long)blockIdx.x * blockDim.x + threadIdx.x) / S; I < nc; I += (long)gridDim.x * blockDim.x / S) {
        const int b = __ldg(rowptr + I), len = __ldg(rowptr + I + 1) - b;
        const long o = __ldg(off + I);
        for (int t0 = lane; t0 < len; t0 += U * S) {
            int c[U];
            double v[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int t = t0 + u * S;
                c[u] = t < len ? __ldcs(pcol + o + t) : 0;
                v[u] = t < len ? __ldcs(pval + o + t) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int t = t0 + u * S;
                if (t < len) {
                    col[b + t] = c[u];
                    val[b + t] = v[u];
                    if (c[u] == (int)I) dpos[I] = b + t;
                }
            }
        }
    }
}

// composite prolongator of the level: P <- P * P_sweep (one entry per row in both).
__global__ void k_compose(int n, int* __restrict__ agg, double* __restrict__ p, const int* __restrict__ agg_s,
    const double* __restrict__ p_s, int first)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        if (first) {
            agg[i] = agg_s[i];
            p[i] = p_s[i];
        } else {
            const int c = agg[i];
            p[i] = __dmul_rn(p[i], p_s[c]);
            agg[i] = agg_s[c];
        }
    }
}

// R = P^T as CSR: counting sort of the rows by aggregate, rows ascending inside.
__global__ void k_count(int n, const int* __restrict__ agg, int* cnt)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) atomicAdd(cnt + agg[i], 1);
}
__global__ void k_scatter(int n, const int* __restrict__ agg, const int* __restrict__ rptr, int* fillpos, int* __restrict__ ridx)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int c = agg[i];
        ridx[rptr[c] + atomicAdd(fillpos + c, 1)] = (int)i;
    }
}
__global__ void k_sort_rrows(int nc, const int* __restrict__ rptr, int* __restrict__ ridx, const double* __restrict__ p,
    double* __restrict__ rval, float* __restrict__ rval32)
{
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (long)gridDim.x * blockDim.x) {
        const int b = rptr[c], e = rptr[c + 1];
        for (int i = b + 1; i < e; i++) {
            const int v = ridx[i];
            int j = i - 1;
            while (j >= b && ridx[j] > v) {
                ridx[j + 1] = ridx[j];
                j--;
            }
            ridx[j + 1] = v;
        }
        for (int i = b; i < e; i++) {
            const double pv = p[ridx[i]];
            rval[i] = pv;
            if (rval32) rval32[i] = (float)pv;
        }
    }
}

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
static std::string err_text(int e)
{
    std::string s;
    if (e & ERR_ROW0) s += "row[0] != 0; ";
    if (e & ERR_ROWN) s += "row[n] != nnz; ";
    if (e & ERR_ROWORDER) s += "row offsets decrease or exceed nnz; ";
    if (e & ERR_COLRANGE) s += "column index out of range; ";
    if (e & ERR_COLSORT) s += "columns not strictly ascending in a row; ";
    if (e & ERR_NODIAG) s += "a row has no diagonal entry; ";
    if (e & ERR_SUITOR_BUDGET) s += "suitor matching exceeded its iteration bound; ";
    if (e & ERR_ASYM_MATCH) s += "matching is not symmetric; ";
    if (e & ERR_BADW) s += "weight vector entry <= DBL_EPSILON; ";
    if (e & ERR_GALERKIN_CAP) s += "Galerkin row exceeds its shared-memory capacity; ";
    if (e & ERR_GALERKIN_OFS) s += "Galerkin candidates exceed the fine matrix's entries; ";
    return s;
}

static int read_err(const int* err, cudaStream_t s)
{
    int e = 0;
    BCMGX_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaStreamSynchronize(s));
    return e;
}

static int row_max_raw(int n, const int* row, cudaStream_t s)
{
    DBuf<int> mx;
    mx.alloc(1, s);
    BCMGX_CUDA(cudaMemsetAsync(mx.p, 0, sizeof(int), s));
    note_launch(); k_row_max<<<gs_grid(n), 256, 0, s>>>(n, row, mx.p);
    BCMGX_CHECK_LAUNCH();
    return read_err(mx.p, s);
}
static int row_max(const DevCsr& A, cudaStream_t s) { return row_max_raw(A.n, A.row.p, s); }

__global__ void k_set_u64(unsigned long long* p, unsigned long long v) { *p = v; }

// SUITOR_EPS / (0.999 min |a_hat|) on the device, with the host form's operations (edge_prep_dev):
// the minimum capped by min_cap and raised to DBL_EPSILON (toMaximumProductMatrix,
// matching.cu:243-245)
__global__ void k_zero_sub(const unsigned long long* min_bits, double min_cap, double* out)
{
    double m = __longlong_as_double((long long)*min_bits);
    m = fmin(m, min_cap);
    if (fabs(m) < DBL_EPSILON) m = DBL_EPSILON;
    *out = __ddiv_rn(kSuitorEps, __dmul_rn(0.999, m));
}

// The inputs of the edge weights: C_r (into C, n doubles), the transposed positions and the
// substitute log argument SUITOR_EPS / (0.999 min |a_hat|) for a_hat == 0; returns it and, when
// min_out_host is set, the minimum.
// min_cap: an upper bound of the minimum (a rank of a row-partitioned set-up that has entries
// outside its own columns takes 99999, makeAH's value for them, into its minimum).
static double edge_prep_dev(int n, int64_t nnz, const int* row, const int* col, const double* val, const double* w,
    double* C, int* tpos, double* min_out_host, cudaStream_t s, double min_cap = DBL_MAX)
{
    DBuf<unsigned long long> mn;
    DBuf<int> err;
    mn.alloc(1, s);
    err.alloc(1, s);
    BCMGX_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    const double dmax = DBL_MAX;
    BCMGX_CUDA(cudaMemcpyAsync(mn.p, &dmax, sizeof(double), cudaMemcpyHostToDevice, s));
    const int S = setup_subwarp(n, nnz);
    note_launch(); k_diag_c<<<gs_grid(n), 256, 0, s>>>(n, row, col, val, w, C, err.p);
    tpos_min_launch(S, n, row, col, tpos, val, w, C, mn.p, s);
    BCMGX_CHECK_LAUNCH();
    double m = 0;
    BCMGX_CUDA(cudaMemcpyAsync(&m, mn.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    int e = read_err(err.p, s);
    if (e) throw Error(BCMGX_ERR_INVALID_INPUT, "edge weights: " + err_text(e));
    m = std::min(m, min_cap);
    if (std::fabs(m) < DBL_EPSILON) m = DBL_EPSILON;   // toMaximumProductMatrix, matching.cu:243-245
    if (min_out_host) *min_out_host = m;
    return kSuitorEps / (0.999 * m);
}

void edge_weights_dev(int n, int64_t nnz, const int* row, const int* col, const double* val, const double* w, double* W,
    int* tpos, double* min_out_host, cudaStream_t s)
{
    DBuf<double> C;
    C.alloc(n, s);
    const double zero_sub = edge_prep_dev(n, nnz, row, col, val, w, C.p, tpos, min_out_host, s);
    BCMGX_SUBWARP_LAUNCH(k_logw, setup_subwarp(n, nnz), n, s, n, row, col, val, w, C.p, tpos, zero_sub, W);
    BCMGX_CHECK_LAUNCH();
}

void validate_csr_dev(int n, int m, int64_t nnz, const int* row, const int* col, bool need_diag, cudaStream_t s)
{
    DBuf<int> err, mx;
    err.alloc(1, s);
    mx.alloc(1, s);
    BCMGX_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    BCMGX_CUDA(cudaMemsetAsync(mx.p, 0, sizeof(int), s));
    note_launch();
    k_validate<<<warp_grid(n), 256, 0, s>>>(n, m, nnz, row, col, err.p, mx.p, need_diag ? 1 : 0);
    BCMGX_CHECK_LAUNCH();
    const int e = read_err(err.p, s);
    if (e) throw Error(BCMGX_ERR_INVALID_INPUT, "input matrix: " + err_text(e));
}

void tpos_dev(int n, int64_t nnz, const int* row, const int* col, int* tpos, cudaStream_t s)
{
    BCMGX_SUBWARP_LAUNCH2(k_tpos, 0, setup_subwarp(n, nnz), n, s, n, row, col, tpos, nullptr, nullptr, nullptr,
        nullptr);
    BCMGX_CHECK_LAUNCH();
}

void suitor_dev(int n, int64_t nnz, const int* row, const int* col, const double* W, const int* tpos, int* M, int max_row,
    cudaStream_t s, const FusedWeights* fw, int* err_out)
{
    if (max_row <= 0) max_row = row_max_raw(n, row, s);
    if (fw && max_row > 32) throw Error(BCMGX_ERR_INTERNAL, "weights formed in the rank kernel need rows of <= 32 entries");
    const bool wide = max_row < 65536;
    DBuf<int> rank, degE, err;
    DBuf<int2> pref, rinfo;
    DBuf<unsigned> offer;
    DBuf<unsigned long long> offer_w;
    const int64_t z = std::max<int64_t>(nnz, 1);
    rank.alloc(z, s);
    degE.alloc(n, s);
    if (!err_out) {
        err.alloc(1, s);
        BCMGX_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    }
    int* errp = err_out ? err_out : err.p;
    if (wide) {
        offer_w.alloc(n, s);
        BCMGX_CUDA(cudaMemsetAsync(offer_w.p, 0, sizeof(unsigned long long) * n, s));
    } else {
        offer.alloc(n, s);
        BCMGX_CUDA(cudaMemsetAsync(offer.p, 0, sizeof(unsigned) * n, s));
    }
    if (fw) {
        note_launch();
        k_rank_w<<<warp_grid(n), 256, 0, s>>>(n, row, col, fw->val, fw->w, fw->C, tpos, fw->zero_sub, rank.p, degE.p,
            fw->zero_sub_dev);
    } else {
        note_launch(); k_rank<<<warp_grid(n), 256, 0, s>>>(n, row, col, W, rank.p, degE.p);
    }
    pref.alloc(z, s);
    rinfo.alloc(n, s);
    BCMGX_SUBWARP_LAUNCH(k_pref, setup_subwarp(n, nnz), n, s, n, row, col, rank.p, tpos, degE.p, pref.p, rinfo.p,
        wide ? 1 : 0);
    BCMGX_CHECK_LAUNCH();
    rank.release();
    static int asc = -1;
    if (asc < 0) {
        const char* e = std::getenv("BCMGX_SUITOR_ASC");
        asc = (e && std::atoi(e) > 0) ? 1 : 0;
    }
    // steps one proposal chain may take: every vertex's list position only moves forward, so no
    // chain needs more than nnz + n. BCMGX_TEST_SUITOR_BUDGET overrides it (fault-path tests:
    // a budget of 0 makes every chain give up at once and the set-up return BCMGX_ERR_TIMEOUT).
    long long budget = (long long)nnz + n + 1024;
    if (const char* tb = std::getenv("BCMGX_TEST_SUITOR_BUDGET"))
        if (*tb) budget = std::max(0LL, std::atoll(tb));
    if (wide) {
        note_launch(); k_suitor_w<<<ceil_div(n, 128), 128, 0, s>>>(n, rinfo.p, pref.p, offer_w.p, budget, errp, asc ? 0 : 1);
        note_launch(); k_suitor_result_w<<<gs_grid(n), 256, 0, s>>>(n, rinfo.p, pref.p, offer_w.p, M);
    } else {
        note_launch(); k_suitor<<<ceil_div(n, 128), 128, 0, s>>>(n, rinfo.p, pref.p, offer.p, budget, errp, asc ? 0 : 1);
        note_launch(); k_suitor_result<<<gs_grid(n), 256, 0, s>>>(n, rinfo.p, pref.p, offer.p, M);
    }
    note_launch(); k_check_symmetric<<<gs_grid(n), 256, 0, s>>>(n, M, errp);
    BCMGX_CHECK_LAUNCH();
    if (err_out) return;
    int e = read_err(err.p, s);
    if (e) throw Error(e & ERR_SUITOR_BUDGET ? BCMGX_ERR_TIMEOUT : BCMGX_ERR_INTERNAL, "suitor matching: " + err_text(e));
}

// One pairwise sweep on A (weights w): matching, prolongator, Galerkin product, coarse weights.
struct SweepOut {
    DevCsr C;
    DBuf<int> agg;
    DBuf<double> p, wc;
    int nc = 0;
};

// The matching and the pairwise prolongator of one sweep on the square matrix A with weights w:
// agg/p per row of A (aggregate ids 0..nc-1, pairs by master then singletons), the fine rows of
// every aggregate (fine0, fine1; -1 for a singleton) and the coarse weights wc = R w. min_cap
// edge_prep_dev without a host round trip: the substitute goes to *zs_dev, the diagonal check's
// error bits to the caller's error word (read with its next round trip).
static void edge_prep_async(int n, int64_t nnz, const int* row, const int* col, const double* val, const double* w,
    double* C, int* tpos, double* zs_dev, unsigned long long* mn, int* err, cudaStream_t s, double min_cap,
    const int* dpos = nullptr)
{
    const int S = setup_subwarp(n, nnz);
    note_launch(); k_set_u64<<<1, 1, 0, s>>>(mn, (unsigned long long)__builtin_bit_cast(long long, DBL_MAX));
    if (dpos) {
        note_launch(); k_diag_c_pos<<<gs_grid(n), 256, 0, s>>>(n, dpos, val, w, C, err);
    } else {
        note_launch(); k_diag_c<<<gs_grid(n), 256, 0, s>>>(n, row, col, val, w, C, err);
    }
    tpos_min_launch(S, n, row, col, tpos, val, w, C, mn, s);
    note_launch(); k_zero_sub<<<1, 1, 0, s>>>(mn, min_cap, zs_dev);
    BCMGX_CHECK_LAUNCH();
}

// bounds the edge weights' minimum (edge_prep_dev).
void sweep_aggregate(bcmgx_hierarchy* H, const DevCsr& A, const double* w, SweepAgg& out, int level, int sweep,
    double min_cap)
{
    cudaStream_t s = H->stream;
    const int n = A.n;
    const int64_t nnz = A.nnz;
    DBuf<double> W, Cd;
    DBuf<int> tpos, M, fm, fs, pofs, sofs, err;
    tpos.alloc(std::max<int64_t>(nnz, 1), s);
    M.alloc(n, s);
    // one error word for the matching and the aggregation, read with the pair / singleton totals
    err.alloc(1, s);
    BCMGX_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    const int amax0 = A.max_row > 0 ? A.max_row : row_max(A, s);
    // the substitute weight and the minimum it comes from stay on the device (no round trip)
    DBuf<double> zs;
    DBuf<unsigned long long> mn;
    zs.alloc(1, s);
    mn.alloc(1, s);
    if (amax0 <= 32) {
        // rows of at most 32 entries: the rank kernel forms the edge weights itself
        Cd.alloc(n, s);
        FusedWeights fw;
        {
            PhaseTimer pt(H, "weights");
            edge_prep_async(n, nnz, A.row.p, A.col.p, A.val.p, w, Cd.p, tpos.p, zs.p, mn.p, err.p, s, min_cap, A.dpos.p);
        }
        fw.val = A.val.p;
        fw.w = w;
        fw.C = Cd.p;
        fw.zero_sub_dev = zs.p;
        PhaseTimer pt(H, "suitor");
        suitor_dev(n, nnz, A.row.p, A.col.p, nullptr, tpos.p, M.p, amax0, s, &fw, err.p);
    } else {
        W.alloc(std::max<int64_t>(nnz, 1), s);
        {
            PhaseTimer pt(H, "weights");
            DBuf<double> C;
            C.alloc(n, s);
            edge_prep_async(n, nnz, A.row.p, A.col.p, A.val.p, w, C.p, tpos.p, zs.p, mn.p, err.p, s, min_cap, A.dpos.p);
            BCMGX_SUBWARP_LAUNCH(k_logw, setup_subwarp(n, nnz), n, s, n, A.row.p, A.col.p, A.val.p, w, C.p, tpos.p,
                0.0, W.p, zs.p);
            BCMGX_CHECK_LAUNCH();
        }
        PhaseTimer pt(H, "suitor");
        suitor_dev(n, nnz, A.row.p, A.col.p, W.p, tpos.p, M.p, amax0, s, nullptr, err.p);
    }
    PhaseTimer pt_p(H, "makeP");
    W.release();
    Cd.release();
    tpos.release();
    fm.alloc(n, s);
    fs.alloc(n, s);
    pofs.alloc(n, s);
    sofs.alloc(n, s);
    note_launch(); k_pair_flags<<<gs_grid(n), 256, 0, s>>>(n, M.p, w, fm.p, fs.p, err.p);
    BCMGX_CHECK_LAUNCH();
    // both scans, then their totals and the error word in one round trip
    DBuf<long long> tots;
    tots.alloc(2, s);
    scan_launch(fm.p, pofs.p, n, false, tots.p, s);
    scan_launch(fs.p, sofs.p, n, false, tots.p + 1, s);
    long long th[2] = { 0, 0 };
    int e = 0;
    BCMGX_CUDA(cudaMemcpyAsync(th, tots.p, 2 * sizeof(long long), cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaStreamSynchronize(s));
    if (e & ERR_NODIAG) throw Error(BCMGX_ERR_INVALID_INPUT, "edge weights: " + err_text(e));
    if (e) throw Error(e & ERR_SUITOR_BUDGET ? BCMGX_ERR_TIMEOUT : BCMGX_ERR_INTERNAL, "aggregation: " + err_text(e));
    const long long npairs = th[0], nsing = th[1];
    const int nc = (int)(npairs + nsing);
    out.nc = nc;
    out.agg.alloc(n, s);
    out.p.alloc(n, s);
    out.wc.alloc(nc, s);
    out.fine0.alloc(nc, s);
    out.fine1.alloc(nc, s);
    note_launch(); k_make_p<<<gs_grid(n), 256, 0, s>>>(n, M.p, w, fm.p, pofs.p, sofs.p, (int)npairs, out.agg.p, out.p.p, out.fine0.p, out.fine1.p, out.wc.p);
    BCMGX_CHECK_LAUNCH();
    if (H->prm.record_sweeps) {
        SweepRecord r;
        r.level = level;
        r.sweep = sweep;
        r.n = n;
        r.nc = nc;
        r.match.resize(n);
        r.agg.resize(n);
        r.p.resize(n);
        r.w.resize(n);
        BCMGX_CUDA(cudaMemcpyAsync(r.match.data(), M.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaMemcpyAsync(r.agg.data(), out.agg.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaMemcpyAsync(r.p.data(), out.p.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaMemcpyAsync(r.w.data(), w, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
        H->rec.push_back(std::move(r));
    }
}

// The Galerkin product C = P^T A P of one sweep: A's rows (columns < A.m), agg/p indexed by A's
// columns with coarse ids < ncols, fine0/fine1 the fine rows of the nc coarse rows of C (rows of
// A). C has nc rows whose columns are agg ids, sorted, and ncols columns.
void galerkin_dev(bcmgx_hierarchy* H, const DevCsr& A, const int* agg, const double* p, const int* fine0,
    const int* fine1, int nc, int ncols, DevCsr& C)
{
    cudaStream_t s = H->stream;
    PhaseTimer pt_g(H, "galerkin");
    DBuf<int> err;
    err.alloc(1, s);
    BCMGX_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    // each coarse row's candidate count (the entries of its fine rows) and their prefix sum, which
    // places the row's output (the counts add up to nnz(A), so the scratch is nnz(A) entries
    // whatever the row lengths); the product of the rows that fit kGalCap candidates per warp,
    // then of the longer ones (listed by the first launch) with one warp per block and shared
    // memory for the longest; then compaction.
    const int amax = A.max_row > 0 ? A.max_row : row_max(A, s);
    constexpr int kGalCap = 512;
    constexpr size_t kGalBytes = 28;   // shared-memory bytes per candidate (keys, products, sort)
    const size_t smem_limit = 200 * 1024;
    const int cap1 = std::min(std::max(2 * amax, 32), kGalCap);
    C.n = nc;
    C.m = ncols;
    C.row.alloc((size_t)nc + 1, s);
    DBuf<int> cand, off, counts, pcol, longr, lstat;
    DBuf<double> pval;
    cand.alloc(std::max(nc, 1), s);
    off.alloc((size_t)nc + 1, s);
    DBuf<int4> span;
    span.alloc(std::max(nc, 1), s);
    note_launch(); k_galerkin_counts<<<gs_grid(nc), 256, 0, s>>>(nc, fine0, fine1, A.row.p, cand.p, span.p);
    BCMGX_CHECK_LAUNCH();
    // the candidates of all coarse rows are entries of A (every row of A is in at most one
    // aggregate); k_galerkin checks each row's range against that before writing
    scan_exclusive_dev(cand.p, off.p, nc, s);
    const long long total = A.nnz;
    cand.release();
    counts.alloc(std::max(nc, 1), s);
    pcol.alloc(std::max<size_t>((size_t)total, 1), s);
    pval.alloc(std::max<size_t>((size_t)total, 1), s);
    const bool may_be_long = 2 * amax > cap1;
    if (may_be_long) {
        longr.alloc(std::max(nc, 1), s);
        lstat.alloc(2, s);
        BCMGX_CUDA(cudaMemsetAsync(lstat.p, 0, 2 * sizeof(int), s));
    }
    // one launch of k_galerkin over `rows` (all coarse rows when NULL) with room for cap candidates
    // per warp; longer rows go to `list` (count and longest in stat[0], stat[1]) when it is given
    auto galerkin = [&](const int* rows, int nrows, int cap, int* list, int* stat) {
        const size_t per_warp = (size_t)cap * kGalBytes;
        const int wpb = (int)std::min<size_t>(8, std::max<size_t>(1, (48 * 1024) / per_warp));
        const size_t smem = per_warp * wpb;
        ensure_smem_limit(k_galerkin, smem);
        const int g = (int)std::max<long>(1, std::min<long>(((long)nrows + wpb - 1) / wpb, (long)num_sms() * 32));
        note_launch();
        k_galerkin<<<g, wpb * 32, smem, s>>>(nrows, rows, fine0, fine1, agg, p, span.p, A.col.p,
            A.val.p, off.p, (long long)total, counts.p, pcol.p, pval.p, cap, list, stat, stat ? stat + 1 : nullptr, err.p,
            ncols);
        BCMGX_CHECK_LAUNCH();
    };
    auto read2 = [&](const int* d, int (&h)[2]) {
        BCMGX_CUDA(cudaMemcpyAsync(h, d, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
    };
    galerkin(nullptr, nc, cap1, may_be_long ? longr.p : nullptr, may_be_long ? lstat.p : nullptr);
    if (may_be_long) {
        int st[2] = { 0, 0 };
        read2(lstat.p, st);
        if (st[0] > 0) {
            const int capmax = (int)(smem_limit / kGalBytes);
            const bool very_long = st[1] > capmax;
            DBuf<int> longr2, lstat2;
            if (very_long) {
                longr2.alloc(st[0], s);
                lstat2.alloc(2, s);
                BCMGX_CUDA(cudaMemsetAsync(lstat2.p, 0, 2 * sizeof(int), s));
            }
            galerkin(longr.p, st[0], std::min(st[1], capmax), very_long ? longr2.p : nullptr,
                very_long ? lstat2.p : nullptr);
            if (very_long) {
                // rows beyond a block's shared memory: candidates in global memory, sorted per row
                // by key with CUB's segmented sort, then summed and written by one block per row
                int st2[2] = { 0, 0 };
                read2(lstat2.p, st2);
                const int n3 = st2[0];
                DBuf<int> cnt3, seg;
                cnt3.alloc(n3, s);
                seg.alloc((size_t)n3 + 1, s);
                note_launch();
                k_galerkin_list_counts<<<gs_grid(n3), 256, 0, s>>>(n3, longr2.p, fine0, fine1, A.row.p, cnt3.p);
                BCMGX_CHECK_LAUNCH();
                const long long total3 = scan_exclusive(cnt3.p, seg.p, n3, true, s);
                DBuf<unsigned long long> k_in, k_out;
                DBuf<double> v_in, v_out;
                k_in.alloc((size_t)total3, s);
                k_out.alloc((size_t)total3, s);
                v_in.alloc((size_t)total3, s);
                v_out.alloc((size_t)total3, s);
                const int g3 = std::min(n3, num_sms() * 4);
                note_launch();
                k_galerkin_long_fill<<<g3, 256, 0, s>>>(n3, longr2.p, fine0, fine1, agg, p, A.row.p,
                    A.col.p, A.val.p, seg.p, k_in.p, v_in.p);
                BCMGX_CHECK_LAUNCH();
                size_t tmp_bytes = 0;
                BCMGX_CUDA(cub::DeviceSegmentedSort::SortPairs(nullptr, tmp_bytes, k_in.p, k_out.p, v_in.p, v_out.p,
                    (int)total3, n3, seg.p, seg.p + 1, s));
                DBuf<unsigned char> tmp;
                tmp.alloc(std::max<size_t>(tmp_bytes, 1), s);
                BCMGX_CUDA(cub::DeviceSegmentedSort::SortPairs(tmp.p, tmp_bytes, k_in.p, k_out.p, v_in.p, v_out.p,
                    (int)total3, n3, seg.p, seg.p + 1, s));
                note_launch();
                k_galerkin_long_rows<<<std::min(n3, num_sms() * 2), 1024, 0, s>>>(n3, longr2.p, fine0, fine1,
                    p, seg.p, k_out.p, v_out.p, off.p, counts.p, pcol.p, pval.p);
                BCMGX_CHECK_LAUNCH();
            }
        }
    }
    // row offsets of C; their total, the longest row and the error word in one round trip
    DBuf<long long> ctot;
    DBuf<int> cmx;
    ctot.alloc(1, s);
    cmx.alloc(1, s);
    BCMGX_CUDA(cudaMemsetAsync(cmx.p, 0, sizeof(int), s));
    scan_launch(counts.p, C.row.p, nc, true, ctot.p, s);
    if (nc > 0) {
        note_launch(); k_row_max<<<gs_grid(nc), 256, 0, s>>>(nc, C.row.p, cmx.p);
        BCMGX_CHECK_LAUNCH();
    }
    long long cnnz = 0;
    int cmax = 0, e = 0;
    BCMGX_CUDA(cudaMemcpyAsync(&cnnz, ctot.p, sizeof(long long), cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaMemcpyAsync(&cmax, cmx.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaStreamSynchronize(s));
    if (e) throw Error(BCMGX_ERR_INTERNAL, "galerkin: " + err_text(e));
    BCMGX_REQUIRE(cnnz <= 0x7fffffffLL, BCMGX_ERR_UNSUPPORTED, "more than 2^31-1 entries (int32 offsets)");
    C.nnz = cnnz;
    C.col.alloc(std::max<int64_t>(C.nnz, 1), s);
    C.val.alloc(std::max<int64_t>(C.nnz, 1), s);
    C.dpos.alloc(std::max(nc, 1), s);
    BCMGX_CUDA(cudaMemsetAsync(C.dpos.p, 0xff, sizeof(int) * (size_t)std::max(nc, 1), s));
    note_launch(); k_compact_rows<<<gs_grid((long)nc * 8), 256, 0, s>>>(nc, off.p, C.row.p, pcol.p, pval.p, C.col.p, C.val.p,
        C.dpos.p);
    BCMGX_CHECK_LAUNCH();
    C.max_row = cmax;
}

static void pairwise_sweep(bcmgx_hierarchy* H, const DevCsr& A, const double* w, SweepOut& out, int level, int sweep)
{
    SweepAgg ag;
    sweep_aggregate(H, A, w, ag, level, sweep, DBL_MAX);
    galerkin_dev(H, A, ag.agg.p, ag.p.p, ag.fine0.p, ag.fine1.p, ag.nc, ag.nc, out.C);
    out.C.m = out.C.n;
    out.nc = ag.nc;
    out.agg = std::move(ag.agg);
    out.p = std::move(ag.p);
    out.wc = std::move(ag.wc);
}

// Largest |col - row| of the matrix (atomicMax of per-thread maxima).
__global__ void k_max_offset(int n, const int* __restrict__ row, const int* __restrict__ col, int* out)
{
    int mx = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        for (int j = row[i]; j < row[i + 1]; j++) mx = max(mx, abs(col[j] - (int)i));
    atomicMax(out, mx);
}

__global__ void k_to_offsets(int n, const int* __restrict__ row, const int* __restrict__ col, short* __restrict__ dcol)
{
    const int lane = threadIdx.x & 31;
    for (long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) / 32; i < n; i += (long)gridDim.x * blockDim.x / 32)
        for (int j = row[i] + lane; j < row[i + 1]; j += 32) dcol[j] = (short)(col[j] - (int)i);
}

// A compact copy of the columns as int16 offsets from the row when every entry lies within
// 32767 of the diagonal: the solve-phase row kernels then stream 2 instead of 4 index bytes per
// entry. BCMGX_INDEX16=0 in the environment keeps int32 columns only.
static void build_offsets(DevCsr& A, cudaStream_t s)
{
    const char* env = std::getenv("BCMGX_INDEX16");
    if (env && env[0] == '0') return;
    if (A.n <= 0 || A.nnz <= 0 || A.dcol.p) return;
    DBuf<int> mx;
    mx.alloc(1, s);
    BCMGX_CUDA(cudaMemsetAsync(mx.p, 0, sizeof(int), s));
    note_launch(); k_max_offset<<<gs_grid(A.n), 256, 0, s>>>(A.n, A.row.p, A.col.p, mx.p);
    BCMGX_CHECK_LAUNCH();
    if (read_err(mx.p, s) > 32767) return;
    A.dcol.alloc(A.nnz, s);
    note_launch(); k_to_offsets<<<warp_grid(A.n), 256, 0, s>>>(A.n, A.row.p, A.col.p, A.dcol.p);
    BCMGX_CHECK_LAUNCH();
}

// ---- value codes (value-indexed CSR) -------------------------------------------------------
// A level whose values take at most kValueCodes distinct FP64 bit patterns (constant-coefficient
// stencils take a handful) stores one byte per entry: the index of its value in a table of them.
// The FP32 table holds the same entries rounded to FP32, so vtab32[vcode[j]] equals the stored
// val32[j]: the coded and the stored forms give the same results bit for bit. Distinct values
// are collected in a hash set of kVcSlots bit patterns (each block first in shared memory, then
// merged into the global set); a block stops as soon as its set passes kValueCodes.
constexpr int kVcSlots = 1024;
constexpr unsigned long long kVcEmpty = ~0ull;   // a NaN pattern; a matrix holding it is not coded
constexpr int64_t kVcMinNnz = 1 << 20;             // smaller levels are launch-bound: no codes

__device__ __forceinline__ unsigned vc_hash(unsigned long long b)
{
    b ^= b >> 33;
    b *= 0xff51afd7ed558ccdULL;
    b ^= b >> 33;
    return (unsigned)b & (kVcSlots - 1);
}

// Inserts bit pattern b into a kVcSlots-slot set (linear probing): 1 when it was new, 0 when it was
// there, -1 when the set is full.
__device__ __forceinline__ int vc_insert(unsigned long long* keys, unsigned long long b)
{
    unsigned h = vc_hash(b);
    for (int probe = 0; probe < kVcSlots; probe++) {
        const unsigned long long k = *(volatile unsigned long long*)(keys + h);
        if (k == b) return 0;
        if (k == kVcEmpty) {
            const unsigned long long old = atomicCAS(keys + h, kVcEmpty, b);
            if (old == kVcEmpty) return 1;
            if (old == b) return 0;
        }
        h = (h + 1) & (kVcSlots - 1);
    }
    return -1;
}

__global__ void k_vc_collect(long nnz, const double* __restrict__ val, unsigned long long* gkeys, int* gcount, int* over)
{
    __shared__ unsigned long long keys[kVcSlots];
    __shared__ int cnt, full;
    for (int i = threadIdx.x; i < kVcSlots; i += blockDim.x) keys[i] = kVcEmpty;
    if (threadIdx.x == 0) {
        cnt = 0;
        full = *(volatile int*)over;
    }
    __syncthreads();
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += (long)gridDim.x * blockDim.x) {
        if (*(volatile int*)&full) break;
        const unsigned long long b = (unsigned long long)__double_as_longlong(__ldcs(val + i));
        const int r = b == kVcEmpty ? -1 : vc_insert(keys, b);
        if (r < 0 || (r > 0 && atomicAdd(&cnt, 1) >= kValueCodes)) *(volatile int*)&full = 1;
    }
    __syncthreads();
    if (full) {
        if (threadIdx.x == 0) atomicExch(over, 1);
        return;
    }
    for (int i = threadIdx.x; i < kVcSlots; i += blockDim.x) {
        const unsigned long long b = keys[i];
        if (b == kVcEmpty) continue;
        const int r = vc_insert(gkeys, b);
        if (r < 0 || (r > 0 && atomicAdd(gcount, 1) >= kValueCodes)) atomicExch(over, 1);
    }
}

// code[i] = the table index of val[i] (every value is in the set)
__global__ void k_vc_encode(long nnz, const double* __restrict__ val, const unsigned long long* __restrict__ gkeys,
    const int* __restrict__ slot_code, unsigned char* __restrict__ code)
{
    __shared__ unsigned long long keys[kVcSlots];
    __shared__ unsigned char sc[kVcSlots];
    for (int i = threadIdx.x; i < kVcSlots; i += blockDim.x) {
        keys[i] = gkeys[i];
        sc[i] = (unsigned char)slot_code[i];
    }
    __syncthreads();
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += (long)gridDim.x * blockDim.x) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(__ldcs(val + i));
        unsigned h = vc_hash(b);
        for (int probe = 0; probe < kVcSlots && keys[h] != b; probe++) h = (h + 1) & (kVcSlots - 1);
        code[i] = sc[h];
    }
}

// Builds A's value codes when its values take at most kValueCodes distinct bit patterns (and the
// level is large enough to be bandwidth-bound); BCMGX_VALUE_CODES=0 in the environment turns this
// off. One host round trip for the distinct values.
static void build_value_codes(DevCsr& A, cudaStream_t s)
{
    A.vcode.release();
    A.vtab64.release();
    A.vtab32.release();
    A.nvalues = 0;
    const char* env = std::getenv("BCMGX_VALUE_CODES");
    if (env && env[0] == '0') return;
    if (A.nnz < kVcMinNnz) return;
    DBuf<unsigned long long> keys;
    DBuf<int> cnt;
    keys.alloc(kVcSlots, s);
    cnt.alloc(2, s);
    BCMGX_CUDA(cudaMemsetAsync(keys.p, 0xff, sizeof(unsigned long long) * kVcSlots, s));
    BCMGX_CUDA(cudaMemsetAsync(cnt.p, 0, 2 * sizeof(int), s));
    note_launch();
    k_vc_collect<<<gs_grid(A.nnz), 256, 0, s>>>(A.nnz, A.val.p, keys.p, cnt.p, cnt.p + 1);
    BCMGX_CHECK_LAUNCH();
    std::vector<unsigned long long> hk(kVcSlots);
    int hc[2] = { 0, 0 };
    BCMGX_CUDA(cudaMemcpyAsync(hk.data(), keys.p, sizeof(unsigned long long) * kVcSlots, cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaMemcpyAsync(hc, cnt.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaStreamSynchronize(s));
    if (hc[1] || hc[0] <= 0 || hc[0] > kValueCodes) return;
    // the table in bit-pattern order (deterministic), the code of every occupied slot
    std::vector<unsigned long long> vals;
    for (unsigned long long k : hk)
        if (k != kVcEmpty) vals.push_back(k);
    std::sort(vals.begin(), vals.end());
    std::vector<double> t64(kValueCodes, 0.0);
    std::vector<float> t32(kValueCodes, 0.0f);
    for (size_t i = 0; i < vals.size(); i++) {
        std::memcpy(&t64[i], &vals[i], sizeof(double));
        t32[i] = (float)t64[i];
    }
    std::vector<int> slot_code(kVcSlots, 0);
    for (int h = 0; h < kVcSlots; h++)
        if (hk[h] != kVcEmpty)
            slot_code[h] = (int)(std::lower_bound(vals.begin(), vals.end(), hk[h]) - vals.begin());
    DBuf<int> sc;
    sc.alloc(kVcSlots, s);
    BCMGX_CUDA(cudaMemcpyAsync(sc.p, slot_code.data(), sizeof(int) * kVcSlots, cudaMemcpyHostToDevice, s));
    A.vtab64.alloc(kValueCodes, s);
    A.vtab32.alloc(kValueCodes, s);
    BCMGX_CUDA(cudaMemcpyAsync(A.vtab64.p, t64.data(), sizeof(double) * kValueCodes, cudaMemcpyHostToDevice, s));
    BCMGX_CUDA(cudaMemcpyAsync(A.vtab32.p, t32.data(), sizeof(float) * kValueCodes, cudaMemcpyHostToDevice, s));
    A.vcode.alloc(A.nnz, s);
    note_launch();
    k_vc_encode<<<gs_grid(A.nnz), 256, 0, s>>>(A.nnz, A.val.p, keys.p, sc.p, A.vcode.p);
    BCMGX_CHECK_LAUNCH();
    // the host vectors above are read by the copies before this returns
    BCMGX_CUDA(cudaStreamSynchronize(s));
    A.nvalues = (int)vals.size();
}

// ---- pattern-indexed rows ------------------------------------------------------------------
// A stencil level's rows repeat a handful of column-offset sequences (a 27-point grid has 27
// boundary types). Each row's sequence gets a 63-bit hash; the distinct hashes are collected and
// numbered with the value codes' hash set (k_vc_collect / k_vc_encode on the hashes' bit patterns),
// one row per number gives the form's offsets, and a check pass compares every row with its form,
// so a hash collision only costs the pattern form, never a wrong column.
__global__ void k_pat_hash(int n, const int* __restrict__ row, const short* __restrict__ dcol,
    unsigned long long* __restrict__ h)
{
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long)gridDim.x * blockDim.x) {
        const int b = row[r], e = row[r + 1];
        unsigned long long v = 1469598103934665603ull ^ (unsigned long long)(e - b);
        for (int j = b; j < e; j++) v = (v ^ (unsigned long long)(unsigned short)dcol[j]) * 1099511628211ull;
        h[r] = v & 0x7fffffffffffffffull;   // never kVcEmpty
    }
}

// rep[id] = some row of form id; len[id] its length. The claim is tried only while the form has
// none (a plain load first): millions of rows share a few forms, and atomics on one word serialise.
__global__ void k_pat_rep(int n, const int* __restrict__ row, const unsigned char* __restrict__ pid, int* rep,
    int* len)
{
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long)gridDim.x * blockDim.x) {
        const int id = pid[r];
        if (ld_cg(rep + id) == -1 && atomicCAS(rep + id, -1, (int)r) == -1) len[id] = row[r + 1] - row[r];
    }
}

// pat[id * W + k] = offset k of form id (0 past its length)
__global__ void k_pat_table(int npat, int W, const int* __restrict__ row, const short* __restrict__ dcol,
    const int* __restrict__ rep, const int* __restrict__ len, short* __restrict__ pat)
{
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < (long)npat * W; t += (long)gridDim.x * blockDim.x) {
        const int id = (int)(t / W), k = (int)(t % W);
        const int r = rep[id];
        pat[t] = (r >= 0 && k < len[id]) ? dcol[row[r] + k] : (short)0;
    }
}

// every row against its form (length and offsets); rows n .. total-1 of the per-slice array take
// row n-1's form
__global__ void k_pat_check(int n, long total, int W, const int* __restrict__ row, const short* __restrict__ dcol,
    unsigned char* __restrict__ pid, const short* __restrict__ pat, const int* __restrict__ len, int* bad)
{
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < total; r += (long)gridDim.x * blockDim.x) {
        if (r >= n) {
            pid[r] = pid[n - 1];
            continue;
        }
        const int id = pid[r];
        const int b = row[r], e = row[r + 1];
        bool ok = e - b == len[id] && e - b <= W;
        for (int j = b; ok && j < e; j++) ok = dcol[j] == pat[(long)id * W + (j - b)];
        if (!ok) atomicOr(bad, 1);
    }
}

void build_patterns(DevCsr& A, cudaStream_t s)
{
    A.sl_pid.release();
    A.sl_pat.release();
    A.npat = A.patw = 0;
    const char* env = std::getenv("BCMGX_SLPAT");
    if (env && env[0] == '0') return;
    const int n = A.n;
    if (n <= 0 || !A.dcol.p || !A.sl_code.p || A.max_row <= 0 || A.max_row > 32) return;
    const long total = ((long)n + 31) / 32 * 32;   // whole 32-row slices
    DBuf<unsigned long long> h, keys;
    DBuf<int> cnt;
    h.alloc(n, s);
    keys.alloc(kVcSlots, s);
    cnt.alloc(2, s);
    note_launch(); k_pat_hash<<<gs_grid(n), 256, 0, s>>>(n, A.row.p, A.dcol.p, h.p);
    BCMGX_CUDA(cudaMemsetAsync(keys.p, 0xff, sizeof(unsigned long long) * kVcSlots, s));
    BCMGX_CUDA(cudaMemsetAsync(cnt.p, 0, 2 * sizeof(int), s));
    note_launch(); k_vc_collect<<<gs_grid(n), 256, 0, s>>>(n, (const double*)h.p, keys.p, cnt.p, cnt.p + 1);
    BCMGX_CHECK_LAUNCH();
    std::vector<unsigned long long> hk(kVcSlots);
    int hc[2] = { 0, 0 };
    BCMGX_CUDA(cudaMemcpyAsync(hk.data(), keys.p, sizeof(unsigned long long) * kVcSlots, cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaMemcpyAsync(hc, cnt.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaStreamSynchronize(s));
    if (hc[1] || hc[0] <= 0 || hc[0] > 255) return;
    std::vector<unsigned long long> forms;
    for (unsigned long long k : hk)
        if (k != kVcEmpty) forms.push_back(k);
    std::sort(forms.begin(), forms.end());
    const int npat = (int)forms.size();
    std::vector<int> slot_id(kVcSlots, 0);
    for (int t = 0; t < kVcSlots; t++)
        if (hk[t] != kVcEmpty) slot_id[t] = (int)(std::lower_bound(forms.begin(), forms.end(), hk[t]) - forms.begin());
    const int W = ((A.max_row + 3) / 4) * 4;
    DBuf<int> sid, rep, len, bad;
    sid.alloc(kVcSlots, s);
    rep.alloc(npat, s);
    len.alloc(npat, s);
    bad.alloc(1, s);
    BCMGX_CUDA(cudaMemcpyAsync(sid.p, slot_id.data(), sizeof(int) * kVcSlots, cudaMemcpyHostToDevice, s));
    BCMGX_CUDA(cudaMemsetAsync(rep.p, 0xff, sizeof(int) * npat, s));
    BCMGX_CUDA(cudaMemsetAsync(len.p, 0, sizeof(int) * npat, s));
    BCMGX_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    A.sl_pid.alloc(total, s);
    A.sl_pat.alloc((size_t)npat * W, s);
    note_launch(); k_vc_encode<<<gs_grid(n), 256, 0, s>>>(n, (const double*)h.p, keys.p, sid.p, A.sl_pid.p);
    note_launch(); k_pat_rep<<<gs_grid(n), 256, 0, s>>>(n, A.row.p, A.sl_pid.p, rep.p, len.p);
    note_launch(); k_pat_table<<<gs_grid((long)npat * W), 256, 0, s>>>(npat, W, A.row.p, A.dcol.p, rep.p, len.p, A.sl_pat.p);
    note_launch(); k_pat_check<<<gs_grid(total), 256, 0, s>>>(n, total, W, A.row.p, A.dcol.p, A.sl_pid.p, A.sl_pat.p, len.p,
        bad.p);
    BCMGX_CHECK_LAUNCH();
    // the host vector above is read by its copy before this returns
    if (read_err(bad.p, s)) {
        A.sl_pid.release();
        A.sl_pat.release();
        return;
    }
    A.npat = npat;
    A.patw = W;
}

void finish_level_matrix(Level& V, bool want_f32, cudaStream_t s)
{
    const int n = V.A.n;
    build_offsets(V.A, s);
    V.M.alloc(n, s);
    if (want_f32) V.M32.alloc(n, s);
    note_launch(); k_abs_row_sum<<<gs_grid(n), 256, 0, s>>>(n, V.A.row.p, V.A.val.p, V.M.p, want_f32 ? V.M32.p : nullptr);
    if (want_f32) {
        V.A.val32.alloc(std::max<int64_t>(V.A.nnz, 1), s);
        note_launch(); k_to_f32<<<gs_grid(V.A.nnz), 256, 0, s>>>(V.A.nnz, V.A.val.p, V.A.val32.p);
    }
    BCMGX_CHECK_LAUNCH();
    build_value_codes(V.A, s);
}

void build_restriction(Level& V, int nc, bool want_f32, cudaStream_t s)
{
    const int n = V.A.n;
    DBuf<int> cnt, fillpos;
    cnt.alloc(std::max(nc, 1), s);
    fillpos.alloc(std::max(nc, 1), s);
    BCMGX_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * std::max(nc, 1), s));
    BCMGX_CUDA(cudaMemsetAsync(fillpos.p, 0, sizeof(int) * std::max(nc, 1), s));
    note_launch(); k_count<<<gs_grid(n), 256, 0, s>>>(n, V.agg.p, cnt.p);
    BCMGX_CHECK_LAUNCH();
    V.rptr.alloc((size_t)nc + 1, s);
    scan_exclusive_dev(cnt.p, V.rptr.p, nc, s);
    V.ridx.alloc(n, s);
    V.rval.alloc(n, s);
    if (want_f32) {
        V.rval32.alloc(n, s);
        V.p32.alloc(n, s);
        note_launch(); k_to_f32<<<gs_grid(n), 256, 0, s>>>(n, V.p.p, V.p32.p);
    }
    note_launch(); k_scatter<<<gs_grid(n), 256, 0, s>>>(n, V.agg.p, V.rptr.p, fillpos.p, V.ridx.p);
    note_launch(); k_sort_rrows<<<gs_grid(nc), 256, 0, s>>>(nc, V.rptr.p, V.ridx.p, V.p.p, V.rval.p, want_f32 ? V.rval32.p : nullptr);
    BCMGX_CHECK_LAUNCH();
}

void compose_prolongator(int n, int* agg, double* p, const int* agg_s, const double* p_s, bool first, cudaStream_t s)
{
    note_launch();
    k_compose<<<gs_grid(n), 256, 0, s>>>(n, agg, p, agg_s, p_s, first ? 1 : 0);
    BCMGX_CHECK_LAUNCH();
}

int row_max_dev(int n, const int* row, cudaStream_t s) { return row_max_raw(n, row, s); }

int setup_grid(long n, int threads) { return gs_grid(n, threads); }

// AMG::ApplyData::setGridSweeps (AMG.cu:306-331).
static std::vector<int> grid_sweeps(int cycle_type, int max_levels)
{
    const int ml = max_levels - 1;
    std::vector<int> g(std::max(ml, 0), 1);
    if (cycle_type == BCMGX_CYCLE_H) {
        for (int i = 0; i < ml; i++)
            if (i % 2 == 0) g[i] = 2;
    } else if (cycle_type == BCMGX_CYCLE_W) {
        for (int i = 0; i < ml - 1; i++) g[i] = 2;
    }
    return g;
}

void build_hierarchy(bcmgx_hierarchy* H, const bcmgx_csr* Ain)
{
    cudaStream_t s = H->stream;
    const bcmgx_params& P = H->prm;
    const bool f32 = P.vcycle_precision == BCMGX_VCYCLE_FP32;
    H->lv.clear();
    H->lv.emplace_back();
    Level& L0 = H->lv[0];
    DevCsr& A = L0.A;
    A.n = Ain->n;
    A.m = Ain->m;
    A.nnz = Ain->nnz;
    A.row.alloc((size_t)A.n + 1, s);
    A.col.alloc(std::max<int64_t>(A.nnz, 1), s);
    A.val.alloc(std::max<int64_t>(A.nnz, 1), s);
    const cudaMemcpyKind kind = Ain->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    BCMGX_CUDA(cudaMemcpyAsync(A.row.p, Ain->row, sizeof(int) * ((size_t)A.n + 1), kind, s));
    BCMGX_CUDA(cudaMemcpyAsync(A.col.p, Ain->col, sizeof(int) * A.nnz, kind, s));
    BCMGX_CUDA(cudaMemcpyAsync(A.val.p, Ain->val, sizeof(double) * A.nnz, kind, s));
    {
        // checks, longest row, largest column offset and the int16 offsets in one pass and one
        // round trip; the offsets are kept when they all fit (build_offsets then has nothing to do)
        DBuf<int> st;
        st.alloc(3, s);
        BCMGX_CUDA(cudaMemsetAsync(st.p, 0, 3 * sizeof(int), s));
        const char* env16 = std::getenv("BCMGX_INDEX16");
        const bool want16 = !(env16 && env16[0] == '0');
        if (want16) A.dcol.alloc(A.nnz, s);
        const bool bcmg = P.preconditioner == BCMGX_PREC_BCMG;
        if (bcmg) A.dpos.alloc(A.n, s);
        note_launch(); k_validate_offsets<<<gs_grid((long)A.n * 8), 256, 0, s>>>(A.n, A.m, A.nnz, A.row.p, A.col.p,
            st.p, st.p + 1, st.p + 2, want16 ? A.dcol.p : nullptr, bcmg ? 1 : 0, bcmg ? A.dpos.p : nullptr);
        BCMGX_CHECK_LAUNCH();
        int h[3] = { 0, 0, 0 };
        BCMGX_CUDA(cudaMemcpyAsync(h, st.p, 3 * sizeof(int), cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
        if (h[0]) throw Error(BCMGX_ERR_INVALID_INPUT, "input matrix: " + err_text(h[0]));
        A.max_row = h[1];
        if (h[2] > 32767) A.dcol.release();
    }
    const int L0n = A.n;
    H->grid_sweeps = grid_sweeps(P.cycle_type, P.max_levels);
    H->ftcoarse = 1;
    // AMG::BuildData::setMaxCoarseSize, AMG.cu:238-241
    H->maxcoarsesize = (int)(40 * std::pow((double)L0n, 1.0 / 3.0));
    if (P.preconditioner == BCMGX_PREC_AFSAI) afsai_build_dev(H);
    if (P.preconditioner == BCMGX_PREC_L1_JACOBI) {
        H->l1d.alloc(L0n, s);
        note_launch(); k_l1_divisor<<<gs_grid(L0n), 256, 0, s>>>(L0n, A.row.p, A.col.p, A.val.p, H->l1d.p);
        BCMGX_CHECK_LAUNCH();
    }
    if (P.preconditioner != BCMGX_PREC_BCMG) {
        finish_level_matrix(L0, false, s);
        H->op_cmplx = 1;
        H->op_wcmplx = 1;
        H->avg_cratio = 1;
        return;
    }
    const int sweepnumber = P.aggrsweeps + 1;
    DBuf<double> w;
    w.alloc(L0n, s);
    note_launch(); k_fill<<<gs_grid(L0n), 256, 0, s>>>(L0n, w.p, 1.0);
    BCMGX_CHECK_LAUNCH();
    double avcoarseratio = 0;
    int level;
    for (level = 1; level < P.max_levels;) {
        const DevCsr* Ai_ = &H->lv[level - 1].A;
        const int nfine = Ai_->n;
        SweepOut prev, cur;
        DBuf<double> wsw;   // weights of the running sweep (moved from the previous one)
        const double* wi_ = w.p;
        DBuf<int> Pagg;
        DBuf<double> Pval;
        Pagg.alloc(nfine, s);
        Pval.alloc(nfine, s);
        for (int i = 0; i < sweepnumber; i++) {
            pairwise_sweep(H, *Ai_, wi_, cur, level - 1, i);
            PhaseTimer pt(H, "compose");
            const double size_precoarse = Ai_->n, size_coarse = cur.nc;
            const double coarse_ratio = size_precoarse / size_coarse;
            if (coarse_ratio <= kCoarseRatioThreshold) H->ftcoarse = kFtcoarseInc;
            compose_prolongator(nfine, Pagg.p, Pval.p, cur.agg.p, cur.p.p, i == 0, s);
            if (size_coarse <= (double)H->ftcoarse * H->maxcoarsesize || i + 1 == sweepnumber) break;
            prev = std::move(cur);
            cur = SweepOut();
            Ai_ = &prev.C;
            wi_ = prev.wc.p;
        }
        w = std::move(cur.wc);
        Level& F = H->lv[level - 1];
        F.agg = std::move(Pagg);
        F.p = std::move(Pval);
        const int nc = cur.C.n;
        PhaseTimer pt(H, "restriction+finish");
        build_restriction(F, nc, f32, s);
        if (level == 1) finish_level_matrix(F, f32, s);
        Level NL;
        NL.A = std::move(cur.C);
        H->lv.push_back(std::move(NL));
        const double size_coarse = H->lv[level].A.n;
        avcoarseratio += H->lv[level - 1].A.n / size_coarse;
        level++;
        if (size_coarse <= (double)H->ftcoarse * H->maxcoarsesize) break;
    }
    if (H->lv.size() == 1) finish_level_matrix(H->lv[0], false, s);
    const int Lc = (int)H->lv.size();
    for (int l = 1; l < Lc; l++) finish_level_matrix(H->lv[l], f32 && l < Lc - 1, s);
    // the coarsest level runs in FP64 even in the FP32 cycle
    if (Lc > 1 && f32) {
        Level& last = H->lv[Lc - 1];
        last.A.val32.release();
        last.M32.release();
    }
    // AMG::Hierarchy::finalize_cmplx / finalize_wcmplx (AMG.cu:144-165)
    double nnz0 = (double)H->lv[0].A.nnz, c = 0, wc = 0;
    for (int l = 0; l < Lc; l++) {
        c += (double)H->lv[l].A.nnz;
        wc += std::pow(2.0, (double)l) * (double)H->lv[l].A.nnz;
    }
    H->op_cmplx = c / nnz0;
    H->op_wcmplx = wc / nnz0;
    H->avg_cratio = level > 1 ? avcoarseratio / (level - 1) : 1;
    BCMGX_CUDA(cudaStreamSynchronize(s));
    if (prof_on()) {
        for (auto& pr : H->prof) std::fprintf(stderr, "[bcmgx setup] %-20s %9.3f ms\n", pr.first.c_str(), pr.second);
        H->prof.clear();
    }
}

}  // namespace bcmgx

// ------------------------------------------------------------------------------------------
// Allocation-free edge weights
// ------------------------------------------------------------------------------------------
// Some callers cannot let this library allocate device memory: a framework whose caching
// allocator already holds (nearly) all of the GPU's memory, so that one more allocation would
// fail, or a process that runs under a fixed device-memory budget. bcmgx_edge_weights_noalloc
// serves them. Its scratch (the per-row C values, the transposed-entry positions, the absolute
// minimum and the error words) lives in the file-scope array below, which holds matrices of at
// most kNoAllocMaxRows rows and kNoAllocMaxNnz entries. Every GPU that loads this library keeps
// these bytes until the process exits. All calls share the one array and it keeps the last
// call's contents: the words that must start from a known value are reset by every call, and
// calls that overlap on the GPU race on the array.
namespace bcmgx {

constexpr int kNoAllocMaxRows = 65536;
constexpr int64_t kNoAllocMaxNnz = 2097152;
constexpr size_t kNoAllocCBytes = sizeof(double) * kNoAllocMaxRows;
constexpr size_t kNoAllocTposBytes = sizeof(int) * kNoAllocMaxNnz;
constexpr size_t kNoAllocBytes = kNoAllocCBytes + kNoAllocTposBytes + 256;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_edge_weights_scratch[kNoAllocBytes];

static std::mutex g_noalloc_mu;
static unsigned char* g_noalloc_addr[kNoAllocMaxDevices];

// Device address of the scratch array on the current device. In host code the array's name only
// stands for it; the address is looked up once per device, with that device current.
static unsigned char* noalloc_scratch()
{
    int dev = 0;
    BCMGX_CUDA(cudaGetDevice(&dev));
    BCMGX_REQUIRE(dev >= 0 && dev < kNoAllocMaxDevices, BCMGX_ERR_UNSUPPORTED, "device ordinal too large");
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_edge_weights_scratch);
        if (e != cudaSuccess)
            throw Error(BCMGX_ERR_CUDA, std::string("cudaGetSymbolAddress of the scratch array failed: ") + cudaGetErrorString(e));
        g_noalloc_addr[dev] = (unsigned char*)p;
    }
    return g_noalloc_addr[dev];
}

__global__ void k_noalloc_reset(unsigned long long* min_bits, int* err, int* max_row)
{
    *min_bits = (unsigned long long)__double_as_longlong(DBL_MAX);
    *err = 0;
    *max_row = 0;
}

static void edge_weights_noalloc(int n, int64_t nnz, const int* row, const int* col, const double* val, const double* w,
    double* W, double* min_out, cudaStream_t s)
{
    BCMGX_REQUIRE(n > 0 && nnz > 0 && row && col && val && w && W, BCMGX_ERR_INVALID_INPUT, "bad argument");
    BCMGX_REQUIRE(n <= kNoAllocMaxRows && nnz <= kNoAllocMaxNnz, BCMGX_ERR_INVALID_INPUT,
        "matrix too large for the allocation-free entry point (at most " + std::to_string(kNoAllocMaxRows) + " rows and " +
            std::to_string(kNoAllocMaxNnz) + " non-zeros; got " + std::to_string(n) + " rows, " + std::to_string(nnz) + ")");
    unsigned char* base = noalloc_scratch();
    double* C = (double*)base;
    int* tpos = (int*)(base + kNoAllocCBytes);
    unsigned long long* minb = (unsigned long long*)(base + kNoAllocCBytes + kNoAllocTposBytes);
    int* err = (int*)(minb + 1);
    int* mx = err + 1;
    note_launch();
    k_noalloc_reset<<<1, 1, 0, s>>>(minb, err, mx);
    note_launch();
    k_validate<<<warp_grid(n), 256, 0, s>>>(n, n, nnz, row, col, err, mx, 1);
    BCMGX_CHECK_LAUNCH();
    int e = read_err(err, s);
    if (e) throw Error(BCMGX_ERR_INVALID_INPUT, "input matrix: " + err_text(e));
    note_launch();
    k_diag_c<<<gs_grid(n), 256, 0, s>>>(n, row, col, val, w, C, err);
    const int S = setup_subwarp(n, nnz);
    tpos_min_launch(S, n, row, col, tpos, val, w, C, minb, s);
    BCMGX_CHECK_LAUNCH();
    double m = 0;
    BCMGX_CUDA(cudaMemcpyAsync(&m, minb, sizeof(double), cudaMemcpyDeviceToHost, s));
    e = read_err(err, s);
    if (e) throw Error(BCMGX_ERR_INVALID_INPUT, "edge weights: " + err_text(e));
    if (std::fabs(m) < DBL_EPSILON) m = DBL_EPSILON;
    BCMGX_SUBWARP_LAUNCH(k_logw, S, n, s, n, row, col, val, w, C, tpos, kSuitorEps / (0.999 * m), W);
    BCMGX_CHECK_LAUNCH();
    BCMGX_CUDA(cudaStreamSynchronize(s));
    if (min_out) *min_out = m;
}

}  // namespace bcmgx

extern "C" int bcmgx_edge_weights_noalloc(int n, int64_t nnz, const int* row, const int* col, const double* val,
    const double* w, double* W, double* min_abs_out, void* stream)
{
    try {
        bcmgx::edge_weights_noalloc(n, nnz, row, col, val, w, W, min_abs_out, (cudaStream_t)stream);
        return BCMGX_OK;
    } catch (const bcmgx::Error& e) {
        bcmgx::set_last_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        bcmgx::set_last_error(e.what());
        return BCMGX_ERR_INTERNAL;
    }
}
