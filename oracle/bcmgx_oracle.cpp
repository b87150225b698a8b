/*
 * bcmgx_oracle.cpp -- CPU oracle for the BCMG-preconditioned FCG path of BootCMatchGX.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker: a plain C++17 (+ OpenMP for the bulk
 * loops) restatement of the reference's single-rank algorithm. It is loaded by tests/ as the
 * parity oracle, by __graft_entry__.smoke() as the checker, and by bench.py as the timed
 * CPU baseline ("port"). The product library (bootcmatchgx_b200) never links, loads or calls it.
 *
 * Every function names the reference file:line it restates (paths inside the BootCMatchGX
 * project). Pins: the golden solutions BCMGX/src/test/data/cmp/lap3d_{7p,27p}_10x10x10_*_sol.txt
 * (compared at 1e-5, the reference's own compareSolutions threshold, launchAndCompare.mk:320-330)
 * and the generator fixtures BCMGX/src/test/data/mtx/lap3d_*.mtx.
 *
 * Floating point: every operation of the set-up phase is rounded on its own (this file is
 * compiled with -ffp-contract=off), so the hierarchy (weights, matching, P, Galerkin sums,
 * weight vectors) is bit-reproducible by a GPU implementation that also avoids contraction.
 * The set-up sums have at most two terms (pairwise aggregation), so their order cannot matter.
 */
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// BCMGX/src/preconditioner/bcmg/suitor.h:8
constexpr double kSuitorEps = 3.885780586188048e-10;
// BCMGX/src/preconditioner/bcmg/matchingAggregation.cu:8-9
constexpr int kFtcoarseInc = 100;
constexpr double kCoarseRatioThreshold = 1.2;

struct Csr {
    int n = 0, m = 0;
    std::vector<int> row, col;
    std::vector<double> val;
    long nnz() const { return (long)col.size(); }
};

// Settings, same meaning and defaults as BCMGX/src/config/Params.h:238-291.
struct Params {
    int solver = 0;          // SolverType: 0 CGHS 1 FCG 2 CGS 3 PIPELINED_CGS 4 CGS_CUBLAS
    int itnlim = 2000;
    double rtol = 1e-6;
    int dispnorm = 1;
    int preconditioner = 0;  // PreconditionerType: 0 NONE 1 L1_JACOBI 2 BCMG 3 AFSAI
    int bootstrap_type = 0;
    int max_hrc = 1;
    double conv_ratio = 0.8;
    int matchtype = 0;
    int aggrsweeps = 2;
    int aggr_type = 0;
    int max_levels = 39;
    int cycle_type = 0;      // 0 V 1 H 2 W 3 VARIABLE_V
    int coarse_solver = 0;
    int relax_type = 0;
    int relaxnumber_coarse = 20;
    int prerelax_sweeps = 4;
    int postrelax_sweeps = 4;
    int l1jacsweeps = 4;
    int sstep = 1;
    int stop_criterion = 1;
    int ru_res = 1;
    int rec_res_int = 0;
};

struct Level {
    Csr A;
    std::vector<int> part;    // row partition over ranks: part[r] .. part[r+1]-1 (np = P set-ups)
    std::vector<double> M;    // absolute row sums (l1-Jacobi divisor)
    std::vector<int> agg;     // composite prolongator to the next level: column of row i
    std::vector<double> p;    // composite prolongator value of row i
    std::vector<int> rptr, ridx;  // R = P^T: fine rows of each aggregate, ascending
    std::vector<double> rval;
};

struct SweepRecord {
    int level, sweep, nc;
    std::vector<int> match;
    std::vector<int> agg;
    std::vector<double> p;
    std::vector<double> w_in;
};

struct Hierarchy {
    Params prm;
    std::vector<Level> lv;
    std::vector<SweepRecord> rec;
    int maxcoarsesize = 0;
    int ftcoarse = 1;
    double op_cmplx = 0, op_wcmplx = 0, avg_cratio = 1;
    std::vector<int> grid_sweeps;
    std::vector<double> l1d;   // standalone l1-Jacobi divisor a_ii + sum_{j != i} |a_ij| (L1_JACOBI)
    Csr G, GT;                 // AFSAI factor and its transpose (AFSAI)
};

// ------------------------------------------------------------------------------------------
// Generators
// ------------------------------------------------------------------------------------------

// Global row number of grid point (gi,gj,gk) when the nx*P x ny*Q x nz*R grid is split in
// P x Q x R blocks of nx x ny x nz points, blocks numbered x-fastest and points inside a block
// numbered x-fastest. Restates BCMGX/src/generator/laplacian.cu:14-25.
long internal_index(long gi, long gj, long gk, long nx, long ny, long nz, long P, long Q, long R)
{
    (void)R;
    long i = gi % nx, j = gj % ny, k = gk % nz;
    long p = gi / nx, q = gj / ny, r = gk / nz;
    return (r * P * Q + q * P + p) * nx * ny * nz + (k * nx * ny + j * nx + i);
}

// 7-point (diagonal 6) or 27-point (diagonal 26) Dirichlet Laplacian, off-diagonals -1, in the
// reference's rank-block-major global order. Restates generateLocalLaplacian3D_7p
// (laplacian.cu:119-334) and generateLocalLaplacian3D_27p (laplacian.cu:336-777) run on
// P*Q*R ranks and stacked in rank order, rows column-sorted as check_and_fix_order does
// (CSR.cu:1895-1918).
Csr lap3d(int stencil, int nx, int ny, int nz, int P, int Q, int R)
{
    const long gnx = (long)nx * P, gny = (long)ny * Q, gnz = (long)nz * R;
    const long N = gnx * gny * gnz;
    const long local = (long)nx * ny * nz;
    Csr A;
    A.n = A.m = (int)N;
    A.row.assign(N + 1, 0);
    auto decode = [&](long row, long& gi, long& gj, long& gk) {
        long blk = row / local, loc = row % local;
        long p = blk % P, q = (blk / P) % Q, r = blk / ((long)P * Q);
        long i = loc % nx, j = (loc / nx) % ny, k = loc / ((long)nx * ny);
        gi = p * nx + i; gj = q * ny + j; gk = r * nz + k;
    };
    auto is_nb = [&](int dx, int dy, int dz) {
        int a = std::abs(dx) + std::abs(dy) + std::abs(dz);
        return stencil == 27 ? true : a <= 1;
    };
#pragma omp parallel for schedule(static)
    for (long row = 0; row < N; row++) {
        long gi, gj, gk;
        decode(row, gi, gj, gk);
        int c = 0;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    if (!is_nb(dx, dy, dz)) continue;
                    long a = gi + dx, b = gj + dy, d = gk + dz;
                    if (a < 0 || a >= gnx || b < 0 || b >= gny || d < 0 || d >= gnz) continue;
                    c++;
                }
        A.row[row + 1] = c;
    }
    for (long r = 0; r < N; r++) A.row[r + 1] += A.row[r];
    A.col.resize(A.row[N]);
    A.val.resize(A.row[N]);
    const double diag = stencil == 27 ? 26.0 : 6.0;
#pragma omp parallel for schedule(static)
    for (long row = 0; row < N; row++) {
        long gi, gj, gk;
        decode(row, gi, gj, gk);
        std::pair<int, double> e[27];
        int c = 0;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    if (!is_nb(dx, dy, dz)) continue;
                    long a = gi + dx, b = gj + dy, d = gk + dz;
                    if (a < 0 || a >= gnx || b < 0 || b >= gny || d < 0 || d >= gnz) continue;
                    int col = (int)internal_index(a, b, d, nx, ny, nz, P, Q, R);
                    e[c++] = { col, (dx | dy | dz) ? -1.0 : diag };
                }
        std::sort(e, e + c);
        long o = A.row[row];
        for (int t = 0; t < c; t++) {
            A.col[o + t] = e[t].first;
            A.val[o + t] = e[t].second;
        }
    }
    return A;
}

// ------------------------------------------------------------------------------------------
// Basic sparse kernels
// ------------------------------------------------------------------------------------------

// M_i = sum_j |a_ij| in column order. Restates _row_sum_2 (CSR.cu:1362-1379), used by
// relaxPrepare (matchingAggregation.cu:40-60).
std::vector<double> abs_row_sum(const Csr& A)
{
    std::vector<double> M(A.n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < A.n; i++) {
        double s = 0.0;
        for (int j = A.row[i]; j < A.row[i + 1]; j++) s += std::fabs(A.val[j]);
        M[i] = s;
    }
    return M;
}

// y = A x. Restates the np=1 branch of CSRVector_product_adaptive_miniwarp_witho
// (CSR.cu:829-846) with alpha=1, beta=0; the sum runs in column order.
void spmv(const Csr& A, const double* x, double* y)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < A.n; i++) {
        double s = 0.0;
        for (int j = A.row[i]; j < A.row[i + 1]; j++) s += A.val[j] * x[A.col[j]];
        y[i] = s;
    }
}

double dot(const double* a, const double* b, long n)
{
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

// ------------------------------------------------------------------------------------------
// Set-up: weights, matching, pairwise aggregation, Galerkin product
// ------------------------------------------------------------------------------------------

// Edge weights of one pairwise sweep, stored on A's own pattern (diagonal slots hold 0).
// Restates makeAH/_makeC/_makeAH_warp (matching.cu:66-171), toMaximumProductMatrix with the
// absolute-minimum reduction and _make_w (matching.cu:188-251), and the symmetrisation
// _write_T_warp (matching.cu:13-64): a lower-triangle entry takes the upper entry's weight.
void edge_weights(const Csr& A, const std::vector<double>& w, std::vector<double>& W, double* min_out)
{
    const int n = A.n;
    std::vector<double> C(n, 0.0);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; r++) {
        for (int j = A.row[r]; j < A.row[r + 1]; j++)
            if (A.col[j] == r) {
                C[r] = A.val[j] * w[r] * w[r];
                break;
            }
    }
    W.assign(A.nnz(), 0.0);
    double mn = DBL_MAX;
#pragma omp parallel for schedule(static) reduction(min : mn)
    for (int r = 0; r < n; r++) {
        for (int j = A.row[r]; j < A.row[r + 1]; j++) {
            int c = A.col[j];
            if (c == r) continue;
            double a = A.val[j];
            double norm = C[r] + C[c];
            double ah;
            if (norm > DBL_EPSILON) {
                double wt = w[r] * w[c];
                ah = 1.0 - ((2.0 * a * wt) / norm);
            } else {
                ah = DBL_EPSILON;
            }
            W[j] = ah;
            mn = std::min(mn, std::fabs(ah));
        }
    }
    if (std::fabs(mn) < DBL_EPSILON) mn = DBL_EPSILON;
    if (min_out) *min_out = mn;
    const double zero_sub = kSuitorEps / (0.999 * mn);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; r++) {
        for (int j = A.row[r]; j < A.row[r + 1]; j++) {
            if (A.col[j] == r) continue;
            double s = std::fabs(W[j]);
            W[j] = std::log(s != 0.0 ? s : zero_sub);
        }
    }
    // lower := upper (reads only c<r rows' upper entries, writes only lower entries)
    std::vector<double> Wu(W);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; r++) {
        for (int j = A.row[r]; j < A.row[r + 1]; j++) {
            int c = A.col[j];
            if (c >= r) break;
            const int* b = A.col.data() + A.row[c];
            const int* e = A.col.data() + A.row[c + 1];
            const int* f = std::lower_bound(b, e, r);
            if (f != e && *f == r) W[j] = Wu[A.row[c] + (f - b)];
        }
    }
}

// Strict total order on edges used by the suitor matching: weight first, then the larger
// endpoint, then the smaller one. Each vertex ranks its candidates by (weight, candidate id)
// and each vertex ranks its suitors by (weight, suitor id) (suitor.cu:104-141); both rankings
// agree with this key, so the suitor result is the greedy matching for it.
struct EdgeKey {
    double w;
    int hi, lo;
    bool operator>(const EdgeKey& o) const
    {
        if (w != o.w) return w > o.w;
        if (hi != o.hi) return hi > o.hi;
        return lo > o.lo;
    }
};

// Greedy matching on edges with weight > 0 visited in decreasing EdgeKey order.
std::vector<int> match_greedy(const Csr& A, const std::vector<double>& W)
{
    struct E { EdgeKey k; };
    std::vector<E> es;
    for (int r = 0; r < A.n; r++)
        for (int j = A.row[r]; j < A.row[r + 1]; j++) {
            int c = A.col[j];
            if (c <= r || !(W[j] > 0)) continue;
            es.push_back({ { W[j], c, r } });
        }
    std::sort(es.begin(), es.end(), [](const E& a, const E& b) { return a.k > b.k; });
    std::vector<int> M(A.n, -1);
    for (auto& e : es)
        if (M[e.k.hi] < 0 && M[e.k.lo] < 0) {
            M[e.k.hi] = e.k.lo;
            M[e.k.lo] = e.k.hi;
        }
    return M;
}

// Sequential suitor algorithm (Manne & Halappanavar). Same result as match_greedy, O(nnz).
// The device kernel it restates is kernel_for_matching/find_Candidate/set_suitor
// (suitor.cu:51-267); weights <= 0 are never proposed (suitor.cu:92-94).
std::vector<int> match_suitor(const Csr& A, const std::vector<double>& W)
{
    const int n = A.n;
    std::vector<int> s(n, -1);
    std::vector<EdgeKey> ws(n, EdgeKey { 0.0, -1, -1 });
    for (int u = 0; u < n; u++) {
        int cur = u;
        bool done = false;
        while (!done) {
            done = true;
            int best = -1;
            EdgeKey bk { 0.0, -1, -1 };
            for (int j = A.row[cur]; j < A.row[cur + 1]; j++) {
                int v = A.col[j];
                if (v == cur || !(W[j] > 0)) continue;
                EdgeKey k { W[j], std::max(v, cur), std::min(v, cur) };
                if (k > bk && k > ws[v]) {
                    bk = k;
                    best = v;
                }
            }
            if (best >= 0) {
                int prev = s[best];
                s[best] = cur;
                ws[best] = bk;
                if (prev >= 0) {
                    cur = prev;
                    done = false;
                }
            }
        }
    }
    return s;
}

// Pairwise prolongator of one sweep: column agg[i] and value p[i] of row i, nc columns.
// Restates makeP_GPU (matchingPairAggregation.cu:24-170): a matched pair v<u whose
// ||(w_v,w_u)|| exceeds DBL_EPSILON is one aggregate with values w/||.||, numbered by the
// rank of v among pair masters (stable select, :127-148); every other vertex is a singleton
// with value w/|w| (:36-40). Singletons are numbered in vertex order after the pairs (the
// makePCol_CPU order, matchingAggregation.cu:62-87) because the device code numbers them in
// atomicAdd order (:38). A vertex with |w| <= DBL_EPSILON gets value 0 in the last column.
int make_pairwise_p(const std::vector<int>& M, const std::vector<double>& w, std::vector<int>& agg,
    std::vector<double>& p, std::vector<int>& fine0, std::vector<int>& fine1)
{
    const int n = (int)M.size();
    agg.assign(n, -1);
    p.assign(n, 0.0);
    std::vector<char> master(n, 0);
    int npairs = 0;
    for (int v = 0; v < n; v++) {
        int u = M[v];
        if (u >= 0 && v < u) {
            double wv = w[v], wu = w[u];
            double nrm = std::sqrt(wv * wv + wu * wu);
            if (nrm > DBL_EPSILON) {
                master[v] = 1;
                agg[v] = agg[u] = npairs++;
                p[v] = wv / nrm;
                p[u] = wu / nrm;
            }
        }
    }
    int nc = npairs;
    std::vector<int> bad;
    for (int v = 0; v < n; v++) {
        if (agg[v] >= 0) continue;
        if (std::fabs(w[v]) > DBL_EPSILON) {
            agg[v] = nc++;
            p[v] = w[v] / std::fabs(w[v]);
        } else {
            bad.push_back(v);
        }
    }
    for (int v : bad) {
        agg[v] = nc > 0 ? nc - 1 : 0;
        p[v] = 0.0;
    }
    if (nc == 0 && !bad.empty()) nc = 1;
    fine0.assign(nc, -1);
    fine1.assign(nc, -1);
    for (int v = 0; v < n; v++) {
        int c = agg[v];
        if (fine0[c] < 0) fine0[c] = v;
        else if (fine1[c] < 0) fine1[c] = v;
    }
    (void)master;
    return nc;
}

// ---- the row-partitioned (np = P) set-up --------------------------------------------------
// At np > 1 every rank holds a block of consecutive rows with global column ids; the matching
// sees only the rank's own columns. The restatement below runs the P ranks' set-ups together on
// the global matrix:
//  * makeAH (matching.cu:66-111) writes 99999 for an entry whose column lies outside the rank's
//    rows, and toMaximumProductMatrix (matching.cu:231-251) takes the absolute minimum over the
//    rank's AH without any reduction over ranks: every block has its own minimum, over its
//    within-block |a_hat| and the 99999 of its cross-block entries;
//  * _write_T_warp (matching.cu:29-64) and find_Candidate (suitor.cu:95-100) skip columns outside
//    the rank's rows: cross-block entries get weight 0 here, which the matching never proposes;
//  * makeP_GPU (matchingPairAggregation.cu:109-170) numbers each rank's aggregates locally (pairs
//    by master, then singletons) and matchingPairAggregation shifts them by the ranks' coarse
//    offsets (matchingPairAggregation.cu:188-222): block b's aggregates follow block b-1's.
// Everything else of the set-up and the whole solve is the same arithmetic as at np = 1 (halo
// exchanges bring remote values; sizes and coarsening tests use the global counts, full_n).

// block of every row of a partition (offsets part[0] = 0 < ... < part[P] = n)
std::vector<int> block_of_rows(const std::vector<int>& part)
{
    std::vector<int> b(part.back());
    for (size_t k = 0; k + 1 < part.size(); k++)
        for (int r = part[k]; r < part[k + 1]; r++) b[r] = (int)k;
    return b;
}

void edge_weights_parts(const Csr& A, const std::vector<double>& w, const std::vector<int>& part, std::vector<double>& W)
{
    const int n = A.n;
    const int P = (int)part.size() - 1;
    const std::vector<int> blk = block_of_rows(part);
    std::vector<double> C(n, 0.0);
    for (int r = 0; r < n; r++)
        for (int j = A.row[r]; j < A.row[r + 1]; j++)
            if (A.col[j] == r) {
                C[r] = A.val[j] * w[r] * w[r];
                break;
            }
    W.assign(A.nnz(), 0.0);
    std::vector<double> mn(P, DBL_MAX);
    for (int r = 0; r < n; r++) {
        const int b = blk[r];
        for (int j = A.row[r]; j < A.row[r + 1]; j++) {
            int c = A.col[j];
            if (c == r) continue;
            if (blk[c] != b) {
                mn[b] = std::min(mn[b], 99999.0);
                continue;
            }
            double a = A.val[j];
            double norm = C[r] + C[c];
            double ah;
            if (norm > DBL_EPSILON) {
                double wt = w[r] * w[c];
                ah = 1.0 - ((2.0 * a * wt) / norm);
            } else {
                ah = DBL_EPSILON;
            }
            W[j] = ah;
            mn[b] = std::min(mn[b], std::fabs(ah));
        }
    }
    for (int b = 0; b < P; b++)
        if (std::fabs(mn[b]) < DBL_EPSILON) mn[b] = DBL_EPSILON;
    for (int r = 0; r < n; r++) {
        const double zero_sub = kSuitorEps / (0.999 * mn[blk[r]]);
        for (int j = A.row[r]; j < A.row[r + 1]; j++) {
            const int c = A.col[j];
            if (c == r || blk[c] != blk[r]) continue;
            double s = std::fabs(W[j]);
            W[j] = std::log(s != 0.0 ? s : zero_sub);
        }
    }
    std::vector<double> Wu(W);
    for (int r = 0; r < n; r++) {
        for (int j = A.row[r]; j < A.row[r + 1]; j++) {
            int c = A.col[j];
            if (c >= r) break;
            if (blk[c] != blk[r]) continue;
            const int* b = A.col.data() + A.row[c];
            const int* e = A.col.data() + A.row[c + 1];
            const int* f = std::lower_bound(b, e, r);
            if (f != e && *f == r) W[j] = Wu[A.row[c] + (f - b)];
        }
    }
}

// make_pairwise_p block by block: block b's pairs (by master), then its singletons, numbered from
// the sum of the earlier blocks' aggregate counts; coarse_part receives the coarse partition.
int make_pairwise_p_parts(const std::vector<int>& M, const std::vector<double>& w, const std::vector<int>& part,
    std::vector<int>& agg, std::vector<double>& p, std::vector<int>& fine0, std::vector<int>& fine1,
    std::vector<int>& coarse_part)
{
    const int n = (int)M.size();
    agg.assign(n, -1);
    p.assign(n, 0.0);
    coarse_part.assign(1, 0);
    int nc = 0;
    for (size_t b = 0; b + 1 < part.size(); b++) {
        const int r0 = part[b], r1 = part[b + 1];
        for (int v = r0; v < r1; v++) {
            int u = M[v];
            if (u >= 0 && v < u) {
                double wv = w[v], wu = w[u];
                double nrm = std::sqrt(wv * wv + wu * wu);
                if (nrm > DBL_EPSILON) {
                    agg[v] = agg[u] = nc++;
                    p[v] = wv / nrm;
                    p[u] = wu / nrm;
                }
            }
        }
        std::vector<int> bad;
        for (int v = r0; v < r1; v++) {
            if (agg[v] >= 0) continue;
            if (std::fabs(w[v]) > DBL_EPSILON) {
                agg[v] = nc++;
                p[v] = w[v] / std::fabs(w[v]);
            } else {
                bad.push_back(v);
            }
        }
        for (int v : bad) {
            agg[v] = nc > coarse_part.back() ? nc - 1 : nc;
            p[v] = 0.0;
        }
        if (nc == coarse_part.back() && !bad.empty()) nc++;
        coarse_part.push_back(nc);
    }
    fine0.assign(nc, -1);
    fine1.assign(nc, -1);
    for (int v = 0; v < n; v++) {
        int c = agg[v];
        if (fine0[c] < 0) fine0[c] = v;
        else if (fine1[c] < 0) fine1[c] = v;
    }
    return nc;
}

// Galerkin product C = P^T A P for a pairwise P. Restates the two nsparse products of
// matchingAggregation.cu:128-131 (AP = A*P, then R*AP) as nsparse evaluates them: every
// product a*b is rounded, then accumulated into a zero-initialised slot
// (kernel_spgemm_hash_d.cu:792-799, nsparse_asm.h:97-114). With one non-zero per row of P and
// at most two rows per aggregate, each slot receives at most two terms, so the sum order
// cannot change the result. Rows come out column-sorted with every structural entry kept.
Csr galerkin_pairwise(const Csr& A, const std::vector<int>& agg, const std::vector<double>& p,
    const std::vector<int>& fine0, const std::vector<int>& fine1, int nc)
{
    Csr C;
    C.n = C.m = nc;
    C.row.assign(nc + 1, 0);
    std::vector<std::vector<std::pair<int, double>>> rows(nc);
#pragma omp parallel
    {
        std::vector<int> slot(nc, -1);
        std::vector<int> touched;
        std::vector<double> ap(nc, 0.0), cv(nc, 0.0);
        std::vector<int> cslot(nc, -1);
        std::vector<int> ctouched;
#pragma omp for schedule(dynamic, 256)
        for (int I = 0; I < nc; I++) {
            ctouched.clear();
            for (int f = 0; f < 2; f++) {
                int i = f == 0 ? fine0[I] : fine1[I];
                if (i < 0) continue;
                touched.clear();
                for (int j = A.row[i]; j < A.row[i + 1]; j++) {
                    int J = agg[A.col[j]];
                    double t = A.val[j] * p[A.col[j]];
                    if (slot[J] < 0) {
                        slot[J] = 1;
                        ap[J] = 0.0;
                        touched.push_back(J);
                    }
                    ap[J] = ap[J] + t;
                }
                for (int J : touched) {
                    double c = p[i] * ap[J];
                    if (cslot[J] < 0) {
                        cslot[J] = 1;
                        cv[J] = 0.0;
                        ctouched.push_back(J);
                    }
                    cv[J] = cv[J] + c;
                    slot[J] = -1;
                }
            }
            std::sort(ctouched.begin(), ctouched.end());
            auto& out = rows[I];
            out.reserve(ctouched.size());
            for (int J : ctouched) {
                out.push_back({ J, cv[J] });
                cslot[J] = -1;
            }
        }
    }
    for (int I = 0; I < nc; I++) C.row[I + 1] = C.row[I] + (int)rows[I].size();
    C.col.resize(C.row[nc]);
    C.val.resize(C.row[nc]);
#pragma omp parallel for schedule(static)
    for (int I = 0; I < nc; I++) {
        long o = C.row[I];
        for (auto& e : rows[I]) {
            C.col[o] = e.first;
            C.val[o] = e.second;
            o++;
        }
    }
    return C;
}

// Weight vector of the coarse sweep: w_c = R w, R = P^T with rows in fine-index order.
// Restates shifted_CSRVector_product_adaptive_miniwarp2 (CSR.cu:1195-1255) for rows of one
// or two entries: each product rounded, then added.
std::vector<double> restrict_weights(const std::vector<double>& w, const std::vector<double>& p,
    const std::vector<int>& fine0, const std::vector<int>& fine1)
{
    const int nc = (int)fine0.size();
    std::vector<double> wc(nc);
    for (int I = 0; I < nc; I++) {
        double t0 = fine0[I] >= 0 ? p[fine0[I]] * w[fine0[I]] : 0.0;
        double t1 = fine1[I] >= 0 ? p[fine1[I]] * w[fine1[I]] : 0.0;
        wc[I] = t0 + t1;
    }
    return wc;
}

// AMG::ApplyData::setGridSweeps (AMG.cu:306-331): coarse-grid visits per level.
std::vector<int> grid_sweeps(int cycle_type, int max_levels)
{
    int ml = max_levels - 1;
    std::vector<int> g(std::max(ml, 0), 1);
    if (cycle_type == 1) {
        for (int i = 0; i < ml; i++)
            if (i % 2 == 0) g[i] = 2;
    } else if (cycle_type == 2) {
        for (int i = 0; i < ml - 1; i++) g[i] = 2;
    }
    return g;
}

void build_restriction(Level& L, int nc)
{
    const int n = (int)L.agg.size();
    L.rptr.assign(nc + 1, 0);
    for (int i = 0; i < n; i++) L.rptr[L.agg[i] + 1]++;
    for (int c = 0; c < nc; c++) L.rptr[c + 1] += L.rptr[c];
    L.ridx.resize(n);
    L.rval.resize(n);
    std::vector<int> pos(L.rptr.begin(), L.rptr.end() - 1);
    for (int i = 0; i < n; i++) {
        int c = L.agg[i];
        L.ridx[pos[c]] = i;
        L.rval[pos[c]] = L.p[i];
        pos[c]++;
    }
}

// ---- AFSAI (adaptive factorized sparse approximate inverse) ---------------------------------
// Restates afsai_setup (preconditioner/afsai/afsai.cu:287-1090) at np = 1 with its kernels
// (kapGradCUDA_WiP.cu, d_gFSA.cu, choldc.cu, scalar_product_atomicAdd.h): 30 steps of one new
// entry per row of the lower-triangular factor G of the diagonally scaled matrix, chosen by the
// largest |gradient| (ties: the smallest column), each step solving the row's small SPD system
// (packed U^T U Cholesky, cudacholdcMix); a row stops when its Kaporin term changes by less than
// 1e-3 relative or stops growing. Applied as v = G^T (G r) (afsai_apply, :1092-1103).
constexpr int kAfsaiSteps = 30;
constexpr double kAfsaiEps = 0.001;

// solve U^T U x = b in place of b, U upper-packed (column j holds rows 0..j) with the diagonal
// stored inverted; false when a pivot is not positive (cudacholdcMix, choldc.cu)
bool afsai_chol_solve(double* l, double* x, int n)
{
    int ooffi = 0;
    for (int i = 0; i < n; i++) {
        int ooffj = ooffi;
        for (int j = i; j < n; j++) {
            double sum = l[i + ooffj];
            for (int k = 0; k < i; k++) sum -= l[ooffi + k] * l[ooffj + k];
            if (i == j) {
                if (sum <= 0.0) return false;
                l[ooffj + i] = 1. / std::sqrt(sum);
            } else {
                l[ooffj + i] = sum * l[ooffi + i];
            }
            ooffj += (j + 1);
        }
        ooffi += (i + 1);
    }
    ooffi = 0;
    for (int i = 0; i < n; i++) {
        double sum = x[i];
        for (int j = i - 1; j >= 0; j--) sum -= l[ooffi + j] * x[j];
        x[i] = sum * l[ooffi + i];
        ooffi += (i + 1);
    }
    ooffi = n * (n - 1) / 2;
    for (int i = n - 1; i >= 0; i--) {
        double sum = x[i];
        int ooffj = ooffi + i;
        for (int j = i + 1; j < n; j++) {
            sum -= l[ooffj + i + 1] * x[j];
            ooffj += (j + 1);
        }
        x[i] = sum * l[ooffi + i];
        ooffi -= i;
    }
    return true;
}

// One row of G: pattern cols (ascending, all < i) and coefficients, plus the Kaporin term.
void afsai_row(const Csr& S, int i, std::vector<int>& iwn, std::vector<double>& x, double& dk)
{
    iwn.clear();
    x.clear();
    dk = 0.0;
    double dk_old = 0.0;
    std::vector<double> M, b;
    for (int step = 0; step < kAfsaiSteps; step++) {
        const int m = (int)iwn.size();
        // gradient g_c = S(i, c) + sum_k x_k S(iwn_k, c) over columns c < i; merge of sorted rows
        std::vector<int> pos(m + 1), end(m + 1), rows(m + 1);
        std::vector<double> fac(m + 1);
        rows[0] = i;
        fac[0] = 1.0;
        for (int k = 0; k < m; k++) {
            rows[k + 1] = iwn[k];
            fac[k + 1] = x[k];
        }
        for (int k = 0; k <= m; k++) {
            pos[k] = S.row[rows[k]];
            end[k] = S.row[rows[k] + 1];
        }
        int best = -1, iw = 0;
        double bestv = 0.0;
        for (;;) {
            int c = INT32_MAX;
            for (int k = 0; k <= m; k++)
                if (pos[k] < end[k] && S.col[pos[k]] < c) c = S.col[pos[k]];
            if (c >= i) break;
            double g = 0.0;
            for (int k = 0; k <= m; k++)
                if (pos[k] < end[k] && S.col[pos[k]] == c) {
                    g += S.val[pos[k]] * fac[k];
                    pos[k]++;
                }
            while (iw < m && iwn[iw] < c) iw++;
            if (iw < m && iwn[iw] == c) continue;   // already in the pattern
            if (std::fabs(g) > bestv) {
                bestv = std::fabs(g);
                best = c;
            }
        }
        if (best < 0) break;   // no new entry: the row is done
        iwn.insert(std::lower_bound(iwn.begin(), iwn.end(), best), best);
        const int n = m + 1;
        // the row's system: M = S(iwn, iwn) upper-packed, b = -S(i, iwn)
        M.assign(n * (n + 1) / 2, 0.0);
        b.assign(n, 0.0);
        for (int r = 0; r < n; r++) {
            const int row = iwn[r];
            int jj = S.row[row];
            const int je = S.row[row + 1];
            for (int cidx = r; cidx < n; cidx++) {
                while (jj < je && S.col[jj] < iwn[cidx]) jj++;
                if (jj == je) break;
                if (S.col[jj] == iwn[cidx]) M[cidx * (cidx + 1) / 2 + r] = S.val[jj];
            }
        }
        for (int jj = S.row[i], r = 0; jj < S.row[i + 1] && r < n && S.col[jj] < i;) {
            if (iwn[r] > S.col[jj]) jj++;
            else if (iwn[r] == S.col[jj]) { b[r] = -S.val[jj]; jj++; r++; }
            else r++;
        }
        x = b;
        if (!afsai_chol_solve(M.data(), x.data(), n)) {   // not reached for SPD matrices
            x.assign(n, 0.0);
            dk = 0.0;
            break;
        }
        double d = 0.0;
        for (int k = 0; k < n; k++) d += b[k] * x[k];
        dk = d;
        const bool conv = std::fabs(dk - dk_old) < kAfsaiEps * dk_old || dk == 0.0;
        dk_old = dk;
        if (conv) break;
    }
}

// G (lower triangular, diagonal last in each row) of the scaled matrix
Csr afsai_build(const Csr& A)
{
    const int n = A.n;
    std::vector<double> d(n);
    for (int i = 0; i < n; i++)
        for (int j = A.row[i]; j < A.row[i + 1]; j++)
            if (A.col[j] == i) d[i] = 1.0 / std::sqrt(A.val[j]);
    Csr S = A;
    std::vector<double> sdiag(n, 0.0);
    for (int i = 0; i < n; i++)
        for (int j = A.row[i]; j < A.row[i + 1]; j++) {
            S.val[j] = (A.val[j] * d[A.col[j]]) * d[i];
            if (A.col[j] == i) sdiag[i] = S.val[j];
        }
    std::vector<std::vector<int>> cols(n);
    std::vector<std::vector<double>> vals(n);
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; i++) {
        std::vector<int> iwn;
        std::vector<double> x;
        double dk;
        afsai_row(S, i, iwn, x, dk);
        const double sf = sdiag[i] - dk;
        if (sf > 0.0) {
            const double s = 1.0 / std::sqrt(sf);
            for (size_t k = 0; k < iwn.size(); k++) {
                cols[i].push_back(iwn[k]);
                vals[i].push_back(s * x[k]);
            }
            cols[i].push_back(i);
            vals[i].push_back(s);
        } else {
            cols[i].push_back(i);
            vals[i].push_back(1.0);
        }
    }
    Csr G;
    G.n = G.m = n;
    G.row.assign(n + 1, 0);
    for (int i = 0; i < n; i++) G.row[i + 1] = G.row[i] + (int)cols[i].size();
    for (int i = 0; i < n; i++) {
        G.col.insert(G.col.end(), cols[i].begin(), cols[i].end());
        G.val.insert(G.val.end(), vals[i].begin(), vals[i].end());
    }
    return G;
}

Csr transpose(const Csr& G)
{
    Csr T;
    T.n = G.m;
    T.m = G.n;
    T.row.assign(T.n + 1, 0);
    for (int c : G.col) T.row[c + 1]++;
    for (int i = 0; i < T.n; i++) T.row[i + 1] += T.row[i];
    T.col.resize(G.col.size());
    T.val.resize(G.col.size());
    std::vector<int> fill(T.row.begin(), T.row.end() - 1);
    for (int i = 0; i < G.n; i++)
        for (int j = G.row[i]; j < G.row[i + 1]; j++) {
            const int t = fill[G.col[j]]++;
            T.col[t] = i;
            T.val[t] = G.val[j];
        }
    return T;
}

// Hierarchy construction. Restates bcmg_setup (bcmg.cu:12-49) -> Bootstrap::bootstrap with one
// hierarchy (bootstrap.cu:11-46) -> adaptiveCoarsening (matchingAggregation.cu:287-466) ->
// matchingAggregation (matchingAggregation.cu:106-269), with the parameters of
// AMG::BootBuildData::initByParams (AMG.cu:366-388): sweepnumber = aggrsweeps+1, w = 1,
// maxcoarsesize = (int)(40 * n^(1/3)) (AMG.cu:238-241).
// part0: the row partition of A0 over P ranks (offsets, P + 1 entries), or empty for np = 1.
Hierarchy* build(const Csr& A0, const Params& prm, bool record, const std::vector<int>& part0 = {})
{
    Hierarchy* H = new Hierarchy();
    H->prm = prm;
    H->maxcoarsesize = (int)(40 * std::pow((double)A0.n, 1.0 / 3.0));
    H->grid_sweeps = grid_sweeps(prm.cycle_type, prm.max_levels);
    H->lv.emplace_back();
    H->lv[0].A = A0;
    const bool parts = part0.size() > 2;
    H->lv[0].part = part0.empty() ? std::vector<int> { 0, A0.n } : part0;
    H->lv[0].M = abs_row_sum(A0);
    if (prm.preconditioner == 1) {
        // set_l1j (l1jacobi.cu:484-493): mydiag + addAbsoluteRowSumNoDiag
        H->l1d.assign(A0.n, 0.0);
        for (int i = 0; i < A0.n; i++) {
            double d = 0.0, off = 0.0;
            for (int j = A0.row[i]; j < A0.row[i + 1]; j++) {
                if (A0.col[j] == i) d = A0.val[j];
                else off += std::fabs(A0.val[j]);
            }
            H->l1d[i] = d + off;
        }
    }
    if (prm.preconditioner == 3) {
        H->G = afsai_build(A0);
        H->GT = transpose(H->G);
    }
    if (prm.preconditioner != 2) return H;
    const int sweepnumber = prm.aggrsweeps + 1;
    std::vector<double> w(A0.n, 1.0);
    H->ftcoarse = 1;
    double avcoarseratio = 0;
    int level;
    for (level = 1; level < prm.max_levels;) {
        const Csr* Ai_ = &H->lv[level - 1].A;
        Csr Ai_own;
        std::vector<double> wi_ = w, wi;
        std::vector<int> Pagg;
        std::vector<double> Pval;
        Csr Ai;
        std::vector<int> part_i = H->lv[level - 1].part, part_c;
        for (int i = 0; i < sweepnumber; i++) {
            std::vector<double> W;
            if (parts) edge_weights_parts(*Ai_, wi_, part_i, W);
            else edge_weights(*Ai_, wi_, W, nullptr);
            std::vector<int> M = match_suitor(*Ai_, W);
            std::vector<int> agg, f0, f1;
            std::vector<double> p;
            int nc;
            if (parts) {
                nc = make_pairwise_p_parts(M, wi_, part_i, agg, p, f0, f1, part_c);
            } else {
                nc = make_pairwise_p(M, wi_, agg, p, f0, f1);
                part_c = { 0, nc };
            }
            if (record) H->rec.push_back({ level - 1, i, nc, M, agg, p, wi_ });
            Ai = galerkin_pairwise(*Ai_, agg, p, f0, f1, nc);
            wi = restrict_weights(wi_, p, f0, f1);
            double size_precoarse = Ai_->n, size_coarse = Ai.n;
            double coarse_ratio = size_precoarse / size_coarse;
            if (coarse_ratio <= kCoarseRatioThreshold) H->ftcoarse = kFtcoarseInc;
            if (i == 0) {
                Pagg = agg;
                Pval = p;
            } else {
                for (size_t r = 0; r < Pagg.size(); r++) {
                    int c = Pagg[r];
                    Pval[r] = Pval[r] * p[c];
                    Pagg[r] = agg[c];
                }
            }
            if (size_coarse <= (double)H->ftcoarse * H->maxcoarsesize || i + 1 == sweepnumber) break;
            Ai_own = std::move(Ai);
            Ai_ = &Ai_own;
            wi_ = wi;
            part_i = part_c;
        }
        w = wi;
        Level& prev = H->lv[level - 1];
        prev.agg = Pagg;
        prev.p = Pval;
        const int nc = Ai.n;
        build_restriction(prev, nc);
        Level nl;
        nl.A = std::move(Ai);
        nl.part = part_c;
        nl.M = abs_row_sum(nl.A);
        H->lv.push_back(std::move(nl));
        double size_coarse = H->lv[level].A.n;
        avcoarseratio += H->lv[level - 1].A.n / size_coarse;
        level++;
        if (size_coarse <= (double)H->ftcoarse * H->maxcoarsesize) break;
    }
    // AMG::Hierarchy::finalize_cmplx / finalize_wcmplx (AMG.cu:144-165)
    double nnz0 = (double)H->lv[0].A.nnz(), c = 0, wc = 0;
    for (size_t i = 0; i < H->lv.size(); i++) {
        c += (double)H->lv[i].A.nnz();
        wc += std::pow(2.0, (double)i) * (double)H->lv[i].A.nnz();
    }
    H->op_cmplx = c / nnz0;
    H->op_wcmplx = wc / nnz0;
    H->avg_cratio = level > 1 ? avcoarseratio / (level - 1) : 1;
    return H;
}

// ------------------------------------------------------------------------------------------
// Solve: l1-Jacobi, V-cycle, FCG
// ------------------------------------------------------------------------------------------

// k sweeps of u <- ((f - A u) / M) + u with ping-pong buffers. Restates l1jacobi_iter
// (l1jacobi.cu:428-479) -> jacobi_adaptive_miniwarp_coarsest (:404-426) -> _jacobi_it_full<0>
// (:345-379).
void l1jacobi(int k, const Csr& A, const std::vector<double>& M, const double* f, double* u, double* tmp)
{
    const int n = A.n;
    double* src = u;
    double* dst = tmp;
    for (int s = 0; s < k; s++) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            double t = 0.0;
            for (int j = A.row[i]; j < A.row[i + 1]; j++) t += A.val[j] * src[A.col[j]];
            dst[i] = ((-t + f[i]) / M[i]) + src[i];
        }
        std::swap(src, dst);
    }
    if (src != u) std::memcpy(u, src, sizeof(double) * n);
}

struct Work {
    std::vector<std::vector<double>> rhs, x, x2;
    std::vector<double> res;
};

// One multigrid cycle on level l (0-based). Restates GAMG_cycle (GAMG_cycle.cu:58-236) at np=1.
void cycle(const Hierarchy& H, Work& wk, int l)
{
    const Params& prm = H.prm;
    const int L = (int)H.lv.size();
    const Level& lv = H.lv[l];
    const int n = lv.A.n;
    if (l == L - 1) {
        l1jacobi(prm.relaxnumber_coarse, lv.A, lv.M, wk.rhs[l].data(), wk.x[l].data(), wk.x2[l].data());
        return;
    }
    const int coeff = prm.cycle_type == 3 ? (1 << l) : 1;
    l1jacobi(prm.prerelax_sweeps * coeff, lv.A, lv.M, wk.rhs[l].data(), wk.x[l].data(), wk.x2[l].data());
    double* res = wk.res.data();
    spmv(lv.A, wk.x[l].data(), res);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) res[i] = wk.rhs[l][i] - res[i];
    const int nc = H.lv[l + 1].A.n;
    std::vector<double>& rc = wk.rhs[l + 1];
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nc; c++) {
        double s = 0.0;
        for (int t = lv.rptr[c]; t < lv.rptr[c + 1]; t++) s += lv.rval[t] * res[lv.ridx[t]];
        rc[c] = s;
    }
    std::fill(wk.x[l + 1].begin(), wk.x[l + 1].end(), 0.0);
    if (L > 2 || prm.relaxnumber_coarse > 0) {
        int visits = l < (int)H.grid_sweeps.size() ? H.grid_sweeps[l] : 1;
        for (int i = 1; i <= visits; i++) {
            cycle(H, wk, l + 1);
            if (l + 1 == L - 1) break;
        }
    }
    const std::vector<double>& xc = wk.x[l + 1];
    double* x = wk.x[l].data();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) x[i] = lv.p[i] * xc[lv.agg[i]] + x[i];
    l1jacobi(prm.postrelax_sweeps * coeff, lv.A, lv.M, wk.rhs[l].data(), x, wk.x2[l].data());
}

void prec_apply(const Hierarchy& H, Work& wk, const double* r, double* v)
{
    const int n = H.lv[0].A.n;
    if (H.prm.preconditioner == 1) {
        // l1jacobi_apply (l1jacobi.cu:513-523): l1jacsweeps sweeps from v (zero at every call site)
        std::vector<double> tmp(n);
        l1jacobi(H.prm.l1jacsweeps, H.lv[0].A, H.l1d, r, v, tmp.data());
        return;
    }
    if (H.prm.preconditioner == 3) {
        std::vector<double> t(n);
        spmv(H.G, r, t.data());
        spmv(H.GT, t.data(), v);
        return;
    }
    if (H.prm.preconditioner != 2) {
        std::memcpy(v, r, sizeof(double) * n);
        return;
    }
    std::memcpy(wk.rhs[0].data(), r, sizeof(double) * n);
    std::memcpy(wk.x[0].data(), v, sizeof(double) * n);
    cycle(H, wk, 0);
    std::memcpy(v, wk.x[0].data(), sizeof(double) * n);
}

struct SolveInfo {
    int niter;
    int retv;
    double delta0;
    double exit_res;
};

// Flexible CG with one reduction per iteration. Restates flexibileConjugateGradients_v3
// (FCG.cu:27-165): start-up :46-100, loop :102-156, niter = iter + 1 :164.
SolveInfo fcg(const Hierarchy& H, const double* b, double* x)
{
    const Csr& A = H.lv[0].A;
    const long n = A.n;
    Work wk;
    for (auto& l : H.lv) {
        wk.rhs.emplace_back(l.A.n, 0.0);
        wk.x.emplace_back(l.A.n, 0.0);
        wk.x2.emplace_back(l.A.n, 0.0);
    }
    wk.res.assign(n, 0.0);
    std::vector<double> v(n, 0.0), w(n), r(b, b + n), d, q;
    spmv(A, x, w.data());
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) r[i] = -1.0 * w[i] + 1.0 * r[i];
    const double delta0 = std::sqrt(dot(r.data(), r.data(), n));
    prec_apply(H, wk, r.data(), v.data());
    spmv(A, v.data(), w.data());
    double alpha = dot(r.data(), v.data(), n);
    double beta = dot(w.data(), v.data(), n);
    double delta = beta;
    double theta = alpha / delta;
    double gamma = 0.0;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) {
        x[i] = theta * v[i] + 1.0 * x[i];
        r[i] = -theta * w[i] + 1.0 * r[i];
    }
    double l2 = std::sqrt(dot(r.data(), r.data(), n));
    d = v;
    q = w;
    int iter = 0;
    const Params& prm = H.prm;
    do {
        const bool even = (iter % 2) == 0;
        std::vector<double>& pv = even ? v : d;   // preconditioned residual (new direction)
        std::vector<double>& pw = even ? w : q;   // A * pv
        std::vector<double>& od = even ? d : v;   // previous direction
        std::vector<double>& oq = even ? q : w;   // A * previous direction
        std::fill(pv.begin(), pv.end(), 0.0);
        prec_apply(H, wk, r.data(), pv.data());
        spmv(A, pv.data(), pw.data());
        double a = 0, bb = 0, g = 0;
#pragma omp parallel for reduction(+ : a, bb, g) schedule(static)
        for (long i = 0; i < n; i++) {
            a += r[i] * pv[i];
            bb += pw[i] * pv[i];
            g += oq[i] * pv[i];
        }
        alpha = a;
        beta = bb;
        gamma = g;
        theta = gamma / delta;
        delta = beta - ((gamma * gamma) / delta);
        const double theta2 = alpha / delta;
        double rr = 0.0;
#pragma omp parallel for reduction(+ : rr) schedule(static)
        for (long i = 0; i < n; i++) {
            double nv = -theta * od[i] + pv[i];
            pv[i] = nv;
            x[i] = theta2 * nv + x[i];
            double nw = -theta * oq[i] + pw[i];
            pw[i] = nw;
            r[i] = -theta2 * nw + r[i];
            rr += r[i] * r[i];
        }
        l2 = std::sqrt(rr);
        if (prm.dispnorm > 1) std::printf("%d) r norm: %.10lf\n", iter, l2);
        iter++;
    } while (l2 > prm.rtol * delta0 && iter < prm.itnlim);
    SolveInfo si;
    si.niter = iter + 1;
    si.retv = iter >= prm.itnlim ? -1 : 0;
    si.delta0 = delta0;
    si.exit_res = l2;
    return si;
}

Work make_work(const Hierarchy& H)
{
    Work wk;
    for (auto& l : H.lv) {
        wk.rhs.emplace_back(l.A.n, 0.0);
        wk.x.emplace_back(l.A.n, 0.0);
        wk.x2.emplace_back(l.A.n, 0.0);
    }
    wk.res.assign(H.lv[0].A.n, 0.0);
    return wk;
}

// Preconditioned CG, Hestenes-Stiefel form. Restates cg_hs (cghs/CG_HS.cu:25-151): delta0 =
// ||r0|| when stop_criterion == 1 else 1; u = B r from a zero guess; stop when ||r|| < rtol *
// delta0 (strict); niter = iter + 1 on convergence, itnlim otherwise.
SolveInfo cghs(const Hierarchy& H, const double* b, double* x)
{
    const Csr& A = H.lv[0].A;
    const long n = A.n;
    const Params& prm = H.prm;
    const bool pre = prm.preconditioner != 0;
    Work wk = make_work(H);
    std::vector<double> s(n, 0.0), p(n), r(b, b + n), u(n, 0.0), w(n);
    spmv(A, x, w.data());
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) r[i] = -1.0 * w[i] + 1.0 * r[i];
    if (pre) prec_apply(H, wk, r.data(), u.data());
    else u = r;
    p = u;
    const double delta0 = prm.stop_criterion == 1 ? std::sqrt(dot(r.data(), r.data(), n)) : 1.0;
    double rho_old = 0.0, l2 = 0.0;
    int iter, excnlim = -1, retv = -1;
    for (iter = 0; iter < prm.itnlim; iter++) {
        if (iter > 0) {
            if (pre) {
                std::fill(u.begin(), u.end(), 0.0);
                prec_apply(H, wk, r.data(), u.data());
            } else {
                u = r;
            }
            const double rho = dot(r.data(), u.data(), n);
            const double beta = rho / rho_old;
#pragma omp parallel for schedule(static)
            for (long i = 0; i < n; i++) p[i] = 1.0 * u[i] + beta * p[i];
        }
        spmv(A, p.data(), s.data());
        const double ur = dot(u.data(), r.data(), n);
        const double ps = dot(p.data(), s.data(), n);
        rho_old = ur;
        const double alpha = ur / ps;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; i++) {
            x[i] = alpha * p[i] + 1.0 * x[i];
            r[i] = -alpha * s[i] + 1.0 * r[i];
        }
        l2 = std::sqrt(dot(r.data(), r.data(), n));
        if (l2 < prm.rtol * delta0) {
            excnlim = 0;
            retv = 0;
            break;
        }
    }
    SolveInfo si;
    si.niter = iter + 1 + excnlim;
    si.retv = retv;
    si.delta0 = delta0;
    si.exit_res = l2;
    return si;
}

// ---- s-step CG (Chronopoulos and Gear) ------------------------------------------------------

// Matrix powers kernel (krylov_base/mpk.cu:10-83). sP is n x 2s column-major. Without a
// preconditioner: columns 0..s hold r, A r, ..., A^s r. With one: columns 0..s-1 hold
// P_j = (B A)^j B r and columns s..2s-1 hold A P_j (B applied from a zero guess).
void mpk(const Hierarchy& H, Work& wk, const double* r, int s, std::vector<double>& sP)
{
    const Csr& A = H.lv[0].A;
    const long n = A.n;
    double* P = sP.data();
    if (H.prm.preconditioner == 0) {
        std::memcpy(P, r, sizeof(double) * n);
        for (int i = 0; i < s; i++) spmv(A, P + i * n, P + (i + 1) * n);
        return;
    }
    std::fill(P, P + n, 0.0);
    prec_apply(H, wk, r, P);
    int pin = 0, pout = s;
    for (int i = 0; i < 2 * s - 1; i++) {
        if (i % 2 == 0) {
            spmv(A, P + pin * n, P + pout * n);
        } else {
            std::fill(P + pout * n, P + (pout + 1) * n, 0.0);
            prec_apply(H, wk, P + pin * n, P + pout * n);
        }
        const int t = pin;
        pin = pout;
        pout = t + 1;
    }
}

// The 2s moments (krylov_base/computevm.cu:6-31).
void computevm(const std::vector<double>& sP, int s, const double* r, long n, bool pre, double* vm)
{
    const double* P = sP.data();
    if (!pre) {
        for (int k = 0; k <= s; k++) vm[k] = dot(P + k * n, r, n);
        for (int k = 0; k < s - 1; k++) vm[s + 1 + k] = dot(P + (1 + k) * n, P + s * n, n);
    } else {
        for (int k = 0; k < s; k++) vm[k] = dot(P + k * n, r, n);
        for (int k = 0; k < s; k++) vm[s + k] = dot(P + k * n, P + (2 * s - 1) * n, n);
    }
}

// Cholesky factor (lower, column-major) in place; the square root is taken in single precision
// as in myChol (op/scalarWorkMO.cu:126-157, the build without LAPACK). Returns 1 when W is not
// positive definite.
int chol_lower(double* W, int n)
{
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < i; j++) {
            double sum = 0.0;
            for (int k = 0; k < j; k++) sum += W[i + k * n] * W[j + k * n];
            W[i + j * n] = (W[i + j * n] - sum) / W[j + j * n];
        }
        double sum = 0.0;
        for (int k = 0; k < i; k++) sum += W[i + k * n] * W[i + k * n];
        const double sq = W[i + i * n] - sum;
        if (sq < 0.0) return 1;
        W[i + i * n] = (double)sqrtf((float)sq);
    }
    return 0;
}

// rhs (n x nrhs, column-major, leading dimension nrhs) <- (L L^T)^{-1} rhs (mysolvem, :159-189).
void chol_solve(const double* L, double* rhs, int n, int nrhs)
{
    std::vector<double> y(n);
    for (int j = 0; j < nrhs; j++) {
        for (int i = 0; i < n; i++) {
            double sum = 0.0;
            for (int k = 0; k < i; k++) sum += L[i + n * k] * y[k];
            y[i] = (rhs[i + nrhs * j] - sum) / L[i + n * i];
        }
        for (int i = n - 1; i >= 0; i--) {
            double sum = 0.0;
            for (int k = i + 1; k < n; k++) sum += L[k + n * i] * rhs[k + nrhs * j];
            rhs[i + nrhs * j] = (y[i] - sum) / L[i + n * i];
        }
    }
}

// alpha (s) and beta (s x s) of one s-step iteration from the moments; W carries the Cholesky
// factor to the next call. Restates scalarWorkMO (op/scalarWorkMO.cu:191-245, no-LAPACK build).
int scalar_work(const double* vm, double* W, double* alpha, double* beta, int s, int iter)
{
    if (iter == 0) {
        for (int i = 0; i < s; i++)
            for (int j = 0; j < s; j++) W[i * s + j] = vm[i + j + 1];
        if (chol_lower(W, s)) return 1;
        std::memcpy(alpha, vm, sizeof(double) * s);
        chol_solve(W, alpha, s, 1);
        return 0;
    }
    std::vector<double> b1(s * s, 0.0), rhs1(2 * s - 1, 0.0);
    for (int i = 0; i < s; i++) {
        rhs1[s - 1 + i] = vm[i];
        for (int j = 0; j < i; j++) rhs1[s - 1 + i] += rhs1[s - 1 + j] * alpha[s - i + j - 1];
        rhs1[s - 1 + i] = -rhs1[s - 1 + i] / alpha[s - 1];
    }
    for (int i = 0; i < s; i++)
        for (int j = 0; j < s; j++) {
            b1[i + j * s] = -rhs1[i + j];
            beta[i + j * s] = -rhs1[i + j];
        }
    chol_solve(W, beta, s, s);
    for (int i = 0; i < s; i++)   // getNewW (:108-124): W = H(vm) - b1^T beta
        for (int j = 0; j < s; j++) {
            W[i + s * j] = vm[i + j + 1];
            for (int k = 0; k < s; k++) W[i + s * j] -= b1[k + s * i] * beta[k + s * j];
        }
    if (chol_lower(W, s)) return 1;
    std::memcpy(alpha, vm, sizeof(double) * s);
    chol_solve(W, alpha, s, 1);
    return 0;
}

// C(:, 0:s) += A(:, 0:s) * B (B s x s column-major); E += f * C(:, 0:s) * D (mydmmv,
// op/basic.cu:378-462). Column-major n x s blocks.
void block_update(const double* A, long n, int s, const double* B, double* C, const double* D, double* E, double f)
{
#pragma omp parallel for schedule(static)
    for (long row = 0; row < n; row++) {
        double e = 0.0;
        for (int col = 0; col < s; col++) {
            double ro = C[col * n + row];
            for (int k = 0; k < s; k++) ro += A[k * n + row] * B[k + s * col];
            C[col * n + row] = ro;
            e += ro * D[col];
        }
        E[row] += f * e;
    }
}

// s-step CG. Restates cgsstep (cgs/CGs.cu:43-224); CGS_CUBLAS (cgs_cublas/CGscublas.cu) and
// PIPELINED_CGS (pipelined_cgs/pipelinedCGs.cu) compute the same iterates in exact arithmetic.
// Each outer iteration advances s CG steps; niter counts outer iterations.
SolveInfo sstep_cg(const Hierarchy& H, const double* b, double* x)
{
    const Csr& A = H.lv[0].A;
    const long n = A.n;
    const Params& prm = H.prm;
    const int s = prm.sstep;
    const bool pre = prm.preconditioner != 0;
    Work wk = make_work(H);
    std::vector<double> r(b, b + n), w(n);
    auto residual = [&] {
        spmv(A, x, w.data());
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; i++) r[i] = -1.0 * w[i] + 1.0 * b[i];
    };
    residual();
    std::vector<double> sP1(n * 2 * s, 0.0), sP2(n * 2 * s, 0.0);
    std::vector<double> sCP1, sCP2;
    if (!pre && prm.ru_res) {
        sCP1.assign(n * s, 0.0);
        sCP2.assign(n * s, 0.0);
    }
    std::vector<double> vm(2 * s), alpha(s, 0.0), beta(s * s, 0.0), W(s * s, 0.0);
    const double delta0 = prm.stop_criterion == 1 ? std::sqrt(dot(r.data(), r.data(), n)) : 1.0;
    double l2 = 0.0;
    int iter, info = 0, excnlim = -1, retv = -1;
    for (iter = 0; iter < prm.itnlim; iter++) {
        if (iter > 0 && info == 0 && prm.ru_res && prm.rec_res_int > 0 && iter % prm.rec_res_int == 0) residual();
        std::vector<double>& cur = (iter % 2 == 0) ? sP2 : sP1;
        std::vector<double>& old = (iter % 2 == 0) ? sP1 : sP2;
        mpk(H, wk, r.data(), s, cur);
        computevm(cur, s, r.data(), n, pre, vm.data());
        info = scalar_work(vm.data(), W.data(), alpha.data(), beta.data(), s, iter);
        if (info != 0) {
            retv = info;
            break;
        }
        std::vector<double>* ccur = nullptr;
        std::vector<double>* cold = nullptr;
        if (prm.ru_res && !pre) {
            ccur = (iter % 2 == 0) ? &sCP2 : &sCP1;
            cold = (iter % 2 == 0) ? &sCP1 : &sCP2;
            std::memcpy(ccur->data(), cur.data() + n, sizeof(double) * n * s);
        }
        block_update(old.data(), n, s, beta.data(), cur.data(), alpha.data(), x, 1.0);
        if (prm.ru_res) {
            if (pre) block_update(old.data() + s * n, n, s, beta.data(), cur.data() + s * n, alpha.data(), r.data(), -1.0);
            else block_update(cold->data(), n, s, beta.data(), ccur->data(), alpha.data(), r.data(), -1.0);
        } else {
            residual();
        }
        l2 = std::sqrt(dot(r.data(), r.data(), n));
        if (l2 < prm.rtol * delta0) {
            excnlim = 0;
            retv = 0;
            break;
        }
    }
    SolveInfo si;
    si.niter = iter + 1 + excnlim;
    si.retv = retv;
    si.delta0 = delta0;
    si.exit_res = l2;
    return si;
}

Csr from_raw(int n, int m, long nnz, const int* row, const int* col, const double* val)
{
    Csr A;
    A.n = n;
    A.m = m;
    A.row.assign(row, row + n + 1);
    A.col.assign(col, col + nnz);
    A.val.assign(val, val + nnz);
    return A;
}

} // namespace

// ------------------------------------------------------------------------------------------
// C interface (ctypes)
// ------------------------------------------------------------------------------------------
extern "C" {

typedef struct orc_params {
    int solver, itnlim;
    double rtol;
    int dispnorm, preconditioner, bootstrap_type, max_hrc;
    double conv_ratio;
    int matchtype, aggrsweeps, aggr_type, max_levels, cycle_type, coarse_solver, relax_type;
    int relaxnumber_coarse, prerelax_sweeps, postrelax_sweeps, l1jacsweeps, sstep;
    int stop_criterion, ru_res, rec_res_int;
} orc_params;

static Params to_params(const orc_params* p)
{
    Params q;
    q.solver = p->solver;
    q.itnlim = p->itnlim;
    q.rtol = p->rtol;
    q.dispnorm = p->dispnorm;
    q.preconditioner = p->preconditioner;
    q.bootstrap_type = p->bootstrap_type;
    q.max_hrc = p->max_hrc;
    q.conv_ratio = p->conv_ratio;
    q.matchtype = p->matchtype;
    q.aggrsweeps = p->aggrsweeps;
    q.aggr_type = p->aggr_type;
    q.max_levels = p->max_levels;
    q.cycle_type = p->cycle_type;
    q.coarse_solver = p->coarse_solver;
    q.relax_type = p->relax_type;
    q.relaxnumber_coarse = p->relaxnumber_coarse;
    q.prerelax_sweeps = p->prerelax_sweeps;
    q.postrelax_sweeps = p->postrelax_sweeps;
    q.l1jacsweeps = p->l1jacsweeps;
    q.sstep = p->sstep;
    q.stop_criterion = p->stop_criterion;
    q.ru_res = p->ru_res;
    q.rec_res_int = p->rec_res_int;
    return q;
}

void orc_params_default(orc_params* p)
{
    Params d;
    p->solver = d.solver;
    p->itnlim = d.itnlim;
    p->rtol = d.rtol;
    p->dispnorm = d.dispnorm;
    p->preconditioner = d.preconditioner;
    p->bootstrap_type = d.bootstrap_type;
    p->max_hrc = d.max_hrc;
    p->conv_ratio = d.conv_ratio;
    p->matchtype = d.matchtype;
    p->aggrsweeps = d.aggrsweeps;
    p->aggr_type = d.aggr_type;
    p->max_levels = d.max_levels;
    p->cycle_type = d.cycle_type;
    p->coarse_solver = d.coarse_solver;
    p->relax_type = d.relax_type;
    p->relaxnumber_coarse = d.relaxnumber_coarse;
    p->prerelax_sweeps = d.prerelax_sweeps;
    p->postrelax_sweeps = d.postrelax_sweeps;
    p->l1jacsweeps = d.l1jacsweeps;
    p->sstep = d.sstep;
    p->stop_criterion = d.stop_criterion;
    p->ru_res = d.ru_res;
    p->rec_res_int = d.rec_res_int;
}

int orc_num_threads(int nt)
{
#ifdef _OPENMP
    if (nt > 0) omp_set_num_threads(nt);
    return omp_get_max_threads();
#else
    (void)nt;
    return 1;
#endif
}

void* orc_matrix_lap3d(int stencil, int nx, int ny, int nz, int P, int Q, int R)
{
    return new Csr(lap3d(stencil, nx, ny, nz, P, Q, R));
}

void* orc_matrix_from_csr(int n, int m, long nnz, const int* row, const int* col, const double* val)
{
    return new Csr(from_raw(n, m, nnz, row, col, val));
}

void orc_matrix_info(void* h, int* n, int* m, long* nnz)
{
    Csr* A = (Csr*)h;
    *n = A->n;
    *m = A->m;
    *nnz = A->nnz();
}

void orc_matrix_export(void* h, int* row, int* col, double* val)
{
    Csr* A = (Csr*)h;
    std::copy(A->row.begin(), A->row.end(), row);
    std::copy(A->col.begin(), A->col.end(), col);
    std::copy(A->val.begin(), A->val.end(), val);
}

void orc_matrix_free(void* h) { delete (Csr*)h; }

void orc_spmv(void* h, const double* x, double* y) { spmv(*(Csr*)h, x, y); }

// Weights of one sweep on A's pattern (diagonal slots 0); returns the clamped |a_hat| minimum.
double orc_edge_weights(void* h, const double* w, double* W)
{
    Csr* A = (Csr*)h;
    std::vector<double> wv(w, w + A->n), Wv;
    double mn = 0;
    edge_weights(*A, wv, Wv, &mn);
    std::copy(Wv.begin(), Wv.end(), W);
    return mn;
}

// method 0: greedy over sorted edges, 1: sequential suitor.
void orc_match(void* h, const double* W, int method, int* M)
{
    Csr* A = (Csr*)h;
    std::vector<double> Wv(W, W + A->nnz());
    std::vector<int> r = method == 0 ? match_greedy(*A, Wv) : match_suitor(*A, Wv);
    std::copy(r.begin(), r.end(), M);
}

void* orc_setup(void* h, const orc_params* p, int record)
{
    return build(*(Csr*)h, to_params(p), record != 0);
}

// The set-up of the reference run on nparts ranks, rank k holding rows part[k] .. part[k+1]-1.
void* orc_setup_parts(void* h, const orc_params* p, int record, int nparts, const int* part)
{
    return build(*(Csr*)h, to_params(p), record != 0, std::vector<int>(part, part + nparts + 1));
}

// Row partition of level l (nparts + 1 offsets).
int orc_hier_level_parts(void* h, int l, int* part)
{
    const std::vector<int>& pt = ((Hierarchy*)h)->lv[l].part;
    if (part) std::copy(pt.begin(), pt.end(), part);
    return (int)pt.size() - 1;
}

void orc_hier_free(void* h) { delete (Hierarchy*)h; }

// The AFSAI factor G (n rows) of an AFSAI hierarchy; row/col/val sized from orc_matrix_info.
void* orc_hier_afsai(void* h) { return &((Hierarchy*)h)->G; }

int orc_hier_levels(void* h) { return (int)((Hierarchy*)h)->lv.size(); }

void orc_hier_stats(void* h, double* out)
{
    Hierarchy* H = (Hierarchy*)h;
    out[0] = H->op_cmplx;
    out[1] = H->op_wcmplx;
    out[2] = H->avg_cratio;
    out[3] = H->maxcoarsesize;
    out[4] = H->ftcoarse;
}

void orc_hier_level_info(void* h, int l, int* n, long* nnz)
{
    Hierarchy* H = (Hierarchy*)h;
    *n = H->lv[l].A.n;
    *nnz = H->lv[l].A.nnz();
}

void* orc_hier_level_matrix(void* h, int l) { return &((Hierarchy*)h)->lv[l].A; }

void orc_hier_level_prolongator(void* h, int l, int* agg, double* p, double* M)
{
    Hierarchy* H = (Hierarchy*)h;
    const Level& L = H->lv[l];
    if (agg) std::copy(L.agg.begin(), L.agg.end(), agg);
    if (p) std::copy(L.p.begin(), L.p.end(), p);
    if (M) std::copy(L.M.begin(), L.M.end(), M);
}

int orc_hier_num_records(void* h) { return (int)((Hierarchy*)h)->rec.size(); }

void orc_hier_record(void* h, int k, int* level, int* sweep, int* n, int* nc)
{
    const SweepRecord& r = ((Hierarchy*)h)->rec[k];
    *level = r.level;
    *sweep = r.sweep;
    *n = (int)r.match.size();
    *nc = r.nc;
}

void orc_hier_record_data(void* h, int k, int* match, int* agg, double* p, double* w_in)
{
    const SweepRecord& r = ((Hierarchy*)h)->rec[k];
    std::copy(r.match.begin(), r.match.end(), match);
    std::copy(r.agg.begin(), r.agg.end(), agg);
    std::copy(r.p.begin(), r.p.end(), p);
    std::copy(r.w_in.begin(), r.w_in.end(), w_in);
}

// Pairwise Galerkin product of a given matching (same numbering as the set-up).
void* orc_galerkin(void* h, const int* M, const double* w, double* w_coarse)
{
    Csr* A = (Csr*)h;
    std::vector<int> Mv(M, M + A->n), agg, f0, f1;
    std::vector<double> wv(w, w + A->n), p;
    int nc = make_pairwise_p(Mv, wv, agg, p, f0, f1);
    if (w_coarse) {
        std::vector<double> wc = restrict_weights(wv, p, f0, f1);
        std::copy(wc.begin(), wc.end(), w_coarse);
    }
    return new Csr(galerkin_pairwise(*A, agg, p, f0, f1, nc));
}

// One V-cycle application v = B r (v is zeroed first, as FCG does before prec_apply).
void orc_vcycle(void* h, const double* r, double* v)
{
    Hierarchy* H = (Hierarchy*)h;
    Work wk;
    for (auto& l : H->lv) {
        wk.rhs.emplace_back(l.A.n, 0.0);
        wk.x.emplace_back(l.A.n, 0.0);
        wk.x2.emplace_back(l.A.n, 0.0);
    }
    wk.res.assign(H->lv[0].A.n, 0.0);
    std::fill(v, v + H->lv[0].A.n, 0.0);
    prec_apply(*H, wk, r, v);
}

// Solve with the hierarchy's solver: FCG (1), CGHS (0), or the s-step CG for CGS (2),
// PIPELINED_CGS (3) and CGS_CUBLAS (4), as solve() dispatches (solver/solve.cu:11-51).
int orc_solve(void* h, const double* b, double* x, int* niter, double* delta0, double* exit_res)
{
    const Hierarchy& H = *(Hierarchy*)h;
    SolveInfo si = H.prm.solver == 1 ? fcg(H, b, x) : H.prm.solver == 0 ? cghs(H, b, x) : sstep_cg(H, b, x);
    *niter = si.niter;
    *delta0 = si.delta0;
    *exit_res = si.exit_res;
    return si.retv;
}

} // extern "C"
