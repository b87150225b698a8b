// afsai.cu -- the AFSAI preconditioner: adaptive factorized sparse approximate inverse.
//
// Restates afsai_setup (BCMGX/src/preconditioner/afsai/afsai.cu:287-1090) at np = 1. On the
// diagonally scaled matrix S = D A D, D = diag(1 / sqrt(a_ii)) (finddiag, scalediag,
// CSRscaleA_0), every row i of the lower-triangular factor G grows one entry per step for up to
// 30 steps (AFSAISTEP, AFSAILFIL = 1):
//   1. gradient g_c = S(i, c) + sum_k x_k S(p_k, c) over the columns c < i, where p is the row's
//      pattern and x its coefficients (d_kapGrad_merge, kapGradCUDA_WiP.cu);
//   2. the column of largest |g_c| outside the pattern joins it (RISortSplit), ties to the
//      smallest column; a row with no candidate stops;
//   3. x = S(p, p)^{-1} (-S(p, i)) by a packed U^T U Cholesky (d_gatherFullSysAdapt, d_gFSA.cu;
//      cudacholdcMix, choldc.cu) and the Kaporin term dk = sum_k b_k x_k (multiscalar_product);
//   4. the row stops once |dk - dk_old| < 1e-3 dk_old or dk = 0 (check_done).
// Then G(i, p) = x / sqrt(S(i, i) - dk) and G(i, i) = 1 / sqrt(S(i, i) - dk) (createprc). The
// preconditioner is v = G^T (G r) (afsai_apply, :1092-1103), with G of the scaled matrix, as in
// the reference.
//
// Rows are independent, so one thread runs a row's whole adaptive loop: the gradient is a
// streaming merge of at most 31 sorted rows (no scratch vector), the small system lives in the
// thread's local memory. All arithmetic is separately rounded (no contraction), so G equals the
// oracle's restatement bit for bit.
#include "internal.h"
#include "common.cuh"

#include <algorithm>
#include <cstdint>

namespace bcmgx {

long long scan_exclusive(const int* in, int* out, long n, bool with_total, cudaStream_t s);
void scan_exclusive_dev(const int* in, int* out, long n, cudaStream_t s);
int num_sms();

namespace {

constexpr int kSteps = 30;            // AFSAISTEP * AFSAILFIL
constexpr int kRowCap = kSteps + 1;   // pattern plus the diagonal
constexpr double kEps = 0.001;        // AFSAIEPSILON

int grid_for(long n, int threads) { return (int)std::max<long>(1, std::min<long>((n + threads - 1) / threads, 1L << 30)); }

// d_i = 1 / sqrt(a_ii); err when a diagonal is missing or not positive
__global__ void k_afsai_diag(int n, const int* __restrict__ row, const int* __restrict__ col, const double* __restrict__ val,
    double* __restrict__ d, int* err)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double a = 0.0;
        for (int j = row[i]; j < row[i + 1]; j++)
            if (col[j] == i) a = val[j];
        if (!(a > 0.0)) atomicExch(err, 1);
        d[i] = __ddiv_rn(1.0, __dsqrt_rn(a));
    }
}

// S_ij = (a_ij d_j) d_i (_CSR_scale_mini_warp<1>, CSR.cu:539-565)
__global__ void k_afsai_scale(int n, const int* __restrict__ row, const int* __restrict__ col, const double* __restrict__ val,
    const double* __restrict__ d, double* __restrict__ S)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double di = d[i];
        for (int j = row[i]; j < row[i + 1]; j++) S[j] = __dmul_rn(__dmul_rn(val[j], d[col[j]]), di);
    }
}

// U^T U x = b in place (U upper-packed by columns, inverted diagonal); false on a pivot <= 0
__device__ bool chol_solve(double* l, double* x, int n)
{
    int ooffi = 0;
    for (int i = 0; i < n; i++) {
        int ooffj = ooffi;
        for (int j = i; j < n; j++) {
            double sum = l[i + ooffj];
            for (int k = 0; k < i; k++) sum = __dsub_rn(sum, __dmul_rn(l[ooffi + k], l[ooffj + k]));
            if (i == j) {
                if (sum <= 0.0) return false;
                l[ooffj + i] = __ddiv_rn(1.0, __dsqrt_rn(sum));
            } else {
                l[ooffj + i] = __dmul_rn(sum, l[ooffi + i]);
            }
            ooffj += j + 1;
        }
        ooffi += i + 1;
    }
    ooffi = 0;
    for (int i = 0; i < n; i++) {
        double sum = x[i];
        for (int j = i - 1; j >= 0; j--) sum = __dsub_rn(sum, __dmul_rn(l[ooffi + j], x[j]));
        x[i] = __dmul_rn(sum, l[ooffi + i]);
        ooffi += i + 1;
    }
    ooffi = n * (n - 1) / 2;
    for (int i = n - 1; i >= 0; i--) {
        double sum = x[i];
        int ooffj = ooffi + i;
        for (int j = i + 1; j < n; j++) {
            sum = __dsub_rn(sum, __dmul_rn(l[ooffj + i + 1], x[j]));
            ooffj += j + 1;
        }
        x[i] = __dmul_rn(sum, l[ooffi + i]);
        ooffi -= i;
    }
    return true;
}

// One row of G per thread; writes len[i] <= kRowCap entries at cols/vals[i * kRowCap ...].
__global__ void __launch_bounds__(128) k_afsai_rows(int n, const int* __restrict__ row, const int* __restrict__ col,
    const double* __restrict__ S, int* __restrict__ len, int* __restrict__ gcol, double* __restrict__ gval)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int iwn[kSteps];
    double x[kSteps], b[kSteps], M[kSteps * (kSteps + 1) / 2];
    int pos[kRowCap], end[kRowCap];
    double fac[kRowCap];
    int m = 0;
    double dk = 0.0, dk_old = 0.0;
    for (int step = 0; step < kSteps; step++) {
        pos[0] = row[i];
        end[0] = row[i + 1];
        fac[0] = 1.0;
        for (int k = 0; k < m; k++) {
            pos[k + 1] = row[iwn[k]];
            end[k + 1] = row[iwn[k] + 1];
            fac[k + 1] = x[k];
        }
        int best = -1, iw = 0;
        double bestv = 0.0;
        for (;;) {
            int c = INT32_MAX;
            for (int k = 0; k <= m; k++)
                if (pos[k] < end[k]) c = min(c, col[pos[k]]);
            if (c >= i) break;
            double g = 0.0;
            for (int k = 0; k <= m; k++)
                if (pos[k] < end[k] && col[pos[k]] == c) {
                    g = __dadd_rn(g, __dmul_rn(S[pos[k]], fac[k]));
                    pos[k]++;
                }
            while (iw < m && iwn[iw] < c) iw++;
            if (iw < m && iwn[iw] == c) continue;
            if (fabs(g) > bestv) {
                bestv = fabs(g);
                best = c;
            }
        }
        if (best < 0) break;
        int at = m;
        while (at > 0 && iwn[at - 1] > best) {
            iwn[at] = iwn[at - 1];
            at--;
        }
        iwn[at] = best;
        m++;
        for (int t = 0; t < m * (m + 1) / 2; t++) M[t] = 0.0;
        for (int r = 0; r < m; r++) {
            b[r] = 0.0;
            int jj = row[iwn[r]];
            const int je = row[iwn[r] + 1];
            for (int cidx = r; cidx < m; cidx++) {
                while (jj < je && col[jj] < iwn[cidx]) jj++;
                if (jj == je) break;
                if (col[jj] == iwn[cidx]) M[cidx * (cidx + 1) / 2 + r] = S[jj];
            }
        }
        for (int jj = row[i], r = 0; jj < row[i + 1] && r < m && col[jj] < i;) {
            if (iwn[r] > col[jj]) {
                jj++;
            } else if (iwn[r] == col[jj]) {
                b[r] = -S[jj];
                jj++;
                r++;
            } else {
                r++;
            }
        }
        for (int r = 0; r < m; r++) x[r] = b[r];
        if (!chol_solve(M, x, m)) {   // not reached for SPD matrices: zero coefficients
            for (int r = 0; r < m; r++) x[r] = 0.0;
            dk = 0.0;
            break;
        }
        double d = 0.0;
        for (int r = 0; r < m; r++) d = __dadd_rn(d, __dmul_rn(b[r], x[r]));
        dk = d;
        const bool conv = fabs(__dsub_rn(dk, dk_old)) < __dmul_rn(kEps, dk_old) || dk == 0.0;
        dk_old = dk;
        if (conv) break;
    }
    double sii = 0.0;
    for (int j = row[i]; j < row[i + 1]; j++)
        if (col[j] == i) sii = S[j];
    const double sf = __dsub_rn(sii, dk);
    int* oc = gcol + i * kRowCap;
    double* ov = gval + i * kRowCap;
    if (sf > 0.0) {
        const double s = __ddiv_rn(1.0, __dsqrt_rn(sf));
        for (int k = 0; k < m; k++) {
            oc[k] = iwn[k];
            ov[k] = __dmul_rn(s, x[k]);
        }
        oc[m] = (int)i;
        ov[m] = s;
        len[i] = m + 1;
    } else {
        oc[0] = (int)i;
        ov[0] = 1.0;
        len[i] = 1;
    }
}

__global__ void k_afsai_compact(int n, const int* __restrict__ rowptr, const int* __restrict__ gcol,
    const double* __restrict__ gval, int* __restrict__ col, double* __restrict__ val)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        for (int t = rowptr[i]; t < rowptr[i + 1]; t++) {
            col[t] = gcol[i * kRowCap + (t - rowptr[i])];
            val[t] = gval[i * kRowCap + (t - rowptr[i])];
        }
}

__global__ void k_count_cols(long nnz, const int* __restrict__ col, int* __restrict__ cnt)
{
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < nnz; t += (long)gridDim.x * blockDim.x) atomicAdd(cnt + col[t], 1);
}

// transpose fill (atomic slots), then each row of the transpose sorted by column
__global__ void k_transpose_fill(int n, const int* __restrict__ row, const int* __restrict__ col, const double* __restrict__ val,
    int* __restrict__ fill, int* __restrict__ tcol, double* __restrict__ tval)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        for (int j = row[i]; j < row[i + 1]; j++) {
            const int t = atomicAdd(fill + col[j], 1);
            tcol[t] = (int)i;
            tval[t] = val[j];
        }
}

__global__ void k_sort_rows(int n, const int* __restrict__ row, int* __restrict__ col, double* __restrict__ val)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        for (int a = row[i] + 1; a < row[i + 1]; a++) {
            const int c = col[a];
            const double v = val[a];
            int b = a - 1;
            while (b >= row[i] && col[b] > c) {
                col[b + 1] = col[b];
                val[b + 1] = val[b];
                b--;
            }
            col[b + 1] = c;
            val[b + 1] = v;
        }
}

}  // namespace

// Builds G and G^T of the hierarchy's level-0 matrix (AFSAI preconditioner set-up).
void afsai_build_dev(bcmgx_hierarchy* H)
{
    cudaStream_t s = H->stream;
    const DevCsr& A = H->lv[0].A;
    const int n = A.n;
    DBuf<double> d, S, gval;
    DBuf<int> len, gcol, err;
    d.alloc(n, s);
    S.alloc(std::max<int64_t>(A.nnz, 1), s);
    err.alloc(1, s);
    BCMGX_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    note_launch(); k_afsai_diag<<<grid_for(n, 256), 256, 0, s>>>(n, A.row.p, A.col.p, A.val.p, d.p, err.p);
    note_launch(); k_afsai_scale<<<grid_for(n, 256), 256, 0, s>>>(n, A.row.p, A.col.p, A.val.p, d.p, S.p);
    BCMGX_CHECK_LAUNCH();
    int e = 0;
    BCMGX_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BCMGX_CUDA(cudaStreamSynchronize(s));
    BCMGX_REQUIRE(e == 0, BCMGX_ERR_INVALID_INPUT, "AFSAI needs a positive diagonal");
    len.alloc((size_t)n + 1, s);
    gcol.alloc((size_t)n * kRowCap, s);
    gval.alloc((size_t)n * kRowCap, s);
    note_launch(); k_afsai_rows<<<grid_for(n, 128), 128, 0, s>>>(n, A.row.p, A.col.p, S.p, len.p, gcol.p, gval.p);
    BCMGX_CHECK_LAUNCH();
    DevCsr& G = H->afsai_G;
    G.n = G.m = n;
    G.row.alloc((size_t)n + 1, s);
    G.nnz = scan_exclusive(len.p, G.row.p, n, true, s);
    G.col.alloc(G.nnz, s);
    G.val.alloc(G.nnz, s);
    note_launch(); k_afsai_compact<<<grid_for(n, 256), 256, 0, s>>>(n, G.row.p, gcol.p, gval.p, G.col.p, G.val.p);
    BCMGX_CHECK_LAUNCH();
    G.tpr = default_tpr(n, G.nnz);
    DevCsr& T = H->afsai_GT;
    T.n = T.m = n;
    T.nnz = G.nnz;
    DBuf<int> cnt, fill;
    cnt.alloc((size_t)n + 1, s);
    BCMGX_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * ((size_t)n + 1), s));
    note_launch(); k_count_cols<<<grid_for(G.nnz, 256), 256, 0, s>>>(G.nnz, G.col.p, cnt.p);
    BCMGX_CHECK_LAUNCH();
    T.row.alloc((size_t)n + 1, s);
    scan_exclusive_dev(cnt.p, T.row.p, n, s);
    fill.alloc((size_t)n + 1, s);
    BCMGX_CUDA(cudaMemcpyAsync(fill.p, T.row.p, sizeof(int) * ((size_t)n + 1), cudaMemcpyDeviceToDevice, s));
    T.col.alloc(T.nnz, s);
    T.val.alloc(T.nnz, s);
    note_launch(); k_transpose_fill<<<grid_for(n, 256), 256, 0, s>>>(n, G.row.p, G.col.p, G.val.p, fill.p, T.col.p, T.val.p);
    note_launch(); k_sort_rows<<<grid_for(n, 256), 256, 0, s>>>(n, T.row.p, T.col.p, T.val.p);
    BCMGX_CHECK_LAUNCH();
    T.tpr = default_tpr(n, T.nnz);
    H->afsai_tmp.alloc(n, s);
    BCMGX_CUDA(cudaStreamSynchronize(s));
}

// v = G^T (G r)
void afsai_apply(bcmgx_hierarchy* H, const double* r, double* v, const int* skip)
{
    rowop_spmv(H->afsai_G, r, H->afsai_tmp.p, skip, H->stream);
    rowop_spmv(H->afsai_GT, H->afsai_tmp.p, v, skip, H->stream);
}

}  // namespace bcmgx
