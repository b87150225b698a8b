// krylov.cu -- the reference's other Krylov solvers on the same kernels and drivers as FCG.
//
//  * CGHS: preconditioned CG in Hestenes-Stiefel form (BCMGX/src/solver/cghs/CG_HS.cu:25-151).
//  * CGS: the s-step CG of Chronopoulos and Gear (BCMGX/src/solver/cgs/CGs.cu:43-224) with its
//    matrix powers kernel (krylov_base/mpk.cu:10-83), moments (krylov_base/computevm.cu:6-31) and
//    small dense work (op/scalarWorkMO.cu:108-245). CGS_CUBLAS (cgs_cublas/CGscublas.cu) and
//    PIPELINED_CGS (pipelined_cgs/pipelinedCGs.cu) compute the same iterates in exact arithmetic:
//    the first does the small dense products with cuBLAS, the second overlaps the moments'
//    MPI_Iallreduce with the next matrix powers kernel, which has nothing to hide on one GPU.
//    All three run this code.
//
// All scalars live on the device (KryState); the s x s Cholesky work runs in a one-thread kernel,
// so an iteration needs no host round trip and the solve is captured as one CUDA graph (start-up,
// then a WHILE conditional node over two iterations), or driven from the host one iteration ahead
// (use_graph = 0), exactly as the FCG solve. Both stop on ||r|| < rtol * delta0 (strict), with
// delta0 = ||r0|| when stop_criterion = 1 and 1 otherwise (CG_HS.cu:80-82, CGs.cu:115-117).
#include "internal.h"
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

namespace bcmgx {

int num_sms();

namespace {

constexpr int kThreads = 256;
constexpr int kBlocksPerSM = 8;
constexpr int kMaxS = 8;          // s-step limit (2s moments in one reduction)

struct KryState {
    double rho, ps, alpha, beta, rnorm2, delta0, tol;
    double vm[2 * kMaxS];
    double W[kMaxS * kMaxS];      // Cholesky factor of the moment matrix, carried between iterations
    double sa[kMaxS];             // alpha (s)
    double sb[kMaxS * kMaxS];     // beta (s x s, column-major)
    int iter, itnlim, done, bad, resid_skip;
    int ticket[4];
};

// grid of a grid-stride kernel over n elements: resident blocks only, at most kBlocksPerSM per SM
// (the size of the reduction partials)
template <typename Kern>
int red_blocks(Kern kern, long n)
{
    return std::min(fit_grid(kern, kThreads, (n + kThreads - 1) / kThreads), num_sms() * kBlocksPerSM);
}

__global__ void k_kry_init(KryState* st, int itnlim)
{
    KryState z {};
    z.itnlim = itnlim;
    *st = z;
}

// delta0 = ||r0|| (stop_criterion 1) or 1, tol = rtol * delta0
__global__ void __launch_bounds__(kThreads) k_kry_norm0(int n, const double* __restrict__ r, KryState* st, double* part,
    double rtol, int stop_criterion)
{
    double acc[1] = { 0.0 };
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) acc[0] += r[i] * r[i];
    double out[1];
    if (grid_sum<1>(acc, part, &st->ticket[0], out) && threadIdx.x == 0) {
        st->delta0 = stop_criterion == 1 ? sqrt(out[0]) : 1.0;
        st->tol = rtol * st->delta0;
    }
}

__global__ void k_kry_copy(long n, const double* __restrict__ a, double* __restrict__ b, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) b[i] = a[i];
}

// ---- CGHS --------------------------------------------------------------------------------

// rho = r . u; in the loop (MODE 1) also beta = rho / rho_previous (CG_HS.cu:94-111)
template <int MODE>
__global__ void __launch_bounds__(kThreads) k_cg_rho(int n, const double* __restrict__ r, const double* __restrict__ u,
    KryState* st, double* part, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    double acc[1] = { 0.0 };
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) acc[0] += r[i] * u[i];
    double out[1];
    if (grid_sum<1>(acc, part, &st->ticket[1], out) && threadIdx.x == 0) {
        if (MODE == 1) st->beta = out[0] / st->rho;
        st->rho = out[0];
    }
}

// p = u + beta p (my_axpby, CG_HS.cu:113-117)
__global__ void k_cg_p(int n, const double* __restrict__ u, double* __restrict__ p, const KryState* st, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    const double beta = st->beta;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        p[i] = 1.0 * u[i] + beta * p[i];
}

// ps = p . s for s = A p (computed before); alpha = rho / ps (CG_HS.cu:120-136)
__global__ void __launch_bounds__(kThreads) k_cg_ps(int n, const double* __restrict__ p, const double* __restrict__ s,
    KryState* st, double* part, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    double acc[1] = { 0.0 };
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) acc[0] += p[i] * s[i];
    double out[1];
    if (grid_sum<1>(acc, part, &st->ticket[2], out) && threadIdx.x == 0) {
        st->ps = out[0];
        st->alpha = st->rho / out[0];
        if (!isfinite(st->alpha)) st->bad = 1;
    }
}

// x += alpha p, r -= alpha s, ||r|| and the stopping test (CG_HS.cu:138-157)
__global__ void __launch_bounds__(kThreads) k_cg_update(int n, const double* __restrict__ p, const double* __restrict__ s,
    double* __restrict__ x, double* __restrict__ r, KryState* st, double* part, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    if (st->bad) {
        if (blockIdx.x == 0 && threadIdx.x == 0) st->done = 1;
        return;
    }
    const double a = st->alpha;
    double acc[1] = { 0.0 };
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        x[i] = a * p[i] + 1.0 * x[i];
        const double ri = -a * s[i] + 1.0 * r[i];
        r[i] = ri;
        acc[0] += ri * ri;
    }
    double out[1];
    if (grid_sum<1>(acc, part, &st->ticket[3], out) && threadIdx.x == 0) {
        st->rnorm2 = out[0];
        st->iter += 1;
        const double l2 = sqrt(out[0]);
        if (!isfinite(l2)) st->bad = 1;
        st->done = (l2 < st->tol || st->iter >= st->itnlim || st->bad) ? 1 : 0;
    }
}

// ---- s-step CG -----------------------------------------------------------------------------

// Pairs of the 2s moments: vm[k] = P[:, ia[k]] . (ib[k] < 0 ? r : P[:, ib[k]]) (computevm.cu:14-20).
struct MomentPairs {
    int np;
    int ia[2 * kMaxS], ib[2 * kMaxS];
};

__global__ void __launch_bounds__(kThreads) k_sstep_moments(int n, const double* __restrict__ P, const double* __restrict__ r,
    MomentPairs mp, KryState* st, double* part, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    double acc[2 * kMaxS];
#pragma unroll
    for (int k = 0; k < 2 * kMaxS; k++) acc[k] = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double ri = r[i];
#pragma unroll
        for (int k = 0; k < 2 * kMaxS; k++) {
            if (k < mp.np) {
                const double bi = mp.ib[k] < 0 ? ri : P[(long)mp.ib[k] * n + i];
                acc[k] += P[(long)mp.ia[k] * n + i] * bi;
            }
        }
    }
    double out[2 * kMaxS];
    if (grid_sum<2 * kMaxS>(acc, part, &st->ticket[0], out) && threadIdx.x == 0)
        for (int k = 0; k < mp.np; k++) st->vm[k] = out[k];
}

// Cholesky factor (lower, column-major) in place, square root in single precision as myChol
// (scalarWorkMO.cu:126-157, the build without LAPACK); false when W is not positive definite.
__device__ bool sstep_chol(double* W, int n)
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
        if (!(sq >= 0.0)) return false;
        W[i + i * n] = (double)sqrtf((float)sq);
    }
    return true;
}

// rhs (n x nrhs, column-major, leading dimension nrhs) <- (L L^T)^{-1} rhs (mysolvem, :159-189)
__device__ void sstep_solve(const double* L, double* rhs, int n, int nrhs)
{
    double y[kMaxS];
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

// alpha and beta of one outer iteration from the moments (scalarWorkMO, :191-245, no-LAPACK
// build). A moment matrix that is not positive definite ends the solve (the reference returns
// info = 1 and breaks, CGs.cu:134-138): bad and done are set and x, r stay unchanged.
__global__ void k_sstep_scalar(KryState* st, int s, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    const double* vm = st->vm;
    double* W = st->W;
    double* alpha = st->sa;
    double* beta = st->sb;
    bool ok = true;
    if (st->iter == 0) {
        for (int i = 0; i < s; i++)
            for (int j = 0; j < s; j++) W[i * s + j] = vm[i + j + 1];
        ok = sstep_chol(W, s);
        if (ok) {
            for (int i = 0; i < s; i++) alpha[i] = vm[i];
            sstep_solve(W, alpha, s, 1);
        }
    } else {
        double b1[kMaxS * kMaxS], rhs1[2 * kMaxS - 1];
        for (int i = 0; i < 2 * s - 1; i++) rhs1[i] = 0.0;
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
        sstep_solve(W, beta, s, s);
        for (int i = 0; i < s; i++)   // getNewW (:108-124): W = H(vm) - b1^T beta
            for (int j = 0; j < s; j++) {
                double w = vm[i + j + 1];
                for (int k = 0; k < s; k++) w -= b1[k + s * i] * beta[k + s * j];
                W[i + s * j] = w;
            }
        ok = sstep_chol(W, s);
        if (ok) {
            for (int i = 0; i < s; i++) alpha[i] = vm[i];
            sstep_solve(W, alpha, s, 1);
        }
    }
    if (!ok) {
        st->bad = 1;
        st->done = 1;
    }
}

// C(:, 0:s) += A(:, 0:s) * beta;  E += f * C(:, 0:s) * alpha  (mydmmv, op/basic.cu:378-462), on
// column-major n x s blocks. NORM: E is the residual; ||E||^2 and the stopping test follow.
template <bool NORM>
__global__ void __launch_bounds__(kThreads) k_sstep_update(int n, int s, const double* __restrict__ A, double* __restrict__ C,
    double* __restrict__ E, double f, KryState* st, double* part, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    __shared__ double sb[kMaxS * kMaxS], sa[kMaxS];
    for (int t = threadIdx.x; t < s * s; t += blockDim.x) sb[t] = st->sb[t];
    for (int t = threadIdx.x; t < s; t += blockDim.x) sa[t] = st->sa[t];
    __syncthreads();
    double acc[1] = { 0.0 };
    for (long row = (long)blockIdx.x * blockDim.x + threadIdx.x; row < n; row += (long)gridDim.x * blockDim.x) {
        double e = 0.0;
        for (int c = 0; c < s; c++) {
            double ro = C[c * (long)n + row];
            for (int k = 0; k < s; k++) ro += A[k * (long)n + row] * sb[k + s * c];
            C[c * (long)n + row] = ro;
            e += ro * sa[c];
        }
        const double v = E[row] + f * e;
        E[row] = v;
        if (NORM) acc[0] += v * v;
    }
    if (!NORM) return;
    double out[1];
    if (grid_sum<1>(acc, part, &st->ticket[3], out) && threadIdx.x == 0) {
        st->rnorm2 = out[0];
        st->iter += 1;
        const double l2 = sqrt(out[0]);
        if (!isfinite(l2)) st->bad = 1;
        st->done = (l2 < st->tol || st->iter >= st->itnlim || st->bad) ? 1 : 0;
    }
}

// ||r||^2 and the stopping test after a recomputed residual (ru_res = 0, CGs.cu:170-174)
__global__ void __launch_bounds__(kThreads) k_sstep_norm_stop(int n, const double* __restrict__ r, KryState* st, double* part,
    const int* __restrict__ skip)
{
    if (skip && *skip) return;
    double acc[1] = { 0.0 };
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) acc[0] += r[i] * r[i];
    double out[1];
    if (grid_sum<1>(acc, part, &st->ticket[3], out) && threadIdx.x == 0) {
        st->rnorm2 = out[0];
        st->iter += 1;
        const double l2 = sqrt(out[0]);
        if (!isfinite(l2)) st->bad = 1;
        st->done = (l2 < st->tol || st->iter >= st->itnlim || st->bad) ? 1 : 0;
    }
}

// resid_skip = done, or not an iteration at which the residual is recomputed (CGs.cu:121-129)
__global__ void k_sstep_resid_flag(KryState* st, int rec_res_int)
{
    const int it = st->iter;
    st->resid_skip = (st->done || !(it > 0 && it % rec_res_int == 0)) ? 1 : 0;
}

__global__ void k_kry_set_while(cudaGraphConditionalHandle h, const KryState* st)
{
    cudaGraphSetConditional(h, st->done ? 0u : 1u);
}

}  // namespace

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
struct KrylovWork {
    int s = 0;
    DBuf<double> u, p, sv;             // CGHS: preconditioned residual, direction, A p
    DBuf<double> P1, P2, C1, C2;       // s-step bases (n x 2s) and copies of the A-columns (n x s)
    DBuf<double> part;
    DBuf<KryState> st;
    KryState* st_host = nullptr;       // two pinned slots
    cudaGraphExec_t graph = nullptr;
    long long startup_kernels = 0, body_kernels = 0;
    ~KrylovWork()
    {
        if (graph) cudaGraphExecDestroy(graph);
        pinned_free(st_host);
    }
};

void free_krylov(KrylovWork* w) { delete w; }

namespace {

bool sstep_solver(int solver)
{
    return solver == BCMGX_SOLVER_CGS || solver == BCMGX_SOLVER_PIPELINED_CGS || solver == BCMGX_SOLVER_CGS_CUBLAS;
}

KrylovWork& krylov_work(bcmgx_hierarchy* H)
{
    if (H->krylov) return *H->krylov;
    H->krylov = new KrylovWork();
    KrylovWork& wk = *H->krylov;
    cudaStream_t s = H->stream;
    const size_t n = (size_t)H->lv[0].A.n;
    const bcmgx_params& P = H->prm;
    if (sstep_solver(P.solver)) {
        wk.s = P.sstep;
        wk.P1.alloc(n * 2 * wk.s, s);
        wk.P2.alloc(n * 2 * wk.s, s);
        if (P.preconditioner == BCMGX_PREC_NONE && P.ru_res) {
            wk.C1.alloc(n * wk.s, s);
            wk.C2.alloc(n * wk.s, s);
        }
    } else {
        wk.u.alloc(n, s);
        wk.p.alloc(n, s);
        wk.sv.alloc(n, s);
    }
    wk.part.alloc((size_t)num_sms() * kBlocksPerSM * 2 * kMaxS, s);
    wk.st.alloc(1, s);
    wk.st_host = (KryState*)pinned_alloc(2 * sizeof(KryState));
    return wk;
}

void startup_common(bcmgx_hierarchy* H, KrylovWork& wk, const double* b, const double* x)
{
    cudaStream_t s = H->stream;
    const DevCsr& A = H->lv[0].A;
    persist_reset_ext(H, s);
    note_launch();
    k_kry_init<<<1, 1, 0, s>>>(wk.st.p, H->prm.itnlim);
    rowop_resid(A, x, b, H->r.p, nullptr, s);   // r = b - A x0
    note_launch();
    k_kry_norm0<<<red_blocks(k_kry_norm0, A.n), kThreads, 0, s>>>(A.n, H->r.p, wk.st.p, wk.part.p, H->prm.rtol, H->prm.stop_criterion);
    BCMGX_CHECK_LAUNCH();
}

// CGHS start-up (CG_HS.cu:56-76): r0, delta0, u = B r0, p = u, rho = r . u
void cghs_startup(bcmgx_hierarchy* H, KrylovWork& wk, const double* b, double* x)
{
    cudaStream_t s = H->stream;
    const int n = H->lv[0].A.n;
    startup_common(H, wk, b, x);
    const bool pre = H->prm.preconditioner != BCMGX_PREC_NONE;
    const double* u = pre ? wk.u.p : H->r.p;
    if (pre) prec_apply_impl(H, H->r.p, wk.u.p, nullptr);
    note_launch();
    k_kry_copy<<<red_blocks(k_kry_copy, n), kThreads, 0, s>>>(n, u, wk.p.p, nullptr);
    note_launch();
    k_cg_rho<0><<<red_blocks(k_cg_rho<0>, n), kThreads, 0, s>>>(n, H->r.p, u, wk.st.p, wk.part.p, nullptr);
    BCMGX_CHECK_LAUNCH();
}

// One CGHS iteration: s = A p, alpha, x and r updated with the stopping test, then the next
// direction from u = B r (CG_HS.cu:91-157, with the direction update moved to the end of the
// loop body so that every iteration runs the same kernels).
void cghs_iteration(bcmgx_hierarchy* H, KrylovWork& wk, double* x, const int* skip)
{
    cudaStream_t s = H->stream;
    const DevCsr& A = H->lv[0].A;
    const int n = A.n;
    const bool pre = H->prm.preconditioner != BCMGX_PREC_NONE;
    const double* u = pre ? wk.u.p : H->r.p;
    rowop_spmv(A, wk.p.p, wk.sv.p, skip, s);
    note_launch();
    k_cg_ps<<<red_blocks(k_cg_ps, n), kThreads, 0, s>>>(n, wk.p.p, wk.sv.p, wk.st.p, wk.part.p, skip);
    note_launch();
    k_cg_update<<<red_blocks(k_cg_update, n), kThreads, 0, s>>>(n, wk.p.p, wk.sv.p, x, H->r.p, wk.st.p, wk.part.p, skip);
    BCMGX_CHECK_LAUNCH();
    if (pre) prec_apply_impl(H, H->r.p, wk.u.p, skip);
    note_launch();
    k_cg_rho<1><<<red_blocks(k_cg_rho<1>, n), kThreads, 0, s>>>(n, H->r.p, u, wk.st.p, wk.part.p, skip);
    note_launch();
    k_cg_p<<<red_blocks(k_cg_p, n), kThreads, 0, s>>>(n, u, wk.p.p, wk.st.p, skip);
    BCMGX_CHECK_LAUNCH();
}

void sstep_startup(bcmgx_hierarchy* H, KrylovWork& wk, const double* b, double* x)
{
    cudaStream_t s = H->stream;
    const size_t n = (size_t)H->lv[0].A.n;
    startup_common(H, wk, b, x);
    BCMGX_CUDA(cudaMemsetAsync(wk.P1.p, 0, sizeof(double) * n * 2 * wk.s, s));
    if (wk.C1.p) BCMGX_CUDA(cudaMemsetAsync(wk.C1.p, 0, sizeof(double) * n * wk.s, s));
}

// Matrix powers kernel into the n x 2s block P (krylov_base/mpk.cu:10-83).
void sstep_mpk(bcmgx_hierarchy* H, KrylovWork& wk, double* P, const int* skip)
{
    cudaStream_t s = H->stream;
    const DevCsr& A = H->lv[0].A;
    const long n = A.n;
    const int S = wk.s;
    if (H->prm.preconditioner == BCMGX_PREC_NONE) {
        note_launch();
        k_kry_copy<<<red_blocks(k_kry_copy, n), kThreads, 0, s>>>(n, H->r.p, P, skip);
        BCMGX_CHECK_LAUNCH();
        for (int i = 0; i < S; i++) rowop_spmv(A, P + i * n, P + (i + 1) * n, skip, s);
        return;
    }
    prec_apply_impl(H, H->r.p, P, skip);
    int pin = 0, pout = S;
    for (int i = 0; i < 2 * S - 1; i++) {
        if (i % 2 == 0) rowop_spmv(A, P + pin * n, P + pout * n, skip, s);
        else prec_apply_impl(H, P + pin * n, P + pout * n, skip);
        const int t = pin;
        pin = pout;
        pout = t + 1;
    }
}

// One outer s-step iteration (CGs.cu:120-175); `cur` receives the new basis, `old` holds the
// previous directions.
void sstep_iteration(bcmgx_hierarchy* H, KrylovWork& wk, bool even, const double* b, double* x, const int* skip)
{
    cudaStream_t s = H->stream;
    const DevCsr& A = H->lv[0].A;
    const long n = A.n;
    const int S = wk.s;
    const bcmgx_params& P = H->prm;
    const bool pre = P.preconditioner != BCMGX_PREC_NONE;
    double* cur = even ? wk.P2.p : wk.P1.p;
    double* old = even ? wk.P1.p : wk.P2.p;
    if (P.ru_res && P.rec_res_int > 0) {
        note_launch();
        k_sstep_resid_flag<<<1, 1, 0, s>>>(wk.st.p, P.rec_res_int);
        BCMGX_CHECK_LAUNCH();
        rowop_resid(A, x, b, H->r.p, &wk.st.p->resid_skip, s);
    }
    sstep_mpk(H, wk, cur, skip);
    MomentPairs mp {};
    if (!pre) {
        mp.np = 2 * S;
        for (int k = 0; k <= S; k++) { mp.ia[k] = k; mp.ib[k] = -1; }
        for (int k = 0; k < S - 1; k++) { mp.ia[S + 1 + k] = 1 + k; mp.ib[S + 1 + k] = S; }
    } else {
        mp.np = 2 * S;
        for (int k = 0; k < S; k++) { mp.ia[k] = k; mp.ib[k] = -1; }
        for (int k = 0; k < S; k++) { mp.ia[S + k] = k; mp.ib[S + k] = 2 * S - 1; }
    }
    note_launch();
    k_sstep_moments<<<red_blocks(k_sstep_moments, n), kThreads, 0, s>>>((int)n, cur, H->r.p, mp, wk.st.p, wk.part.p, skip);
    note_launch();
    k_sstep_scalar<<<1, 1, 0, s>>>(wk.st.p, S, skip);
    BCMGX_CHECK_LAUNCH();
    double* ccur = even ? wk.C2.p : wk.C1.p;
    const double* cold = even ? wk.C1.p : wk.C2.p;
    if (P.ru_res && !pre) {
        note_launch();
        k_kry_copy<<<red_blocks(k_kry_copy, n * S), kThreads, 0, s>>>(n * S, cur + n, ccur, skip);
    }
    note_launch();
    k_sstep_update<false><<<red_blocks(k_sstep_update<false>, n), kThreads, 0, s>>>((int)n, S, old, cur, x, 1.0, wk.st.p, wk.part.p, skip);
    BCMGX_CHECK_LAUNCH();
    if (P.ru_res) {
        const double* Aold = pre ? old + S * n : cold;
        double* Acur = pre ? cur + S * n : ccur;
        note_launch();
        k_sstep_update<true><<<red_blocks(k_sstep_update<true>, n), kThreads, 0, s>>>((int)n, S, Aold, Acur, H->r.p, -1.0, wk.st.p, wk.part.p, skip);
    } else {
        rowop_resid(A, x, b, H->r.p, skip, s);
        note_launch();
        k_sstep_norm_stop<<<red_blocks(k_sstep_norm_stop, n), kThreads, 0, s>>>((int)n, H->r.p, wk.st.p, wk.part.p, skip);
    }
    BCMGX_CHECK_LAUNCH();
}

void startup(bcmgx_hierarchy* H, KrylovWork& wk, const double* b, double* x)
{
    if (sstep_solver(H->prm.solver)) sstep_startup(H, wk, b, x);
    else cghs_startup(H, wk, b, x);
}

void iteration(bcmgx_hierarchy* H, KrylovWork& wk, bool even, const double* b, double* x, const int* skip)
{
    if (sstep_solver(H->prm.solver)) sstep_iteration(H, wk, even, b, x, skip);
    else cghs_iteration(H, wk, x, skip);
}

// The whole solve as one graph on the hierarchy's own b / x buffers: start-up, then a WHILE node
// over two iterations and the kernel that sets the loop condition from `done`.
void build_graph(bcmgx_hierarchy* H, KrylovWork& wk)
{
    cudaStream_t s = H->stream;
    const int n = H->lv[0].A.n;
    if (!H->gb.p) {
        H->gb.alloc(n, s);
        H->gx.alloc(n, s);
    }
    BCMGX_CUDA(cudaStreamSynchronize(s));
    cudaGraph_t g = nullptr;
    BCMGX_CUDA(cudaGraphCreate(&g, 0));
    const long long c0 = launch_count();
    BCMGX_CUDA(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    startup(H, wk, H->gb.p, H->gx.p);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    BCMGX_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &ndeps));
    std::vector<cudaGraphNode_t> tail(deps, deps + ndeps);
    cudaGraph_t gg = g;
    BCMGX_CUDA(cudaStreamEndCapture(s, &gg));
    const long long c1 = launch_count();
    cudaGraphConditionalHandle h;
    BCMGX_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wn;
    BCMGX_CUDA(cudaGraphAddNode(&wn, g, tail.data(), tail.size(), &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    BCMGX_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    iteration(H, wk, true, H->gb.p, H->gx.p, &wk.st.p->done);
    iteration(H, wk, false, H->gb.p, H->gx.p, &wk.st.p->done);
    note_launch();
    k_kry_set_while<<<1, 1, 0, s>>>(h, wk.st.p);
    BCMGX_CHECK_LAUNCH();
    BCMGX_CUDA(cudaStreamEndCapture(s, &body));
    const long long c2 = launch_count();
    wk.startup_kernels = c1 - c0;
    wk.body_kernels = c2 - c1;
    note_launches(-(c2 - c0));   // captured, not launched
    BCMGX_CUDA(cudaGraphInstantiate(&wk.graph, g, 0));
    BCMGX_CUDA(cudaGraphDestroy(g));
}

int finish(bcmgx_hierarchy* H, const KryState& S, float ms, bcmgx_solve_info* info)
{
    const bool converged = !S.bad && S.rnorm2 >= 0.0 && std::sqrt(S.rnorm2) < S.tol;
    if (info) {
        info->niter = S.iter;
        info->retv = converged ? 0 : (S.bad ? 1 : -1);
        info->delta0 = S.delta0;
        info->exit_res = std::sqrt(S.rnorm2);
        info->solve_ms = ms;
        info->full_n = H->lv[0].A.n;
    }
    if (S.bad) return BCMGX_ERR_NOT_SPD;
    return converged ? BCMGX_OK : BCMGX_ERR_NO_CONVERGENCE;
}

}  // namespace

// CGHS or s-step CG on device vectors b, x (x: x0 in, solution out).
int krylov_solve(bcmgx_hierarchy* H, const double* b, double* x, bcmgx_solve_info* info)
{
    ensure_solve_workspace(H);
    KrylovWork& wk = krylov_work(H);
    cudaStream_t s = H->stream;
    const int n = H->lv[0].A.n;
    const bcmgx_params& P = H->prm;
    if (P.use_graph == 1 && !P.dispnorm) {
        if (!wk.graph) build_graph(H, wk);
        BCMGX_CUDA(cudaMemcpyAsync(H->gb.p, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        BCMGX_CUDA(cudaMemcpyAsync(H->gx.p, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        BCMGX_CUDA(cudaEventRecord(H->ev0, s));
        BCMGX_CUDA(cudaGraphLaunch(wk.graph, s));
        BCMGX_CUDA(cudaEventRecord(H->ev1, s));
        BCMGX_CUDA(cudaMemcpyAsync(x, H->gx.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        BCMGX_CUDA(cudaMemcpyAsync(wk.st_host, wk.st.p, sizeof(KryState), cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
        const long long bodies = std::max(1LL, (long long)(wk.st_host->iter + 1) / 2 + (wk.st_host->bad ? 1 : 0));
        note_launches(wk.startup_kernels + wk.body_kernels * bodies);
    } else {
        BCMGX_CUDA(cudaEventRecord(H->ev0, s));
        startup(H, wk, b, x);
        KryState* ring = wk.st_host;
        const int* done = &wk.st.p->done;
        auto enqueue = [&](int k) {
            iteration(H, wk, (k % 2) == 0, b, x, done);
            BCMGX_CUDA(cudaMemcpyAsync(ring + (k % 2), wk.st.p, sizeof(KryState), cudaMemcpyDeviceToHost, s));
            BCMGX_CUDA(cudaEventRecord(H->ev_it[k % 2], s));
        };
        enqueue(0);
        int k = 0;
        for (;;) {
            enqueue(k + 1);
            BCMGX_CUDA(cudaEventSynchronize(H->ev_it[k % 2]));
            const KryState& S = ring[k % 2];
            if (P.dispnorm && !S.bad) std::printf("%d) r norm: %.10lf\n", S.iter - 1, std::sqrt(S.rnorm2));
            if (S.done) break;
            k++;
        }
        BCMGX_CUDA(cudaEventRecord(H->ev1, s));
        BCMGX_CUDA(cudaMemcpyAsync(wk.st_host, wk.st.p, sizeof(KryState), cudaMemcpyDeviceToHost, s));
        BCMGX_CUDA(cudaStreamSynchronize(s));
    }
    float ms = 0;
    BCMGX_CUDA(cudaEventElapsedTime(&ms, H->ev0, H->ev1));
    return finish(H, *wk.st_host, ms, info);
}

}  // namespace bcmgx
