// generators.cpp -- input plumbing of the driver: 3D Laplacian generators, the laplacian .cfg
// reader, a MatrixMarket reader, and the heterogeneous-diffusion generator used by the
// benchmarks. Host code (OpenMP over rows).
#include "internal.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace bcmgx {
namespace {

struct Grid {
    long nx, ny, nz, P, Q, R;
    long gnx() const { return nx * P; }
    long gny() const { return ny * Q; }
    long gnz() const { return nz * R; }
    long local() const { return nx * ny * nz; }
    long rows() const { return gnx() * gny() * gnz(); }
    // Global number of point (gi,gj,gk): blocks of nx*ny*nz points numbered x-fastest over the
    // P x Q x R block grid, points x-fastest inside a block (internal_index, laplacian.cu:14-25).
    long index(long gi, long gj, long gk) const
    {
        const long p = gi / nx, q = gj / ny, r = gk / nz;
        const long i = gi % nx, j = gj % ny, k = gk % nz;
        return (r * P * Q + q * P + p) * local() + (k * nx * ny + j * nx + i);
    }
    void point(long row, long& gi, long& gj, long& gk) const
    {
        const long blk = row / local(), loc = row % local();
        gi = (blk % P) * nx + loc % nx;
        gj = ((blk / P) % Q) * ny + (loc / nx) % ny;
        gk = (blk / (P * Q)) * nz + loc / (nx * ny);
    }
    bool inside(long a, long b, long c) const { return a >= 0 && a < gnx() && b >= 0 && b < gny() && c >= 0 && c < gnz(); }
};

void check_grid(int stencil, int nx, int ny, int nz, int P, int Q, int R)
{
    BCMGX_REQUIRE(stencil == 7 || stencil == 27, BCMGX_ERR_INVALID_INPUT, "stencil must be 7 or 27");
    BCMGX_REQUIRE(nx > 0 && ny > 0 && nz > 0 && P > 0 && Q > 0 && R > 0, BCMGX_ERR_INVALID_INPUT, "grid sizes must be positive");
    const double rows = (double)nx * ny * nz * P * Q * R;
    BCMGX_REQUIRE(rows * stencil < 2147483647.0, BCMGX_ERR_UNSUPPORTED, "grid too large for int32 CSR offsets");
}

// row length of the point, counting in-domain neighbours of the stencil
inline int stencil_len(const Grid& g, int stencil, long gi, long gj, long gk)
{
    const int cx = 1 + (gi > 0) + (gi + 1 < g.gnx());
    const int cy = 1 + (gj > 0) + (gj + 1 < g.gny());
    const int cz = 1 + (gk > 0) + (gk + 1 < g.gnz());
    if (stencil == 27) return cx * cy * cz;
    return 1 + (cx - 1) + (cy - 1) + (cz - 1);
}

}  // namespace
}  // namespace bcmgx

using namespace bcmgx;

extern "C" {

int bcmgx_laplacian_3d_size(int stencil, int nx, int ny, int nz, int P, int Q, int R, int64_t* n, int64_t* nnz)
{
    try {
        check_grid(stencil, nx, ny, nz, P, Q, R);
        Grid g { nx, ny, nz, P, Q, R };
        // separable count: per axis, points with a lower / upper neighbour
        auto axis = [](long N, long& one, long& two, long& three) {
            three = std::max(N - 2, 0L);
            two = N >= 2 ? 2 : 0;
            one = N == 1 ? 1 : 0;
        };
        long a1, a2, a3, b1, b2, b3, c1, c2, c3;
        axis(g.gnx(), a1, a2, a3);
        axis(g.gny(), b1, b2, b3);
        axis(g.gnz(), c1, c2, c3);
        const long sx = a1 * 1 + a2 * 2 + a3 * 3, sy = b1 * 1 + b2 * 2 + b3 * 3, sz = c1 * 1 + c2 * 2 + c3 * 3;
        const long N = g.rows();
        long z;
        if (stencil == 27) {
            z = sx * sy * sz;
        } else {
            // 1 + (cx-1) + (cy-1) + (cz-1) summed over the grid
            z = N + (sx - g.gnx()) * g.gny() * g.gnz() + (sy - g.gny()) * g.gnx() * g.gnz() + (sz - g.gnz()) * g.gnx() * g.gny();
        }
        if (n) *n = N;
        if (nnz) *nnz = z;
        return BCMGX_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
}

// 7-point (diagonal 6) / 27-point (diagonal 26) Dirichlet Laplacian with off-diagonals -1 in the
// reference's global row order, rows column-sorted. Same matrix as generateLocalLaplacian3D_7p
// (laplacian.cu:119-334) / _27p (:336-777) on P*Q*R ranks stacked in rank-block order, followed
// by check_and_fix_order (CSR.cu:1895-1918); with P = Q = R = 1 and nx = ny = nz = n it is also
// the -a n matrix of generateLocalLaplacian3D (laplacian.cu:27-117). Arrays are caller-owned,
// sized by bcmgx_laplacian_3d_size.
int bcmgx_laplacian_3d(int stencil, int nx, int ny, int nz, int P, int Q, int R, int* row, int* col, double* val)
{
    try {
        check_grid(stencil, nx, ny, nz, P, Q, R);
        BCMGX_REQUIRE(row && col && val, BCMGX_ERR_INVALID_INPUT, "NULL output array");
        const Grid g { nx, ny, nz, P, Q, R };
        const long N = g.rows();
        // row offsets: lengths, then a serial prefix sum
#pragma omp parallel for schedule(static)
        for (long r = 0; r < N; r++) {
            long gi, gj, gk;
            g.point(r, gi, gj, gk);
            row[r + 1] = stencil_len(g, stencil, gi, gj, gk);
        }
        row[0] = 0;
        for (long r = 0; r < N; r++) row[r + 1] += row[r];
        const double diag = stencil == 27 ? 26.0 : 6.0;
#pragma omp parallel for schedule(static)
        for (long r = 0; r < N; r++) {
            long gi, gj, gk;
            g.point(r, gi, gj, gk);
            int cols[27];
            int c = 0;
            for (int dz = -1; dz <= 1; dz++)
                for (int dy = -1; dy <= 1; dy++)
                    for (int dx = -1; dx <= 1; dx++) {
                        if (stencil == 7 && std::abs(dx) + std::abs(dy) + std::abs(dz) > 1) continue;
                        if (!g.inside(gi + dx, gj + dy, gk + dz)) continue;
                        cols[c++] = (int)g.index(gi + dx, gj + dy, gk + dz);
                    }
            std::sort(cols, cols + c);
            const long o = row[r];
            for (int t = 0; t < c; t++) {
                col[o + t] = cols[t];
                val[o + t] = cols[t] == (int)r ? diag : -1.0;
            }
        }
        return BCMGX_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
}

// "name = value" lines for nx ny nz P Q R; '#' lines skipped (read_laplacian_file,
// laplacian.cu:974-1017). out = {nx, ny, nz, P, Q, R}.
int bcmgx_read_laplacian_cfg(const char* path, int* out)
{
    FILE* fp = path ? std::fopen(path, "r") : nullptr;
    if (!fp) {
        set_last_error(std::string("[ERROR] - Laplacian file not found! (") + (path ? path : "NULL") + ")");
        return BCMGX_ERR_INVALID_INPUT;
    }
    const char* names[6] = { "nx", "ny", "nz", "P", "Q", "R" };
    int got[6] = { 0, 0, 0, 0, 0, 0 };
    char buf[1024];
    int rc = BCMGX_OK;
    while (std::fgets(buf, sizeof buf, fp)) {
        size_t len = std::strlen(buf);
        if (len == 0 || buf[0] == '#') continue;
        bool blank = true;
        for (size_t i = 0; i < len; i++)
            if (!std::isspace((unsigned char)buf[i])) blank = false;
        if (blank) continue;
        char opt[64];
        int v = 0;
        if (std::sscanf(buf, "%63s = %d", opt, &v) != 2) {
            set_last_error(std::string("[ERROR] Error reading file ") + path);
            rc = BCMGX_ERR_INVALID_INPUT;
            break;
        }
        for (int i = 0; i < 6; i++)
            if (std::strstr(opt, names[i]) != nullptr) {
                out[i] = v;
                got[i] = 1;
                break;
            }
    }
    std::fclose(fp);
    if (rc == BCMGX_OK) {
        for (int i = 0; i < 6; i++)
            if (!got[i]) {
                set_last_error(std::string("laplacian cfg: missing ") + names[i]);
                return BCMGX_ERR_INVALID_INPUT;
            }
    }
    return rc;
}

// MatrixMarket "coordinate real general|symmetric" reader (readMTXDouble, CSR.cu:1973-2120):
// 1-based indices, symmetric entries mirrored, rows column-sorted (stable). Arrays are malloc'ed
// by the library and released with bcmgx_host_free.
int bcmgx_read_matrix_market(const char* path, int* n_out, int* m_out, int64_t* nnz_out, int** row_out, int** col_out,
    double** val_out)
{
    try {
        BCMGX_REQUIRE(path && n_out && m_out && nnz_out && row_out && col_out && val_out, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        FILE* fp = std::fopen(path, "r");
        BCMGX_REQUIRE(fp != nullptr, BCMGX_ERR_INVALID_INPUT, std::string("Error opening file ") + path + ": " + std::strerror(errno));
        char banner[64] = { 0 }, mtx[64] = { 0 }, crd[64] = { 0 }, dtype[64] = { 0 }, scheme[64] = { 0 };
        char buf[4096];
        if (!std::fgets(buf, sizeof buf, fp) || std::sscanf(buf, "%63s %63s %63s %63s %63s", banner, mtx, crd, dtype, scheme) != 5) {
            std::fclose(fp);
            throw Error(BCMGX_ERR_INVALID_INPUT, "MatrixMarket: bad banner");
        }
        if (std::strcmp(dtype, "real") != 0 || std::strcmp(crd, "coordinate") != 0) {
            std::fclose(fp);
            throw Error(BCMGX_ERR_INVALID_INPUT, std::string("MatrixMarket: only coordinate real matrices are read, not '") + dtype + "'");
        }
        const bool sym = std::strcmp(scheme, "symmetric") == 0;
        if (!sym && std::strcmp(scheme, "general") != 0) {
            std::fclose(fp);
            throw Error(BCMGX_ERR_INVALID_INPUT, std::string("MatrixMarket: unhandled storage scheme '") + scheme + "'");
        }
        do {
            if (!std::fgets(buf, sizeof buf, fp)) {
                std::fclose(fp);
                throw Error(BCMGX_ERR_INVALID_INPUT, "MatrixMarket: missing size line");
            }
        } while (buf[0] == '%');
        unsigned long nr = 0, nc = 0, nz = 0;
        if (std::sscanf(buf, "%lu %lu %lu", &nr, &nc, &nz) != 3) {
            std::fclose(fp);
            throw Error(BCMGX_ERR_INVALID_INPUT, "MatrixMarket: bad size line");
        }
        std::vector<int> ri, cj;
        std::vector<double> vv;
        ri.reserve(sym ? 2 * nz : nz);
        cj.reserve(sym ? 2 * nz : nz);
        vv.reserve(sym ? 2 * nz : nz);
        for (unsigned long k = 0; k < nz; k++) {
            unsigned long a, b;
            double v;
            if (!std::fgets(buf, sizeof buf, fp) || std::sscanf(buf, "%lu %lu %le", &a, &b, &v) != 3 || a < 1 || b < 1 || a > nr || b > nc) {
                std::fclose(fp);
                throw Error(BCMGX_ERR_INVALID_INPUT, "MatrixMarket: bad record " + std::to_string(k + 1));
            }
            ri.push_back((int)(a - 1));
            cj.push_back((int)(b - 1));
            vv.push_back(v);
            if (sym && a != b) {
                ri.push_back((int)(b - 1));
                cj.push_back((int)(a - 1));
                vv.push_back(v);
            }
        }
        std::fclose(fp);
        const long Z = (long)ri.size();
        int* row = (int*)std::calloc(nr + 1, sizeof(int));
        int* col = (int*)std::malloc(sizeof(int) * std::max(Z, 1L));
        double* val = (double*)std::malloc(sizeof(double) * std::max(Z, 1L));
        if (!row || !col || !val) {
            std::free(row);
            std::free(col);
            std::free(val);
            throw std::bad_alloc();
        }
        for (long k = 0; k < Z; k++) row[ri[k] + 1]++;
        for (unsigned long r = 0; r < nr; r++) row[r + 1] += row[r];
        std::vector<int> pos(row, row + nr);
        for (long k = 0; k < Z; k++) {
            const int o = pos[ri[k]]++;
            col[o] = cj[k];
            val[o] = vv[k];
        }
        for (unsigned long r = 0; r < nr; r++) {
            std::vector<std::pair<int, double>> e;
            for (int j = row[r]; j < row[r + 1]; j++) e.push_back({ col[j], val[j] });
            std::stable_sort(e.begin(), e.end(), [](const std::pair<int, double>& a, const std::pair<int, double>& b) { return a.first < b.first; });
            for (int j = row[r], t = 0; j < row[r + 1]; j++, t++) {
                col[j] = e[t].first;
                val[j] = e[t].second;
            }
        }
        *n_out = (int)nr;
        *m_out = (int)nc;
        *nnz_out = Z;
        *row_out = row;
        *col_out = col;
        *val_out = val;
        return BCMGX_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return BCMGX_ERR_OOM;
    }
}

void bcmgx_host_free(void* p) { std::free(p); }

// 7-point cell-centred finite-volume diffusion on an nx*ny*nz grid (x fastest) with per-cell
// coefficient kappa > 0: the face coefficient between cells i and j is the harmonic mean
// 2 k_i k_j / (k_i + k_j); a boundary face contributes 2 k_i to the diagonal (Dirichlet value 0
// on the boundary, half-cell distance). The result is symmetric positive definite. Arrays are
// caller-owned and sized like the 7-point Laplacian of the same grid.
int bcmgx_diffusion_7p(int nx, int ny, int nz, const double* kappa, int* row, int* col, double* val)
{
    try {
        check_grid(7, nx, ny, nz, 1, 1, 1);
        BCMGX_REQUIRE(kappa && row && col && val, BCMGX_ERR_INVALID_INPUT, "NULL argument");
        const Grid g { nx, ny, nz, 1, 1, 1 };
        const long N = g.rows();
#pragma omp parallel for schedule(static)
        for (long r = 0; r < N; r++) {
            long gi, gj, gk;
            g.point(r, gi, gj, gk);
            row[r + 1] = stencil_len(g, 7, gi, gj, gk);
        }
        row[0] = 0;
        for (long r = 0; r < N; r++) row[r + 1] += row[r];
        int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
        for (long r = 0; r < N; r++) {
            long gi, gj, gk;
            g.point(r, gi, gj, gk);
            const double ki = kappa[r];
            if (!(ki > 0.0) || !std::isfinite(ki)) bad = 1;
            const long nb[6][3] = { { 0, 0, -1 }, { 0, -1, 0 }, { -1, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } };
            double diag = 0.0;
            long o = row[r];
            // neighbours in ascending column order: -z, -y, -x, (diag), +x, +y, +z
            long dpos = -1;
            for (int t = 0; t < 6; t++) {
                if (t == 3) dpos = o++;
                const long a = gi + nb[t][0], b = gj + nb[t][1], c = gk + nb[t][2];
                if (!g.inside(a, b, c)) {
                    diag += 2.0 * ki;
                    continue;
                }
                const long j = g.index(a, b, c);
                const double kj = kappa[j];
                const double t_ij = 2.0 * ki * kj / (ki + kj);
                col[o] = (int)j;
                val[o] = -t_ij;
                diag += t_ij;
                o++;
            }
            col[dpos] = (int)r;
            val[dpos] = diag;
        }
        BCMGX_REQUIRE(!bad, BCMGX_ERR_INVALID_INPUT, "kappa must be positive and finite");
        return BCMGX_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
}

}  // extern "C"
