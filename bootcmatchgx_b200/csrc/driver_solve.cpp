// driver_solve.cpp -- command-line driver with the flags, defaults and outputs of the reference's
// driverSolve (BCMGX/src/example/driverSolve.cu:59-406), on one GPU through the C ABI.
//
// Input: -m MatrixMarket file | -l laplacian .cfg with -g 7p|27p | -a n; settings with -s
// (.properties, else the legacy positional format). Right-hand side 1, x0 = 0 (:243-247), as
// the reference; extensions: --rhs-xstar SEED (b = A x*, x* uniform[-1,1] from SEED),
// --vcycle fp32|fp64, and "-l 7p|27p --grid NXxNYxNZ" in place of a .cfg file.
// Output: the info file (-i, SolverOut.cu:9-97 layout plus the profile table of
// profiling.cu:194-360 for the prec_setup and solve regions) and the solution (-o, one "%g"
// value per line, Vector::print, vector.cu:378-410).
#include "bcmgx.h"

#include <chrono>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <getopt.h>
#include <random>
#include <string>
#include <vector>

#define USAGE                                                                                                               \
    "Usage: %s [--matrix <FILE_NAME> | --laplacian <SIZE> | --laplacian-3d <FILE_NAME>] --settings <FILE_NAME>\n\n"         \
    "\tYou can specify only one out of the three available options: --matrix, --laplacian-3d and --laplacian\n\n"           \
    "\t-a, --laplacian <SIZE>                      Generate a matrix whose size is <SIZE>^3.\n"                             \
    "\t-B, --out-prefix <STRING>                   Use <PREFIX> when writing additional files to output dir.\n"             \
    "\t-d, --dump-matrix <FILE_NAME>               Write the input matrix to <FILE_NAME>0.\n"                               \
    "\t-e, --errlog <FILE_NAME>                    Write log to <FILE_NAME>0.\n"                                            \
    "\t-g, --laplacian-3d-generator [ 7p | 27p ]   Choose laplacian 3d generator (7 points or 27 points).\n"                \
    "\t-h, --help                                  Print this message.\n"                                                   \
    "\t-i, --info <FILE_NAME>                      Write info to <FILE_NAME>.\n"                                            \
    "\t-l, --laplacian-3d <FILE_NAME>              Read generation parameters from file <FILE_NAME> (or 7p|27p with --grid).\n" \
    "\t-m, --matrix <FILE_NAME>                    Read the matrix from file <FILE_NAME>.\n"                                \
    "\t-M, --detailed-metrics <FILE_NAME>          Accepted for compatibility.\n"                                           \
    "\t-o, --out <FILE_NAME>                       Write solution to <FILE_NAME>.\n"                                        \
    "\t-O, --out-dir <DIR>                         Write additional files to <DIR>.\n"                                      \
    "\t-p, --summary-prof <FILE_NAME>              Write summary profile log to <FILE_NAME>0.\n"                            \
    "\t-P, --detailed-prof <FILE_NAME>             Write detailed profile log to <FILE_NAME>0.\n"                           \
    "\t-s, --settings <FILE_NAME>                  Read settings from file <FILE_NAME>.\n"                                  \
    "\t-S, --out-suffix <STRING>                   Use <SUFFIX> when writing additional files to output dir.\n"             \
    "\t-x, --extended-prof                         Write extended profile info inside the info-file.\n"                     \
    "\t    --grid <NXxNYxNZ>                       Grid for -l 7p|27p (single block).\n"                                   \
    "\t    --rhs-xstar <SEED>                      b = A x*, x* uniform[-1,1] (std::mt19937_64(SEED)).\n"                   \
    "\t    --vcycle [ fp64 | fp32 ]                V-cycle arithmetic (default fp64).\n\n"

static void logf2(FILE* fp, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
static void logf2(FILE* fp, const char* fmt, ...)
{
    va_list a;
    va_start(a, fmt);
    vprintf(fmt, a);
    va_end(a);
    if (fp) {
        va_start(a, fmt);
        vfprintf(fp, fmt, a);
        va_end(a);
    }
}

static const char* solver_s(int v)
{
    static const char* t[] = { "CGHS", "FCG", "CGS", "PIPELINED_CGS", "CGS_CUBLAS", "INVALID" };
    return (v >= 0 && v < 6) ? t[v] : "INVALID";
}
static const char* prec_s(int v)
{
    static const char* t[] = { "NONE", "L1_JACOBI", "BCMG", "AFSAI", "INVALID" };
    return (v >= 0 && v < 5) ? t[v] : "INVALID";
}
static const char* cycle_s(int v)
{
    static const char* t[] = { "V_CYCLE", "H_CYCLE", "W_CYCLE", "VARIABLE_V_CYCLE", "INVALID" };
    return (v >= 0 && v < 5) ? t[v] : "INVALID";
}
static const char* boot_s(int v)
{
    static const char* t[] = { "MULTIPLICATIVE", "SYMMETRIZED_MULTIPLICATIVE", "ADDITIVE", "INVALID" };
    return (v >= 0 && v < 4) ? t[v] : "INVALID";
}

static int fail(const char* what, int rc)
{
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, bcmgx_last_error_string());
    return 1;
}

int main(int argc, char** argv)
{
    enum { MTX, LAP_3D, LAP, NONE } opt = NONE;
    std::string mtx_file, lap_3d_file, settings_file, info_file, out_file, grid, vcycle = "fp64";
    std::string summary_prof, detailed_prof, dump_matrix;
    int stencil = 27;   // driverSolve.cu:73 (LAP_27P)
    bool bad_gen = false;
    int n_lap = 0;
    long xstar_seed = -1;
    static struct option long_options[] = {
        { "laplacian", required_argument, nullptr, 'a' },
        { "out-prefix", required_argument, nullptr, 'B' },
        { "dump-matrix", required_argument, nullptr, 'd' },
        { "errlog", required_argument, nullptr, 'e' },
        { "laplacian-3d-generator", required_argument, nullptr, 'g' },
        { "help", no_argument, nullptr, 'h' },
        { "info", required_argument, nullptr, 'i' },
        { "laplacian-3d", required_argument, nullptr, 'l' },
        { "matrix", required_argument, nullptr, 'm' },
        { "detailed-metrics", required_argument, nullptr, 'M' },
        { "out", required_argument, nullptr, 'o' },
        { "out-dir", required_argument, nullptr, 'O' },
        { "summary-prof", required_argument, nullptr, 'p' },
        { "detailed-prof", required_argument, nullptr, 'P' },
        { "settings", required_argument, nullptr, 's' },
        { "out-suffix", required_argument, nullptr, 'S' },
        { "extended-prof", no_argument, nullptr, 'x' },
        { "grid", required_argument, nullptr, 1001 },
        { "rhs-xstar", required_argument, nullptr, 1002 },
        { "vcycle", required_argument, nullptr, 1003 },
        { nullptr, 0, nullptr, 0 },
    };
    int ch;
    while ((ch = getopt_long(argc, argv, "a:B:d:e:g:hi:l:m:M:o:O:p:P:s:S:x", long_options, nullptr)) != -1) {
        switch (ch) {
        case 'a': n_lap = std::atoi(optarg); opt = LAP; break;
        case 'd': dump_matrix = optarg; break;
        case 'g':
            if (!std::strcmp(optarg, "7p")) stencil = 7;
            else if (!std::strcmp(optarg, "27p")) stencil = 27;
            else bad_gen = true;
            break;
        case 'i': info_file = optarg; break;
        case 'l':
            lap_3d_file = optarg;
            opt = LAP_3D;
            break;
        case 'm': mtx_file = optarg; opt = MTX; break;
        case 'o': out_file = optarg; break;
        case 'p': summary_prof = optarg; break;
        case 'P': detailed_prof = optarg; break;
        case 's': settings_file = optarg; break;
        case 'B': case 'e': case 'M': case 'O': case 'S': case 'x': break;
        case 1001: grid = optarg; break;
        case 1002: xstar_seed = std::atol(optarg); break;
        case 1003: vcycle = optarg; break;
        case 'h':
        default: std::printf(USAGE, argv[0]); return EXIT_FAILURE;
        }
    }
    if (opt == NONE || settings_file.empty() || bad_gen) {
        std::printf(USAGE, argv[0]);
        return EXIT_FAILURE;
    }

    // settings (driverSolve.cu:211-220)
    bcmgx_params p;
    const bool props = settings_file.size() >= 11 && settings_file.compare(settings_file.size() - 11, 11, ".properties") == 0;
    std::printf("Reading setting file %s\n", settings_file.c_str());
    int rc = props ? bcmgx_params_from_properties(settings_file.c_str(), &p) : bcmgx_params_from_legacy_file(settings_file.c_str(), &p);
    if (rc) return fail("reading settings", rc);
    if (p.error != 0) return -1;
    if (vcycle == "fp32") p.vcycle_precision = BCMGX_VCYCLE_FP32;

    // matrix (driverSolve.cu:222-229)
    int n = 0, m = 0;
    int64_t nnz = 0;
    std::vector<int> row, col;
    std::vector<double> val;
    if (opt == MTX) {
        int *r = nullptr, *c = nullptr;
        double* v = nullptr;
        rc = bcmgx_read_matrix_market(mtx_file.c_str(), &n, &m, &nnz, &r, &c, &v);
        if (rc) return fail("reading the matrix", rc);
        row.assign(r, r + n + 1);
        col.assign(c, c + nnz);
        val.assign(v, v + nnz);
        bcmgx_host_free(r);
        bcmgx_host_free(c);
        bcmgx_host_free(v);
    } else {
        int g[6];
        if (opt == LAP) {
            g[0] = g[1] = g[2] = n_lap;
            g[3] = g[4] = g[5] = 1;
            stencil = 7;
        } else if (lap_3d_file == "7p" || lap_3d_file == "27p") {
            stencil = lap_3d_file == "7p" ? 7 : 27;
            if (std::sscanf(grid.c_str(), "%dx%dx%d", &g[0], &g[1], &g[2]) != 3) {
                std::fprintf(stderr, "--grid NXxNYxNZ is required with -l 7p|27p\n");
                return EXIT_FAILURE;
            }
            g[3] = g[4] = g[5] = 1;
        } else {
            rc = bcmgx_read_laplacian_cfg(lap_3d_file.c_str(), g);
            if (rc) return fail("reading the laplacian file", rc);
            std::fprintf(stderr, "Using laplacian 3d %d points generator.\n", stencil);
        }
        int64_t n64 = 0;
        rc = bcmgx_laplacian_3d_size(stencil, g[0], g[1], g[2], g[3], g[4], g[5], &n64, &nnz);
        if (rc) return fail("sizing the laplacian", rc);
        n = m = (int)n64;
        row.resize((size_t)n + 1);
        col.resize(nnz);
        val.resize(nnz);
        rc = bcmgx_laplacian_3d(stencil, g[0], g[1], g[2], g[3], g[4], g[5], row.data(), col.data(), val.data());
        if (rc) return fail("generating the laplacian", rc);
    }
    if (!dump_matrix.empty()) {
        std::string fn = dump_matrix + "0.mtx";
        FILE* f = std::fopen(fn.c_str(), "w");
        if (f) {
            std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%d %d %lld\n", n, m, (long long)nnz);
            for (int i = 0; i < n; i++)
                for (int j = row[i]; j < row[i + 1]; j++) std::fprintf(f, "%d %d %.17g\n", i + 1, col[j] + 1, val[j]);
            std::fclose(f);
        }
    }

    // rhs = 1, x0 = 0 (driverSolve.cu:243-247)
    std::vector<double> b(n, 1.0), x(n, 0.0);
    if (xstar_seed >= 0) {
        std::mt19937_64 gen((unsigned long long)xstar_seed);
        std::uniform_real_distribution<double> U(-1.0, 1.0);
        std::vector<double> xs(n);
        for (auto& e : xs) e = U(gen);
        for (int i = 0; i < n; i++) {
            double s = 0;
            for (int j = row[i]; j < row[i + 1]; j++) s += val[j] * xs[col[j]];
            b[i] = s;
        }
    }

    bcmgx_csr A { n, m, nnz, row.data(), col.data(), val.data(), 0 };
    std::printf("Setting preconditioner\n");
    bcmgx_hierarchy* h = nullptr;
    auto t0 = std::chrono::steady_clock::now();
    rc = bcmgx_setup(&A, &p, &h);
    auto t1 = std::chrono::steady_clock::now();
    if (rc) return fail("prec_setup", rc);
    std::printf("Solving\n");
    bcmgx_solve_info si {};
    rc = bcmgx_solve(h, b.data(), x.data(), 0, &si);
    auto t2 = std::chrono::steady_clock::now();
    if (rc && rc != BCMGX_ERR_NO_CONVERGENCE) {
        fail("solve", rc);
        bcmgx_free(h);
        return 1;
    }
    const unsigned long setup_ns = (unsigned long)std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count();
    const unsigned long solve_ns = (unsigned long)std::chrono::duration_cast<std::chrono::nanoseconds>(t2 - t1).count();

    bcmgx_hierarchy_info hi {};
    bcmgx_hierarchy_get_info(h, &hi);
    if (!info_file.empty()) {
        std::printf("Dumping output\n");
        FILE* fp = std::fopen(info_file.c_str(), "w");
        if (!fp) std::printf("File %s opening failed.\n", info_file.c_str());
        logf2(fp, "nprocs                                       : %d\n", 1);
        logf2(fp, "Solver                                       : %s\n", solver_s(p.solver));
        logf2(fp, "Tolerance                                    : %g\n", p.rtol);
        logf2(fp, "Preconditioner                               : %s\n", prec_s(p.preconditioner));
        if (si.retv < 0) logf2(fp, "*** Exceeded max iter ***\n");
        logf2(fp, "Total iterations                             : %d\n", si.niter);
        logf2(fp, "Global dimension (number of rows)            : %ld\n", (long)n);
        logf2(fp, "Local dimension (number of rows)             : %d\n", n);
        logf2(fp, "Initial residual                             : %.10lf\n", si.delta0);
        logf2(fp, "Final residual                               : %.10lf\n", si.exit_res);
        if (p.preconditioner == BCMGX_PREC_BCMG) {
            logf2(fp, "Number of hierarchies                        : %d\n", 1);
            logf2(fp, "Estimated ratio                              : %f\n", 1.0);
            logf2(fp, "max_hrc                                      : %d\n", p.max_hrc);
            logf2(fp, "conv_ratio                                   : %f\n", p.conv_ratio);
            logf2(fp, "bootstrap_composition_type                   : %s\n", boot_s(p.bootstrap_type));
            logf2(fp, "solver_it                                    : %d\n", 15);
            logf2(fp, "ncycle_type                                  : %s\n", cycle_s(p.cycle_type));
            logf2(fp, "relax_type                                   : %s\n", "L1_JACOBI");
            logf2(fp, "relaxnumber_coarse                           : %d\n", p.relaxnumber_coarse);
            logf2(fp, "prerelax_number                              : %d\n", p.prerelax_sweeps);
            logf2(fp, "postrelax_number                             : %d\n", p.postrelax_sweeps);
            logf2(fp, "relax_weight                                 : %f\n", 1.0);
            logf2(fp, "Number of levels                             : %d\n", hi.num_levels);
            for (int l = 0; l < hi.num_levels; l++)
                logf2(fp, "A%-44d: n: %ld nnz: %lld avg_nnz: %f\n", l, (long)hi.n[l], (long long)hi.nnz[l], (float)hi.nnz[l] / (float)hi.n[l]);
            logf2(fp, "Current cmplx for V-cycle                    : %lf\n", hi.op_cmplx);
            logf2(fp, "Current cmplx for W-cycle                    : %lf\n", hi.op_wcmplx);
            logf2(fp, "Average Coarsening Ratio                     : %lf\n", hi.avg_cratio);
        }
        logf2(fp, "\n");
        logf2(fp, "|%-130s|%15s|%15s|%15s|%10s|%10s|%10s|%6s|\n", "PATH", "MIN [ns]", "MAX [ns]", "AVG [ns]", "# MIN", "# MAX", "# AVG", "# PROC");
        logf2(fp, "|%-130s|%15lu|%15lu|%15.2lf|%10lu|%10lu|%10.2lf|%6d|\n", "prec_setup", setup_ns, setup_ns, (double)setup_ns, 1UL, 1UL, 1.0, 1);
        logf2(fp, "|%-130s|%15lu|%15lu|%15.2lf|%10lu|%10lu|%10.2lf|%6d|\n", "solve", solve_ns, solve_ns, (double)solve_ns, 1UL, 1UL, 1.0, 1);
        logf2(fp, "\nTOTAL SOLVE TIME [s]: %lf\n", (double)solve_ns * 1e-9);
        logf2(fp, "DEVICE SETUP TIME [ms]: %lf\nDEVICE SOLVE TIME [ms]: %lf\n", hi.setup_ms, si.solve_ms);
        if (fp) std::fclose(fp);
    }
    for (const std::string& pf : { summary_prof, detailed_prof }) {
        if (pf.empty()) continue;
        FILE* f = std::fopen((pf + "0").c_str(), "w");
        if (!f) continue;
        std::fprintf(f, "prec_setup %lu ns\nsolve %lu ns\n", setup_ns, solve_ns);
        std::fclose(f);
    }
    std::printf("Finalizing preconditioner\n");
    bcmgx_free(h);
    if (!out_file.empty()) {
        std::printf("Dumping solution\n");
        FILE* f = std::fopen(out_file.c_str(), "w");
        if (!f) {
            std::printf("Error opening %s for writing\n", out_file.c_str());
        } else {
            for (int i = 0; i < n; i++) std::fprintf(f, "%g\n", x[i]);
            std::fclose(f);
            std::printf("...done.\n");
        }
    }
    std::printf("Shutdown\n");
    return 0;
}
