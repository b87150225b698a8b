// params.cpp -- settings: defaults, the .properties reader, the legacy positional reader, dump.
// Behaviour follows BCMGX/src/config/Params.cu and Params.h of the reference.
#include "internal.h"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>

namespace bcmgx {

namespace {

const char* const kSolvers[] = { "CGHS", "FCG", "CGS", "PIPELINED_CGS", "CGS_CUBLAS", "INVALID" };
const char* const kPrecs[] = { "NONE", "L1_JACOBI", "BCMG", "AFSAI", "INVALID" };
const char* const kBoots[] = { "MULTIPLICATIVE", "SYMMETRIZED_MULTIPLICATIVE", "ADDITIVE", "INVALID" };
const char* const kMatch[] = { "SUITOR", "INVALID" };
const char* const kCycles[] = { "V_CYCLE", "H_CYCLE", "W_CYCLE", "VARIABLE_V_CYCLE", "INVALID" };
const char* const kRelax[] = { "L1_JACOBI", "INVALID" };

// string -> enum; an unknown string maps to the INVALID member (Params.cu:16-260).
template <size_t N>
int lookup(const char* const (&tab)[N], const std::string& s)
{
    for (size_t i = 0; i + 1 < N; i++)
        if (s == tab[i]) return (int)i;
    return (int)N - 1;
}

template <size_t N>
const char* name_of(const char* const (&tab)[N], int v)
{
    return (v >= 0 && v < (int)N) ? tab[v] : "INVALID";
}

// trim/ltrim/rtrim of BCMGX/src/utility/string.cu:7-29 (std::isspace on both ends).
std::string trim(std::string s)
{
    auto notsp = [](unsigned char c) { return !std::isspace(c); };
    s.erase(std::find_if(s.rbegin(), s.rend(), notsp).base(), s.end());
    s.erase(s.begin(), std::find_if(s.begin(), s.end(), notsp));
    return s;
}

int to_int(const std::string& key, const std::string& v)
{
    try {
        size_t pos = 0;
        int r = std::stoi(v, &pos);
        return r;
    } catch (...) {
        throw Error(BCMGX_ERR_INVALID_INPUT, "settings: value of '" + key + "' is not an integer: '" + v + "'");
    }
}

double to_double(const std::string& key, const std::string& v)
{
    try {
        return std::stod(v);
    } catch (...) {
        throw Error(BCMGX_ERR_INVALID_INPUT, "settings: value of '" + key + "' is not a number: '" + v + "'");
    }
}

constexpr int kBufSize = 1024;

}  // namespace

const char* solver_name(int v) { return name_of(kSolvers, v); }
const char* prec_name(int v) { return name_of(kPrecs, v); }
const char* cycle_name(int v) { return name_of(kCycles, v); }
const char* boot_name(int v) { return name_of(kBoots, v); }

// Defaults of struct params, BCMGX/src/config/Params.h:238-291.
void params_default(bcmgx_params* p)
{
    std::memset(p, 0, sizeof(*p));
    p->solver = BCMGX_SOLVER_CGHS;
    p->itnlim = 2000;
    p->rtol = 1.e-6;
    p->dispnorm = 1;
    p->preconditioner = BCMGX_PREC_NONE;
    p->bootstrap_type = BCMGX_BOOT_MULTIPLICATIVE;
    p->max_hrc = 1;
    p->conv_ratio = 0.8;
    p->matchtype = BCMGX_MATCH_SUITOR;
    p->aggrsweeps = 2;
    p->aggr_type = 0;
    p->max_levels = 39;
    p->cycle_type = BCMGX_CYCLE_V;
    p->coarse_solver = BCMGX_L1_JACOBI;
    p->relax_type = BCMGX_L1_JACOBI;
    p->relaxnumber_coarse = 20;
    p->prerelax_sweeps = 4;
    p->postrelax_sweeps = 4;
    p->l1jacsweeps = 4;
    p->sstep = 1;
    p->stop_criterion = 1;
    p->ru_res = 1;
    p->rec_res_int = 0;
    p->error = 0;
    p->vcycle_precision = BCMGX_VCYCLE_FP64;
    p->record_sweeps = 0;
    p->use_graph = 1;
    p->device = -1;
    p->autotune = 1;
    p->stream = nullptr;
}

// key = value reader. Restates parse_properties_file (Params.cu:272-327): the text after '#'
// is ignored when looking for '=', the last '=' before it splits key and value, a line of
// spaces only is skipped, a non-blank line without '=' is an error. The value runs to the end
// of the physical line (Params.cu:311) and is trimmed, so numbers tolerate a trailing comment
// and enumerations do not. Keys as in Params::initFromPropertiesFile (Params.cu:330-402);
// unknown keys are ignored.
void params_from_properties(const char* path, bcmgx_params* p)
{
    params_default(p);
    FILE* fp = std::fopen(path, "r");
    if (!fp)
        throw Error(BCMGX_ERR_INVALID_INPUT, std::string("Error opening setting file ") + path + ": " + std::strerror(errno));
    char buf[kBufSize + 1];
    int line = 0;
    try {
        while (std::fgets(buf, kBufSize, fp) != nullptr) {
            line++;
            const char* hash = std::strchr(buf, '#');
            int len = hash ? (int)(hash - buf) : (int)std::strlen(buf);
            if (len > 0 && buf[len - 1] == '\n') len--;
            bool empty = true;
            int eq = -1;
            for (int i = 0; i < len; i++) {
                if (buf[i] != ' ') empty = false;
                if (buf[i] == '=') eq = i;
            }
            if (empty) continue;
            if (eq < 0)
                throw Error(BCMGX_ERR_INVALID_INPUT, std::string("Error reading setting file ") + path +
                        ": could not find '=' at line " + std::to_string(line));
            std::string key = trim(std::string(buf, eq));
            std::string value = trim(std::string(buf + eq + 1));
            if (key == "rhsfile" || key == "solfile") {
                // parsed and unused by the reference's solve path
            } else if (key == "solver") p->solver = lookup(kSolvers, value);
            else if (key == "itnlim") p->itnlim = to_int(key, value);
            else if (key == "rtol") p->rtol = to_double(key, value);
            else if (key == "dispnorm") p->dispnorm = to_int(key, value);
            else if (key == "preconditioner") p->preconditioner = lookup(kPrecs, value);
            else if (key == "bootstrap_type") p->bootstrap_type = lookup(kBoots, value);
            else if (key == "max_hrc") p->max_hrc = to_int(key, value);
            else if (key == "conv_ratio") p->conv_ratio = to_double(key, value);
            else if (key == "matchtype") p->matchtype = lookup(kMatch, value);
            else if (key == "aggrsweeps") p->aggrsweeps = to_int(key, value);
            else if (key == "aggr_type") p->aggr_type = to_int(key, value);
            else if (key == "max_levels") p->max_levels = to_int(key, value);
            else if (key == "cycle_type") p->cycle_type = lookup(kCycles, value);
            else if (key == "coarse_solver") p->coarse_solver = lookup(kRelax, value);
            else if (key == "relax_type") p->relax_type = lookup(kRelax, value);
            else if (key == "relaxnumber_coarse") p->relaxnumber_coarse = to_int(key, value);
            else if (key == "prerelax_sweeps") p->prerelax_sweeps = to_int(key, value);
            else if (key == "postrelax_sweeps") p->postrelax_sweeps = to_int(key, value);
            else if (key == "l1jacsweeps") p->l1jacsweeps = to_int(key, value);
            else if (key == "sstep") p->sstep = to_int(key, value);
            else if (key == "stop_criterion") p->stop_criterion = to_int(key, value);
            else if (key == "ru_res") p->ru_res = to_int(key, value);
            else if (key == "rec_res_int") p->rec_res_int = to_int(key, value);
            // extensions (not in the reference's key set)
            else if (key == "vcycle_precision") p->vcycle_precision = (value == "FP32" || value == "1") ? BCMGX_VCYCLE_FP32 : BCMGX_VCYCLE_FP64;
        }
    } catch (...) {
        std::fclose(fp);
        throw;
    }
    std::fclose(fp);
}

namespace {
// get_*_param of Params.cu:223-270: one value per line, first '%'-delimited token.
std::string legacy_token(FILE* fp, const char* what)
{
    char buf[kBufSize + 1];
    if (std::fgets(buf, kBufSize, fp) == nullptr)
        throw Error(BCMGX_ERR_INVALID_INPUT, std::string("ERROR: reading param ") + what + " from conf file");
    char* save = nullptr;
    char* tok = strtok_r(buf, "%", &save);
    return tok ? std::string(tok) : std::string();
}
int legacy_int(FILE* fp, const char* what)
{
    int v = 0;
    std::sscanf(legacy_token(fp, what).c_str(), "%d", &v);
    return v;
}
double legacy_double(FILE* fp, const char* what)
{
    double v = 0;
    std::sscanf(legacy_token(fp, what).c_str(), "%lf", &v);
    return v;
}
std::string legacy_string(FILE* fp, const char* what) { return trim(legacy_token(fp, what)); }
}  // namespace

// Positional settings file, fixed line order of Params::initFromFile (Params.cu:406-474).
void params_from_legacy(const char* path, bcmgx_params* p)
{
    params_default(p);
    FILE* fp = std::fopen(path, "r");
    if (!fp)
        throw Error(BCMGX_ERR_INVALID_INPUT, std::string("Error opening setting file ") + path + ": " + std::strerror(errno));
    try {
        legacy_string(fp, "rhsfile");
        legacy_string(fp, "solfile");
        p->solver = lookup(kSolvers, legacy_string(fp, "solver_type"));
        p->bootstrap_type = lookup(kBoots, legacy_string(fp, "bootstrap_composition_type"));
        p->max_hrc = legacy_int(fp, "max_hrc");
        p->conv_ratio = legacy_double(fp, "conv_ratio");
        p->matchtype = lookup(kMatch, legacy_string(fp, "matchtype"));
        p->aggrsweeps = legacy_int(fp, "aggrsweeps");
        p->aggr_type = legacy_int(fp, "aggrtype");
        p->max_levels = legacy_int(fp, "max_levels");
        p->cycle_type = lookup(kCycles, legacy_string(fp, "cycle_type"));
        p->coarse_solver = lookup(kRelax, legacy_string(fp, "coarse_solver"));
        p->relax_type = lookup(kRelax, legacy_string(fp, "relax_type"));
        p->relaxnumber_coarse = legacy_int(fp, "relaxnumber_coarse");
        legacy_int(fp, "coarsesolver_type");
        p->prerelax_sweeps = legacy_int(fp, "prerelax_sweeps");
        p->postrelax_sweeps = legacy_int(fp, "postrelax_sweeps");
        p->itnlim = legacy_int(fp, "itnlim");
        p->rtol = legacy_double(fp, "rtol");
        p->sstep = legacy_int(fp, "sstep");
        p->stop_criterion = legacy_int(fp, "stop_criterion");
        p->ru_res = legacy_int(fp, "ru_res");
        p->preconditioner = lookup(kPrecs, legacy_string(fp, "sprec"));
        p->l1jacsweeps = legacy_int(fp, "l1jacsweeps");
        p->rec_res_int = legacy_int(fp, "rec_res_int");
        p->dispnorm = legacy_int(fp, "dispnorm");
        legacy_int(fp, "detailedtiming");
    } catch (...) {
        std::fclose(fp);
        throw;
    }
    std::fclose(fp);
    if (p->max_hrc != 1) p->error = 1;   // "[ERROR] bootstrap not yet supported" (Params.cu:463-466)
    if (p->aggr_type != 0) p->error = 1; // "[ERROR] aggr_type value not supported" (:467-470)
}

// Params::dump (Params.cu:476-506), same lines and formats.
void params_dump(const bcmgx_params* p, FILE* out)
{
    std::fprintf(out, "\trhsfile: %s\n", "NONE");
    std::fprintf(out, "\tsolfile: %s\n", "NONE");
    std::fprintf(out, "\tsolver_type: %s\n", solver_name(p->solver));
    std::fprintf(out, "\tbootstrap_composition_type: %s\n", boot_name(p->bootstrap_type));
    std::fprintf(out, "\tmax_hrc: %d\n", p->max_hrc);
    std::fprintf(out, "\tconv_ratio: %f\n", p->conv_ratio);
    std::fprintf(out, "\tmatchtype %s\n", name_of(kMatch, p->matchtype));
    std::fprintf(out, "\taggrsweeps: %d\n", p->aggrsweeps);
    std::fprintf(out, "\taggrtype: %d\n", p->aggr_type);
    std::fprintf(out, "\tmax_levels: %d\n", p->max_levels);
    std::fprintf(out, "\tcycle_type: %s\n", cycle_name(p->cycle_type));
    std::fprintf(out, "\tcoarse_solver_type: %s\n", name_of(kRelax, p->coarse_solver));
    std::fprintf(out, "\trelax_type: %s\n", name_of(kRelax, p->relax_type));
    std::fprintf(out, "\tprerelax_sweeps: %d\n", p->prerelax_sweeps);
    std::fprintf(out, "\tpostrelax_sweeps: %d\n", p->postrelax_sweeps);
    std::fprintf(out, "\titnlim: %d\n", p->itnlim);
    std::fprintf(out, "\trtol: %f\n", p->rtol);
    std::fprintf(out, "\trelaxnumber_coarse: %d\n", p->relaxnumber_coarse);
    std::fprintf(out, "\tmem_alloc_size: %d\n", 2000000);
    std::fprintf(out, "\terror: %d\n", p->error);
    std::fprintf(out, "\tsstep: %d\n", p->sstep);
    std::fprintf(out, "\tstop_criterion: %d\n", p->stop_criterion);
    std::fprintf(out, "\tru_res: %d\n", p->ru_res);
    std::fprintf(out, "\tpreconditioner_type: %s\n", prec_name(p->preconditioner));
    std::fprintf(out, "\tl1jacsweeps: %d\n", p->l1jacsweeps);
    std::fprintf(out, "\trec_res_int: %d\n", p->rec_res_int);
    std::fprintf(out, "\tdispnorm: %d\n", p->dispnorm);
}

}  // namespace bcmgx
