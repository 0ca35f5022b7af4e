// Host-side restatement of the reference's Fortran driver, calling the ext_* C ABI of a
// backend library loaded with dlopen.  Each routine cites the Fortran it follows
// (paths relative to the reference project; 2D and 3D drivers share their logic).
// Compile with -ffp-contract=off: the scalar recurrences (alpha = rro/pw, ...) must
// round exactly as the Fortran's.

#include "tea_driver.h"

#include <dlfcn.h>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tea_b200.h"
#include "tea_eigen.h"

namespace {

thread_local std::string g_last_error;

struct DriverError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

[[noreturn]] void fail(const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    throw DriverError(buf);
}

// ----------------------------------------------------------------------------- deck

enum { G_RECT = 1, G_CIRC = 2, G_POINT = 3 };  // tealeaf_2d/data.f90:62-64
enum { FIELD_DENSITY = 1, FIELD_ENERGY0, FIELD_ENERGY1, FIELD_U, FIELD_P, FIELD_SD };
constexpr int NUM_FIELDS = 6;
constexpr int CONDUCTIVITY = 1, RECIP_CONDUCTIVITY = 2;
// g_small is a REAL(8) PARAMETER initialised from a default-real literal
// (tealeaf_2d/data.f90:30).
constexpr double G_SMALL = (double)1.0e-16f;

struct State {
    bool defined = false;
    double density = 0.0, energy = 0.0;
    double xmin = 0.0, xmax = 0.0, ymin = 0.0, ymax = 0.0, zmin = 0.0, zmax = 0.0;
    double radius = 0.0;
    int geometry = 0;
};

struct Config {
    int dim = 2;
    double xmin = 0.0, ymin = 0.0, zmin = 0.0, xmax = 100.0, ymax = 100.0, zmax = 100.0;
    int x_cells = 10, y_cells = 10, z_cells = 10;
    // Defaults of tealeaf_2d/read_input.f90:39-80.  dtinit, eps and tl_ch_cg_epslim are
    // assigned from default-real (single precision) literals there.
    double dtinit = (double)0.1f;
    int max_iters = 1000;
    double eps = (double)1.0e-10f;
    double end_time = 10.0;
    int end_step = 640000;  // g_ibig, tealeaf_2d/data.f90:28
    int summary_frequency = 10;
    int visit_frequency = 0;
    int coefficient = CONDUCTIVITY;
    bool profiler_on = false;
    bool tl_ch_cg_errswitch = false;
    int tl_ch_cg_presteps = 30;
    double tl_ch_cg_epslim = (double)1e-5f;
    bool tl_check_result = false;
    int tl_ppcg_inner_steps = 10;
    bool tl_preconditioner_on = false;
    int solver = TEA_SOLVER_JACOBI;
    int test_problem = 0;
    bool use_ext_kernels = true;
    // Additive keywords (not in the reference).
    double tl_eps_rel = 0.0;  // relative target: eps = tl_eps_rel^2 * sum(u0^2) per solve
    bool use_fused_solve = false;
    int precision = 0;          // tl_precision fp64 | fp32 (whole-solve path only)
    int inner_max_iters = 0;    // tl_inner_max_iters
    double inner_tol = 0.0;     // tl_inner_tol
    int inner_solver = 0;       // tl_inner_solver deck | chebyshev
    std::vector<State> states;  // states[0] is state 1
};

// Line preprocessing of parse_getline (tealeaf_2d/parse.f90:143-247): control characters
// become blanks, '!' and ';' start comments, the line is lower-cased and '=' and ','
// become blanks.  Only lines inside the *tea ... *endtea block are returned.
std::vector<std::vector<std::string>> deck_lines(const std::string& text)
{
    std::vector<std::vector<std::string>> out;
    std::istringstream in(text);
    std::string raw;
    bool inside = false;
    while (std::getline(in, raw)) {
        std::string l = raw;
        for (char& ch : l) {
            unsigned char u = (unsigned char)ch;
            if (u < 32 || u > 128) ch = ' ';
        }
        size_t s = l.find('!');
        if (s != std::string::npos) l = l.substr(0, s);
        s = l.find(';');
        if (s != std::string::npos) l = l.substr(0, s);
        for (char& ch : l) ch = (char)std::tolower((unsigned char)ch);
        size_t b = l.find_first_not_of(' ');
        if (b == std::string::npos) continue;
        l = l.substr(b);
        if (l[0] == '*') {
            std::string nugget = l.substr(0, l.find(' '));
            if (nugget == "*tea") inside = true;
            else if (nugget == "*endtea") inside = false;
            continue;
        }
        if (!inside) continue;
        for (char& ch : l)
            if (ch == '=' || ch == ',') ch = ' ';
        std::vector<std::string> words;
        std::istringstream ws(l);
        std::string w;
        while (ws >> w) words.push_back(w);
        if (!words.empty()) out.push_back(words);
    }
    return out;
}

// parse_getival: READ(word, '(I7)').
int getival(const std::string& w)
{
    std::string t = w.substr(0, 7);
    char* end = nullptr;
    long v = std::strtol(t.c_str(), &end, 10);
    if (end == t.c_str() || *end != '\0') fail("Error attempting to convert to integer:%s", w.c_str());
    return (int)v;
}

// parse_getrval: integers get ".0" appended, then READ(word, '(E27.20)').
double getrval(const std::string& w)
{
    std::string t = w.substr(0, 27);
    char* end = nullptr;
    double v = std::strtod(t.c_str(), &end);
    if (end == t.c_str()) fail("Error attempting to convert to real:%s", w.c_str());
    return v;
}

// read_input, tealeaf_2d/read_input.f90:24-299 (3D: tealeaf_3d/read_input.f90).
Config parse_deck(const std::string& text, int dim)
{
    Config cfg;
    cfg.dim = dim;
    auto lines = deck_lines(text);
    // A value may sit on the next line (parse_getword(.TRUE.) wraps).
    size_t li = 0, wi = 0;
    auto next_word = [&](bool wrap) -> std::string {
        while (li < lines.size()) {
            if (wi < lines[li].size()) return lines[li][wi++];
            if (!wrap) return std::string();
            ++li;
            wi = 0;
        }
        return std::string();
    };
    int state_max = 0;
    for (auto& l : lines)
        for (size_t k = 0; k < l.size(); ++k)
            if (l[k] == "state") {
                if (k + 1 < l.size()) state_max = std::max(state_max, getival(l[k + 1]));
                break;
            }
    if (state_max < 1) fail("read_input: No states defined.");
    cfg.states.assign(state_max, State());

    // One cursor over the words: a keyword reads its value with wrap, after which the
    // remaining words come from the line the value was taken from, as in the Fortran.
    li = 0;
    wi = 0;
    while (li < lines.size()) {
        {
            std::string word = next_word(false);
            if (word.empty()) {
                ++li;
                wi = 0;
                continue;
            }
            if (word == "initial_timestep") cfg.dtinit = getrval(next_word(true));
            else if (word == "end_time") cfg.end_time = getrval(next_word(true));
            else if (word == "end_step") cfg.end_step = getival(next_word(true));
            else if (word == "xmin") cfg.xmin = getrval(next_word(true));
            else if (word == "xmax") cfg.xmax = getrval(next_word(true));
            else if (word == "ymin") cfg.ymin = getrval(next_word(true));
            else if (word == "ymax") cfg.ymax = getrval(next_word(true));
            else if (word == "zmin" && dim == 3) cfg.zmin = getrval(next_word(true));
            else if (word == "zmax" && dim == 3) cfg.zmax = getrval(next_word(true));
            else if (word == "x_cells") cfg.x_cells = getival(next_word(true));
            else if (word == "y_cells") cfg.y_cells = getival(next_word(true));
            else if (word == "z_cells" && dim == 3) cfg.z_cells = getival(next_word(true));
            else if (word == "visit_frequency") cfg.visit_frequency = getival(next_word(true));
            else if (word == "summary_frequency") cfg.summary_frequency = getival(next_word(true));
            else if (word == "tl_ch_cg_presteps") cfg.tl_ch_cg_presteps = getival(next_word(true));
            else if (word == "tl_ppcg_inner_steps") cfg.tl_ppcg_inner_steps = getival(next_word(true));
            else if (word == "tl_ch_cg_epslim") cfg.tl_ch_cg_epslim = getrval(next_word(true));
            else if (word == "tl_check_result") cfg.tl_check_result = true;
            else if (word == "tl_ch_cg_errswitch") cfg.tl_ch_cg_errswitch = true;
            else if (word == "tl_preconditioner_on") cfg.tl_preconditioner_on = true;
            else if (word == "use_fortran_kernels") cfg.use_ext_kernels = false;
            else if (word == "use_ext_kernels") cfg.use_ext_kernels = true;
            else if (word == "tl_use_jacobi") cfg.solver = TEA_SOLVER_JACOBI;
            else if (word == "tl_use_cg") cfg.solver = TEA_SOLVER_CG;
            else if (word == "tl_use_ppcg") cfg.solver = TEA_SOLVER_PPCG;
            else if (word == "tl_use_chebyshev") cfg.solver = TEA_SOLVER_CHEBYSHEV;
            else if (word == "profiler_on") cfg.profiler_on = true;
            else if (word == "tl_max_iters") cfg.max_iters = getival(next_word(true));
            else if (word == "tl_eps") cfg.eps = getrval(next_word(true));
            else if (word == "tl_coefficient_density") cfg.coefficient = CONDUCTIVITY;
            else if (word == "tl_coefficient_inverrse_density") cfg.coefficient = RECIP_CONDUCTIVITY;
            else if (word == "test_problem") cfg.test_problem = getival(next_word(true));
            else if (word == "tl_eps_rel") cfg.tl_eps_rel = getrval(next_word(true));
            else if (word == "use_fused_solve") cfg.use_fused_solve = true;
            else if (word == "tl_precision") {
                std::string v = next_word(true);
                if (v == "fp64") cfg.precision = TEA_PRECISION_FP64;
                else if (v == "fp32") cfg.precision = TEA_PRECISION_FP32_REFINED;
                else fail("read_input: tl_precision must be fp64 or fp32, not %s", v.c_str());
            } else if (word == "tl_inner_tol") cfg.inner_tol = getrval(next_word(true));
            else if (word == "tl_inner_solver") {
                const std::string v = next_word(true);
                if (v == "deck") cfg.inner_solver = TEA_INNER_DECK;
                else if (v == "chebyshev") cfg.inner_solver = TEA_INNER_CHEBYSHEV;
                else fail("read_input: tl_inner_solver must be deck or chebyshev, not %s", v.c_str());
            }
            else if (word == "tl_inner_max_iters") cfg.inner_max_iters = getival(next_word(true));
            else if (word == "state") {
                int s = getival(next_word(true));
                if (s < 1 || s > state_max) fail("read_input: bad state %d", s);
                State& st = cfg.states[s - 1];
                if (st.defined) fail("read_input: State defined twice.");
                st.defined = true;
                for (;;) {
                    std::string k = next_word(false);
                    if (k.empty()) break;
                    if (k == "xmin") st.xmin = getrval(next_word(true));
                    else if (k == "ymin") st.ymin = getrval(next_word(true));
                    else if (k == "zmin" && dim == 3) st.zmin = getrval(next_word(true));
                    else if (k == "xmax") st.xmax = getrval(next_word(true));
                    else if (k == "ymax") st.ymax = getrval(next_word(true));
                    else if (k == "zmax" && dim == 3) st.zmax = getrval(next_word(true));
                    else if (k == "radius") st.radius = getrval(next_word(true));
                    else if (k == "density") st.density = getrval(next_word(true));
                    else if (k == "energy") st.energy = getrval(next_word(true));
                    else if (k == "geometry") {
                        std::string g = next_word(true);
                        if ((dim == 2 && g == "rectangle") || (dim == 3 && g == "cuboid")) st.geometry = G_RECT;
                        else if (g == "circle") st.geometry = G_CIRC;
                        else if (g == "point") st.geometry = G_POINT;
                    }
                }
            }
        }
    }
    if (!cfg.use_ext_kernels) fail("read_input: use_fortran_kernels is not available; the ext_* kernels are the product path");
    // Shrink states 2..N by a hundredth of a cell (tealeaf_2d/read_input.f90:290-297).
    // float(x_cells) is a default-real conversion, exact for any realistic size.
    const double dx = (cfg.xmax - cfg.xmin) / (double)(float)cfg.x_cells;
    const double dy = (cfg.ymax - cfg.ymin) / (double)(float)cfg.y_cells;
    const double dz = (cfg.zmax - cfg.zmin) / (double)(float)cfg.z_cells;
    for (size_t n = 1; n < cfg.states.size(); ++n) {
        State& s = cfg.states[n];
        s.xmin = s.xmin + (dx / 100.0);
        s.ymin = s.ymin + (dy / 100.0);
        s.xmax = s.xmax - (dx / 100.0);
        s.ymax = s.ymax - (dy / 100.0);
        if (dim == 3) {
            s.zmin = s.zmin + (dz / 100.0);
            s.zmax = s.zmax - (dz / 100.0);
        }
    }
    return cfg;
}

// ----------------------------------------------------------------------------- backend

struct Backend {
    void* handle = nullptr;
    int dim = 2;
    void* init = nullptr;
    void (*finalise)() = nullptr;
    void* initialise_chunk = nullptr;
    void* generate_chunk = nullptr;
    void (*field_summary)(const int*, double*, double*, double*, double*) = nullptr;
    void (*set_field)(const int*) = nullptr;
    void (*copy_u)(const int*) = nullptr;
    void (*calc_residual)(const int*) = nullptr;
    void (*calc_2norm)(const int*, double*, const void*) = nullptr;
    void (*finalise_solve)(const int*) = nullptr;
    void (*update_halo)(const int*, const int*, const int*, const int*) = nullptr;
    void* pack = nullptr;  // ext_pack_message_ (2D and 3D signatures differ)
    // tea_pack_face_: the same packing with the 2D bottom/top faces on the inner columns
    void (*pack_face)(const int*, const int*, const int*, const int*, const int*, double*, const void*) = nullptr;
    void (*jacobi_init)(const int*, const int*, const double*) = nullptr;
    void (*jacobi_solve)(const int*, double*) = nullptr;
    void (*cg_init)(const int*, const int*, const int*, double*, double*) = nullptr;
    void (*cg_calc_w)(const int*, double*) = nullptr;
    void (*cg_calc_ur)(const int*, const double*, double*) = nullptr;
    void (*cg_calc_p)(const int*, const double*) = nullptr;
    void (*cheby_init)(const int*, double*, double*, const double*, const int*, const int*) = nullptr;
    void (*cheby_iterate)(const int*, const int*) = nullptr;
    void (*ppcg_init)(const int*, double*, double*, const double*, const int*) = nullptr;
    void (*ppcg_init_sd)(const int*) = nullptr;
    void (*ppcg_inner)(const int*, int*) = nullptr;
    void (*whole_solve)(const int*, const tea_solve_params*, tea_solve_result*) = nullptr;
    void (*get_status)(int*) = nullptr;
    int (*transfer_bytes)(const int*, long long*, long long*) = nullptr;
    int (*ws_record)(const int*, const int*) = nullptr;
    int (*ws_attach)(const int*, const int*) = nullptr;
    int (*chunk_dims)(const int*, int*) = nullptr;             // tea_chunk_dims_ (visit output)
    int (*read_field)(const int*, const int*, double*) = nullptr;  // tea_read_field_

    template <class F>
    void bind(F& fp, const char* name, bool required = true)
    {
        void* s = dlsym(handle, name);
        if (!s && required) fail("backend lacks symbol %s", name);
        fp = reinterpret_cast<F>(s);
    }

    void open(const char* path, int d)
    {
        dim = d;
        handle = dlopen(path, RTLD_NOW | RTLD_LOCAL);
        if (!handle) fail("dlopen(%s): %s", path, dlerror());
        init = dlsym(handle, "ext_init_");
        initialise_chunk = dlsym(handle, "ext_initialise_chunk_");
        generate_chunk = dlsym(handle, "ext_generate_chunk_");
        if (!init || !initialise_chunk || !generate_chunk) fail("backend lacks the set-up symbols");
        bind(finalise, "ext_finalise_");
        bind(field_summary, "ext_field_summary_kernel_");
        bind(set_field, "ext_set_field_kernel_");
        bind(copy_u, "ext_solver_copy_u_");
        bind(calc_residual, "ext_calculate_residual_");
        bind(calc_2norm, "ext_calculate_2norm_");
        bind(finalise_solve, "ext_solver_finalise_");
        bind(update_halo, "ext_update_halo_kernel_");
        pack = dlsym(handle, "ext_pack_message_");
        bind(pack_face, "tea_pack_face_", false);
        bind(jacobi_init, "ext_jacobi_kernel_init_");
        bind(jacobi_solve, "ext_jacobi_kernel_solve_");
        bind(cg_init, "ext_cg_solver_init_");
        bind(cg_calc_w, "ext_cg_calc_w_");
        bind(cg_calc_ur, "ext_cg_calc_ur_");
        bind(cg_calc_p, "ext_cg_calc_p_");
        bind(cheby_init, "ext_cheby_solver_init_");
        bind(cheby_iterate, "ext_cheby_solver_iterate_");
        bind(ppcg_init, "ext_ppcg_init_");
        bind(ppcg_init_sd, "ext_ppcg_init_sd_");
        bind(ppcg_inner, "ext_ppcg_inner_");
        bind(whole_solve, "ext_tea_leaf_solve_", false);
        bind(get_status, "ext_get_status_", false);
        bind(transfer_bytes, "tea_transfer_bytes_", false);
        bind(ws_record, "tea_ws_record_", false);
        bind(ws_attach, "tea_ws_attach_", false);
        bind(chunk_dims, "tea_chunk_dims_", false);
        bind(read_field, "tea_read_field_", false);
    }

    void close()
    {
        // The library stays loaded (dlclose would unload CUDA state mid-process);
        // the handle is reference counted by the loader.
        handle = nullptr;
    }

    void check_status(const char* where)
    {
        if (!get_status) return;
        int st = 0;
        get_status(&st);
        if (st != TEA_OK && st != TEA_ERR_NOT_CONVERGED && st != TEA_ERR_NONFINITE) fail("backend status %d after %s", st, where);
    }
};

// ----------------------------------------------------------------------------- output

// v in Fortran's E12.4 edit descriptor (right-justified in 12 characters, mantissa
// 0.dddd, exponent E+dd, or +ddd without the E beyond two digits), the format of the
// reference's graphics files.  out holds at least 13 characters.
void fortran_e12_4(char* out, double v)
{
    if (std::isnan(v)) {
        std::snprintf(out, 13, "%12s", "NaN");
        return;
    }
    if (std::isinf(v)) {
        std::snprintf(out, 13, "%12s", v > 0 ? "Infinity" : "-Infinity");
        return;
    }
    const char* sign = std::signbit(v) ? "-" : "";
    char body[32];
    if (v == 0.0) {
        std::snprintf(body, sizeof(body), "%s0.0000E+00", sign);
    } else {
        char m[32];
        std::snprintf(m, sizeof(m), "%.3E", std::fabs(v));  // d.dddE+xx, rounded to 4 digits
        const char digits[5] = {m[0], m[2], m[3], m[4], 0};
        const int e = std::atoi(m + 6) + 1;  // 0.dddd x 10^e
        const int ae = e < 0 ? -e : e;
        if (ae <= 99) std::snprintf(body, sizeof(body), "%s0.%sE%c%02d", sign, digits, e < 0 ? '-' : '+', ae);
        else std::snprintf(body, sizeof(body), "%s0.%s%c%03d", sign, digits, e < 0 ? '-' : '+', ae);
    }
    std::snprintf(out, 13, "%12.12s", body);  // body has at most 11 characters
}

struct Log {
    FILE* file = nullptr;
    bool echo = true;
    void line(const char* fmt, ...)
    {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        if (file) fprintf(file, "%s\n", buf);
        if (echo) printf("%s\n", buf);
    }
};

double now_seconds()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Known answers of tealeaf_2d/field_summary.f90:92-143 and tealeaf_3d/field_summary.f90:93-169.
// 3D test 6 is compared against a default-real literal in the reference.
bool known_answer(int dim, int test, double* expected)
{
    static const double kat2d[] = {103.88639125996923, 177.00175203427580, 139.97102840522848,
                                   118.33195538063963, 108.12687625327908, 103.46970921076068,
                                   101.21009327612924, 100.16633923123922, 99.695059768963887,
                                   99.756584330021866, 106.22536751207716, 103.75236286020100,
                                   102.95322957172701, 102.61257379535277, 101.99792927438858,
                                   101.93825682423312, 101.54636465546844, 101.51302189154072};
    static const double kat3d[] = {157.550841832793,   116.067951160930,   95.4865103390698,
                                   166.838315378708,   116.482111627676,   (double)57.275950005439007f,
                                   56.905915016570454, 70.914754278021732, 58.156372502592568,
                                   57.571559142436392, 58.442896702081427, 57.788169431988784,
                                   57.847149250777079, 58.633563819463340, 59.336123231095804,
                                   60.219852602894704, 58.374475944856059, 58.605123548564777,
                                   58.322724309579144, 58.529888354664266, 59.029784947717950,
                                   59.496231543737323, 57.788169432006349, 58.922579985226299,
                                   59.629007203000995, 58.421562127057406, 59.093728049719466,
                                   58.222880800927285, 59.225127737540063};
    if (dim == 2 && test >= 6 && test <= 23) { *expected = kat2d[test - 6]; return true; }
    if (dim == 3 && test >= 1 && test <= 29) { *expected = kat3d[test - 1]; return true; }
    return false;
}

// ----------------------------------------------------------------------------- run

struct Runner {
    Config cfg;
    Backend be;
    Log log;
    const tea_run_options* opt;
    const tea_comm* comm = nullptr;  // several ranks: slabs (tea_run_deck_comm)
    int chunk = 1;
    int neighbours[6] = {-1, -1, -1, -1, -1, -1};  // every face EXTERNAL_FACE on one rank
    int lx = 0, ly = 0, lz = 0;                    // this rank's chunk, inner cells
    double cx0 = 0.0, cy0 = 0.0, cz0 = 0.0;        // this rank's chunk: first vertex
    double cdx = 0.0, cdy = 0.0, cdz = 0.0;        // and cell widths
    bool visit_started = false;
    std::vector<double> snd, rcv;

    bool split() const { return comm && comm->size > 1; }

    // tea_allsum (tealeaf_2d/tea.f90:1249-1267): every global scalar is a sum over ranks.
    void allsum(double* v, int n)
    {
        if (split()) comm->allreduce_sum(v, n, comm->ctx);
    }

    // tea_exchange (tealeaf_2d/tea.f90:246-407, tealeaf_3d/tea.f90): pack the selected
    // fields' faces towards each internal neighbour, swap, unpack.  Slabs have internal
    // faces only across the split axis (bottom/top in 2D, back/front in 3D).  The 2D
    // bottom/top packer of the reference (tealeaf_2d/ext_pack_kernel.hpp:17-44) starts at
    // padded column 0, so it sends columns 0..nx-1 and the last two inner columns of every
    // exchanged halo row stay stale; a backend that exports tea_pack_face_ packs the inner
    // columns and is used instead.
    void exchange(const int* fields, int depth)
    {
        if (!split()) return;
        if (be.pack_face) {
            exchange_with(fields, depth, [&](int face, double* buf, int pk) {
                be.pack_face(&chunk, fields, cur_offsets, &depth, &face, buf, &pk);
                be.check_status("tea_pack_face_");
            });
            return;
        }
        if (!be.pack) fail("backend lacks ext_pack_message_");
        exchange_with(fields, depth, [&](int face, double* buf, int pk) {
            const int cell_data = 1;
            if (cfg.dim == 2)
                reinterpret_cast<void (*)(const int*, const int*, const int*, const int*, const int*, double*,
                                          const void*)>(be.pack)(&chunk, fields, cur_offsets, &depth, &face, buf, &pk);
            else
                reinterpret_cast<void (*)(const int*, const int*, const int*, const int*, const int*, const int*,
                                          double*, const void*)>(be.pack)(&chunk, fields, cur_offsets, &depth, &face,
                                                                          &cell_data, buf, &pk);
            be.check_status("ext_pack_message_");
        });
    }

    int cur_offsets[NUM_FIELDS] = {};

    template <class Pack>
    void exchange_with(const int* fields, int depth, Pack&& pack)
    {
        const int face_lo = cfg.dim == 2 ? 3 : 5, face_hi = face_lo + 1;  // CHUNK_BOTTOM/TOP, BACK/FRONT
        const int per_depth = cfg.dim == 2 ? lx + 5 : (lx + 5) * (ly + 5);
        int end = 0;
        for (int f = 0; f < NUM_FIELDS; ++f) {
            cur_offsets[f] = fields[f] ? end : (cfg.dim == 2 ? 0 : -1);
            if (fields[f]) end += depth * per_depth;
        }
        if (end == 0) return;
        snd.assign(end, 0.0);
        rcv.assign(end, 0.0);
        for (int face : {face_lo, face_hi}) {
            const int nb = neighbours[face - 1];
            if (nb < 0) continue;  // external
            const int peer = comm->rank + (face == face_lo ? -1 : 1);
            pack(face, snd.data(), 1);
            comm->sendrecv(snd.data(), end, peer, rcv.data(), end, peer, comm->ctx);
            pack(face, rcv.data(), 0);
        }
    }
    double time = 0.0, dt = 0.0;
    int step = 0;
    bool complete = false;
    double rx_unused = 0.0;

    void update_halo(const int* fields, int depth)
    {
        // update_halo (tealeaf_2d/update_halo.f90:27-66): tea_exchange (a no-op on one rank),
        // then the reflective update of the external faces.
        exchange(fields, depth);
        be.update_halo(&chunk, neighbours, fields, &depth);
    }

    void halo(std::initializer_list<int> ids, int depth)
    {
        int fields[NUM_FIELDS] = {0, 0, 0, 0, 0, 0};
        for (int id : ids) fields[id - 1] = 1;
        update_halo(fields, depth);
    }

    void field_summary(tea_run_summary* sum, bool print_kat, double* out4)
    {
        // tealeaf_2d/field_summary.f90:27-161.
        double vol = 0, mass = 0, ie = 0, temp = 0;
        be.field_summary(&chunk, &vol, &mass, &ie, &temp);
        {
            double v4[4] = {vol, mass, ie, temp};
            allsum(v4, 4);
            vol = v4[0];
            mass = v4[1];
            ie = v4[2];
            temp = v4[3];
        }
        log.line("");
        log.line(" Time %.16g", time);
        log.line("                       Volume            Mass         Density          Energy               U");
        log.line(" step:%7d%16.7E%16.7E%16.7E%16.7E%16.7E", step, vol, mass, mass / vol, ie, temp);
        if (out4) { out4[0] = vol; out4[1] = mass; out4[2] = ie; out4[3] = temp; }
        if (sum) { sum->vol = vol; sum->mass = mass; sum->ie = ie; sum->temp = temp; }
        if (print_kat && complete && cfg.test_problem >= 1 && sum) {
            double expected = 0.0;
            sum->test_problem = cfg.test_problem;
            if (known_answer(cfg.dim, cfg.test_problem, &expected)) {
                double qa = std::fabs((100.0 * (temp / expected)) - 100.0);
                sum->kat_available = 1;
                sum->kat_expected = expected;
                sum->qa_diff = qa;
                sum->kat_passed = qa < 0.001;
                log.line("Test problem %4d is within %16.7E%% of the expected solution", cfg.test_problem, qa);
                log.line(sum->kat_passed ? " This test is considered PASSED" : " This test is considered NOT PASSED");
            }
        }
    }

    void start(tea_run_summary* sum)
    {
        // start.f90:24-162.
        time = 0.0;
        step = 0;
        dt = cfg.dtinit;
        int x = cfg.x_cells, y = cfg.y_cells, z = cfg.z_cells, rank = split() ? comm->rank : 0;
        // tea_decompose (tealeaf_2d/tea.f90:115-212) restricted to slabs of the slowest axis:
        // first cell and count of this rank, the remainder going to the first ranks.
        int first = 1;
        if (split()) {
            const int total = cfg.dim == 2 ? y : z, n = comm->size, r = comm->rank;
            const int delta = total / n, mod = total % n;
            first = r * delta + 1 + std::min(r, mod);
            const int count = delta + (r < mod ? 1 : 0);
            if (count < 1) fail("%d ranks for %d cells along the split axis", n, total);
            (cfg.dim == 2 ? y : z) = count;
            const int lo = cfg.dim == 2 ? 2 : 4;  // CHUNK_BOTTOM / CHUNK_BACK, 0-based
            neighbours[lo] = r > 0 ? r : -1;          // the neighbour's chunk id (1-based)
            neighbours[lo + 1] = r < n - 1 ? r + 2 : -1;
        }
        lx = x;
        ly = y;
        lz = z;
        if (cfg.dim == 2) reinterpret_cast<void (*)(int*, int*, int*)>(be.init)(&x, &y, &rank);
        else reinterpret_cast<void (*)(int*, int*, int*, int*)>(be.init)(&x, &y, &z, &rank);
        be.check_status("ext_init_");
        // initialise_chunk.f90:33-36 (x/ymin + d * (left/bottom - 1)).
        double dx = (cfg.xmax - cfg.xmin) / (double)(float)cfg.x_cells;
        double dy = (cfg.ymax - cfg.ymin) / (double)(float)cfg.y_cells;
        double dz = (cfg.zmax - cfg.zmin) / (double)(float)cfg.z_cells;
        const double off = (double)(first - 1);
        double xmin = cfg.xmin + dx * 0.0;
        double ymin = cfg.ymin + dy * (cfg.dim == 2 ? off : 0.0);
        double zmin = cfg.zmin + dz * (cfg.dim == 3 ? off : 0.0);
        cx0 = xmin; cy0 = ymin; cz0 = zmin;
        cdx = dx; cdy = dy; cdz = dz;
        if (cfg.dim == 2)
            reinterpret_cast<void (*)(const int*, const double*, const double*, const double*, const double*)>(
                be.initialise_chunk)(&chunk, &xmin, &ymin, &dx, &dy);
        else
            reinterpret_cast<void (*)(const int*, const double*, const double*, const double*, const double*,
                                      const double*, const double*)>(be.initialise_chunk)(&chunk, &xmin, &ymin,
                                                                                         &zmin, &dx, &dy, &dz);
        // generate_chunk.f90:34-85.
        int ns = (int)cfg.states.size();
        std::vector<double> den(ns), en(ns), x0(ns), x1(ns), y0(ns), y1(ns), z0(ns), z1(ns), rad(ns);
        std::vector<int> geo(ns);
        for (int s = 0; s < ns; ++s) {
            const State& st = cfg.states[s];
            den[s] = st.density; en[s] = st.energy;
            x0[s] = st.xmin; x1[s] = st.xmax; y0[s] = st.ymin; y1[s] = st.ymax;
            z0[s] = st.zmin; z1[s] = st.zmax; rad[s] = st.radius; geo[s] = st.geometry;
        }
        int rect = G_RECT, circ = G_CIRC, point = G_POINT;
        if (cfg.dim == 2)
            reinterpret_cast<void (*)(const int*, const int*, const double*, const double*, const double*,
                                      const double*, const double*, const double*, const double*, const int*,
                                      const int*, const int*, const int*)>(be.generate_chunk)(
                &chunk, &ns, den.data(), en.data(), x0.data(), x1.data(), y0.data(), y1.data(), rad.data(),
                geo.data(), &rect, &circ, &point);
        else
            reinterpret_cast<void (*)(const int*, const int*, const double*, const double*, const double*,
                                      const double*, const double*, const double*, const double*, const double*,
                                      const double*, const int*, const int*, const int*, const int*)>(
                be.generate_chunk)(&chunk, &ns, den.data(), en.data(), x0.data(), x1.data(), y0.data(),
                                   y1.data(), z0.data(), z1.data(), rad.data(), geo.data(), &rect, &circ, &point);
        be.check_status("ext_generate_chunk_");
        halo({FIELD_DENSITY, FIELD_ENERGY0, FIELD_ENERGY1}, 2);
        field_summary(sum, false, nullptr);
        if (opt->ws_net && opt->ws_mode == 2) {
            if (!be.ws_attach || be.ws_attach(&chunk, &opt->ws_net) != 0) fail("warm start: cannot attach network");
        }
    }

    // tea_leaf(), tealeaf_2d/tea_solve.f90:36-605, one implicit solve per timestep.
    void tea_leaf(tea_step_record* rec)
    {
        const int max_iters = cfg.max_iters;
        const bool cg_like = cfg.solver == TEA_SOLVER_CG || cfg.solver == TEA_SOLVER_CHEBYSHEV ||
                             cfg.solver == TEA_SOLVER_PPCG;
        const bool use_cheby = cfg.solver == TEA_SOLVER_CHEBYSHEV;
        const bool use_ppcg = cfg.solver == TEA_SOLVER_PPCG;
        int precond = cfg.tl_preconditioner_on ? 1 : 0;
        int coefficient = cfg.coefficient;
        double eps = cfg.eps;

        if (coefficient != RECIP_CONDUCTIVITY && coefficient != CONDUCTIVITY)
            fail("tea_leaf: unknown coefficient option");

        if (cfg.use_fused_solve && be.whole_solve) {
            tea_solve_params p;
            std::memset(&p, 0, sizeof(p));
            p.solver = cfg.solver;
            p.coefficient = coefficient;
            p.preconditioner = precond;
            p.max_iters = max_iters;
            p.ch_cg_presteps = cfg.tl_ch_cg_presteps;
            p.ch_cg_errswitch = cfg.tl_ch_cg_errswitch;
            p.ppcg_inner_steps = cfg.tl_ppcg_inner_steps;
            p.check_result = cfg.tl_check_result;
            p.dt = dt;
            p.eps = eps;
            p.ch_cg_epslim = cfg.tl_ch_cg_epslim;
            p.eps_rel = cfg.tl_eps_rel;
            p.precision = cfg.precision;
            p.inner_max_iters = cfg.inner_max_iters;
            p.inner_tol = cfg.inner_tol;
            p.inner_solver = cfg.inner_solver;
            tea_solve_result r;
            std::memset(&r, 0, sizeof(r));
            be.whole_solve(&chunk, &p, &r);
            be.check_status("ext_tea_leaf_solve_");
            if (r.switch_step > 0) {
                log.line("Switching after %3d steps, error %15.7E", r.switch_step, 0.0);
                log.line("     eigmin     eigmax         cn      error");
                log.line("%11.5f%11.5f%11.4E", r.eigmin, r.eigmax, r.eigmax / r.eigmin);
            }
            log.line("Conduction error %14.7E", r.error);
            if (cfg.tl_check_result) log.line("EXACT error calculated as%14.7E", r.exact_error);
            log.line("Iteration count %8d", r.iterations);
            rec->iterations = r.iterations;
            rec->error = r.error;
            rec->exact_error = r.exact_error;
            rec->eps_used = r.eps_used;
            rec->status = r.status;
            rec->cheby_steps = r.cheby_steps;
            rec->switch_step = r.switch_step;
            rec->est_itc = r.est_itc;
            rec->corrections = r.corrections;
            rec->inner_solver = r.inner_solver;
            rec->warm_start_used = r.warm_start_used;
            rec->warm_r0_plain = r.warm_r0_plain;
            rec->warm_r0_guess = r.warm_r0_guess;
            if (opt->ws_net && opt->ws_mode == 1) {
                if (!be.ws_record || be.ws_record(&opt->ws_net, &chunk) != 0) fail("warm start: cannot record pair");
            }
            return;
        }

        double error = 1e10, exact_error = 0.0;
        double rro = 0.0, pw = 0.0, rrn = 0.0, alpha = 0.0, beta = 0.0;
        double eigmin = 0.0, eigmax = 0.0, theta = 0.0, cn = 0.0;
        std::vector<double> cg_alphas(max_iters + 2, 0.0), cg_betas(max_iters + 2, 0.0);
        std::vector<double> ch_alphas(max_iters + 2, 0.0), ch_betas(max_iters + 2, 0.0);
        int est_itc = 0, cheby_calc_steps = 0, max_cheby_iters = 0, switch_step = 0;
        int fields[NUM_FIELDS] = {0, 0, 0, 0, 0, 0};

        // INIT (:79-164)
        halo({FIELD_ENERGY1, FIELD_DENSITY}, 2);
        if (cg_like) {
            be.cg_init(&chunk, &coefficient, &precond, &dt, &rro);
            allsum(&rro, 1);
            std::fill(fields, fields + NUM_FIELDS, 0);
            fields[FIELD_U - 1] = 1;
            fields[FIELD_P - 1] = 1;
            update_halo(fields, 1);
        } else {
            be.jacobi_init(&chunk, &coefficient, &dt);
            std::fill(fields, fields + NUM_FIELDS, 0);
            fields[FIELD_U - 1] = 1;
        }
        be.copy_u(&chunk);
        if (cfg.tl_eps_rel > 0.0) {
            // Additive relative target: sum r^2 < tl_eps_rel^2 * sum u0^2.
            double bb = 0.0;
            int zero = 0;
            be.calc_2norm(&chunk, &bb, &zero); allsum(&bb, 1);
            eps = cfg.tl_eps_rel * cfg.tl_eps_rel * bb;
        }
        be.check_status("solver init");

        int n;
        for (n = 1; n <= max_iters; ++n) {
            bool ch_switch_check;
            if (cfg.tl_ch_cg_errswitch)
                ch_switch_check = (cheby_calc_steps > 0) || ((error <= cfg.tl_ch_cg_epslim) && (n >= 20));
            else
                ch_switch_check = (n >= cfg.tl_ch_cg_presteps) && (error <= 1.0);

            if ((use_cheby || use_ppcg) && ch_switch_check) {
                if (cheby_calc_steps == 0) {
                    max_cheby_iters = max_iters - n + 2;
                    rro = error;
                    int info = tea::tea_calc_eigenvalues(cg_alphas.data() + 1, cg_betas.data() + 1, n - 1,
                                                         &eigmin, &eigmax);
                    if (info != 0) fail("tea_leaf: Error in calculating eigenvalues");
                    eigmin = eigmin * tea::kEigMinScale;
                    eigmax = eigmax * tea::kEigMaxScale;
                    if ((int)ch_alphas.size() < max_cheby_iters + 1) {
                        ch_alphas.resize(max_cheby_iters + 1, 0.0);
                        ch_betas.resize(max_cheby_iters + 1, 0.0);
                    }
                    if (use_cheby) {
                        tea::tea_calc_ch_coefs(ch_alphas.data(), ch_betas.data(), eigmin, eigmax, &theta,
                                               max_cheby_iters);
                        std::fill(fields, fields + NUM_FIELDS, 0);
                        fields[FIELD_U - 1] = 1;
                    } else {
                        tea::tea_calc_ch_coefs(ch_alphas.data(), ch_betas.data(), eigmin, eigmax, &theta,
                                               cfg.tl_ppcg_inner_steps);
                    }
                    cn = eigmax / eigmin;
                    log.line("Switching after %3d steps, error %15.7E", n, rro);
                    log.line("     eigmin     eigmax         cn      error");
                    log.line("%11.5f%11.5f%11.4E%11.4E", eigmin, eigmax, cn, error);
                }
                if (use_cheby) {
                    if (cheby_calc_steps == 0) {
                        // tea_leaf_cheby_first_step, :658-750.
                        double bb = 0.0;
                        int zero = 0, one = 1;
                        be.calc_2norm(&chunk, &bb, &zero); allsum(&bb, 1);
                        be.cheby_init(&chunk, ch_alphas.data(), ch_betas.data(), &theta, &precond,
                                      &max_cheby_iters);
                        update_halo(fields, 1);
                        be.cheby_iterate(&chunk, &max_cheby_iters);
                        be.calc_2norm(&chunk, &error, &one); allsum(&error, 1);
                        est_itc = tea::tea_cheby_est_itc(bb, error, cn);
                        log.line("    est itc");
                        log.line("%11d", est_itc);
                        cheby_calc_steps = 1;
                        switch_step = n;
                    } else {
                        be.cheby_iterate(&chunk, &cheby_calc_steps);
                        if ((n >= est_itc) && (n % 10 == 0)) {
                            int one = 1;
                            be.calc_2norm(&chunk, &error, &one); allsum(&error, 1);
                        }
                    }
                } else {
                    if (cheby_calc_steps == 0) {
                        cheby_calc_steps = 1;
                        switch_step = n;
                        be.ppcg_init(&chunk, ch_alphas.data(), ch_betas.data(), &theta, &max_cheby_iters);
                        be.calc_residual(&chunk);
                        update_halo(fields, 1);
                    }
                    be.cg_calc_w(&chunk, &pw); allsum(&pw, 1);
                    alpha = rro / pw;
                    be.cg_calc_ur(&chunk, &alpha, &rrn); allsum(&rrn, 1);
                    // tea_leaf_run_ppcg_inner_steps, :607-656.
                    be.ppcg_init_sd(&chunk);
                    int sd_fields[NUM_FIELDS] = {0, 0, 0, 0, 0, 1};
                    for (int k = 1; k <= cfg.tl_ppcg_inner_steps; ++k) {
                        update_halo(sd_fields, 1);
                        be.ppcg_inner(&chunk, &k);
                    }
                    int one = 1;
                    be.calc_2norm(&chunk, &rrn, &one); allsum(&rrn, 1);
                    beta = rrn / rro;
                    be.cg_calc_p(&chunk, &beta);
                    error = rrn;
                    rro = rrn;
                }
                cheby_calc_steps = cheby_calc_steps + 1;
            } else if (cg_like) {
                fields[FIELD_P - 1] = 1;
                be.cg_calc_w(&chunk, &pw); allsum(&pw, 1);
                alpha = rro / pw;
                if (use_cheby || use_ppcg) cg_alphas[n] = alpha;
                be.cg_calc_ur(&chunk, &alpha, &rrn); allsum(&rrn, 1);
                beta = rrn / rro;
                if (use_cheby || use_ppcg) cg_betas[n] = beta;
                be.cg_calc_p(&chunk, &beta);
                error = rrn;
                rro = rrn;
            } else {
                be.jacobi_solve(&chunk, &error); allsum(&error, 1);
                if (n % 50 == 0) {
                    update_halo(fields, 1);
                    int one = 1;
                    be.calc_residual(&chunk);
                    be.calc_2norm(&chunk, &error, &one); allsum(&error, 1);
                }
            }
            update_halo(fields, 1);
            if (std::fabs(error) < eps) break;
        }
        if (n > max_iters) n = max_iters + 1;
        if (cfg.tl_check_result) {
            int one = 1;
            be.calc_residual(&chunk);
            be.calc_2norm(&chunk, &exact_error, &one); allsum(&exact_error, 1);
        }
        be.check_status("solve");
        log.line("Conduction error %14.7E", error);
        if (cfg.tl_check_result) log.line("EXACT error calculated as%14.7E", exact_error);
        log.line("Iteration count %8d", n - 1);
        be.finalise_solve(&chunk);
        halo({FIELD_ENERGY1}, 1);
        rec->iterations = n - 1;
        rec->error = error;
        rec->exact_error = exact_error;
        rec->eps_used = eps;
        rec->status = TEA_OK;
        rec->cheby_steps = cheby_calc_steps > 0 ? cheby_calc_steps - 1 : 0;
        rec->switch_step = switch_step;
        rec->est_itc = est_itc;
    }

    // visit(), tealeaf_2d/visit.f90:23-112 and tealeaf_3d/visit.f90: graphics output into
    // the working directory.  Rank 0 keeps the index tea.visit ("!NBLOCKS n" once, then
    // one line per rank's file at each call) and every rank writes its chunk as the
    // legacy-VTK rectilinear grid tea.<rank+1>.<step>.vtk (five-digit fields), with the
    // reference's header lines and Fortran E12.4 numbers.  The reference's files stop
    // after declaring two field arrays without values (and print an unset z extent in
    // 2D); these carry the cells' density, energy and temperature (u) as CELL_DATA, read
    // from the backend, and a 2D grid is one cell deep in z, so VTK readers accept them.
    // The index lists every rank's file, where the reference lists rank 0's chunks only.
    void visit()
    {
        if (!be.chunk_dims || !be.read_field) fail("visit output needs tea_chunk_dims_ and tea_read_field_");
        const int nranks = split() ? comm->size : 1, rank = split() ? comm->rank : 0;
        const int tag = step % 100000;  // the five digits of WRITE(i6) step+100000
        if (rank == 0) {
            FILE* f = std::fopen("tea.visit", visit_started ? "a" : "w");
            if (!f) fail("cannot write tea.visit");
            if (!visit_started) std::fprintf(f, "!NBLOCKS %5d\n", nranks);
            for (int r = 0; r < nranks; ++r) std::fprintf(f, "tea.%05d.%05d.vtk\n", (r + 1) % 100000, tag);
            std::fclose(f);
        }
        visit_started = true;
        int dims[3] = {0, 0, 0};
        if (be.chunk_dims(&chunk, dims) != 0) fail("visit: tea_chunk_dims_ failed");
        const size_t padded = (size_t)dims[0] * dims[1] * dims[2];
        const int nz = cfg.dim == 3 ? lz : 1;
        const long ncells = (long)lx * ly * nz;
        char name[64];
        std::snprintf(name, sizeof(name), "tea.%05d.%05d.vtk", (rank + 1) % 100000, tag);
        FILE* f = std::fopen(name, "w");
        if (!f) fail("cannot write %s", name);
        char num[32];
        auto put = [&](double v) {
            fortran_e12_4(num, v);
            std::fputs(num, f);
            std::fputc('\n', f);
        };
        std::fprintf(f, "# vtk DataFile Version 3.0\nvtk output\nASCII\nDATASET RECTILINEAR_GRID\n");
        std::fprintf(f, "DIMENSIONS%12d%12d%12d\n", lx + 1, ly + 1, cfg.dim == 3 ? lz + 1 : 1);
        std::fprintf(f, "X_COORDINATES %5d double\n", lx + 1);
        for (int k = 0; k <= lx; ++k) put(cx0 + cdx * (double)k);
        std::fprintf(f, "Y_COORDINATES %5d double\n", ly + 1);
        for (int k = 0; k <= ly; ++k) put(cy0 + cdy * (double)k);
        if (cfg.dim == 3) {
            std::fprintf(f, "Z_COORDINATES %5d double\n", lz + 1);
            for (int k = 0; k <= lz; ++k) put(cz0 + cdz * (double)k);
        } else {
            std::fprintf(f, "Z_COORDINATES %5d double\n", 1);
            put(0.0);
        }
        std::fprintf(f, "CELL_DATA %ld\nFIELD FieldData 3\n", ncells);
        std::vector<double> buf(padded);
        const int kPad = 2;  // the flat arrays hold two halo cells before the inner ones
        const struct { const char* name; int id; } out[3] = {
            {"density", FIELD_DENSITY}, {"energy", FIELD_ENERGY1}, {"temperature", FIELD_U}};
        for (const auto& o : out) {
            if (be.read_field(&chunk, &o.id, buf.data()) != 0) fail("visit: tea_read_field_(%d) failed", o.id);
            std::fprintf(f, "%s 1 %ld double\n", o.name, ncells);
            for (int ii = 0; ii < nz; ++ii)
                for (int jj = 0; jj < ly; ++jj)
                    for (int kk = 0; kk < lx; ++kk) {
                        const size_t zi = cfg.dim == 3 ? (size_t)(ii + kPad) : 0;
                        put(buf[(size_t)(kk + kPad) + (size_t)dims[0] * ((size_t)(jj + kPad) + (size_t)dims[1] * zi)]);
                    }
        }
        if (std::fclose(f) != 0) fail("cannot write %s", name);
        be.check_status("visit");
    }

    int run(tea_run_summary* sum, tea_step_record* steps, int max_steps)
    {
        start(sum);
        if (opt->end_step_override > 0) cfg.end_step = opt->end_step_override;
        // diffuse, tealeaf_2d/diffuse.f90:23-160.
        const double t0 = now_seconds();
        double solve_total = 0.0;
        long iters_total = 0;
        be.set_field(&chunk);
        for (;;) {
            step = step + 1;
            // timestep()/calc_dt(): dt = min(dt, dtinit) (tealeaf_2d/timestep.f90:44-52).
            double dtlp = cfg.dtinit;
            if (dtlp <= dt) dt = dtlp;
            log.line(" Step %7d time %11.7f timestep  %9.2E", step, time, dt);
            tea_step_record rec;
            std::memset(&rec, 0, sizeof(rec));
            const double s0 = now_seconds();
            tea_leaf(&rec);
            const double s1 = now_seconds();
            solve_total += s1 - s0;
            iters_total += rec.iterations;
            time = time + dt;
            rec.step = step;
            rec.time = time;
            rec.dt = dt;
            rec.solve_seconds = s1 - s0;
            bool summarised = false;
            if (cfg.summary_frequency != 0 && step % cfg.summary_frequency == 0) {
                double v[4];
                field_summary(sum, false, v);
                rec.vol = v[0]; rec.mass = v[1]; rec.ie = v[2]; rec.temp = v[3];
                rec.has_summary = 1;
                summarised = true;
            }
            if (cfg.visit_frequency != 0 && step % cfg.visit_frequency == 0) visit();
            const double wall = now_seconds() - t0;
            log.line(" Wall clock %.15g", wall);
            const double cells = (double)cfg.x_cells * cfg.y_cells * (cfg.dim == 3 ? cfg.z_cells : 1);
            log.line(" Average time per cell %.15g", wall / (step * cells));
            bool last = (time + G_SMALL > cfg.end_time) || (step >= cfg.end_step);
            if (last) {
                complete = true;
                double v[4];
                field_summary(sum, true, v);
                rec.vol = v[0]; rec.mass = v[1]; rec.ie = v[2]; rec.temp = v[3];
                rec.has_summary = 1;
                summarised = true;
                if (cfg.visit_frequency != 0) visit();
            } else if (opt->summary_every_step && !summarised) {
                double v[4];
                be.field_summary(&chunk, &v[0], &v[1], &v[2], &v[3]);
                rec.vol = v[0]; rec.mass = v[1]; rec.ie = v[2]; rec.temp = v[3];
                rec.has_summary = 1;
            }
            rec.wall_end = now_seconds() - t0;
            if (be.transfer_bytes) be.transfer_bytes(&chunk, &rec.h2d_bytes, &rec.d2h_bytes);
            if (steps && step - 1 < max_steps) steps[step - 1] = rec;
            if (last) break;
        }
        sum->steps = step;
        sum->wall_seconds = now_seconds() - t0;
        sum->solve_seconds = solve_total;
        sum->total_iterations = iters_total;
        sum->x_cells = cfg.x_cells;
        sum->y_cells = cfg.y_cells;
        sum->z_cells = cfg.dim == 3 ? cfg.z_cells : 1;
        sum->solver = cfg.solver;
        log.line("");
        log.line(" Calculation complete");
        log.line(" Tea is finishing");
        if (!opt->keep_chunk) be.finalise();
        return 0;
    }
};

}  // namespace

extern "C" int tea_run_deck(const char* deck_text, const tea_run_options* options, tea_run_summary* summary,
                            tea_step_record* steps, int max_steps)
{
    return tea_run_deck_comm(deck_text, options, nullptr, summary, steps, max_steps);
}

extern "C" int tea_run_deck_comm(const char* deck_text, const tea_run_options* options, const tea_comm* comm,
                                 tea_run_summary* summary, tea_step_record* steps, int max_steps)
{
    g_last_error.clear();
    tea_run_summary local;
    if (!summary) summary = &local;
    std::memset(summary, 0, sizeof(*summary));
    Runner r;
    try {
        if (!options || !options->backend) fail("no backend given");
        if (options->dim != 2 && options->dim != 3) fail("dim must be 2 or 3");
        r.opt = options;
        r.comm = comm;
        if (comm && (comm->size < 1 || comm->rank < 0 || comm->rank >= comm->size ||
                     (comm->size > 1 && (!comm->allreduce_sum || !comm->sendrecv))))
            fail("invalid communicator");
        r.cfg = parse_deck(deck_text ? deck_text : "", options->dim);
        if (options->use_fused_solve) r.cfg.use_fused_solve = true;
        if (options->precision > 0) r.cfg.precision = options->precision;
        if (r.cfg.precision != TEA_PRECISION_FP64 && !r.cfg.use_fused_solve)
            fail("tl_precision fp32 needs the whole-solve path (use_fused_solve)");
        if (r.split() && r.cfg.use_fused_solve)
            fail("the whole-solve path runs one chunk: several ranks use the per-call path");
        if (options->eps_override > 0.0) r.cfg.eps = options->eps_override;
        if (options->eps_rel_override > 0.0) r.cfg.tl_eps_rel = options->eps_rel_override;
        r.log.echo = !options->quiet && !(comm && comm->rank != 0);
        if (options->out_path && !(comm && comm->rank != 0)) {
            r.log.file = fopen(options->out_path, "w");
            if (!r.log.file) fail("cannot open %s", options->out_path);
        }
        r.be.open(options->backend, options->dim);
        if (r.cfg.use_fused_solve && !r.be.whole_solve) fail("backend has no ext_tea_leaf_solve_");
        int rc = r.run(summary, steps, max_steps);
        if (r.log.file) fclose(r.log.file);
        return rc;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        if (r.log.file) fclose(r.log.file);
        return 1;
    }
}

extern "C" const char* tea_driver_last_error(void) { return g_last_error.c_str(); }

// The switch-time scalar algorithms, exported for host-side tests.
extern "C" int tea_calc_eigenvalues_c(const double* cg_alphas, const double* cg_betas, int n, double* eigmin,
                                      double* eigmax)
{
    return tea::tea_calc_eigenvalues(cg_alphas, cg_betas, n, eigmin, eigmax);
}

extern "C" int tea_tridiag_extremes_c(const double* cg_alphas, const double* cg_betas, int n, double* eigmin,
                                      double* eigmax)
{
    return tea::tea_tridiag_extremes(cg_alphas, cg_betas, n, eigmin, eigmax);
}

extern "C" void tea_calc_ch_coefs_c(double* ch_alphas, double* ch_betas, double eigmin, double eigmax,
                                    double* theta, int n)
{
    tea::tea_calc_ch_coefs(ch_alphas, ch_betas, eigmin, eigmax, theta, n);
}

extern "C" int tea_cheby_est_itc_c(double bb, double error, double cn) { return tea::tea_cheby_est_itc(bb, error, cn); }
