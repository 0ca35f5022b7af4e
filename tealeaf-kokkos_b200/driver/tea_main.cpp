// tea_leaf executable: the command-line entry of the reference (tealeaf_2d/tea_leaf.f90:35-104)
// restated over the C++ driver.  Usage:
//   tea_leaf [--dim 2|3] [--backend LIB] [--fused] [--out FILE | --no-out] [--quiet]
//            [--summary-every-step] [--end-step N] [--json FILE] [deck [output]]
// As in the reference (tea_leaf.f90:68-85), the deck defaults to ./tea.in and the output
// log to ./tea.out; a missing deck is replaced by the reference's default one.  --json
// writes the run summary and per-step records.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "tea_driver.h"

#include <cmath>

// JSON number for a double: NaN/Inf are written as Python's json module reads them.
static std::string num(double v)
{
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "Infinity" : "-Infinity";
    char b[40];
    std::snprintf(b, sizeof(b), "%.17g", v);
    return b;
}

// initialise.f90:69-97 (tealeaf_2d, tealeaf_3d): when the input deck cannot be opened, the
// reference writes this default one in its place and runs it -- a 10 x 10 (x 2 in 3D)
// mesh with five states, Jacobi, test_problem 1.  The lines are the reference's, the 3D
// deck's "rectangle" included (the 3D parser knows only "cuboid", so those states keep
// no geometry there, and here).
static void write_default_deck(const std::string& path, int dim)
{
    std::vector<std::string> lines = {
        "*tea",
        " state 1 density=100.0 energy=0.0001",
        " state 2 density=0.1 energy=25.0 geometry=rectangle xmin=0.0 xmax=1.0 ymin=1.0 ymax=2.0",
        " state 3 density=0.1 energy=0.1 geometry=rectangle xmin=1.0 xmax=6.0 ymin=1.0 ymax=2.0",
        " state 4 density=0.1 energy=0.1 geometry=rectangle xmin=5.0 xmax=6.0 ymin=1.0 ymax=8.0",
        " state 5 density=0.1 energy=0.1 geometry=rectangle xmin=5.0 xmax=10.0 ymin=7.0 ymax=8.0",
        " x_cells=10",
        " y_cells=10"};
    if (dim == 3) lines.push_back(" z_cells=2");
    lines.push_back(" xmin=0.0");
    lines.push_back(" ymin=0.0");
    if (dim == 3) lines.push_back(" zmin=0.0");
    lines.push_back(" xmax=10.0");
    lines.push_back(" ymax=10.0");
    if (dim == 3) lines.push_back(" zmax=10.0");
    for (const char* l : {" initial_timestep=0.004", " end_step=10", " tl_max_iters=1000", " test_problem 1",
                          " tl_use_jacobi", " tl_eps=1.0e-15", "*endtea"})
        lines.push_back(l);
    std::ofstream out(path);
    for (const auto& l : lines) out << l << "\n";
}

int main(int argc, char** argv)
{
    tea_run_options opt;
    std::memset(&opt, 0, sizeof(opt));
    opt.dim = 2;
    std::string deck_path = "tea.in", backend, out_path = "tea.out", json_path;
    int positional = 0;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto need = [&](const char* what) -> std::string {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "missing value for %s\n", what);
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--dim") opt.dim = std::atoi(need("--dim").c_str());
        else if (a == "--backend") backend = need("--backend");
        else if (a == "--fused") opt.use_fused_solve = 1;
        else if (a == "--out") out_path = need("--out");
        else if (a == "--no-out") out_path.clear();
        else if (a == "--quiet") opt.quiet = 1;
        else if (a == "--summary-every-step") opt.summary_every_step = 1;
        else if (a == "--end-step") opt.end_step_override = std::atoi(need("--end-step").c_str());
        else if (a == "--json") json_path = need("--json");
        else if (positional++ == 0) deck_path = a;
        else out_path = a;
    }
    if (backend.empty()) {
        std::fprintf(stderr, "--backend LIB is required (libtea2d_b200.so / libtea3d_b200.so)\n");
        return 2;
    }
    if (!std::ifstream(deck_path)) write_default_deck(deck_path, opt.dim);
    std::ifstream in(deck_path);
    if (!in) {
        std::fprintf(stderr, "cannot read %s\n", deck_path.c_str());
        return 2;
    }
    std::stringstream ss;
    ss << in.rdbuf();
    opt.backend = backend.c_str();
    opt.out_path = out_path.empty() ? nullptr : out_path.c_str();
    const int max_steps = 100000;
    std::vector<tea_step_record> steps(max_steps);
    tea_run_summary sum;
    int rc = tea_run_deck(ss.str().c_str(), &opt, &sum, steps.data(), max_steps);
    if (rc != 0) {
        std::fprintf(stderr, "tea_leaf: %s\n", tea_driver_last_error());
        return 1;
    }
    if (!json_path.empty()) {
        FILE* f = std::fopen(json_path.c_str(), "w");
        if (!f) return 1;
        std::fprintf(f, "{\"steps\": %d, \"test_problem\": %d, \"kat_available\": %d, \"kat_passed\": %d, "
                        "\"qa_diff\": %s, \"vol\": %s, \"mass\": %s, \"ie\": %s, \"temp\": %s, "
                        "\"wall_seconds\": %.9g, \"solve_seconds\": %.9g, \"total_iterations\": %ld, \"records\": [",
                     sum.steps, sum.test_problem, sum.kat_available, sum.kat_passed, num(sum.qa_diff).c_str(),
                     num(sum.vol).c_str(), num(sum.mass).c_str(), num(sum.ie).c_str(), num(sum.temp).c_str(),
                     sum.wall_seconds, sum.solve_seconds, sum.total_iterations);
        int n = sum.steps < max_steps ? sum.steps : max_steps;
        for (int s = 0; s < n; ++s) {
            const tea_step_record& r = steps[s];
            std::fprintf(f, "%s{\"step\": %d, \"iterations\": %d, \"error\": %s, \"exact_error\": %s, "
                            "\"eps_used\": %s, \"solve_seconds\": %.9g, \"has_summary\": %d, \"vol\": %s, "
                            "\"mass\": %s, \"ie\": %s, \"temp\": %s, \"switch_step\": %d, \"est_itc\": %d, "
                            "\"cheby_steps\": %d}",
                         s ? ", " : "", r.step, r.iterations, num(r.error).c_str(), num(r.exact_error).c_str(),
                         num(r.eps_used).c_str(), r.solve_seconds, r.has_summary, num(r.vol).c_str(),
                         num(r.mass).c_str(), num(r.ie).c_str(), num(r.temp).c_str(), r.switch_step, r.est_itc,
                         r.cheby_steps);
        }
        std::fprintf(f, "]}\n");
        std::fclose(f);
    }
    return 0;
}
