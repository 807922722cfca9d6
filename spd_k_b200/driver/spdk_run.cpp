// spdk_run: the athinput-driven driver (the reference's src/main.cpp) on
// top of the C ABI of libspdk_cuda.so.
//
//   spdk_run [-i deck.athinput] [block/name=value ...]
//
// Reads the same parameters with the same defaults (src/main.cpp:126-189),
// builds the hydro solver (job/system = hydro) or the induction solver
// (job/system = induction), runs time_evolution to time/tlim with the
// reference's output clamping, and writes, when output/dt > 0, the
// reference's output files into $SPD_OUTPUT_DIR (default ./output):
//   hydro:     W_cv_N<N>p<p>_<n>_0.dat in the reference's
//              (1, 6, Nz, Ny, Nx, nz, ny, nx) layout with ghost elements;
//              the driver fills the ghost elements with NaN (the reference
//              leaves 0/0 there) and the bookkeeping slot 5 with 0
//   induction: B2_cv_N<N>p<p>_<n>_0.dat (+ troubles) exactly as the
//              reference writes them
//   X/Y/Z_N<N>p<p>_0.dat: FV face coordinates of each direction.
// It prints the reference's "evolution:" line (steps, seconds, ms/step,
// zone-cycles/s) with the evolution timed without output I/O.
// Additions for hydro runs (no reference counterpart): output/checkpoint_dt
// > 0 writes checkpoint_<step>.spdk (spdk_hydro_checkpoint_async) into the
// output directory every checkpoint_dt of simulated time, and
// job/restart=<file> resumes a run from one; the resumed run's states and
// output files equal the uninterrupted run's. For induction runs,
// fallback/apply=true applies the upwind-EMF fallback where the corrector
// detects troubles (the reference only detects).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "spdk.h"
#include "spdk_induction.h"

namespace {

// <block> name = value (last assignment wins), '#' comments
// (src/parameter_input.cpp:24-73)
struct Params {
    std::map<std::string, std::map<std::string, std::string>> v;
    static std::string trim(const std::string& s) {
        const size_t a = s.find_first_not_of(" \t\r\n");
        if (a == std::string::npos) return "";
        return s.substr(a, s.find_last_not_of(" \t\r\n") - a + 1);
    }
    void load(const std::string& path) {
        std::ifstream f(path);
        if (!f) throw std::runtime_error("cannot open input file '" + path + "'");
        std::string line, block;
        while (std::getline(f, line)) {
            line = trim(line.substr(0, line.find('#')));
            if (line.empty()) continue;
            if (line[0] == '<') {
                block = trim(line.substr(1, line.find('>') - 1));
                continue;
            }
            const size_t eq = line.find('=');
            if (eq == std::string::npos) throw std::runtime_error("malformed line: " + line);
            v[block][trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
        }
    }
    void override_(const std::string& o) {
        const size_t s = o.find('/'), e = o.find('=');
        v[trim(o.substr(0, s))][trim(o.substr(s + 1, e - s - 1))] = trim(o.substr(e + 1));
    }
    bool has(const std::string& b, const std::string& n) const {
        auto it = v.find(b);
        return it != v.end() && it->second.count(n);
    }
    std::string str(const std::string& b, const std::string& n, const std::string& d) const {
        return has(b, n) ? v.at(b).at(n) : d;
    }
    double real(const std::string& b, const std::string& n, double d) const {
        return has(b, n) ? std::stod(v.at(b).at(n)) : d;
    }
    int integer(const std::string& b, const std::string& n, int d) const {
        return has(b, n) ? std::stoi(v.at(b).at(n)) : d;
    }
    bool boolean(const std::string& b, const std::string& n, bool d) const {
        if (!has(b, n)) return d;
        const std::string s = v.at(b).at(n);
        if (s == "true" || s == "yes" || s == "on" || s == "1") return true;
        if (s == "false" || s == "no" || s == "off" || s == "0") return false;
        throw std::runtime_error("not a boolean: " + s);
    }
};

struct Problem {
    const char* name;
    int id;
    double pp[10];  // amp, v1, v2, v3, d0, d1, p0, p1, radius, sigma
};
// src/main.cpp:31-65 (ids 10-12: the project's extra problems)
const Problem kProblems[] = {
    {"sine_wave", SPDK_IC_SINE_WAVE, {0.125, 1.0, 1.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 0.0}},
    {"sedov", SPDK_IC_SEDOV, {0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.1, 0.0}},
    {"spherical_blast", SPDK_IC_SPHERICAL_BLAST, {0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 10.0, 0.1, 0.1, 0.0}},
    {"square", SPDK_IC_SQUARE, {0.0, 1.0, 1.0, 0.0, 1.0, 2.0, 1.0, 0.0, 0.25, 0.0}},
    {"sod_shock_tube", SPDK_IC_SOD, {0.0, 0.0, 0.0, 0.0, 1.0, 0.125, 1.0, 0.1, 0.5, 0.0}},
    {"shu_osher", SPDK_IC_SHU_OSHER, {0.2, 0.0, 0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 0.0}},
    {"kelvin_helmholtz", SPDK_IC_KELVIN_HELMHOLTZ, {0.1, 0.5, 0.0, 0.0, 1.0, 2.0, 2.5, 0.0, 0.0, 0.05 / std::sqrt(2.0)}},
    {"implosion", SPDK_IC_IMPLOSION, {0.0, 0.0, 0.0, 0.0, 1.0, 0.125, 1.0, 0.14, 0.15, 0.0}},
    {"rti", SPDK_IC_RTI, {0.025, 0.0, 0.0, 0.0, 2.0, 1.0, 1.0, 0.0, 0.5, 0.0}},
    {"user", SPDK_IC_USER, {0.5, 1.0, 0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.5, 0.1}},
    {"kh_noise", SPDK_IC_KH_NOISE, {0.01, 0.5, 0.0, 0.0, 1.0, 2.0, 2.5, 0.0, 0.25, 0.0}},
    {"quadrant", SPDK_IC_QUADRANT, {0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0, 0.0, 0.0}},
    {"rti_top", SPDK_IC_RTI_TOP, {0.01, 0.0, 0.0, 0.0, 2.0, 1.0, 2.5, 0.0, 0.75, 0.0}},
};

int bc_id(const std::string& s) {
    if (s == "periodic") return SPDK_BC_PERIODIC;
    if (s == "gradfree") return SPDK_BC_GRADFREE;
    if (s == "reflective") return SPDK_BC_REFLECTIVE;
    throw std::runtime_error("unknown boundary '" + s + "'");
}

void integrator(const std::string& s, int* kind, int* order) {
    if (s == "ader") { *kind = SPDK_INTEGRATOR_ADER; *order = 3; return; }
    if (s.size() == 3 && s.compare(0, 2, "rk") == 0 && s[2] >= '1' && s[2] <= '3') {
        *kind = SPDK_INTEGRATOR_RK;
        *order = s[2] - '0';
        return;
    }
    throw std::runtime_error("unknown integrator '" + s + "' (ader, rk1, rk2, rk3)");
}

void check(int rc) {
    if (rc != 0) throw std::runtime_error(std::string("spdk error ") + std::to_string(rc) + ": " + spdk_last_error());
}

std::string out_dir() {
    const char* e = std::getenv("SPD_OUTPUT_DIR");
    std::string d = e ? e : "output";
    mkdir(d.c_str(), 0755);
    return d + "/";
}

void write_file(const std::string& path, const double* a, size_t n) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(a), (std::streamsize)(n * sizeof(double)));
}

// FV face coordinates of one direction (src/structs.hpp:40-75)
std::vector<double> fv_faces(int N, int p, double L, bool active) {
    std::vector<double> f(active ? (size_t)N * (p + 1) + 5 : 1);
    check(spdk_fv_faces(N, p, L, active, f.data(), f.size()));
    return f;
}

int run_hydro(const Params& P, int p, const int N[3], const double L[3], double tlim, bool outputs, double dt_out) {
    spdk_hydro_config c{};
    c.p = p;
    for (int d = 0; d < 3; d++) {
        c.N[d] = N[d];
        c.L[d] = L[d];
    }
    c.bc[0] = bc_id(P.str("mesh", "x1_bc", "periodic"));
    c.bc[1] = bc_id(P.str("mesh", "x2_bc", "periodic"));
    c.bc[2] = bc_id(P.str("mesh", "x3_bc", "periodic"));
    integrator(P.str("time", "integrator", "ader"), &c.integrator, &c.rk_order);
    c.fallback = P.boolean("job", "fallback", true);
    c.gamma = P.real("hydro", "gamma", 1.4);
    c.cfl = P.real("time", "cfl", 0.8);
    c.g[0] = P.real("hydro", "g1", 0.0);
    c.g[1] = P.real("hydro", "g2", 0.0);
    c.g[2] = P.real("hydro", "g3", 0.0);
    c.nad_tolerance = P.real("fallback", "tolerance", 1e-5);
    c.nad_delta = P.str("fallback", "NAD", "relative") == "delta";
    c.nad_moore = P.str("fallback", "NAD_neighbors", "2nd") == "2nd";
    c.sed = P.boolean("fallback", "SED", true);
    c.blending = P.boolean("fallback", "blending", true);
    // src/main.cpp:233-240: viscosity is opt-in (hydro/nu > 0), beta = -2/3 nu by default
    c.nu = P.real("hydro", "nu", 0.0);
    c.beta = P.real("hydro", "beta", -2. / 3 * c.nu);
    if (c.nu > 0.0) std::cout << "viscosity on: nu = " << c.nu << ", beta = " << c.beta << std::endl;
    const std::string prob = P.str("problem", "problem", "sine_wave");
    const Problem* pr = nullptr;
    for (const Problem& q : kProblems)
        if (prob == q.name) pr = &q;
    if (!pr) throw std::runtime_error("unknown problem '" + prob + "'");
    c.problem = pr->id;
    const char* names[10] = {"amp", "v1", "v2", "v3", "d0", "d1", "p0", "p1", "radius", "sigma"};
    double* dst[10] = {&c.amp, &c.v1, &c.v2, &c.v3, &c.d0, &c.d1, &c.p0, &c.p1, &c.radius, &c.sigma};
    for (int q = 0; q < 10; q++) *dst[q] = P.real("problem", names[q], pr->pp[q]);
    c.dir = P.integer("problem", "dir", 0);
    c.cx = 0.5 * L[0];
    c.cy = 0.5 * L[1];
    c.cz = 0.5 * L[2];
    for (int q = 0; q < 16; q++) c.q[q] = P.real("problem", "q" + std::to_string(q), 0.0);
    c.seed = (unsigned long long)P.integer("problem", "seed", 0);
    c.precision = P.str("job", "precision", "fp64") == "fp32" ? SPDK_PRECISION_FP32 : SPDK_PRECISION_FP64;
    c.device = 0;

    spdk_hydro* h = nullptr;
    check(spdk_hydro_create(&c, &h));
    spdk_hydro_info info{};
    check(spdk_hydro_get_info(h, &info));
    const int D = info.ndim, n = p + 1, V = info.nvar;
    const int gz = D == 3 ? 1 : 0;
    const int Ez = N[2] + 2 * gz, Ey = N[1] + 2, Ex = N[0] + 2, nz = D == 3 ? n : 1;
    const size_t state = (size_t)info.n_elements * V * info.n_points;
    const size_t cells = (size_t)info.n_elements * info.n_points;
    std::vector<double> w(state), tr(cells);
    const std::string dir = outputs ? out_dir() : "";
    int n_output = 0;
    auto write_outputs = [&]() {
        check(spdk_hydro_read(h, SPDK_FIELD_W_CV, w.data(), state));
        // reference layout (1, 6, Ez, Ey, Ex, nz, n, n); ghost elements NaN
        std::vector<double> f((size_t)6 * Ez * Ey * Ex * nz * n * n, std::numeric_limits<double>::quiet_NaN());
        const int slot_of[5] = {0, 1, 2, D == 3 ? 3 : -1, D == 3 ? 4 : 3};
        for (int s = 0; s < 6; s++)
            for (int k = 0; k < Ez; k++)
                for (int j = 0; j < Ey; j++)
                    for (int i = 0; i < Ex; i++) {
                        const bool active = (k >= gz && k < Ez - gz) && j >= 1 && j < Ey - 1 && i >= 1 && i < Ex - 1;
                        const long long e = active ? ((long long)(k - gz) * N[1] + (j - 1)) * N[0] + (i - 1) : -1;
                        for (int q = 0; q < nz * n * n; q++) {
                            double val;
                            if (s == 5) val = 0.0;
                            else if (!active) val = std::numeric_limits<double>::quiet_NaN();
                            else if (slot_of[s] < 0) val = 0.0;  // m_z of a 2D run
                            else val = w[((size_t)e * V + slot_of[s]) * info.n_points + q];
                            f[((((size_t)s * Ez + k) * Ey + j) * Ex + i) * nz * n * n + q] = val;
                        }
                    }
        write_file(dir + "W_cv_N" + std::to_string(N[0]) + "p" + std::to_string(p) + "_" + std::to_string(n_output) +
                       "_0.dat",
                   f.data(), f.size());
        n_output++;
    };
    // time_evolution (src/hydro_ader.hpp:215-273), optionally resumed from
    // a checkpoint (job/restart) and writing checkpoints every
    // output/checkpoint_dt of simulated time, asynchronously and without
    // changing any dt, so a run and its restarts step identically
    double t = 0, dt = 0, t_output = dt_out, t_io = 0;
    long long steps = 0;
    const std::string restart = P.str("job", "restart", "");
    if (!restart.empty()) {
        spdk_checkpoint_info ci{};
        check(spdk_hydro_restore(h, restart.c_str(), &ci));
        t = ci.t;
        t_output = ci.t_output;
        steps = ci.steps;
        n_output = (int)ci.outputs;
        std::printf("restarted from %s: t = %.17g, step %lld\n", restart.c_str(), t, steps);
    } else if (outputs) {
        write_outputs();
    }
    const double ckpt_dt = P.real("output", "checkpoint_dt", -1.0);
    const std::string ckpt_dir = ckpt_dt > 0 ? out_dir() : "";
    double t_ckpt = t + ckpt_dt;
    check(spdk_hydro_get_dt(h, &dt));
    const auto t0 = std::chrono::steady_clock::now();
    while (t < tlim) {
        check(spdk_hydro_step(h));
        t += dt;
        steps++;
        check(spdk_hydro_get_dt(h, &dt));
        if (outputs) {
            if (t >= t_output) {
                t_output = t + dt_out;
                const auto a = std::chrono::steady_clock::now();
                write_outputs();
                t_io += std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
            }
            if (t + dt > t_output) {
                dt = t_output - t;
                check(spdk_hydro_set_dt(h, dt));
            }
        }
        if (ckpt_dt > 0 && t >= t_ckpt && t < tlim) {
            const spdk_checkpoint_info ci{t, t_output, steps, n_output};
            check(spdk_hydro_checkpoint_async(h, (ckpt_dir + "checkpoint_" + std::to_string(steps) + ".spdk").c_str(),
                                              &ci));
            t_ckpt = t + ckpt_dt;
        }
    }
    check(spdk_hydro_sync(h));
    check(spdk_hydro_checkpoint_wait(h));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() - t_io;
    std::printf("\nevolution: %lld steps, %g s (%g ms/step), %g zone-cycles/s\n", steps, secs,
                steps ? secs / steps * 1e3 : 0.0, secs > 0 ? (double)info.n_dof * steps / secs : 0.0);
    spdk_hydro_destroy(h);
    return 0;
}

int run_induction(const Params& P, int p, const int N[3], const double L[3], double tlim, bool outputs,
                  double dt_out) {
    spdk_induction_config c{};
    c.p = p;
    for (int d = 0; d < 3; d++) {
        c.N[d] = N[d];
        c.L[d] = L[d];
    }
    c.bc[0] = bc_id(P.str("mesh", "x1_bc", "periodic"));
    c.bc[1] = bc_id(P.str("mesh", "x2_bc", "periodic"));
    c.bc[2] = bc_id(P.str("mesh", "x3_bc", "periodic"));
    integrator(P.str("time", "integrator", "ader"), &c.integrator, &c.rk_order);
    c.fallback = P.boolean("job", "fallback", true);
    c.cfl = P.real("time", "cfl", 0.8);
    c.nu = P.real("induction", "nu", 0.0025);
    c.nad_tolerance = P.real("fallback", "tolerance", 1e-5);
    c.nad_delta = P.str("fallback", "NAD", "relative") == "delta";
    c.nad_moore = P.str("fallback", "NAD_neighbors", "2nd") == "2nd";
    c.sed = P.boolean("fallback", "SED", true);
    c.fallback_apply = P.boolean("fallback", "apply", false);  // no reference counterpart
    spdk_induction* s = nullptr;
    check(spdk_induction_create(&c, &s));
    const std::string dir = outputs ? out_dir() : "";
    int n_output = 0;
    const int F = N[0] * (p + 1) + 4;
    auto write_outputs = [&]() {
        size_t cnt = 0;
        check(spdk_induction_field_size(s, SPDK_IND_FIELD_B2_CV, &cnt));
        std::vector<double> b(cnt);
        check(spdk_induction_read(s, SPDK_IND_FIELD_B2_CV, b.data(), cnt));
        if (c.fallback) {
            size_t ct = 0;
            check(spdk_induction_field_size(s, SPDK_IND_FIELD_TROUBLES, &ct));
            std::vector<double> tr(ct);
            check(spdk_induction_read(s, SPDK_IND_FIELD_TROUBLES, tr.data(), ct));
            write_file(dir + "troubles_N" + std::to_string(F) + "_" + std::to_string(n_output) + "_0.dat", tr.data(),
                       ct);
        }
        write_file(dir + "B2_cv_N" + std::to_string(N[0]) + "p" + std::to_string(p) + "_" + std::to_string(n_output) +
                       "_0.dat",
                   b.data(), cnt);
        n_output++;
    };
    if (outputs) write_outputs();
    // time_evolution (src/induction_ader.hpp:222-272)
    double t = 0, t_output = dt_out, t_io = 0, dt = 0;
    long long steps = 0;
    const auto t0 = std::chrono::steady_clock::now();
    check(spdk_induction_get_dt(s, &dt));
    while (t < tlim) {
        check(spdk_induction_step(s));
        t += dt;
        steps++;
        check(spdk_induction_get_dt(s, &dt));
        if (outputs) {
            if (t >= t_output) {
                t_output = t + dt_out;
                const auto a = std::chrono::steady_clock::now();
                write_outputs();
                t_io += std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
            }
            if (t + dt > t_output) {
                dt = t_output - t;
                check(spdk_induction_set_dt(s, dt));
            }
        }
    }
    size_t cnt = 0;
    check(spdk_induction_field_size(s, SPDK_IND_FIELD_BX_FP, &cnt));
    std::vector<double> sink(cnt);
    check(spdk_induction_read(s, SPDK_IND_FIELD_BX_FP, sink.data(), cnt));  // waits for the last step
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() - t_io;
    const double zones = (double)N[0] * (p + 1) * N[1] * (p + 1) * N[2] * (p + 1);
    std::printf("\nevolution: %lld steps, %g s (%g ms/step), %g zone-cycles/s\n", steps, secs,
                steps ? secs / steps * 1e3 : 0.0, secs > 0 ? zones * steps / secs : 0.0);
    spdk_induction_destroy(s);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        Params P;
        std::vector<std::string> ov;
        std::string deck;
        for (int a = 1; a < argc; a++) {
            const std::string arg = argv[a];
            if (arg == "-i" && a + 1 < argc) deck = argv[++a];
            else if (arg.find('/') != std::string::npos && arg.find('=') != std::string::npos) ov.push_back(arg);
            else throw std::runtime_error("unrecognized argument '" + arg + "'");
        }
        if (!deck.empty()) P.load(deck);
        for (const auto& o : ov) P.override_(o);
        const int p = P.integer("mesh", "p", 3);
        const int N[3] = {P.integer("mesh", "nx1", 8), P.integer("mesh", "nx2", 8), P.integer("mesh", "nx3", 8)};
        const double L[3] = {P.real("mesh", "x1len", 1.0), P.real("mesh", "x2len", 1.0), P.real("mesh", "x3len", 1.0)};
        if (N[0] < 2) throw std::runtime_error("the x-direction must be active (nx1>1)");
        const double tlim = P.real("time", "tlim", 0.1);
        const bool outputs = P.has("output", "dt") && P.real("output", "dt", -1) > 0.0;
        const double dt_out = outputs ? P.real("output", "dt", -1) : tlim;
        const std::string system = P.str("job", "system", "hydro");
        std::printf("system = %s, p = %d, N = (%d,%d,%d), integrator = %s, outputs = %s\n", system.c_str(), p, N[0],
                    N[1], N[2], P.str("time", "integrator", "ader").c_str(), outputs ? "on" : "off");
        if (outputs) {
            const std::string dir = out_dir();
            const char* axes[3] = {"X", "Y", "Z"};
            for (int d = 0; d < 3; d++) {
                const bool act = N[d] > 1;
                const std::vector<double> f = fv_faces(N[d], p, L[d], act);
                write_file(dir + axes[d] + "_N" + std::to_string(N[d]) + "p" + std::to_string(act ? p : 0) + "_0.dat",
                           f.data(), f.size());
            }
        }
        if (system == "hydro") return run_hydro(P, p, N, L, tlim, outputs, dt_out);
        if (system == "induction") return run_induction(P, p, N, L, tlim, outputs, dt_out);
        throw std::runtime_error("unknown system '" + system + "'");
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ERROR: %s\n", e.what());
        return 1;
    }
}
