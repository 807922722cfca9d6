// Host-only entry points of the C ABI: set-up that needs no GPU, used by
// drivers that want the matrices or the initial state before a solver
// exists, and by the CPU test suite.
#include <cstring>
#include <string>
#include <vector>

#include "spdk.h"
#include "spdk_setup.h"

namespace spdk {
int fail(int code, const std::string& msg);
}

extern "C" int spdk_build_matrices(int p, int ader, double* sp_to_fp, double* dfp_to_sp, double* sp_to_cv,
                                   double* cv_to_sp, double* invader, double* wt) {
    if (p < 1 || p > spdk::kMaxP) return spdk::fail(SPDK_E_ARG, "p must be in 1..7");
    spdk::Matrices m;
    spdk::build_matrices(p, ader != 0, &m);
    const int n = p + 1, nf = p + 2;
    if (sp_to_fp) std::memcpy(sp_to_fp, m.sp_to_fp, sizeof(double) * nf * n);
    if (dfp_to_sp) std::memcpy(dfp_to_sp, m.dfp_to_sp, sizeof(double) * n * nf);
    if (sp_to_cv) std::memcpy(sp_to_cv, m.sp_to_cv, sizeof(double) * n * n);
    if (cv_to_sp) std::memcpy(cv_to_sp, m.cv_to_sp, sizeof(double) * n * n);
    if (invader) std::memcpy(invader, m.invader, sizeof(double) * m.nt * m.nt);
    if (wt) std::memcpy(wt, m.wt, sizeof(double) * m.nt);
    return 0;
}

extern "C" int spdk_initial_wcv(const spdk_hydro_config* cfg, double* out, size_t count) {
    if (!cfg || !out) return spdk::fail(SPDK_E_ARG, "null argument");
    const spdk_hydro_config& c = *cfg;
    if (c.p < 1 || c.p > spdk::kMaxP || c.N[0] < 2 || c.N[1] < 2) return spdk::fail(SPDK_E_ARG, "bad mesh");
    const int D = c.N[2] > 1 ? 3 : 2;
    spdk::Matrices m;
    spdk::build_matrices(c.p, c.integrator == SPDK_INTEGRATOR_ADER, &m);
    spdk::Axis ax[3];
    const int N[3] = {c.N[0], c.N[1], D == 3 ? c.N[2] : 1};
    for (int d = 0; d < 3; d++) spdk::build_axis(N[d], c.p, c.L[d], m.x_fp, d < D, &ax[d]);
    std::vector<double> w;
    spdk::initial_wcv(c, m, ax, D, &w);
    if (count != w.size()) return spdk::fail(SPDK_E_ARG, "count must be " + std::to_string(w.size()));
    std::memcpy(out, w.data(), sizeof(double) * w.size());
    return 0;
}

extern "C" int spdk_fv_faces(int N, int p, double L, int active, double* out, size_t count) {
    if (!out || N < 1 || p < 1 || p > spdk::kMaxP || !(L > 0)) return spdk::fail(SPDK_E_ARG, "bad argument");
    spdk::Matrices m;
    spdk::build_matrices(p, true, &m);
    if (!active) {
        // one face at (0 - NGH + x_fp[0]) h, h = L (src/structs.hpp:60-63)
        if (count != 1) return spdk::fail(SPDK_E_ARG, "count must be 1 for an inactive direction");
        out[0] = (0 + 0 - 1 + m.x_fp[0]) * L;
        return 0;
    }
    spdk::Axis a;
    spdk::build_axis(N, p, L, m.x_fp, true, &a);
    if (count != a.fv_faces.size()) return spdk::fail(SPDK_E_ARG, "count must be " + std::to_string(a.fv_faces.size()));
    std::memcpy(out, a.fv_faces.data(), sizeof(double) * a.fv_faces.size());
    return 0;
}
