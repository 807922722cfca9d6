// Host-side setup of the spd_K B200 solver: quadrature nodes, transform
// matrices, sub-grid geometry and initial conditions. All of it runs once
// before the time loop, on the CPU, with the same operation order as the
// reference so the matrices and the initial state are bit-identical.
#pragma once
#include <cstdint>
#include <vector>

#include "spdk.h"

namespace spdk {

constexpr int kMaxP = 7;
constexpr int kMaxN = kMaxP + 1;
constexpr int kMaxNF = kMaxP + 2;

struct Matrices {
    int p = 0, n = 0, nf = 0, nt = 0;
    double x_gl[kMaxN] = {}, w_gl[kMaxN] = {};  // GL(p) on [0,1] (flux-point nodes)
    double x_fp[kMaxNF] = {}, x_sp[kMaxN] = {};
    double xx[kMaxN + 1] = {}, wx[kMaxN + 1] = {};  // GL(p+1) on [0,1]
    double xt[kMaxN] = {}, wt[kMaxN] = {};
    double sp_to_fp[kMaxNF * kMaxN] = {};   // [nf][n]
    double dfp_to_sp[kMaxN * kMaxNF] = {};  // [n][nf]
    double sp_to_cv[kMaxN * kMaxN] = {};
    double cv_to_sp[kMaxN * kMaxN] = {};
    double fp_to_cv[kMaxN * kMaxNF] = {};   // [n][nf] (src/induction_ader.hpp:149)
    double ader[kMaxN * kMaxN] = {};
    double invader[kMaxN * kMaxN] = {};
};

// src/polynomials.cpp + src/hydro_ader.hpp:92-141
void build_matrices(int p, bool ader, Matrices* m);

// FV sub-grid coordinates of one direction in the reference's frame
// indexing (two ghost cells per side; src/structs.hpp:40-75)
struct Axis {
    int N = 1, n = 1, nf = 1, fvn = 1;
    bool active = false;
    double h = 1.0;
    std::vector<double> sd_faces;    // (N+2) x nf, ghost elements included
    std::vector<double> sd_centers;  // (N+2) x n, sub-cell centres
    std::vector<double> fv_faces;    // fvn + 1
    std::vector<double> fv_centers;  // fvn
};
// N elements of an axis of N_all elements over length L, starting at element
// `lo` of it (a slab; lo = 0, N_all = N for the whole axis)
void build_axis(int N, int p, double L, const double* x_fp, bool active, Axis* a, int lo = 0, int N_all = 0);

// Initial state: W_cv (primitive sub-cell averages) of the active elements
// in the solver layout [element][var][point], V = D+2 slots, evaluated by
// the reference's GL quadrature of the point ICs
// (src/initial_conditions.cpp:179-228).
void initial_wcv(const spdk_hydro_config& c, const Matrices& m, const Axis ax[3], int D,
                 std::vector<double>* wcv);

}  // namespace spdk
