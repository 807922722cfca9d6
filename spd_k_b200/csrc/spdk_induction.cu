// The induction solver (src/induction_ader.hpp, src/induction.cpp) on
// device arrays in the reference's own layout, ghost elements included, so
// that every output is the reference's bytes: face fields B_x (x flux
// points), B_y, B_z; edge fields E_x (y and z flux points, x solution
// points), E_y, E_z with the reference's 8 slots (E, b1, b2, v1, v2, Ed,
// b1d, b2d); FV sub-cell arrays with the two-cell ghost frame. One thread
// per output point (or face, or FV cell), reference operation order,
// built without FMA contraction.
//
// The initial vector potential and its curl, and the dt, are computed on
// the host exactly as the reference's constructor does; every per-step
// operation runs on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "spdk.h"
#include "spdk_induction.h"
#include "spdk_reflayout.cuh"
#include "spdk_setup.h"

namespace {

using namespace spdk;

constexpr int kNGH = 2;  // FV ghost layers
constexpr int kEVars = 8;

// src/induction.cpp:18-24: v = (1, 1, 0) (the rest of velocity() follows an
// unconditional return and never runs)
__host__ __device__ __forceinline__ double velocity(int var) { return var < 2 ? 1.0 : 0.0; }

// src/induction.cpp:487-491
__device__ __forceinline__ double upwind(double left, double right, double vel) {
    if (vel == 0) return 0.5 * (left + right);
    return (vel > 0 ? left : right);
}

#define GRID_LOOP(o, n) \
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < (n); o += (long long)gridDim.x * blockDim.x)

// src/induction.cpp:123-200: E at the edge points of every element and slice
__global__ void k_compute_E(SDa E, SDa B1, SDa B2, const double* __restrict__ M, int n, int dim) {
    const int q = choose(dim, E.e[7], E.e[6], E.e[5]);
    const int nader = E.e[0];
    const int dim1 = choose(dim, 1, 2, 0), dim2 = choose(dim1, 1, 2, 0);
    GRID_LOOP(o, E.pts() * nader) {
        const int t = (int)(o % nader);
        int c[6];
        point_of(E, o / nader, c);
        const int k = c[0], j = c[1], i = c[2], kk = c[3], jj = c[4], ii = c[5];
        double b1 = 0, b2 = 0;
        for (int ll = 0; ll < q; ll++) {
            if (dim == 2) {
                b1 += B1.at(t, 0, k, j, i, kk, ll, ii) * M[jj * n + ll];
                b2 += B2.at(t, 0, k, j, i, kk, jj, ll) * M[ii * n + ll];
            } else if (dim == 1) {
                b1 += B1.at(t, 0, k, j, i, kk, jj, ll) * M[ii * n + ll];
                b2 += B2.at(t, 0, k, j, i, ll, jj, ii) * M[kk * n + ll];
            } else {
                b1 += B1.at(t, 0, k, j, i, ll, jj, ii) * M[kk * n + ll];
                b2 += B2.at(t, 0, k, j, i, kk, ll, ii) * M[jj * n + ll];
            }
        }
        const double v1 = velocity(dim1), v2 = velocity(dim2);
        E.at(t, 0, k, j, i, kk, jj, ii) = v1 * b2 - v2 * b1;
        E.at(t, 1, k, j, i, kk, jj, ii) = b1;
        E.at(t, 2, k, j, i, kk, jj, ii) = b2;
        E.at(t, 3, k, j, i, kk, jj, ii) = v1;
        E.at(t, 4, k, j, i, kk, jj, ii) = v2;
        E.at(t, 5, k, j, i, kk, jj, ii) = 0;
        E.at(t, 6, k, j, i, kk, jj, ii) = b1;
        E.at(t, 7, k, j, i, kk, jj, ii) = b2;
    }
}

// src/induction.cpp:494-558: upwind by max(v_L, v_R) of slot v1 on slots
// 0..nvar-4, the average on the last two
__global__ void k_E_riemann(SDa E, int dim, int v1) {
    const int Nx = E.e[4] - (dim == 0), Ny = E.e[3] - (dim == 1), Nz = E.e[2] - (dim == 2);
    const int px = dim == 0 ? 1 : E.e[7], py = dim == 1 ? 1 : E.e[6], pz = dim == 2 ? 1 : E.e[5];
    const int n = choose(dim, E.e[7], E.e[6], E.e[5]);
    const int nader = E.e[0], nvar = E.e[1];
    GRID_LOOP(o, (long long)Nz * Ny * Nx * pz * py * px) {
        long long r = o;
        const int ii = (int)(r % px); r /= px;
        const int jj = (int)(r % py); r /= py;
        const int kk = (int)(r % pz); r /= pz;
        const int i = (int)(r % Nx); r /= Nx;
        const int j = (int)(r % Ny); r /= Ny;
        const int k = (int)r;
        const int l = choose(dim, i, j, k);
        const int kL = dim == 2 ? l : k, jL = dim == 1 ? l : j, iL = dim == 0 ? l : i;
        const int kR = dim == 2 ? l + 1 : k, jR = dim == 1 ? l + 1 : j, iR = dim == 0 ? l + 1 : i;
        const int kkL = dim == 2 ? n - 1 : kk, jjL = dim == 1 ? n - 1 : jj, iiL = dim == 0 ? n - 1 : ii;
        const int kkR = dim == 2 ? 0 : kk, jjR = dim == 1 ? 0 : jj, iiR = dim == 0 ? 0 : ii;
        for (int t = 0; t < nader; t++) {
            const double v = smax(E.at(t, v1, kL, jL, iL, kkL, jjL, iiL), E.at(t, v1, kR, jR, iR, kkR, jjR, iiR));
            for (int var = 0; var < nvar - 3; var++) {
                double& L = E.at(t, var, kL, jL, iL, kkL, jjL, iiL);
                double& R = E.at(t, var, kR, jR, iR, kkR, jjR, iiR);
                const double e = upwind(L, R, v);
                L = e;
                R = e;
            }
            for (int var = nvar - 2; var < nvar; var++) {
                double& L = E.at(t, var, kL, jL, iL, kkL, jjL, iiL);
                double& R = E.at(t, var, kR, jR, iR, kkR, jjR, iiR);
                const double e = upwind(L, R, 0.0);
                L = e;
                R = e;
            }
        }
    }
}

// src/induction.cpp:303-418: dB/dt = curl E at the face points of the
// active elements; predict: B_ader(t) = B - sum_l dBdt(l) invader(t,l) w(l)
// dt, else B -= sum_t dBdt(t) w(t) dt
__global__ void k_update_B(SDa B, SDa Ba, SDa E1, SDa E2, const double* __restrict__ Dm, int nfc,
                           const double* __restrict__ inv, const double* __restrict__ w, double d1, double d2,
                           double dt, int dim, int nader, int predict) {
    const int q = choose(dim, B.e[7], B.e[6], B.e[5]);
    const int Mx = B.e[4] - 2, My = B.e[3] - 2, Mz = B.e[2] - 2;
    const int px = B.e[7], py = B.e[6], pz = B.e[5];
    GRID_LOOP(o, (long long)Mz * My * Mx * pz * py * px) {
        long long r = o;
        const int ii = (int)(r % px); r /= px;
        const int jj = (int)(r % py); r /= py;
        const int kk = (int)(r % pz); r /= pz;
        const int i = 1 + (int)(r % Mx); r /= Mx;
        const int j = 1 + (int)(r % My); r /= My;
        const int k = 1 + (int)r;
        double dBdt[16];
        double dB = 0;
        for (int t = 0; t < nader; t++) {
            double s = 0;
            for (int ll = 0; ll < q; ll++) {
                double E;
                if (dim == 0) {
                    E = E1.at(t, 0, k, j, i, ll, jj, ii);
                    s += E * Dm[kk * nfc + ll] / d2;
                    E = E2.at(t, 0, k, j, i, kk, ll, ii);
                    s -= E * Dm[jj * nfc + ll] / d1;
                } else if (dim == 1) {
                    E = E1.at(t, 0, k, j, i, kk, jj, ll);
                    s += E * Dm[ii * nfc + ll] / d2;
                    E = E2.at(t, 0, k, j, i, ll, jj, ii);
                    s -= E * Dm[kk * nfc + ll] / d1;
                } else {
                    E = E1.at(t, 0, k, j, i, kk, ll, ii);
                    s += E * Dm[jj * nfc + ll] / d2;
                    E = E2.at(t, 0, k, j, i, kk, jj, ll);
                    s -= E * Dm[ii * nfc + ll] / d1;
                }
            }
            dBdt[t] = s;
            if (!predict) dB += s * w[t] * dt;
        }
        if (predict) {
            const double b_old = B.at(0, 0, k, j, i, kk, jj, ii);
            for (int t = 0; t < nader; t++) {
                double d = 0;
                for (int ll = 0; ll < nader; ll++) d += dBdt[ll] * inv[t * nader + ll] * w[ll] * dt;
                Ba.at(t, 0, k, j, i, kk, jj, ii) = b_old - d;
            }
        } else {
            B.at(0, 0, k, j, i, kk, jj, ii) -= dB;
        }
    }
}

// src/induction.cpp:420-455: sub-cell averages of B and |B|^2 (all elements)
__global__ void k_B2_cv(SDa B2, SDa Bx, SDa By, SDa Bz, const double* __restrict__ F, const double* __restrict__ S,
                        int n, int nf) {
    const int q = Bx.e[7];
    const int px = B2.e[7], py = B2.e[6], pz = B2.e[5];
    GRID_LOOP(o, B2.pts()) {
        int c[6];
        point_of(B2, o, c);
        const int k = c[0], j = c[1], i = c[2], kk = c[3], jj = c[4], ii = c[5];
        double bx = 0, by = 0, bz = 0;
        for (int nn = 0; nn < pz; nn++)
            for (int mm = 0; mm < py; mm++)
                for (int ll = 0; ll < q; ll++)
                    bx += Bx.at(0, 0, k, j, i, nn, mm, ll) * S[kk * n + nn] * S[jj * n + mm] * F[ii * nf + ll];
        for (int nn = 0; nn < pz; nn++)
            for (int mm = 0; mm < q; mm++)
                for (int ll = 0; ll < px; ll++)
                    by += By.at(0, 0, k, j, i, nn, mm, ll) * S[kk * n + nn] * F[jj * nf + mm] * S[ii * n + ll];
        for (int nn = 0; nn < q; nn++)
            for (int mm = 0; mm < py; mm++)
                for (int ll = 0; ll < px; ll++)
                    bz += Bz.at(0, 0, k, j, i, nn, mm, ll) * F[kk * nf + nn] * S[jj * n + mm] * S[ii * n + ll];
        B2.at(0, 0, k, j, i, kk, jj, ii) = bx;
        B2.at(0, 1, k, j, i, kk, jj, ii) = by;
        B2.at(0, 2, k, j, i, kk, jj, ii) = bz;
        B2.at(0, 3, k, j, i, kk, jj, ii) = bx * bx + by * by + bz * bz;
    }
}

// src/induction.cpp:457-485: FV cell averages from the sub-cell face averages
__global__ void k_B_cv_from_cf(FVa B, SDa Bx, SDa By, SDa Bz, const double* __restrict__ F, int nf) {
    const int px = Bx.e[7] - 1, py = Bx.e[6], pz = Bx.e[5];
    const int q = px + 1;
    const int Mx = Bx.e[4] - 2, My = Bx.e[3] - 2, Mz = Bx.e[2] - 2;
    GRID_LOOP(o, (long long)Mz * My * Mx * pz * py * px) {
        long long r = o;
        const int ii = (int)(r % px); r /= px;
        const int jj = (int)(r % py); r /= py;
        const int kk = (int)(r % pz); r /= pz;
        const int i = 1 + (int)(r % Mx); r /= Mx;
        const int j = 1 + (int)(r % My); r /= My;
        const int k = 1 + (int)r;
        const int I = ii + kNGH + (i - 1) * px, J = jj + kNGH + (j - 1) * py, K = kk + kNGH + (k - 1) * pz;
        double bx = 0, by = 0, bz = 0;
        for (int ll = 0; ll < q; ll++) {
            bx += Bx.at(0, 0, k, j, i, kk, jj, ll) * F[ii * nf + ll];
            by += By.at(0, 0, k, j, i, kk, ll, ii) * F[jj * nf + ll];
            bz += Bz.at(0, 0, k, j, i, ll, jj, ii) * F[kk * nf + ll];
        }
        B.at(0, K, J, I) = bx;
        B.at(1, K, J, I) = by;
        B.at(2, K, J, I) = bz;
        B.at(3, K, J, I) = bx * bx + by * by + bz * bz;
    }
}

// src/induction.cpp:594-651: E along the sub-cell edges of slice t; the
// range takes the right ghost element in the directions normal to the edge
// and drops each element's last face there (it repeats the next element's
// first)
__global__ void k_edge_integral(SDa Eep, FVa E, const double* __restrict__ S, int n, int t, int dim) {
    const int Nx = Eep.e[4] + (dim == 0 ? 0 : 1), Ny = Eep.e[3] + (dim == 1 ? 0 : 1), Nz = Eep.e[2] + (dim == 2 ? 0 : 1);
    const int px = Eep.e[7] - (dim == 0 ? 0 : 1), py = Eep.e[6] - (dim == 1 ? 0 : 1), pz = Eep.e[5] - (dim == 2 ? 0 : 1);
    const int q = choose(dim, px, py, pz);
    const int Mx = Nx - 2, My = Ny - 2, Mz = Nz - 2;
    GRID_LOOP(o, (long long)Mz * My * Mx * pz * py * px) {
        long long r = o;
        const int ii = (int)(r % px); r /= px;
        const int jj = (int)(r % py); r /= py;
        const int kk = (int)(r % pz); r /= pz;
        const int i = 1 + (int)(r % Mx); r /= Mx;
        const int j = 1 + (int)(r % My); r /= My;
        const int k = 1 + (int)r;
        const int I = ii + kNGH + (i - 1) * px, J = jj + kNGH + (j - 1) * py, K = kk + kNGH + (k - 1) * pz;
        const int id = choose(dim, ii, jj, kk);
        double e = 0;
        for (int ll = 0; ll < q; ll++) {
            const int n0 = dim == 0 ? ll : ii, n1 = dim == 1 ? ll : jj, n2 = dim == 2 ? ll : kk;
            double s = Eep.at(t, 0, k, j, i, n2, n1, n0);
            s *= S[id * n + ll];
            e += s;
        }
        if (K < E.e[1] && J < E.e[2] && I < E.e[3]) E.at(0, K, J, I) = e;
    }
}

// src/induction.cpp:653-720: sub-cell face update of one B component from
// the edge E of the two transverse directions
__global__ void k_fv_update_B(FVa Bn, FVa Bo, SDa B, FVa E1, FVa E2, const double* __restrict__ f1,
                              const double* __restrict__ f2, const double* __restrict__ w, double dt, int t, int dim,
                              int update) {
    const int px = B.e[7], py = B.e[6], pz = B.e[5];
    const int qx = px - (dim == 0), qy = py - (dim == 1), qz = pz - (dim == 2);
    const int dim1 = choose(dim, 1, 2, 0), dim2 = choose(dim1, 1, 2, 0);
    const int Mx = B.e[4] - 2, My = B.e[3] - 2, Mz = B.e[2] - 2;
    GRID_LOOP(o, (long long)Mz * My * Mx * pz * py * px) {
        long long r = o;
        const int ii = (int)(r % px); r /= px;
        const int jj = (int)(r % py); r /= py;
        const int kk = (int)(r % pz); r /= pz;
        const int i = 1 + (int)(r % Mx); r /= Mx;
        const int j = 1 + (int)(r % My); r /= My;
        const int k = 1 + (int)r;
        const int I = ii + kNGH + (i - 1) * qx, J = jj + kNGH + (j - 1) * qy, K = kk + kNGH + (k - 1) * qz;
        const double b_old = B.at(0, 0, k, j, i, kk, jj, ii);
        if (K < Bn.e[1] && J < Bn.e[2] && I < Bn.e[3]) {
            Bo.at(0, K, J, I) = b_old;
            double ep = E1.at(0, K + (dim2 == 2), J + (dim2 == 1), I + (dim2 == 0));
            int id = choose(dim2, I, J, K);
            double h = (f2[id + 1] - f2[id]);
            double dBdt = (ep - E1.at(0, K, J, I)) / h;
            ep = E2.at(0, K + (dim1 == 2), J + (dim1 == 1), I + (dim1 == 0));
            id = choose(dim1, I, J, K);
            h = (f1[id + 1] - f1[id]);
            dBdt -= (ep - E2.at(0, K, J, I)) / h;
            const double b_new = b_old - dBdt * w[t] * dt;
            Bn.at(0, K, J, I) = b_new;
            if (update) B.at(0, 0, k, j, i, kk, jj, ii) = b_new;
        }
    }
}

// src/boundary.cpp:123-190 for the induction's FV arrays. The reference
// loops over the transverse extents of its boundary buffers, which for a
// cell-centred array run one row past the array (and one past a staggered
// array's cell extent); those accesses land, through the row-major layout,
// in the next row or the next variable's first layer. The passes below
// index the array flat with its own extents, so they touch the same
// elements; the accesses past the end of the allocation are dropped.
// Pass 0 reads into buf (the reference's BoundaryL/R). Two iterations can
// then write one element with different values (a wrapped row lands on a
// ghost cell another iteration also fills); the reference's loop runs
// (k, j, i) in order with var, then L before R, inside, so the later
// iteration's value stands. Pass 1 claims each element for the latest
// writer (atomicMax of its sequence number, tagged with a per-call epoch),
// pass 2 lets only that writer store.
__global__ void k_fv_bc(FVa U, double* __restrict__ buf, unsigned long long* __restrict__ win, unsigned epoch, int dim,
                        int type, int N, int shift, int Lx, int Ly, int Lz, int pass) {
    const long long total = (long long)U.e[0] * U.cells();
    GRID_LOOP(o, (long long)Lz * Ly * Lx * U.e[0]) {
        long long r = o;
        const int var = (int)(r % U.e[0]); r /= U.e[0];
        const int i = (int)(r % Lx); r /= Lx;
        const int j = (int)(r % Ly); r /= Ly;
        const int k = (int)r;
        const int l = choose(dim, i, j, k);
        auto off = [&](int L) {
            const int kk = dim == 2 ? L : k, jj = dim == 1 ? L : j, ii = dim == 0 ? L : i;
            return (((long long)var * U.e[1] + kk) * U.e[2] + jj) * U.e[3] + ii;
        };
        if (pass == 0) {
            long long sL, sR;
            double sgn = 1.0;
            if (type == kPeriodic) { sL = off(N - 2 * kNGH + l - shift); sR = off(kNGH + l + shift); }
            else if (type == kGradfree) { sL = off(kNGH + l + shift); sR = off(N - 2 * kNGH + l - shift); }
            else {
                sgn = (var == 1 + dim) ? -1.0 : 1.0;
                sL = off(2 * kNGH - 1 - l);
                sR = off(N - kNGH - 1 - l);
            }
            buf[2 * o] = sL < total ? sgn * U.p[sL] : 0.0;
            buf[2 * o + 1] = sR < total ? sgn * U.p[sR] : 0.0;
        } else {
            const long long dL = off(l), dR = off(N - kNGH + l);
            // iteration order: flat (k, j, i), then var, then L / R
            const unsigned long long f = (((unsigned long long)k * Ly + j) * Lx + i) * U.e[0] + var;
            const unsigned long long keyL = ((unsigned long long)epoch << 32) | (2 * f);
            const unsigned long long keyR = ((unsigned long long)epoch << 32) | (2 * f + 1);
            if (pass == 1) {
                if (dL < total) atomicMax(&win[dL], keyL);
                if (dR < total) atomicMax(&win[dR], keyR);
            } else {
                if (dL < total && win[dL] == keyL) U.p[dL] = buf[2 * o];
                if (dR < total && win[dR] == keyR) U.p[dR] = buf[2 * o + 1];
            }
        }
    }
}

// src/trouble_detection.cpp:35-104 (nvar = slots - 1, one-layer range)
__global__ void k_ind_nad(FVa Un, FVa U, FVa Tr, double tol, int moore, int delta, int mask) {
    const int nvar = U.e[0] - 1;
    const int Mx = U.e[3] - 2, My = U.e[2] - 2, Mz = U.e[1] - 2;
    GRID_LOOP(o, (long long)Mz * My * Mx) {
        const int i = 1 + (int)(o % Mx), j = 1 + (int)((o / Mx) % My), k = 1 + (int)(o / Mx / My);
        for (int var = 0; var < nvar; var++) {
            if (!((mask >> var) & 1)) continue;
            const double un = Un.at(var, k, j, i);
            double mx = U.at(var, k, j, i), mn = mx;
            if (moore) {
                for (int dk = -1; dk <= 1; dk++)
                    for (int dj = -1; dj <= 1; dj++)
                        for (int di = -1; di <= 1; di++) {
                            const double u = U.at(var, k + dk, j + dj, i + di);
                            mx = smax(mx, u);
                            mn = smin(mn, u);
                        }
            } else {
                for (int d = 0; d < 3; d++) {
                    const double uL = U.at(var, k - (d == 2), j - (d == 1), i - (d == 0));
                    const double uR = U.at(var, k + (d == 2), j + (d == 1), i + (d == 0));
                    mx = smax(smax(uL, mx), uR);
                    mn = smin(smin(uL, mn), uR);
                }
            }
            if (delta) {
                const double eps = tol * (mx - mn);
                mn -= eps;
                mx += eps;
            } else {
                mn -= fabs(mn) * tol;
                mx += fabs(mx) * tol;
            }
            Tr.at(var, k, j, i) = (un > mx || un < mn) ? 1 : 0;
        }
    }
}

// src/trouble_detection.cpp:107-148 (two-layer range)
__global__ void k_ind_sed(FVa U, FVa A, const double* __restrict__ c, const double* __restrict__ f, int dim,
                          int mask) {
    const int nvar = U.e[0] - 1;
    const int Mx = U.e[3] - 4, My = U.e[2] - 4, Mz = U.e[1] - 4;
    const int ox = dim == 0, oy = dim == 1, oz = dim == 2;
    GRID_LOOP(o, (long long)Mz * My * Mx) {
        const int i = 2 + (int)(o % Mx), j = 2 + (int)((o / Mx) % My), k = 2 + (int)(o / Mx / My);
        const int l = choose(dim, i, j, k);
        for (int var = 0; var < nvar; var++) {
            if (!((mask >> var) & 1)) continue;
            const double u = U.at(var, k, j, i);
            const double h = (c[l + 1] - c[l - 1]);
            const double hp = (c[l + 2] - c[l]);
            const double hm = (c[l] - c[l - 2]);
            const double du = (U.at(var, k + oz, j + oy, i + ox) - U.at(var, k - oz, j - oy, i - ox)) / h;
            const double dup = (U.at(var, k + 2 * oz, j + 2 * oy, i + 2 * ox) - u) / hp;
            const double dum = (u - U.at(var, k - 2 * oz, j - 2 * oy, i - 2 * ox)) / hm;
            const double d2u = (dup - dum) / (c[l + 1] - c[l - 1]);
            const double dv = 0.5 * d2u * (f[l + 1] - f[l]);
            A.at(var, k, j, i) = sed_alpha(dv, dum, du, dup);
        }
    }
}

// src/trouble_detection.cpp:152-183 (aggregate into the last slot)
__global__ void k_ind_relax(FVa Tr, FVa Ax, FVa Ay, FVa Az, int mask, int use_sed) {
    const int nvar = Tr.e[0] - 1;
    const int Mx = Tr.e[3] - 2, My = Tr.e[2] - 2, Mz = Tr.e[1] - 2;
    GRID_LOOP(o, (long long)Mz * My * Mx) {
        const int i = 1 + (int)(o % Mx), j = 1 + (int)((o / Mx) % My), k = 1 + (int)(o / Mx / My);
        for (int var = 0; var < nvar; var++) {
            if (!((mask >> var) & 1)) continue;
            double alpha = smin(smin(Ax.at(var, k, j, i - 1), Ax.at(var, k, j, i)), Ax.at(var, k, j, i + 1));
            alpha = smin(alpha, smin(smin(Ay.at(var, k, j - 1, i), Ay.at(var, k, j, i)), Ay.at(var, k, j + 1, i)));
            alpha = smin(alpha, smin(smin(Az.at(var, k - 1, j, i), Az.at(var, k, j, i)), Az.at(var, k + 1, j, i)));
            const double trouble = Tr.at(var, k, j, i);
            if (use_sed) Tr.at(var, k, j, i) = alpha < 1 ? trouble : 0;
        }
        double trouble = 0;
        for (int var = 0; var < nvar; var++)
            if ((mask >> var) & 1) trouble = smax(trouble, Tr.at(var, k, j, i));
        Tr.at(nvar, k, j, i) = trouble;
    }
}

// Fallback EMF (no counterpart in the reference, whose corrector detects
// troubles but applies no fallback): on every sub-cell edge of direction
// dim that touches a troubled cell (the aggregate slot of the detection),
// the first-order upwind EMF v1 b2 - v2 b1 of the slice-start face averages
// replaces the high-order edge EMF; b2 (faces normal to dim2) is upwinded
// along dim1 by v1, b1 (normal to dim1) along dim2 by v2, with the
// reference's upwind() rule. Edge (K, J, I) is the low corner, in the two
// directions other than dim, of cell (K, J, I); the loop covers the edges
// the face update of the active cells reads. Edges without a troubled cell
// keep their value bit for bit.
__global__ void k_ind_fallback_emf(FVa E, FVa B1, FVa B2, FVa Tr, int dim, int fx, int fy, int fz) {
    const int dim1 = choose(dim, 1, 2, 0), dim2 = choose(dim1, 1, 2, 0);
    const int Mx = (dim == 0 ? fx - 3 : fx - 2) - kNGH + 1;
    const int My = (dim == 1 ? fy - 3 : fy - 2) - kNGH + 1;
    const int Mz = (dim == 2 ? fz - 3 : fz - 2) - kNGH + 1;
    const int agg = Tr.e[0] - 1;
    const int o1[3] = {dim1 == 0, dim1 == 1, dim1 == 2}, o2[3] = {dim2 == 0, dim2 == 1, dim2 == 2};
    GRID_LOOP(o, (long long)Mz * My * Mx) {
        const int I = kNGH + (int)(o % Mx), J = kNGH + (int)((o / Mx) % My), K = kNGH + (int)(o / Mx / My);
        double tr = 0;
        for (int s1 = 0; s1 < 2; s1++)
            for (int s2 = 0; s2 < 2; s2++)
                tr = smax(tr, Tr.at(agg, K - s1 * o1[2] - s2 * o2[2], J - s1 * o1[1] - s2 * o2[1],
                                    I - s1 * o1[0] - s2 * o2[0]));
        if (tr > 0) {
            const double b2L = B2.at(0, K - o1[2], J - o1[1], I - o1[0]), b2R = B2.at(0, K, J, I);
            const double b1L = B1.at(0, K - o2[2], J - o2[1], I - o2[0]), b1R = B1.at(0, K, J, I);
            const double v1 = velocity(dim1), v2 = velocity(dim2);
            E.at(0, K, J, I) = v1 * upwind(b2L, b2R, v1) - v2 * upwind(b1L, b1R, v2);
        }
    }
}

#undef GRID_LOOP

// src/initial_conditions.cpp:235-249
double magnetic_loop(int var, double x, double y, double z) {
    (void)z;
    x = x - 0.5;
    y = y - 0.5;
    const double r = std::sqrt(x * x + y * y);
    const double A0 = 0.001;
    const double R = 0.3;
    if (var == 2) {
        if (r <= R) return A0 * (R - r);
        return 0;
    }
    return 0;
}

// host view of a reference-layout array
struct HostSD {
    std::vector<double> v;
    int e[8];
    HostSD(int nt, int nv, int Nz, int Ny, int Nx, int nz, int ny, int nx) : e{nt, nv, Nz, Ny, Nx, nz, ny, nx} {
        v.assign((size_t)nt * nv * Nz * Ny * Nx * nz * ny * nx, 0.0);
    }
    double& at(int t, int var, int k, int j, int i, int kk, int jj, int ii) {
        size_t o = (((((size_t)t * e[1] + var) * e[2] + k) * e[3] + j) * e[4] + i);
        o = ((o * e[5] + kk) * e[6] + jj) * e[7] + ii;
        return v[o];
    }
};

}  // namespace

struct spdk_induction {
    spdk_induction_config cfg{};
    Matrices m;
    Axis ax[3];
    int n = 0, nf = 0, nt = 1, nstages = 1, fvn[3] = {0, 0, 0};
    double rk_a[3] = {0, 0, 0};
    double Dt = 0, dt = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    // device matrices / vectors
    double *sp_to_fp = nullptr, *dfp_to_sp = nullptr, *sp_to_cv = nullptr, *cv_to_sp = nullptr, *fp_to_cv = nullptr;
    double *invader = nullptr, *wt = nullptr, *fvf[3] = {nullptr, nullptr, nullptr}, *fvc[3] = {nullptr, nullptr, nullptr};
    double* bcbuf = nullptr;
    unsigned long long* bcwin = nullptr;  // last-writer claims of the FV ghost fill
    unsigned epoch = 0;
    SDa Bfp[3], Bader[3], B0[3], Ecc[3], Bcv[3], Bsave[3], Tfp[3], B2;
    FVa Bold[3], Bnew[3], Bo4, Bn4, troubles, alpha[3], Efv[3];
};

namespace {

int dalloc(spdk_induction* s, double** p, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, count * sizeof(double)) != cudaSuccess) return fail(SPDK_E_NOMEM, "induction: device allocation");
    s->allocs.push_back(q);
    if (cudaMemset(q, 0, count * sizeof(double)) != cudaSuccess) return fail(SPDK_E_CUDA, "induction: memset");
    *p = (double*)q;
    return 0;
}
int make_sd(spdk_induction* s, SDa* a, int nt, int nv, int nz, int ny, int nx) {
    const int E[3] = {s->cfg.N[2] + 2, s->cfg.N[1] + 2, s->cfg.N[0] + 2};
    int ext[8] = {nt, nv, E[0], E[1], E[2], nz, ny, nx};
    size_t c = 1;
    for (int q = 0; q < 8; q++) {
        a->e[q] = ext[q];
        c *= (size_t)ext[q];
    }
    return dalloc(s, &a->p, c);
}
int make_fv(spdk_induction* s, FVa* a, int nv, int sz, int sy, int sx) {
    a->e[0] = nv;
    a->e[1] = s->fvn[2] + sz;
    a->e[2] = s->fvn[1] + sy;
    a->e[3] = s->fvn[0] + sx;
    return dalloc(s, &a->p, (size_t)nv * a->e[1] * a->e[2] * a->e[3]);
}
int upload(spdk_induction* s, double** d, const double* h, size_t count) {
    int rc = dalloc(s, d, count);
    if (rc) return rc;
    if (cudaMemcpy(*d, h, count * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(SPDK_E_CUDA, "induction: upload");
    return 0;
}

// the flux-point extent along d when the array is staggered there
inline int ext_of(const spdk_induction* s, bool fp) { return fp ? s->nf : s->n; }

void release(spdk_induction* s) {
    for (void* p : s->allocs) cudaFree(p);
    s->allocs.clear();
    if (s->stream) cudaStreamDestroy(s->stream);
    s->stream = nullptr;
}

// Solve_E (src/induction_ader.hpp:350-360, inviscid)
int solve_E(spdk_induction* s) {
    cudaStream_t st = s->stream;
    const int n = s->n;
    // ElectricField (:392-420): Ez from (Bx, By), Ey from (Bz, Bx), Ex from (By, Bz)
    const int pairs[3][2] = {{1, 2}, {2, 0}, {0, 1}};  // (B1, B2) of E_dim
    const int order[3] = {2, 1, 0};
    for (int q = 0; q < 3; q++) {
        const int d = order[q];
        k_compute_E<<<blocks_for(s->Ecc[d].pts() * s->nt), kBlock, 0, st>>>(s->Ecc[d], s->Bader[pairs[d][0]],
                                                                             s->Bader[pairs[d][1]], s->sp_to_fp, n, d);
    }
    // apply_boundaries (:422-436)
    const int bcs[6][2] = {{1, 0}, {2, 0}, {0, 1}, {2, 1}, {0, 2}, {1, 2}};  // (E component, direction)
    for (auto& b : bcs) {
        const SDa& E = s->Ecc[b[0]];
        k_boundaries_sd<<<blocks_for(E.pts() * E.e[0] * E.e[1]), kBlock, 0, st>>>(E, b[1], s->cfg.bc[b[1]]);
    }
    // Riemann_Solver (:437-449)
    const int rs[6][3] = {{1, 0, 4}, {2, 0, 3}, {2, 1, 4}, {0, 1, 3}, {0, 2, 4}, {1, 2, 3}};
    for (auto& r : rs) {
        const SDa& E = s->Ecc[r[0]];
        k_E_riemann<<<blocks_for(E.pts()), kBlock, 0, st>>>(E, r[1], r[2]);
    }
    return launched("induction: Solve_E");
}

// Update_prediction / Update_solution (:468-483): component d from E_{d+1}
// (dim2 derivative) and E_{d+2} (dim1 derivative)
int update_B(spdk_induction* s, bool predict) {
    const double h[3] = {s->ax[0].h, s->ax[1].h, s->ax[2].h};
    for (int d = 0; d < 3; d++) {
        const int e1 = (d + 1) % 3, e2 = (d + 2) % 3;
        const double d1 = h[(d + 1) % 3], d2 = h[(d + 2) % 3];
        const SDa& B = s->Bfp[d];
        k_update_B<<<blocks_for(B.pts()), kBlock, 0, s->stream>>>(B, s->Bader[d], s->Ecc[e1], s->Ecc[e2], s->dfp_to_sp,
                                                                  s->nf, s->invader, s->wt, d1, d2, s->dt, d,
                                                                  s->nt, predict ? 1 : 0);
    }
    return launched("induction: update_B");
}

// transform_a_to_b_2d (src/transforms.cpp:226-249): the two directions
// transverse to dim, ping-ponging through T so the last sweep lands in b
void transform_2d(spdk_induction* s, const SDa& a, const SDa& b, const SDa& T, const double* M, int dim) {
    const int dim1 = choose(dim, 1, 2, 0), dim2 = choose(dim1, 1, 2, 0);
    const int dims[2] = {dim1, dim2};
    const SDa* src = &a;
    for (int q = 0; q < 2; q++) {
        const SDa* dst = ((2 - 1 - q) % 2 == 0) ? &b : &T;
        k_transform_1d<<<blocks_for(dst->pts() * a.e[0] * a.e[1]), kBlock, 0, s->stream>>>(*src, *dst, M, s->n,
                                                                                         dims[q], -1);
        src = dst;
    }
}

// boundaries(comm, BC_d, U, alignment, a_dim) for the induction's FV arrays
void fv_bc(spdk_induction* s, const FVa& U, int dim, int alignment, int a_dim) {
    const int shift = alignment * (a_dim == dim);
    // BC_x / BC_y / BC_z extents (src/induction_ader.hpp:255-257)
    int B[3] = {s->fvn[0] + 1, s->fvn[1] + 1, s->fvn[2] + 1};
    B[dim] = kNGH;
    const int Lx = B[0] - (a_dim == 0) * (alignment - shift);
    const int Ly = B[1] - (a_dim == 1) * (alignment - shift);
    const int Lz = B[2] - (a_dim == 2) * (alignment - shift);
    const long long cnt = (long long)Lz * Ly * Lx * U.e[0];
    const unsigned epoch = ++s->epoch;
    for (int pass = 0; pass < 3; pass++)
        k_fv_bc<<<blocks_for(cnt), kBlock, 0, s->stream>>>(U, s->bcbuf, s->bcwin, epoch, dim, s->cfg.bc[dim],
                                                          s->fvn[dim], shift, Lx, Ly, Lz, pass);
}

// FV_Update_solution (src/induction_ader.hpp:530-576)
int fv_update(spdk_induction* s) {
    cudaStream_t st = s->stream;
    // Transform_to_cv
    for (int d = 0; d < 3; d++) transform_2d(s, s->Bfp[d], s->Bcv[d], s->Tfp[d], s->sp_to_cv, d);
    k_B_cv_from_cf<<<blocks_for(s->Bcv[0].pts()), kBlock, 0, st>>>(s->Bo4, s->Bcv[0], s->Bcv[1], s->Bcv[2],
                                                                   s->fp_to_cv, s->nf);
    const int mask = 0b0111;
    const bool use_sed = s->cfg.sed && s->cfg.p > 1;
    for (int t = 0; t < s->nt; t++) {
        for (int d = 0; d < 3; d++)
            k_edge_integral<<<blocks_for(s->Ecc[d].pts() * 2), kBlock, 0, st>>>(s->Ecc[d], s->Efv[d], s->sp_to_cv,
                                                                               s->n, t, d);
        // with the fallback applied, the slice-start faces are kept: the
        // candidate update below is what the detection judges, and the
        // faces are updated again from the kept ones once the EMFs of
        // troubled edges are replaced
        const bool apply = s->cfg.fallback_apply != 0;
        auto face_update = [&]() {
            for (int d = 0; d < 3; d++) {
                const int e1 = (d + 1) % 3, e2 = (d + 2) % 3;
                const int dim1 = (d + 1) % 3, dim2 = (d + 2) % 3;
                k_fv_update_B<<<blocks_for(s->Bcv[d].pts()), kBlock, 0, st>>>(s->Bnew[d], s->Bold[d], s->Bcv[d],
                                                                             s->Efv[e1], s->Efv[e2], s->fvf[dim1],
                                                                             s->fvf[dim2], s->wt, s->dt, t, d, 1);
            }
        };
        auto copy_faces = [&](SDa* dst, SDa* src) {
            for (int d = 0; d < 3; d++)
                cudaMemcpyAsync(dst[d].p, src[d].p, (size_t)src[d].pts() * sizeof(double), cudaMemcpyDeviceToDevice,
                                st);
        };
        if (apply) copy_faces(s->Bsave, s->Bcv);
        face_update();
        k_B_cv_from_cf<<<blocks_for(s->Bcv[0].pts()), kBlock, 0, st>>>(s->Bn4, s->Bcv[0], s->Bcv[1], s->Bcv[2],
                                                                       s->fp_to_cv, s->nf);
        // apply_fv_boundaries (:614-643)
        for (int d = 0; d < 3; d++) {
            fv_bc(s, s->Bo4, d, 0, 0);
            for (int c = 0; c < 3; c++) fv_bc(s, s->Bold[c], d, 1, c);
        }
        // detect_troubles(B_new, B_old, troubles, alphas, ..., PAD = 0, 0b0111)
        const FVa& U = s->Bo4;
        k_ind_nad<<<blocks_for(U.cells()), kBlock, 0, st>>>(s->Bn4, U, s->troubles, s->cfg.nad_tolerance,
                                                            s->cfg.nad_moore, s->cfg.nad_delta, mask);
        if (use_sed)
            for (int d = 0; d < 3; d++)
                k_ind_sed<<<blocks_for(U.cells()), kBlock, 0, st>>>(s->Bn4, s->alpha[d], s->fvc[d], s->fvf[d], d, mask);
        k_ind_relax<<<blocks_for(U.cells()), kBlock, 0, st>>>(s->troubles, s->alpha[0], s->alpha[1], s->alpha[2], mask,
                                                              use_sed ? 1 : 0);
        if (apply) {
            // upwind EMFs on the troubled edges (slice-start FV faces, ghosts
            // filled above), then the face update of the kept slice-start
            // faces from the blended edges
            for (int d = 0; d < 3; d++) {
                const int dim1 = (d + 1) % 3, dim2 = (d + 2) % 3;
                const long long edges = (long long)s->Efv[d].cells();
                k_ind_fallback_emf<<<blocks_for(edges), kBlock, 0, st>>>(s->Efv[d], s->Bold[dim1], s->Bold[dim2],
                                                                        s->troubles, d, s->fvn[0], s->fvn[1],
                                                                        s->fvn[2]);
            }
            copy_faces(s->Bcv, s->Bsave);
            face_update();
        }
    }
    // Transform_to_sp
    for (int d = 0; d < 3; d++) transform_2d(s, s->Bcv[d], s->Bfp[d], s->Tfp[d], s->cv_to_sp, d);
    return launched("induction: FV update");
}

void copy_ader(spdk_induction* s) {
    for (int d = 0; d < 3; d++) {
        const size_t bytes = (size_t)s->Bfp[d].pts() * sizeof(double);
        for (int t = 0; t < s->nt; t++)
            cudaMemcpyAsync(s->Bader[d].p + (size_t)t * s->Bfp[d].pts(), s->Bfp[d].p, bytes, cudaMemcpyDeviceToDevice,
                            s->stream);
    }
}

int enqueue_step(spdk_induction* s) {
    int rc = 0;
    if (s->cfg.integrator == SPDK_INTEGRATOR_RK) {
        // RK_step (src/induction_ader.hpp:374-391)
        for (int d = 0; d < 3; d++)
            cudaMemcpyAsync(s->B0[d].p, s->Bfp[d].p, (size_t)s->Bfp[d].pts() * sizeof(double),
                            cudaMemcpyDeviceToDevice, s->stream);
        for (int st = 0; st < s->nstages; st++) {
            copy_ader(s);
            if ((rc = solve_E(s))) return rc;
            rc = s->cfg.fallback ? fv_update(s) : update_B(s, false);
            if (rc) return rc;
            if (s->rk_a[st] > 0)
                for (int d = 0; d < 3; d++)
                    k_combine<<<blocks_for(s->Bfp[d].pts()), kBlock, 0, s->stream>>>(s->Bfp[d], s->B0[d], s->rk_a[st]);
        }
    } else {
        // ADER_step (:362-372)
        copy_ader(s);
        for (int a = 0; a < s->nt; a++) {
            if ((rc = solve_E(s))) return rc;
            if (a < s->nt - 1 && (rc = update_B(s, true))) return rc;
        }
        rc = s->cfg.fallback ? fv_update(s) : update_B(s, false);
        if (rc) return rc;
    }
    return launched("induction: step");
}

}  // namespace

extern "C" {

int spdk_induction_create(const spdk_induction_config* cfg, spdk_induction** out) {
    if (!cfg || !out) return fail(SPDK_E_ARG, "null argument");
    *out = nullptr;
    const spdk_induction_config& c = *cfg;
    if (c.p < 1 || c.p > kMaxP) return fail(SPDK_E_ARG, "p must be in 1..7");
    if (c.fallback_apply && !c.fallback) return fail(SPDK_E_ARG, "fallback_apply needs fallback = 1");
    for (int d = 0; d < 3; d++) {
        if (c.N[d] < 2) return fail(SPDK_E_ARG, "the induction solver needs three active directions (nx1, nx2, nx3 > 1)");
        if (c.bc[d] < 0 || c.bc[d] > 2) return fail(SPDK_E_ARG, "unknown boundary type");
        if (!(c.L[d] > 0)) return fail(SPDK_E_ARG, "box lengths must be positive");
    }
    const bool ader = c.integrator == SPDK_INTEGRATOR_ADER;
    if (!ader && c.integrator != SPDK_INTEGRATOR_RK) return fail(SPDK_E_ARG, "unknown integrator");
    if (!ader && (c.rk_order < 1 || c.rk_order > 3)) return fail(SPDK_E_ARG, "rk_order must be 1, 2 or 3");
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(SPDK_E_CUDA, "cudaSetDevice failed");

    spdk_induction* s = new spdk_induction;
    s->cfg = c;
    build_matrices(c.p, ader, &s->m);
    s->n = c.p + 1;
    s->nf = c.p + 2;
    s->nt = ader ? s->n : 1;
    s->nstages = ader ? 1 : c.rk_order;
    if (c.rk_order == 2 && !ader) s->rk_a[1] = 0.5;
    if (c.rk_order == 3 && !ader) { s->rk_a[1] = 0.75; s->rk_a[2] = 1.0 / 3.0; }
    for (int d = 0; d < 3; d++) {
        build_axis(c.N[d], c.p, c.L[d], s->m.x_fp, true, &s->ax[d]);
        s->fvn[d] = s->ax[d].fvn;
    }
    const int n = s->n, nf = s->nf, nt = s->nt;
    int rc = 0;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) rc = fail(SPDK_E_CUDA, "stream");
    // matrices
    if (!rc) rc = upload(s, &s->sp_to_fp, s->m.sp_to_fp, (size_t)nf * n);
    if (!rc) rc = upload(s, &s->dfp_to_sp, s->m.dfp_to_sp, (size_t)n * nf);
    if (!rc) rc = upload(s, &s->sp_to_cv, s->m.sp_to_cv, (size_t)n * n);
    if (!rc) rc = upload(s, &s->cv_to_sp, s->m.cv_to_sp, (size_t)n * n);
    if (!rc) rc = upload(s, &s->fp_to_cv, s->m.fp_to_cv, (size_t)n * nf);
    if (!rc) rc = upload(s, &s->invader, s->m.invader, (size_t)nt * nt);
    if (!rc) rc = upload(s, &s->wt, s->m.wt, (size_t)nt);
    for (int d = 0; d < 3 && !rc; d++) {
        rc = upload(s, &s->fvf[d], s->ax[d].fv_faces.data(), s->ax[d].fv_faces.size());
        if (!rc) rc = upload(s, &s->fvc[d], s->ax[d].fv_centers.data(), s->ax[d].fv_centers.size());
    }
    // face fields (B_d at the flux points of d), their slices and stage copies
    for (int d = 0; d < 3 && !rc; d++) {
        const int ez = ext_of(s, d == 2), ey = ext_of(s, d == 1), ex = ext_of(s, d == 0);
        rc = make_sd(s, &s->Bfp[d], 1, 1, ez, ey, ex);
        if (!rc) rc = make_sd(s, &s->Bader[d], nt, 1, ez, ey, ex);
        if (!rc && !ader) rc = make_sd(s, &s->B0[d], 1, 1, ez, ey, ex);
        // edge fields: E_d at the flux points of the two other directions
        if (!rc) rc = make_sd(s, &s->Ecc[d], nt, kEVars, ext_of(s, d != 2), ext_of(s, d != 1), ext_of(s, d != 0));
        if (!rc && c.fallback) {
            rc = make_sd(s, &s->Bcv[d], 1, 1, ez, ey, ex);
            if (!rc) rc = make_sd(s, &s->Tfp[d], 1, 1, ez, ey, ex);
            if (!rc && c.fallback_apply) rc = make_sd(s, &s->Bsave[d], 1, 1, ez, ey, ex);
            if (!rc) rc = make_fv(s, &s->Bold[d], 1, d == 2, d == 1, d == 0);
            if (!rc) rc = make_fv(s, &s->Bnew[d], 1, d == 2, d == 1, d == 0);
            if (!rc) rc = make_fv(s, &s->Efv[d], 1, d != 2, d != 1, d != 0);
            if (!rc) rc = make_fv(s, &s->alpha[d], 4, 0, 0, 0);
        }
    }
    if (!rc) rc = make_sd(s, &s->B2, 1, 4, n, n, n);
    if (!rc && c.fallback) {
        rc = make_fv(s, &s->Bo4, 4, 0, 0, 0);
        if (!rc) rc = make_fv(s, &s->Bn4, 4, 0, 0, 0);
        if (!rc) rc = make_fv(s, &s->troubles, 4, 0, 0, 0);
        int mx = 0;
        for (int d = 0; d < 3; d++) mx = std::max(mx, s->fvn[d] + 1);
        if (!rc) rc = dalloc(s, &s->bcbuf, (size_t)2 * 4 * mx * mx * kNGH);
        // one claim word per element of the largest FV array (4 slots)
        double* w = nullptr;
        if (!rc) rc = dalloc(s, &w, (size_t)4 * mx * mx * mx);
        s->bcwin = reinterpret_cast<unsigned long long*>(w);
    }
    if (!rc) {
        // initial condition (src/induction_ader.hpp:168-181): A at the edge
        // points, B = curl A by rotational_a_to_b over every element
        const int Nz = c.N[2] + 2, Ny = c.N[1] + 2, Nx = c.N[0] + 2;
        const Axis &X = s->ax[0], &Y = s->ax[1], &Z = s->ax[2];
        auto faces = [&](const Axis& a, int e, int q) { return a.sd_faces[(size_t)e * nf + q]; };
        auto centers = [&](const Axis& a, int e, int q) { return a.sd_centers[(size_t)e * n + q]; };
        HostSD Ax(1, 1, Nz, Ny, Nx, nf, nf, n), Ay(1, 1, Nz, Ny, Nx, nf, n, nf), Az(1, 1, Nz, Ny, Nx, n, nf, nf);
        for (int k = 0; k < Nz; k++)
            for (int j = 0; j < Ny; j++)
                for (int i = 0; i < Nx; i++) {
                    for (int kk = 0; kk < nf; kk++)
                        for (int jj = 0; jj < nf; jj++)
                            for (int ii = 0; ii < n; ii++)
                                Ax.at(0, 0, k, j, i, kk, jj, ii) =
                                    magnetic_loop(0, centers(X, i, ii), faces(Y, j, jj), faces(Z, k, kk));
                    for (int kk = 0; kk < nf; kk++)
                        for (int jj = 0; jj < n; jj++)
                            for (int ii = 0; ii < nf; ii++)
                                Ay.at(0, 0, k, j, i, kk, jj, ii) =
                                    magnetic_loop(1, faces(X, i, ii), centers(Y, j, jj), faces(Z, k, kk));
                    for (int kk = 0; kk < n; kk++)
                        for (int jj = 0; jj < nf; jj++)
                            for (int ii = 0; ii < nf; ii++)
                                Az.at(0, 0, k, j, i, kk, jj, ii) =
                                    magnetic_loop(2, faces(X, i, ii), faces(Y, j, jj), centers(Z, k, kk));
                }
        const double* da = s->m.dfp_to_sp;  // (n, nf)
        HostSD* A[3] = {&Ax, &Ay, &Az};
        const double hh[3] = {X.h, Y.h, Z.h};
        for (int d = 0; d < 3 && !rc; d++) {
            // src/induction.cpp:93-121: B_d = d1 A_{d+2} / h1 - d2 A_{d+1} / h2
            HostSD& A1 = *A[(d + 1) % 3];
            HostSD& A2 = *A[(d + 2) % 3];
            const double d1 = hh[(d + 1) % 3], d2 = hh[(d + 2) % 3];
            const int ez = ext_of(s, d == 2), ey = ext_of(s, d == 1), ex = ext_of(s, d == 0);
            const int q = d == 0 ? ex : (d == 1 ? ey : ez);
            HostSD B(1, 1, Nz, Ny, Nx, ez, ey, ex);
            for (int k = 0; k < Nz; k++)
                for (int j = 0; j < Ny; j++)
                    for (int i = 0; i < Nx; i++)
                        for (int kk = 0; kk < ez; kk++)
                            for (int jj = 0; jj < ey; jj++)
                                for (int ii = 0; ii < ex; ii++) {
                                    double d1a2 = 0, d2a1 = 0;
                                    for (int ll = 0; ll < q; ll++) {
                                        if (d == 0) {
                                            d1a2 += A2.at(0, 0, k, j, i, kk, ll, ii) * da[jj * nf + ll];
                                            d2a1 += A1.at(0, 0, k, j, i, ll, jj, ii) * da[kk * nf + ll];
                                        } else if (d == 1) {
                                            d1a2 += A2.at(0, 0, k, j, i, ll, jj, ii) * da[kk * nf + ll];
                                            d2a1 += A1.at(0, 0, k, j, i, kk, jj, ll) * da[ii * nf + ll];
                                        } else {
                                            d1a2 += A2.at(0, 0, k, j, i, kk, jj, ll) * da[ii * nf + ll];
                                            d2a1 += A1.at(0, 0, k, j, i, kk, ll, ii) * da[jj * nf + ll];
                                        }
                                    }
                                    B.at(0, 0, k, j, i, kk, jj, ii) = d1a2 / d1 - d2a1 / d2;
                                }
            if (cudaMemcpy(s->Bfp[d].p, B.v.data(), B.v.size() * sizeof(double), cudaMemcpyHostToDevice) !=
                cudaSuccess)
                rc = fail(SPDK_E_CUDA, "induction: upload B");
        }
        // Induction_compute_dt (src/induction.cpp:52-91): min over active
        // points of cfl dx_min / |v| / n, capped by the resistive limit
        double red = 1.7976931348623157e308;
        for (long long q = 0; q < (long long)c.N[0] * c.N[1] * c.N[2] * n * n * n; q++) {
            double v_max = 0, dx_min = 1;
            v_max += std::fabs(velocity(0));
            dx_min = std::min(dx_min, X.h);
            v_max += std::fabs(velocity(1));
            dx_min = std::min(dx_min, Y.h);
            v_max += std::fabs(velocity(2));
            dx_min = std::min(dx_min, Z.h);
            const double dt_min = c.cfl * dx_min / v_max / n;
            red = red < dt_min ? red : dt_min;
        }
        double Dt = 1E6;
        if (c.nu > 0.0) Dt = 0.5 * c.cfl * (X.h * X.h / c.nu) / (3) / (3) / (c.p + 1) / (c.p + 1);
        s->Dt = std::min(red, Dt);
        s->dt = s->Dt;
        cudaError_t e = cudaDeviceSynchronize();
        if (!rc && e != cudaSuccess) rc = fail(SPDK_E_CUDA, std::string("induction set-up: ") + cudaGetErrorString(e));
    }
    if (rc) {
        release(s);
        delete s;
        return rc;
    }
    *out = s;
    return 0;
}

int spdk_induction_destroy(spdk_induction* s) {
    if (!s) return 0;
    if (s->stream) cudaStreamSynchronize(s->stream);
    release(s);
    delete s;
    return 0;
}

int spdk_induction_get_dt(spdk_induction* s, double* dt) {
    if (!s || !dt) return fail(SPDK_E_ARG, "null argument");
    *dt = s->dt;
    return 0;
}

int spdk_induction_set_dt(spdk_induction* s, double dt) {
    if (!s) return fail(SPDK_E_ARG, "null argument");
    if (!(dt > 0)) return fail(SPDK_E_ARG, "dt must be positive");
    s->dt = dt;
    return 0;
}

int spdk_induction_step(spdk_induction* s) {
    if (!s) return fail(SPDK_E_ARG, "null argument");
    int rc = enqueue_step(s);
    s->dt = s->Dt;
    return rc;
}

int spdk_induction_evolve(spdk_induction* s, double t_end, double dt_output, long long* steps, double* t_out) {
    if (!s) return fail(SPDK_E_ARG, "null argument");
    double t = 0;
    long long ns = 0;
    const bool outputs = dt_output > 0;
    double t_output = dt_output;
    while (t < t_end) {
        const double dt = s->dt;
        int rc = enqueue_step(s);
        if (rc) return rc;
        t += dt;
        ns++;
        s->dt = s->Dt;
        if (outputs) {
            if (t >= t_output) t_output = t + dt_output;
            if (t + s->dt > t_output) s->dt = t_output - t;
        }
    }
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) return fail(SPDK_E_CUDA, "induction: evolve");
    if (steps) *steps = ns;
    if (t_out) *t_out = t;
    return 0;
}

int spdk_induction_field_size(spdk_induction* s, int field, size_t* count) {
    if (!s || !count) return fail(SPDK_E_ARG, "null argument");
    switch (field) {
    case SPDK_IND_FIELD_B2_CV: *count = (size_t)s->B2.pts() * 4; return 0;
    case SPDK_IND_FIELD_TROUBLES:
        if (!s->cfg.fallback) return fail(SPDK_E_STATE, "fallback is off");
        *count = (size_t)s->troubles.cells() * 4;
        return 0;
    case SPDK_IND_FIELD_BX_FP:
    case SPDK_IND_FIELD_BY_FP:
    case SPDK_IND_FIELD_BZ_FP: *count = (size_t)s->Bfp[field - SPDK_IND_FIELD_BX_FP].pts(); return 0;
    }
    return fail(SPDK_E_ARG, "unknown field");
}

int spdk_induction_read(spdk_induction* s, int field, double* host, size_t count) {
    if (!s || !host) return fail(SPDK_E_ARG, "null argument");
    size_t need = 0;
    int rc = spdk_induction_field_size(s, field, &need);
    if (rc) return rc;
    if (count != need) return fail(SPDK_E_ARG, "count must be " + std::to_string(need));
    const double* src = nullptr;
    if (field == SPDK_IND_FIELD_B2_CV) {
        // compute_B2_cv (src/induction.cpp:420-455), as Write_outputs does
        k_B2_cv<<<blocks_for(s->B2.pts()), kBlock, 0, s->stream>>>(s->B2, s->Bfp[0], s->Bfp[1], s->Bfp[2], s->fp_to_cv,
                                                                   s->sp_to_cv, s->n, s->nf);
        if ((rc = launched("induction: compute_B2_cv"))) return rc;
        src = s->B2.p;
    } else if (field == SPDK_IND_FIELD_TROUBLES) {
        src = s->troubles.p;
    } else {
        src = s->Bfp[field - SPDK_IND_FIELD_BX_FP].p;
    }
    if (cudaMemcpyAsync(host, src, need * sizeof(double), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess)
        return fail(SPDK_E_CUDA, "induction: read");
    return 0;
}

}  // extern "C"
