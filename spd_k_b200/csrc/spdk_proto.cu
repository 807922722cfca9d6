// Prototype-level C ABI: the free functions of the reference's
// src/prototypes.hpp on device arrays in the reference's own layout
// (declarations and argument meaning in include/spdk_proto.h).
//
// These are the drop-in for a host that drives the reference's functions one
// by one; the fused per-pass kernels (spdk_kernels.cuh, spdk_fallback.cuh)
// are the fast path. Each kernel maps one thread to one output point (or one
// face / one FV cell) and evaluates the reference's operations in the
// reference's order, so with -fmad=false the results are bit-identical to
// the reference's CPU build. Where the reference updates an array variable
// by variable in place (the gravity source of update_prediction and of
// fv_update_solution reads the already-updated density/momentum of the same
// point), one thread owns the point and walks the variables in the same
// order, which reproduces that behaviour exactly.
#include <cuda_runtime.h>

#include <string>

#include "spdk.h"
#include "spdk_physics.cuh"
#include "spdk_proto.h"
#include "spdk_reflayout.cuh"

namespace {

using namespace spdk;

constexpr int kVX = 1, kVY = 2, kVZ = 3, kVP = 4;  // reference slots (src/define.hpp:36-44)
constexpr int kNV = 5;                             // physics slots
constexpr int kNGH = 2;                            // FV ghost layers (src/define.hpp)

struct Cfg {
    int p, act[3];
    double gm, cfl, g[3], tol;
    int nad_delta, nad_moore, sed, grav;
};

SDa sd(const spdk_sd* a) {
    SDa r{a->data, {}};
    for (int q = 0; q < 8; q++) r.e[q] = a->ext[q];
    return r;
}
FVa fv(const spdk_fv* a) {
    FVa r{a->data, {}};
    for (int q = 0; q < 4; q++) r.e[q] = a->ext[q];
    return r;
}
Cfg cfgof(const spdk_proto_cfg* c) {
    Cfg r{};
    r.p = c->p;
    for (int d = 0; d < 3; d++) {
        r.act[d] = c->active[d] ? 1 : 0;
        r.g[d] = c->g[d];
    }
    r.gm = c->gamma;
    r.cfl = c->cfl;
    r.tol = c->nad_tolerance;
    r.nad_delta = c->nad_delta;
    r.nad_moore = c->nad_moore;
    r.sed = c->sed;
    r.grav = (c->g[0] != 0.0 || c->g[1] != 0.0 || c->g[2] != 0.0) ? 1 : 0;
    return r;
}

bool ok_sd(const spdk_sd* a) {
    if (!a || !a->data) return false;
    for (int q = 0; q < 8; q++)
        if (a->ext[q] < 1) return false;
    return true;
}
bool ok_fv(const spdk_fv* a) {
    if (!a || !a->data) return false;
    for (int q = 0; q < 4; q++)
        if (a->ext[q] < 1) return false;
    return true;
}
bool ok_mat(const spdk_mat* m) { return m && m->data && m->rows > 0 && m->cols > 0; }
bool ok_vec(const spdk_vec* v) { return v && v->data && v->n > 0; }

// src/transforms.cpp:16-27: gravity source of one variable at one point
__device__ __forceinline__ double grav_src(const SDa& U, const Cfg& C, int var, int t, int k, int j, int i, int kk,
                                           int jj, int ii) {
    if (var == kVX) return U.at(t, 0, k, j, i, kk, jj, ii) * C.g[0];
    if (var == kVY) return U.at(t, 0, k, j, i, kk, jj, ii) * C.g[1];
    if (var == kVZ) return U.at(t, 0, k, j, i, kk, jj, ii) * C.g[2];
    if (var == kVP)
        return U.at(t, kVX, k, j, i, kk, jj, ii) * C.g[0] + U.at(t, kVY, k, j, i, kk, jj, ii) * C.g[1] +
               U.at(t, kVZ, k, j, i, kk, jj, ii) * C.g[2];
    return 0.0;
}

// flux divergence of slice t at one solution point (src/transforms.cpp:297-309)
__device__ __forceinline__ double divergence(const SDa& Fx, const SDa& Fy, const SDa& Fz, const double* D, int nfc,
                                             const Cfg& C, int t, int var, int k, int j, int i, int kk, int jj,
                                             int ii, double dx, double dy, double dz) {
    const int q = Fx.e[7];
    double dudt = 0;
    for (int ll = 0; ll < q; ll++) {
        if (C.act[0]) dudt += Fx.at(t, var, k, j, i, kk, jj, ll) * D[ii * nfc + ll] / dx;
        if (C.act[1]) dudt += Fy.at(t, var, k, j, i, kk, ll, ii) * D[jj * nfc + ll] / dy;
        if (C.act[2]) dudt += Fz.at(t, var, k, j, i, ll, jj, ii) * D[kk * nfc + ll] / dz;
    }
    return dudt;
}

// src/transforms.cpp:263-325
__global__ void k_update_prediction(SDa U, SDa Ua, SDa Fx, SDa Fy, SDa Fz, const double* __restrict__ D, int nfc,
                                    const double* __restrict__ inv, const double* __restrict__ w, double dt,
                                    double dx, double dy, double dz, Cfg C) {
    const int nader = Fx.e[0];
    const long long n = U.pts();
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
        int c[6];
        point_of(U, o, c);
        const int k = c[0], j = c[1], i = c[2], kk = c[3], jj = c[4], ii = c[5];
        for (int var = 0; var < kNV; var++) {
            double dudt[16];
            const double u_old = U.at(0, var, k, j, i, kk, jj, ii);
            for (int t = 0; t < nader; t++) {
                dudt[t] = divergence(Fx, Fy, Fz, D, nfc, C, t, var, k, j, i, kk, jj, ii, dx, dy, dz);
                if (C.grav) dudt[t] -= grav_src(Ua, C, var, t, k, j, i, kk, jj, ii);
            }
            for (int t = 0; t < nader; t++) {
                double du = 0;
                for (int ll = 0; ll < nader; ll++) du += dudt[ll] * inv[t * nader + ll] * w[ll] * dt;
                Ua.at(t, var, k, j, i, kk, jj, ii) = u_old - du;
            }
        }
    }
}

// src/transforms.cpp:327-374
__global__ void k_update_solution(SDa U, SDa Ua, SDa Fx, SDa Fy, SDa Fz, const double* __restrict__ D, int nfc,
                                  const double* __restrict__ w, double dt, double dx, double dy, double dz, Cfg C) {
    const int nader = Fx.e[0];
    const long long n = U.pts();
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
        int c[6];
        point_of(U, o, c);
        const int k = c[0], j = c[1], i = c[2], kk = c[3], jj = c[4], ii = c[5];
        for (int var = 0; var < kNV; var++) {
            double du = 0;
            for (int t = 0; t < nader; t++) {
                double dudt = divergence(Fx, Fy, Fz, D, nfc, C, t, var, k, j, i, kk, jj, ii, dx, dy, dz);
                if (C.grav) dudt -= grav_src(Ua, C, var, t, k, j, i, kk, jj, ii);
                du += dudt * w[t] * dt;
            }
            U.at(0, var, k, j, i, kk, jj, ii) -= du;
        }
    }
}

// ---- pointwise physics: src/hydro.cpp:34-206 -------------------------------
// mode 0: primitives, 1: conservatives, 2: fluxes along slot v1
__global__ void k_pointwise(double* __restrict__ in, int in_nv, double* __restrict__ out, int out_nv, long long npts,
                            int nt, int mode, int v1, double gm) {
    const long long n = npts * nt;
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
        const long long t = o / npts, q = o % npts;
        double a[kNV], b[kNV], w[kNV];
#pragma unroll
        for (int v = 0; v < kNV; v++) a[v] = in[(t * in_nv + v) * npts + q];
        if (mode == 0) primitives<3>(a, b, gm);
        else if (mode == 1) conservatives<3>(a, b, gm);
        else {
            primitives<3>(a, w, gm);
            euler_flux<3>(a, w, b, v1 - 1);
        }
#pragma unroll
        for (int v = 0; v < kNV; v++) out[(t * out_nv + v) * npts + q] = b[v];
    }
}

// src/hydro.cpp:208-262 over active points; min via the ordered bit pattern
// of positive doubles
__global__ void k_dt_arm(unsigned long long* out) { *out = 0x7FEFFFFFFFFFFFFFULL; }
__global__ void k_compute_dt(SDa W, double dx, double dy, double dz, double nu, Cfg C, unsigned long long* out) {
    const int gz = C.act[2], gy = C.act[1], gx = C.act[0];
    const int Nz = W.e[2] - 2 * gz, Ny = W.e[3] - 2 * gy, Nx = W.e[4] - 2 * gx;
    const long long n = (long long)Nz * Ny * Nx * W.e[5] * W.e[6] * W.e[7];
    const int px = W.e[7];
    double red = 1.7976931348623157e308;
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
        long long r = o;
        const int ii = (int)(r % W.e[7]); r /= W.e[7];
        const int jj = (int)(r % W.e[6]); r /= W.e[6];
        const int kk = (int)(r % W.e[5]); r /= W.e[5];
        const int i = gx + (int)(r % Nx); r /= Nx;
        const int j = gy + (int)(r % Ny); r /= Ny;
        const int k = gz + (int)r;
        const double cs = sound_speed(W.at(0, 0, k, j, i, kk, jj, ii), W.at(0, kVP, k, j, i, kk, jj, ii), C.gm);
        double cmax = 0, dxmin = 1;
        if (C.act[0]) { cmax += (fabs(W.at(0, kVX, k, j, i, kk, jj, ii)) + cs); dxmin = smin(dxmin, dx); }
        if (C.act[1]) { cmax += (fabs(W.at(0, kVY, k, j, i, kk, jj, ii)) + cs); dxmin = smin(dxmin, dy); }
        if (C.act[2]) { cmax += (fabs(W.at(0, kVZ, k, j, i, kk, jj, ii)) + cs); dxmin = smin(dxmin, dz); }
        double dtm = C.cfl * dxmin / cmax / px;
        if (nu > 0.0) {
            // src/hydro.cpp:245-254: diffusion limit on the sub-cell spacing
            const double dx_sub = dxmin / px;
            const double dt_visc = 0.25 * C.cfl * dx_sub * dx_sub / nu;
            dtm = dtm < dt_visc ? dtm : dt_visc;
        }
        red = red < dtm ? red : dtm;
    }
    for (int s = 16; s > 0; s >>= 1) red = smin(red, __shfl_xor_sync(0xffffffffu, red, s));
    if ((threadIdx.x & 31) == 0) atomicMin(out, (unsigned long long)__double_as_longlong(red));
}

// ---- SD boundaries and Riemann solver: src/boundary.cpp:48-113, src/hydro.cpp:368-418
__global__ void k_riemann(SDa U, SDa F, int D, int v1, double gm, int viscous) {
    const int Nx = U.e[4] - (D == 0), Ny = U.e[3] - (D == 1), Nz = U.e[2] - (D == 2);
    const int px = D == 0 ? 1 : U.e[7], py = D == 1 ? 1 : U.e[6], pz = D == 2 ? 1 : U.e[5];
    const int n = choose(D, U.e[7], U.e[6], U.e[5]);
    const long long cnt = (long long)Nz * Ny * Nx * pz * py * px * U.e[0];
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < cnt; o += (long long)gridDim.x * blockDim.x) {
        long long r = o;
        const int t = (int)(r % U.e[0]); r /= U.e[0];
        const int ii = (int)(r % px); r /= px;
        const int jj = (int)(r % py); r /= py;
        const int kk = (int)(r % pz); r /= pz;
        const int i = (int)(r % Nx); r /= Nx;
        const int j = (int)(r % Ny); r /= Ny;
        const int k = (int)r;
        const int l = choose(D, i, j, k);
        const int kL = D == 2 ? l : k, jL = D == 1 ? l : j, iL = D == 0 ? l : i;
        const int kR = D == 2 ? l + 1 : k, jR = D == 1 ? l + 1 : j, iR = D == 0 ? l + 1 : i;
        const int kkL = D == 2 ? n - 1 : kk, jjL = D == 1 ? n - 1 : jj, iiL = D == 0 ? n - 1 : ii;
        const int kkR = D == 2 ? 0 : kk, jjR = D == 1 ? 0 : jj, iiR = D == 0 ? 0 : ii;
        double uL[kNV], uR[kNV], f[kNV];
        for (int v = 0; v < kNV; v++) {
            uL[v] = U.at(t, v, kL, jL, iL, kkL, jjL, iiL);
            uR[v] = U.at(t, v, kR, jR, iR, kkR, jjR, iiR);
        }
        riemann_llf<3>(f, uL, uR, v1 - 1, gm);
        for (int v = 0; v < kNV; v++) {
            F.at(t, v, kL, jL, iL, kkL, jjL, iiL) = f[v];
            F.at(t, v, kR, jR, iR, kkR, jjR, iiR) = f[v];
        }
        if (viscous) {
            // central interface state, read only by the diffusive terms
            for (int v = 0; v < U.e[1]; v++) {
                const double a = U.at(t, v, kL, jL, iL, kkL, jjL, iiL), b = U.at(t, v, kR, jR, iR, kkR, jjR, iiR);
                const double m = wind_mix(a, b, 0.5);
                U.at(t, v, kL, jL, iL, kkL, jjL, iiL) = m;
                U.at(t, v, kR, jR, iR, kkR, jjR, iiR) = m;
            }
        }
    }
}

// ---- viscous terms: src/hydro.cpp:420-572 --------------------------------
// sd_rusanov_solver: F at both flux points of an interface += the
// wind-weighted (-0.5) mean of the two sides' viscous fluxes, the right
// element's value taken as the left state
__global__ void k_rusanov(SDa U, SDa F, int D) {
    const int Nx = U.e[4] - (D == 0), Ny = U.e[3] - (D == 1), Nz = U.e[2] - (D == 2);
    const int px = D == 0 ? 1 : U.e[7], py = D == 1 ? 1 : U.e[6], pz = D == 2 ? 1 : U.e[5];
    const int n = choose(D, U.e[7], U.e[6], U.e[5]);
    const long long cnt = (long long)Nz * Ny * Nx * pz * py * px * U.e[0];
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < cnt; o += (long long)gridDim.x * blockDim.x) {
        long long r = o;
        const int t = (int)(r % U.e[0]); r /= U.e[0];
        const int ii = (int)(r % px); r /= px;
        const int jj = (int)(r % py); r /= py;
        const int kk = (int)(r % pz); r /= pz;
        const int i = (int)(r % Nx); r /= Nx;
        const int j = (int)(r % Ny); r /= Ny;
        const int k = (int)r;
        const int l = choose(D, i, j, k);
        const int kL = D == 2 ? l : k, jL = D == 1 ? l : j, iL = D == 0 ? l : i;
        const int kR = D == 2 ? l + 1 : k, jR = D == 1 ? l + 1 : j, iR = D == 0 ? l + 1 : i;
        const int kkL = D == 2 ? n - 1 : kk, jjL = D == 1 ? n - 1 : jj, iiL = D == 0 ? n - 1 : ii;
        const int kkR = D == 2 ? 0 : kk, jjR = D == 1 ? 0 : jj, iiR = D == 0 ? 0 : ii;
        for (int v = 0; v < U.e[1]; v++) {
            const double a = U.at(t, v, kR, jR, iR, kkR, jjR, iiR), b = U.at(t, v, kL, jL, iL, kkL, jjL, iiL);
            const double f = wind_mix(a, b, -0.5);
            F.at(t, v, kL, jL, iL, kkL, jjL, iiL) += f;
            F.at(t, v, kR, jR, iR, kkR, jjR, iiR) += f;
        }
    }
}

// compute_gradient: dU = d/d(dim) of the flux-point values at the solution
// points of the active elements (one thread per output value)
__global__ void k_gradient(SDa U, SDa dU, double h, const double* __restrict__ M, int nfc, int dim, Cfg C) {
    const int gz = C.act[2], gy = C.act[1], gx = C.act[0];
    const int Nz = dU.e[2] - 2 * gz, Ny = dU.e[3] - 2 * gy, Nx = dU.e[4] - 2 * gx;
    const long long cnt = (long long)Nz * Ny * Nx * dU.e[5] * dU.e[6] * dU.e[7] * dU.e[0] * dU.e[1];
    const int q = choose(dim, dU.e[7], dU.e[6], dU.e[5]);
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < cnt; o += (long long)gridDim.x * blockDim.x) {
        long long r = o;
        const int var = (int)(r % dU.e[1]); r /= dU.e[1];
        const int t = (int)(r % dU.e[0]); r /= dU.e[0];
        const int ii = (int)(r % dU.e[7]); r /= dU.e[7];
        const int jj = (int)(r % dU.e[6]); r /= dU.e[6];
        const int kk = (int)(r % dU.e[5]); r /= dU.e[5];
        const int i = gx + (int)(r % Nx); r /= Nx;
        const int j = gy + (int)(r % Ny); r /= Ny;
        const int k = gz + (int)r;
        const int id = choose(dim, ii, jj, kk);
        double du = 0;
        for (int ll = 0; ll < q + 1; ll++) {
            const double u = dim == 0 ? U.at(t, var, k, j, i, kk, jj, ll)
                           : dim == 1 ? U.at(t, var, k, j, i, kk, ll, ii) : U.at(t, var, k, j, i, ll, jj, ii);
            du += u * M[id * nfc + ll] / h;
        }
        dU.at(t, var, k, j, i, kk, jj, ii) = du;
    }
}

// compute_viscous_flux: the gradients interpolated to every flux point of
// direction dim (ghost elements included), the viscous flux written over U
__global__ void k_viscous_flux(SDa U, SDa dU1, SDa dU2, SDa dU3, int v1, int v2, int v3,
                               const double* __restrict__ M, int mcols, double nu, double beta, int dim, double gm) {
    const int q = choose(dim, U.e[7], U.e[6], U.e[5]);
    const long long cnt = U.pts() * U.e[0];
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < cnt; o += (long long)gridDim.x * blockDim.x) {
        const int t = (int)(o % U.e[0]);
        int c[6];
        point_of(U, o / U.e[0], c);
        const int k = c[0], j = c[1], i = c[2], kk = c[3], jj = c[4], ii = c[5];
        const int id = choose(dim, ii, jj, kk);
        // momentum gradients by component (slot - 1) and the velocities
        double du1[3], du2[3], du3[3], w[3];
        for (int a = 0; a < 3; a++) {
            du1[a] = 0;
            du2[a] = 0;
            du3[a] = 0;
            for (int ll = 0; ll < q - 1; ll++) {
                const int nk = dim == 2 ? ll : kk, nj = dim == 1 ? ll : jj, ni = dim == 0 ? ll : ii;
                du1[a] += dU1.at(t, 1 + a, k, j, i, nk, nj, ni) * M[id * mcols + ll];
                du2[a] += dU2.at(t, 1 + a, k, j, i, nk, nj, ni) * M[id * mcols + ll];
                du3[a] += dU3.at(t, 1 + a, k, j, i, nk, nj, ni) * M[id * mcols + ll];
            }
        }
        const double rho = U.at(t, 0, k, j, i, kk, jj, ii);
        for (int a = 0; a < 3; a++) w[a] = U.at(t, 1 + a, k, j, i, kk, jj, ii) / rho;
        double fm[3], fe;
        viscous_flux(du1, du2, du3, w, v1 - 1, v2 - 1, v3 - 1, nu, beta, fm, fe);
        for (int v = 0; v < U.e[1]; v++)
            U.at(t, v, k, j, i, kk, jj, ii) = (v >= 1 && v <= 3) ? fm[v - 1] : (v == kVP ? fe : 0.0);
    }
}

// ---- FV boundaries: src/boundary.cpp:123-190 --------------------------------
// cell-centred arrays (the reference's alignment 0, shift 0): the ghost
// layers of direction dim over every transverse cell, ghost rows included
__global__ void k_boundaries_fv(FVa U, int dim, int type) {
    const int shift = 0;
    const int N = choose(dim, U.e[3], U.e[2], U.e[1]);
    const int Nx = dim == 0 ? kNGH : U.e[3];
    const int Ny = dim == 1 ? kNGH : U.e[2];
    const int Nz = dim == 2 ? kNGH : U.e[1];
    const long long cnt = (long long)Nz * Ny * Nx * U.e[0];
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < cnt; o += (long long)gridDim.x * blockDim.x) {
        long long r = o;
        const int var = (int)(r % U.e[0]); r /= U.e[0];
        const int i = (int)(r % Nx); r /= Nx;
        const int j = (int)(r % Ny); r /= Ny;
        const int k = (int)r;
        const int l = choose(dim, i, j, k);
        auto at = [&](int L) -> double& { return U.at(var, dim == 2 ? L : k, dim == 1 ? L : j, dim == 0 ? L : i); };
        double vL, vR;
        if (type == kPeriodic) { vL = at(N - 2 * kNGH + l - shift); vR = at(kNGH + l + shift); }
        else if (type == kGradfree) { vL = at(kNGH + l + shift); vR = at(N - 2 * kNGH + l - shift); }
        else {
            const double sgn = (var == 1 + dim) ? -1.0 : 1.0;
            vL = sgn * at(2 * kNGH - 1 - l);
            vR = sgn * at(N - kNGH - 1 - l);
        }
        at(l) = vL;
        at(N - kNGH + l) = vR;
    }
}

// ---- face integral: src/transforms.cpp:378-481 ------------------------------
__global__ void k_face_integral(SDa Ff, FVa F, SDa T, const double* __restrict__ M, int n, int dim, int tid,
                                Cfg C) {
    const int gz = C.act[2], gy = C.act[1], gx = C.act[0];
    const int Nx = Ff.e[4] + (dim == 0), Ny = Ff.e[3] + (dim == 1), Nz = Ff.e[2] + (dim == 2);
    const int px = Ff.e[7] - (dim == 0), py = Ff.e[6] - (dim == 1), pz = Ff.e[5] - (dim == 2);
    const int dim1 = choose(dim, 1, 2, 0), dim2 = choose(dim1, 1, 2, 0);
    const int q1 = choose(dim1, px, py, pz), q2 = choose(dim2, px, py, pz);
    const int a1 = C.act[dim1], a2 = C.act[dim2];
    const bool both = a1 && a2;
    const int ex = Nx - 2 * gx, ey = Ny - 2 * gy, ez = Nz - 2 * gz;
    const long long cnt = (long long)ez * ey * ex * pz * py * px * kNV;
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < cnt; o += (long long)gridDim.x * blockDim.x) {
        long long r = o;
        const int var = (int)(r % kNV); r /= kNV;
        const int ii = (int)(r % px); r /= px;
        const int jj = (int)(r % py); r /= py;
        const int kk = (int)(r % pz); r /= pz;
        const int i = gx + (int)(r % ex); r /= ex;
        const int j = gy + (int)(r % ey); r /= ey;
        const int k = gz + (int)r;
        const int I = ii + 2 * gx + (i - gx) * px;
        const int J = jj + 2 * gy + (j - gy) * py;
        const int K = kk + 2 * gz + (k - gz) * pz;
        const int id1 = choose(dim1, ii, jj, kk), id2 = choose(dim2, ii, jj, kk);
        double f = 0;
        int nid[3];
        if (!both) {
            for (int nn = 0; nn < q2; nn++) {
                nid[0] = ii; nid[1] = jj; nid[2] = kk;
                nid[dim2] = nn;
                for (int ll = 0; ll < q1; ll++) {
                    nid[dim1] = ll;
                    double sv = Ff.at(tid, var, k, j, i, nid[2], nid[1], nid[0]);
                    if (a1) sv *= M[id1 * n + ll];
                    if (a2) sv *= M[id2 * n + nn];
                    f += sv;
                }
            }
        } else {
            for (int nn = 0; nn < q2; nn++) {
                nid[0] = ii; nid[1] = jj; nid[2] = kk;
                nid[dim2] = nn;
                f += T.at(0, var, k, j, i, nid[2], nid[1], nid[0]) * M[id2 * n + nn];
            }
        }
        if (K < F.e[1] && J < F.e[2] && I < F.e[3]) F.at(var, K, J, I) = f;
    }
}

// ---- fv_update_solution: src/transforms.cpp:483-543 -------------------------
__global__ void k_fv_update(FVa Uo, FVa Un, SDa Ucv, FVa Fx, const double* __restrict__ xf, FVa Fy,
                            const double* __restrict__ yf, FVa Fz, const double* __restrict__ zf,
                            const double* __restrict__ w, int tid, double dt, int update, Cfg C) {
    const int gz = C.act[2], gy = C.act[1], gx = C.act[0];
    const int px = Ucv.e[7], py = Ucv.e[6], pz = Ucv.e[5];
    const int ex = Ucv.e[4] - 2 * gx, ey = Ucv.e[3] - 2 * gy, ez = Ucv.e[2] - 2 * gz;
    const long long cnt = (long long)ez * ey * ex * pz * py * px;
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < cnt; o += (long long)gridDim.x * blockDim.x) {
        long long r = o;
        const int ii = (int)(r % px); r /= px;
        const int jj = (int)(r % py); r /= py;
        const int kk = (int)(r % pz); r /= pz;
        const int i = gx + (int)(r % ex); r /= ex;
        const int j = gy + (int)(r % ey); r /= ey;
        const int k = gz + (int)r;
        const int I = ii + 2 * gx + (i - gx) * px;
        const int J = jj + 2 * gy + (j - gy) * py;
        const int K = kk + 2 * gz + (k - gz) * pz;
        for (int var = 0; var < kNV; var++) {
            double F = 0, h;
            Uo.at(var, K, J, I) = Ucv.at(0, var, k, j, i, kk, jj, ii);
            if (C.act[0]) {
                h = xf[I + 1] - xf[I];
                F += (Fx.at(var, K, J, I + 1) - Fx.at(var, K, J, I)) / h;
            }
            if (C.act[1]) {
                h = yf[J + 1] - yf[J];
                F += (Fy.at(var, K, J + 1, I) - Fy.at(var, K, J, I)) / h;
            }
            if (C.act[2]) {
                h = zf[K + 1] - zf[K];
                F += (Fz.at(var, K + 1, J, I) - Fz.at(var, K, J, I)) / h;
            }
            if (C.grav) F -= grav_src(Ucv, C, var, 0, k, j, i, kk, jj, ii);
            const double u_new = Uo.at(var, K, J, I) - w[tid] * dt * F;
            Un.at(var, K, J, I) = u_new;
            if (update) Ucv.at(0, var, k, j, i, kk, jj, ii) = u_new;
        }
    }
}

// ---- trouble detection: src/trouble_detection.cpp:35-290 --------------------
// cell (k, j, i) of the range that leaves `layers` ghost layers in every
// active direction (src/define.hpp:286-306)
__device__ __forceinline__ bool cell_in(const FVa& U, const Cfg& C, int layers, long long o, int* k, int* j, int* i) {
    const int lx = C.act[0] * layers, ly = C.act[1] * layers, lz = C.act[2] * layers;
    const int nx = U.e[3] - 2 * lx, ny = U.e[2] - 2 * ly, nz = U.e[1] - 2 * lz;
    if (nx <= 0 || ny <= 0 || nz <= 0 || o >= (long long)nx * ny * nz) return false;
    *i = lx + (int)(o % nx);
    o /= nx;
    *j = ly + (int)(o % ny);
    *k = lz + (int)(o / ny);
    return true;
}

// NAD over the one-layer range, smooth-extrema alphas over the two-layer range
__global__ void k_nad_sed(FVa Wn, FVa Wo, FVa Tr, FVa Ax, FVa Ay, FVa Az, const double* __restrict__ xc,
                          const double* __restrict__ xf, const double* __restrict__ yc, const double* __restrict__ yf,
                          const double* __restrict__ zc, const double* __restrict__ zf, int mask, int use_sed,
                          Cfg C) {
    const long long cnt = Wo.cells();
    const int ax = C.act[0], ay = C.act[1], az = C.act[2];
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < cnt; o += (long long)gridDim.x * blockDim.x) {
        int k, j, i;
        if (cell_in(Wo, C, 1, o, &k, &j, &i)) {
            for (int var = 0; var < kNV; var++) {
                if (!((mask >> var) & 1)) continue;
                const double un = Wn.at(var, k, j, i);
                double mx = Wo.at(var, k, j, i), mn = mx;
                if (C.nad_moore) {
                    for (int dk = -az; dk <= az; dk++)
                        for (int dj = -ay; dj <= ay; dj++)
                            for (int di = -ax; di <= ax; di++) {
                                const double u = Wo.at(var, k + dk, j + dj, i + di);
                                mx = smax(mx, u);
                                mn = smin(mn, u);
                            }
                } else {
                    for (int d = 0; d < 3; d++) {
                        if (!C.act[d]) continue;
                        const double uL = Wo.at(var, k - (d == 2), j - (d == 1), i - (d == 0));
                        const double uR = Wo.at(var, k + (d == 2), j + (d == 1), i + (d == 0));
                        mx = smax(smax(uL, mx), uR);
                        mn = smin(smin(uL, mn), uR);
                    }
                }
                if (C.nad_delta) {
                    const double eps = C.tol * (mx - mn);
                    mn -= eps;
                    mx += eps;
                } else {
                    mn -= fabs(mn) * C.tol;
                    mx += fabs(mx) * C.tol;
                }
                Tr.at(var, k, j, i) = (un > mx || un < mn) ? 1 : 0;
            }
        }
        if (use_sed && cell_in(Wo, C, 2, o, &k, &j, &i)) {
            for (int dim = 0; dim < 3; dim++) {
                if (!C.act[dim]) continue;
                const FVa& A = dim == 0 ? Ax : (dim == 1 ? Ay : Az);
                const double* c = dim == 0 ? xc : (dim == 1 ? yc : zc);
                const double* f = dim == 0 ? xf : (dim == 1 ? yf : zf);
                const int ox = dim == 0, oy = dim == 1, oz = dim == 2;
                const int l = choose(dim, i, j, k);
                for (int var = 0; var < kNV; var++) {
                    if (!((mask >> var) & 1)) continue;
                    const double u = Wn.at(var, k, j, i);
                    const double h = (c[l + 1] - c[l - 1]);
                    const double hp = (c[l + 2] - c[l]);
                    const double hm = (c[l] - c[l - 2]);
                    const double du = (Wn.at(var, k + oz, j + oy, i + ox) - Wn.at(var, k - oz, j - oy, i - ox)) / h;
                    const double dup = (Wn.at(var, k + 2 * oz, j + 2 * oy, i + 2 * ox) - u) / hp;
                    const double dum = (u - Wn.at(var, k - 2 * oz, j - 2 * oy, i - 2 * ox)) / hm;
                    const double d2u = (dup - dum) / (c[l + 1] - c[l - 1]);
                    const double dv = 0.5 * d2u * (f[l + 1] - f[l]);
                    A.at(var, k, j, i) = sed_alpha(dv, dum, du, dup);
                }
            }
        }
    }
}

// relax_NAD + aggregate (slot kNV) + PAD, one-layer range
__global__ void k_relax_pad(FVa Tr, FVa Ax, FVa Ay, FVa Az, FVa Wn, int mask, int use_sed, int pad, Cfg C) {
    const long long cnt = Tr.cells();
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < cnt; o += (long long)gridDim.x * blockDim.x) {
        int k, j, i;
        if (!cell_in(Tr, C, 1, o, &k, &j, &i)) continue;
        for (int var = 0; var < kNV; var++) {
            if (!((mask >> var) & 1)) continue;
            double alpha = 1;
            if (C.act[0]) alpha = smin(smin(Ax.at(var, k, j, i - 1), Ax.at(var, k, j, i)), Ax.at(var, k, j, i + 1));
            if (C.act[1])
                alpha = smin(alpha, smin(smin(Ay.at(var, k, j - 1, i), Ay.at(var, k, j, i)), Ay.at(var, k, j + 1, i)));
            if (C.act[2])
                alpha = smin(alpha, smin(smin(Az.at(var, k - 1, j, i), Az.at(var, k, j, i)), Az.at(var, k + 1, j, i)));
            const double trouble = Tr.at(var, k, j, i);
            if (use_sed) Tr.at(var, k, j, i) = alpha < 1 ? trouble : 0;
        }
        double trouble = 0;
        for (int var = 0; var < kNV; var++)
            if ((mask >> var) & 1) trouble = smax(trouble, Tr.at(var, k, j, i));
        Tr.at(kNV, k, j, i) = trouble;
        if (pad) {
            const double rho = Wn.at(0, k, j, i), p = Wn.at(kVP, k, j, i);
            if (rho < kRhoMin || rho > kRhoMax) Tr.at(kNV, k, j, i) = 1;
            if (p < kPMin || p > kPMax) Tr.at(kNV, k, j, i) = 1;
        }
    }
}

// mode 0: apply_blending (src/trouble_detection.cpp:191-210),
// 1: blending_ring (:226-242)
__global__ void k_blend(FVa In, int in_slot, FVa Out, int mode, Cfg C) {
    const double wts[4] = {1.0, 0.75, 0.5, 0.375};
    const int ax = C.act[0], ay = C.act[1], az = C.act[2];
    const long long cnt = In.cells();
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < cnt; o += (long long)gridDim.x * blockDim.x) {
        int k, j, i;
        if (!cell_in(In, C, 1, o, &k, &j, &i)) continue;
        if (mode == 0) {
            double t = 0;
            for (int dk = -az; dk <= az; dk++)
                for (int dj = -ay; dj <= ay; dj++)
                    for (int di = -ax; di <= ax; di++) {
                        const int n0 = (di != 0) + (dj != 0) + (dk != 0);
                        t = smax(t, wts[n0] * In.at(in_slot, k + dk, j + dj, i + di));
                    }
            Out.at(0, k, j, i) = t;
        } else {
            const double t = In.at(0, k, j, i);
            double ring = 0;
            for (int dk = -az; dk <= az; dk++)
                for (int dj = -ay; dj <= ay; dj++)
                    for (int di = -ax; di <= ax; di++)
                        if (In.at(0, k + dk, j + dj, i + di) > 0) ring = 0.25;
            Out.at(0, k, j, i) = smax(t, ring);
        }
    }
}

// src/trouble_detection.cpp:213-221: theta = aggregate trouble slot
__global__ void k_theta_copy(FVa Tr, FVa Th) {
    const long long n = Tr.cells();
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x)
        Th.p[o] = Tr.p[(long long)kNV * n + o];
}

// ---- MUSCL-Hancock fallback fluxes: src/hydro.cpp:591-788 -------------------
struct Geo {
    const double *xc, *xf, *yc, *yf, *zc, *zf;
};
// slopes of every active direction, Hancock half step, the two face states
// of direction D (src/hydro.cpp:622-681)
__device__ void slopes_d(const FVa& W, const Geo& G, const Cfg& C, int D, int k, int j, int i, double* WL,
                         double* WR, double dt) {
    double w[kNV], dW[3][kNV], dwt[kNV];
    for (int v = 0; v < kNV; v++) {
        w[v] = W.at(v, k, j, i);
        double wL = W.at(v, k, j, i - 1), wR = W.at(v, k, j, i + 1);
        dW[0][v] = minmod((wR - w[v]) / (G.xc[i + 1] - G.xc[i]), (w[v] - wL) / (G.xc[i] - G.xc[i - 1]), G.xf[i],
                          G.xf[i + 1]);
        dW[1][v] = 0;
        dW[2][v] = 0;
        if (C.act[1]) {
            wL = W.at(v, k, j - 1, i);
            wR = W.at(v, k, j + 1, i);
            dW[1][v] = minmod((wR - w[v]) / (G.yc[j + 1] - G.yc[j]), (w[v] - wL) / (G.yc[j] - G.yc[j - 1]),
                              G.yf[j], G.yf[j + 1]);
        }
        if (C.act[2]) {
            wL = W.at(v, k - 1, j, i);
            wR = W.at(v, k + 1, j, i);
            dW[2][v] = minmod((wR - w[v]) / (G.zc[k + 1] - G.zc[k]), (w[v] - wL) / (G.zc[k] - G.zc[k - 1]),
                              G.zf[k], G.zf[k + 1]);
        }
    }
    hancock<3>(w, dwt, dW, C.gm);
    for (int v = 0; v < kNV; v++) {
        const double h = (D == 0 ? G.xf[i + 1] - G.xf[i] : (D == 1 ? G.yf[j + 1] - G.yf[j] : G.zf[k + 1] - G.zf[k]));
        const double dw = dW[D][v];
        WR[v] = w[v] - dw + dwt[v] * dt / h;
        WL[v] = w[v] + dw + dwt[v] * dt / h;
    }
}

__device__ void fallback_face(const FVa& W, const FVa& Th, const FVa& F, const Geo& G, const Cfg& C, int D, int k,
                              int j, int i, double dt) {
    double wL[2][kNV], wR[2][kNV], uL[kNV], uR[kNV], fL[kNV];
    for (int l = -1; l < 1; l++)
        slopes_d(W, G, C, D, k + (D == 2 ? l : 0), j + (D == 1 ? l : 0), i + (D == 0 ? l : 0), wL[l + 1], wR[l + 1],
                 dt);
    conservatives<3>(wL[0], uL, C.gm);
    conservatives<3>(wR[1], uR, C.gm);
    riemann_hllc<3>(fL, uL, uR, D, C.gm);
    const double th = smax(Th.at(0, k, j, i), Th.at(0, k - (D == 2), j - (D == 1), i - (D == 0)));
    for (int v = 0; v < kNV; v++) {
        double f = F.at(v, k, j, i);
        f = f + th * (fL[v] - f);
        F.at(v, k, j, i) = f;
    }
}

// faces of the range that starts at the first active cell and runs one cell
// past the active region in every active direction (fv_for_faces)
__global__ void k_fallback(FVa W, FVa Th, FVa Fx, FVa Fy, FVa Fz, Geo G, const double* __restrict__ w, int ader,
                           double dt, Cfg C) {
    const double dtw = w[ader] * dt;
    int lo[3], cnt3[3];
    const int n[3] = {W.e[3], W.e[2], W.e[1]};
    for (int d = 0; d < 3; d++) {
        const int g = C.act[d] ? kNGH : 0;
        lo[d] = g;
        cnt3[d] = (n[d] - 2 * g + (g > 0) + g) - g;
    }
    const long long cnt = (long long)cnt3[0] * cnt3[1] * cnt3[2];
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < cnt; o += (long long)gridDim.x * blockDim.x) {
        long long r = o;
        const int i = lo[0] + (int)(r % cnt3[0]); r /= cnt3[0];
        const int j = lo[1] + (int)(r % cnt3[1]); r /= cnt3[1];
        const int k = lo[2] + (int)r;
        fallback_face(W, Th, Fx, G, C, 0, k, j, i, dtw);
        if (C.act[1]) fallback_face(W, Th, Fy, G, C, 1, k, j, i, dtw);
        if (C.act[2]) fallback_face(W, Th, Fz, G, C, 2, k, j, i, dtw);
    }
}

int check_physics_slots(const spdk_sd* a) {
    return a->ext[1] < kNV ? fail(SPDK_E_ARG, "SD array needs at least 5 variable slots") : 0;
}

}  // namespace

extern "C" {

int spdk_transform_a_to_b_1d(const spdk_sd* a, const spdk_sd* b, const spdk_mat* m, int dim, void* stream) {
    if (!ok_sd(a) || !ok_sd(b) || !ok_mat(m) || dim < 0 || dim > 2) return fail(SPDK_E_ARG, "transform_a_to_b_1d: bad argument");
    SDa A = sd(a), B = sd(b);
    const long long n = B.pts() * A.e[0] * A.e[1];
    k_transform_1d<<<blocks_for(n), kBlock, 0, (cudaStream_t)stream>>>(A, B, m->data, m->cols, dim, -1);
    return launched("transform_a_to_b_1d");
}

int spdk_transform_a_to_b_1d_slice(const spdk_sd* a, const spdk_sd* b, const spdk_mat* m, int dim, int t,
                                   void* stream) {
    if (!ok_sd(a) || !ok_sd(b) || !ok_mat(m) || dim < 0 || dim > 2 || t < 0 || t >= a->ext[0])
        return fail(SPDK_E_ARG, "transform_a_to_b_1d_slice: bad argument");
    SDa A = sd(a), B = sd(b);
    const long long n = B.pts() * A.e[1];
    k_transform_1d<<<blocks_for(n), kBlock, 0, (cudaStream_t)stream>>>(A, B, m->data, m->cols, dim, t);
    return launched("transform_a_to_b_1d_slice");
}

int spdk_transform_a_to_b(const spdk_sd* a, const spdk_sd* b, const spdk_sd* tmp, const spdk_mat* m,
                          const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_sd(a) || !ok_sd(b) || !ok_sd(tmp) || !ok_mat(m)) return fail(SPDK_E_ARG, "transform_a_to_b: bad argument");
    int dims[3], nd = 0;
    for (int d = 0; d < 3; d++)
        if (cfg->active[d]) dims[nd++] = d;
    const spdk_sd* src = a;
    for (int q = 0; q < nd; q++) {
        const spdk_sd* dst = ((nd - 1 - q) % 2 == 0) ? b : tmp;
        int rc = spdk_transform_a_to_b_1d(src, dst, m, dims[q], stream);
        if (rc) return rc;
        src = dst;
    }
    return 0;
}

int spdk_combine_solution(const spdk_sd* u, const spdk_sd* u0, double a, void* stream) {
    if (!ok_sd(u) || !ok_sd(u0)) return fail(SPDK_E_ARG, "combine_solution: bad argument");
    SDa U = sd(u), U0 = sd(u0);
    k_combine<<<blocks_for((long long)U.e[1] * U.pts()), kBlock, 0, (cudaStream_t)stream>>>(U, U0, a);
    return launched("combine_solution");
}

int spdk_update_prediction(const spdk_sd* u, const spdk_sd* u_ader, const spdk_sd* fx, const spdk_sd* fy,
                           const spdk_sd* fz, const spdk_mat* dfp_to_sp, const spdk_mat* invader, const spdk_vec* w,
                           double dt, double dx, double dy, double dz, const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_sd(u) || !ok_sd(u_ader) || !ok_sd(fx) || !ok_sd(fy) || !ok_sd(fz) || !ok_mat(dfp_to_sp) ||
        !ok_mat(invader) || !ok_vec(w) || fx->ext[0] > 16)
        return fail(SPDK_E_ARG, "update_prediction: bad argument");
    if (int rc = check_physics_slots(u)) return rc;
    SDa U = sd(u);
    k_update_prediction<<<blocks_for(U.pts()), kBlock, 0, (cudaStream_t)stream>>>(
        U, sd(u_ader), sd(fx), sd(fy), sd(fz), dfp_to_sp->data, dfp_to_sp->cols, invader->data, w->data, dt, dx, dy,
        dz, cfgof(cfg));
    return launched("update_prediction");
}

int spdk_update_solution(const spdk_sd* u, const spdk_sd* u_ader, const spdk_sd* fx, const spdk_sd* fy,
                         const spdk_sd* fz, const spdk_mat* dfp_to_sp, const spdk_vec* w, double dt, double dx,
                         double dy, double dz, const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_sd(u) || !ok_sd(u_ader) || !ok_sd(fx) || !ok_sd(fy) || !ok_sd(fz) || !ok_mat(dfp_to_sp) ||
        !ok_vec(w))
        return fail(SPDK_E_ARG, "update_solution: bad argument");
    if (int rc = check_physics_slots(u)) return rc;
    SDa U = sd(u);
    k_update_solution<<<blocks_for(U.pts()), kBlock, 0, (cudaStream_t)stream>>>(
        U, sd(u_ader), sd(fx), sd(fy), sd(fz), dfp_to_sp->data, dfp_to_sp->cols, w->data, dt, dx, dy, dz,
        cfgof(cfg));
    return launched("update_solution");
}

static int pointwise_sd(const spdk_sd* in, const spdk_sd* out, int mode, int v1, const spdk_proto_cfg* cfg,
                        void* stream, const char* what) {
    if (!cfg || !ok_sd(in) || !ok_sd(out) || in->ext[1] < kNV || out->ext[1] < kNV) return fail(SPDK_E_ARG, std::string(what) + ": bad argument");
    SDa A = sd(in), B = sd(out);
    for (int q = 2; q < 8; q++)
        if (A.e[q] != B.e[q]) return fail(SPDK_E_ARG, std::string(what) + ": extents differ");
    const int nt = A.e[0] < B.e[0] ? A.e[0] : B.e[0];
    k_pointwise<<<blocks_for(A.pts() * nt), kBlock, 0, (cudaStream_t)stream>>>(A.p, A.e[1], B.p, B.e[1], A.pts(), nt,
                                                                              mode, v1, cfg->gamma);
    return launched(what);
}
static int pointwise_fv(const spdk_fv* in, const spdk_fv* out, int mode, const spdk_proto_cfg* cfg, void* stream,
                        const char* what) {
    if (!cfg || !ok_fv(in) || !ok_fv(out) || in->ext[0] < kNV || out->ext[0] < kNV) return fail(SPDK_E_ARG, std::string(what) + ": bad argument");
    FVa A = fv(in), B = fv(out);
    if (A.cells() != B.cells()) return fail(SPDK_E_ARG, std::string(what) + ": extents differ");
    k_pointwise<<<blocks_for(A.cells()), kBlock, 0, (cudaStream_t)stream>>>(A.p, A.e[0], B.p, B.e[0], A.cells(), 1,
                                                                           mode, 1, cfg->gamma);
    return launched(what);
}

int spdk_compute_conservatives(const spdk_sd* w, const spdk_sd* u, const spdk_proto_cfg* cfg, void* stream) {
    return pointwise_sd(w, u, 1, 1, cfg, stream, "compute_conservatives");
}
int spdk_compute_primitives(const spdk_sd* u, const spdk_sd* w, const spdk_proto_cfg* cfg, void* stream) {
    return pointwise_sd(u, w, 0, 1, cfg, stream, "compute_primitives");
}
int spdk_fv_compute_conservatives(const spdk_fv* w, const spdk_fv* u, const spdk_proto_cfg* cfg, void* stream) {
    return pointwise_fv(w, u, 1, cfg, stream, "compute_conservatives (FV)");
}
int spdk_fv_compute_primitives(const spdk_fv* u, const spdk_fv* w, const spdk_proto_cfg* cfg, void* stream) {
    return pointwise_fv(u, w, 0, cfg, stream, "compute_primitives (FV)");
}

int spdk_compute_fluxes(const spdk_sd* u, const spdk_sd* f, int v1, int v2, int v3, const spdk_proto_cfg* cfg,
                        void* stream) {
    // the flux depends only on which slot is normal; the other two are the
    // remaining momentum slots
    if (v1 < 1 || v1 > 3 || v2 < 1 || v2 > 3 || v3 < 1 || v3 > 3 || v1 == v2 || v1 == v3 || v2 == v3)
        return fail(SPDK_E_ARG, "compute_fluxes: v1, v2, v3 must be a permutation of the momentum slots 1..3");
    return pointwise_sd(u, f, 2, v1, cfg, stream, "compute_fluxes");
}

int spdk_compute_dt(const spdk_sd* w, double dx, double dy, double dz, double nu, double* dt_out,
                    const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_sd(w) || !dt_out || w->ext[1] < kNV) return fail(SPDK_E_ARG, "compute_dt: bad argument");
    if (!(nu >= 0.0)) return fail(SPDK_E_ARG, "compute_dt: nu must be >= 0");
    SDa W = sd(w);
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long* out = reinterpret_cast<unsigned long long*>(dt_out);
    k_dt_arm<<<1, 1, 0, s>>>(out);
    k_compute_dt<<<blocks_for(W.pts()), kBlock, 0, s>>>(W, dx, dy, dz, nu, cfgof(cfg), out);
    return launched("compute_dt");
}

int spdk_sd_riemann_solver(const spdk_sd* u, const spdk_sd* f, int v1, int v2, int v3, int dim, int viscous,
                           const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_sd(u) || !ok_sd(f) || dim < 0 || dim > 2 || u->ext[1] < kNV)
        return fail(SPDK_E_ARG, "sd_riemann_solver: bad argument");
    if (v1 != 1 + dim || v2 < 1 || v2 > 3 || v3 < 1 || v3 > 3 || v2 == v3 || v2 == v1 || v3 == v1)
        return fail(SPDK_E_ARG, "sd_riemann_solver: v1 must be the normal momentum slot 1+dim");
    SDa U = sd(u);
    const long long n = U.pts() * U.e[0];
    k_riemann<<<blocks_for(n), kBlock, 0, (cudaStream_t)stream>>>(U, sd(f), dim, v1, cfg->gamma, viscous ? 1 : 0);
    return launched("sd_riemann_solver");
}

int spdk_sd_rusanov_solver(const spdk_sd* u, const spdk_sd* f, int dim, void* stream) {
    if (!ok_sd(u) || !ok_sd(f) || dim < 0 || dim > 2 || u->ext[1] != f->ext[1] || u->ext[0] != f->ext[0])
        return fail(SPDK_E_ARG, "sd_rusanov_solver: bad argument");
    for (int q = 2; q < 8; q++)
        if (u->ext[q] != f->ext[q]) return fail(SPDK_E_ARG, "sd_rusanov_solver: U and F extents differ");
    if (choose(dim, u->ext[4], u->ext[3], u->ext[2]) < 2)
        return fail(SPDK_E_ARG, "sd_rusanov_solver: direction has no interfaces");
    SDa U = sd(u);
    k_rusanov<<<blocks_for(U.pts() * U.e[0]), kBlock, 0, (cudaStream_t)stream>>>(U, sd(f), dim);
    return launched("sd_rusanov_solver");
}

int spdk_compute_gradient(const spdk_sd* u, const spdk_sd* du, double h, const spdk_mat* dfp_to_sp, int dim,
                          const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_sd(u) || !ok_sd(du) || !ok_mat(dfp_to_sp) || dim < 0 || dim > 2 || !(h > 0.0))
        return fail(SPDK_E_ARG, "compute_gradient: bad argument");
    const int n = choose(dim, du->ext[7], du->ext[6], du->ext[5]);
    if (choose(dim, u->ext[7], u->ext[6], u->ext[5]) != n + 1 || dfp_to_sp->rows < n || dfp_to_sp->cols != n + 1 ||
        u->ext[0] != du->ext[0] || u->ext[1] < du->ext[1])
        return fail(SPDK_E_ARG, "compute_gradient: U must hold n+1 flux points along dim for the n solution points of dU");
    for (int q = 2; q < 5; q++)
        if (u->ext[q] != du->ext[q]) return fail(SPDK_E_ARG, "compute_gradient: element extents differ");
    SDa dU = sd(du);
    k_gradient<<<blocks_for(dU.pts() * dU.e[0] * dU.e[1]), kBlock, 0, (cudaStream_t)stream>>>(
        sd(u), dU, h, dfp_to_sp->data, dfp_to_sp->cols, dim, cfgof(cfg));
    return launched("compute_gradient");
}

int spdk_compute_viscous_flux(const spdk_sd* u, const spdk_sd* du1, int v1, const spdk_sd* du2, int v2,
                              const spdk_sd* du3, int v3, const spdk_mat* sp_to_fp, double nu, double beta, int dim,
                              const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_sd(u) || !ok_sd(du1) || !ok_sd(du2) || !ok_sd(du3) || !ok_mat(sp_to_fp) || dim < 0 || dim > 2 ||
        u->ext[1] < kNV)
        return fail(SPDK_E_ARG, "compute_viscous_flux: bad argument");
    if (v1 != 1 + dim || v2 < 1 || v2 > 3 || v3 < 1 || v3 > 3 || v2 == v3 || v2 == v1 || v3 == v1)
        return fail(SPDK_E_ARG, "compute_viscous_flux: v1 must be the normal momentum slot 1+dim");
    const int n = choose(dim, du1->ext[7], du1->ext[6], du1->ext[5]);
    if (choose(dim, u->ext[7], u->ext[6], u->ext[5]) != n + 1 || sp_to_fp->cols != n || sp_to_fp->rows < n + 1)
        return fail(SPDK_E_ARG, "compute_viscous_flux: U must hold n+1 flux points along dim");
    const spdk_sd* g[3] = {du1, du2, du3};
    for (int a = 0; a < 3; a++) {
        if (g[a]->ext[0] != u->ext[0] || g[a]->ext[1] < 4) return fail(SPDK_E_ARG, "compute_viscous_flux: gradient extents");
        for (int q = 2; q < 8; q++) {
            const bool along = (q == 7 && dim == 0) || (q == 6 && dim == 1) || (q == 5 && dim == 2);
            if (!along && g[a]->ext[q] != u->ext[q])
                return fail(SPDK_E_ARG, "compute_viscous_flux: gradient extents differ from U");
        }
    }
    SDa U = sd(u);
    k_viscous_flux<<<blocks_for(U.pts() * U.e[0]), kBlock, 0, (cudaStream_t)stream>>>(
        U, sd(du1), sd(du2), sd(du3), v1, v2, v3, sp_to_fp->data, sp_to_fp->cols, nu, beta, dim, cfg->gamma);
    return launched("compute_viscous_flux");
}

int spdk_boundaries_sd(const spdk_sd* u, int dim, int type, void* stream) {
    if (!ok_sd(u) || dim < 0 || dim > 2 || type < 0 || type > 2) return fail(SPDK_E_ARG, "boundaries (SD): bad argument");
    if (choose(dim, u->ext[4], u->ext[3], u->ext[2]) < 3) return fail(SPDK_E_ARG, "boundaries (SD): direction has no ghost elements");
    SDa U = sd(u);
    k_boundaries_sd<<<blocks_for(U.pts() * U.e[0] * U.e[1]), kBlock, 0, (cudaStream_t)stream>>>(U, dim, type);
    return launched("boundaries (SD)");
}

int spdk_boundaries_fv(const spdk_fv* u, int dim, int type, int alignment, int a_dim, void* stream) {
    if (!ok_fv(u) || dim < 0 || dim > 2 || type < 0 || type > 2 || a_dim < 0 || a_dim > 2)
        return fail(SPDK_E_ARG, "boundaries (FV): bad argument");
    if (alignment != 0)
        return fail(SPDK_E_ARG, "boundaries (FV): only cell-centred arrays (alignment 0) are supported");
    const int ext = dim == 0 ? u->ext[3] : (dim == 1 ? u->ext[2] : u->ext[1]);
    if (ext < 2 * kNGH + 2) return fail(SPDK_E_ARG, "boundaries (FV): direction too short");
    FVa U = fv(u);
    k_boundaries_fv<<<blocks_for(U.cells() * U.e[0]), kBlock, 0, (cudaStream_t)stream>>>(U, dim, type);
    return launched("boundaries (FV)");
}

int spdk_face_integral(const spdk_sd* f_fp, const spdk_fv* f, const spdk_sd* tmp, const spdk_mat* sp_to_cv, int dim,
                       int t, const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_sd(f_fp) || !ok_fv(f) || !ok_mat(sp_to_cv) || dim < 0 || dim > 2 || t < 0 || t >= f_fp->ext[0] ||
        f_fp->ext[1] < kNV || f->ext[0] < kNV)
        return fail(SPDK_E_ARG, "face_integral: bad argument");
    const int dim1 = dim == 0 ? 1 : (dim == 1 ? 2 : 0), dim2 = dim1 == 0 ? 1 : (dim1 == 1 ? 2 : 0);
    const bool both = cfg->active[dim1] && cfg->active[dim2];
    if (both) {
        if (!ok_sd(tmp)) return fail(SPDK_E_ARG, "face_integral: a temporary is needed with two transverse directions");
        int rc = spdk_transform_a_to_b_1d_slice(f_fp, tmp, sp_to_cv, dim1, t, stream);
        if (rc) return rc;
    }
    SDa Ff = sd(f_fp);
    SDa T = both ? sd(tmp) : Ff;
    const long long n = Ff.pts() * 2 * kNV;  // grid-stride loop bounds the true count
    k_face_integral<<<blocks_for(n), kBlock, 0, (cudaStream_t)stream>>>(Ff, fv(f), T, sp_to_cv->data, sp_to_cv->cols,
                                                                       dim, t, cfgof(cfg));
    return launched("face_integral");
}

int spdk_fv_update_solution(const spdk_fv* u_old, const spdk_fv* u_new, const spdk_sd* u_cv, const spdk_fv* fx,
                            const spdk_vec* x_f, const spdk_fv* fy, const spdk_vec* y_f, const spdk_fv* fz,
                            const spdk_vec* z_f, const spdk_vec* w, int t, double dt, int update,
                            const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_fv(u_old) || !ok_fv(u_new) || !ok_sd(u_cv) || !ok_vec(w) || t < 0 || t >= w->n)
        return fail(SPDK_E_ARG, "fv_update_solution: bad argument");
    const spdk_fv* F[3] = {fx, fy, fz};
    const spdk_vec* X[3] = {x_f, y_f, z_f};
    for (int d = 0; d < 3; d++)
        if (cfg->active[d] && (!ok_fv(F[d]) || !ok_vec(X[d])))
            return fail(SPDK_E_ARG, "fv_update_solution: missing flux or faces of an active direction");
    if (int rc = check_physics_slots(u_cv)) return rc;
    FVa dummy = fv(u_old);
    SDa Ucv = sd(u_cv);
    k_fv_update<<<blocks_for(Ucv.pts()), kBlock, 0, (cudaStream_t)stream>>>(
        fv(u_old), fv(u_new), Ucv, cfg->active[0] ? fv(fx) : dummy, cfg->active[0] ? x_f->data : nullptr,
        cfg->active[1] ? fv(fy) : dummy, cfg->active[1] ? y_f->data : nullptr, cfg->active[2] ? fv(fz) : dummy,
        cfg->active[2] ? z_f->data : nullptr, w->data, t, dt, update, cfgof(cfg));
    return launched("fv_update_solution");
}

int spdk_detect_troubles(const spdk_fv* w_new, const spdk_fv* w_old, const spdk_fv* troubles,
                         const spdk_fv* alpha_x, const spdk_fv* alpha_y, const spdk_fv* alpha_z,
                         const spdk_vec* x_c, const spdk_vec* x_f, const spdk_vec* y_c, const spdk_vec* y_f,
                         const spdk_vec* z_c, const spdk_vec* z_f, int pad, int limit_mask,
                         const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_fv(w_new) || !ok_fv(w_old) || !ok_fv(troubles) || troubles->ext[0] < kNV + 1 ||
        w_new->ext[0] < kNV || w_old->ext[0] < kNV)
        return fail(SPDK_E_ARG, "detect_troubles: bad argument");
    const int use_sed = cfg->sed && cfg->p > 1;
    const spdk_fv* A[3] = {alpha_x, alpha_y, alpha_z};
    const spdk_vec* Cc[3] = {x_c, y_c, z_c};
    const spdk_vec* Ff[3] = {x_f, y_f, z_f};
    if (use_sed)
        for (int d = 0; d < 3; d++)
            if (cfg->active[d] && (!ok_fv(A[d]) || !ok_vec(Cc[d]) || !ok_vec(Ff[d])))
                return fail(SPDK_E_ARG, "detect_troubles: missing alpha, centres or faces of an active direction");
    FVa dummy = fv(w_old);
    FVa Ax = (use_sed && cfg->active[0]) ? fv(alpha_x) : dummy;
    FVa Ay = (use_sed && cfg->active[1]) ? fv(alpha_y) : dummy;
    FVa Az = (use_sed && cfg->active[2]) ? fv(alpha_z) : dummy;
    auto dptr = [&](int d, const spdk_vec* v) { return (use_sed && cfg->active[d]) ? v->data : nullptr; };
    const Cfg C = cfgof(cfg);
    FVa Wo = fv(w_old);
    k_nad_sed<<<blocks_for(Wo.cells()), kBlock, 0, (cudaStream_t)stream>>>(
        fv(w_new), Wo, fv(troubles), Ax, Ay, Az, dptr(0, x_c), dptr(0, x_f), dptr(1, y_c), dptr(1, y_f), dptr(2, z_c),
        dptr(2, z_f), limit_mask, use_sed, C);
    if (int rc = launched("detect_troubles (NAD, SED)")) return rc;
    k_relax_pad<<<blocks_for(Wo.cells()), kBlock, 0, (cudaStream_t)stream>>>(fv(troubles), Ax, Ay, Az, fv(w_new),
                                                                            limit_mask, use_sed, pad ? 1 : 0, C);
    return launched("detect_troubles (relax, PAD)");
}

int spdk_apply_blending(const spdk_fv* troubles, const spdk_fv* theta, const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_fv(troubles) || !ok_fv(theta) || troubles->ext[0] < kNV + 1)
        return fail(SPDK_E_ARG, "apply_blending: bad argument");
    FVa T = fv(troubles);
    k_blend<<<blocks_for(T.cells()), kBlock, 0, (cudaStream_t)stream>>>(T, kNV, fv(theta), 0, cfgof(cfg));
    return launched("apply_blending");
}

int spdk_blending_ring(const spdk_fv* theta_in, const spdk_fv* theta_out, const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_fv(theta_in) || !ok_fv(theta_out)) return fail(SPDK_E_ARG, "blending_ring: bad argument");
    FVa T = fv(theta_in);
    k_blend<<<blocks_for(T.cells()), kBlock, 0, (cudaStream_t)stream>>>(T, 0, fv(theta_out), 1, cfgof(cfg));
    return launched("blending_ring");
}

int spdk_theta_from_troubles(const spdk_fv* troubles, const spdk_fv* theta, void* stream) {
    if (!ok_fv(troubles) || !ok_fv(theta) || troubles->ext[0] < kNV + 1) return fail(SPDK_E_ARG, "theta_from_troubles: bad argument");
    FVa T = fv(troubles);
    k_theta_copy<<<blocks_for(T.cells()), kBlock, 0, (cudaStream_t)stream>>>(T, fv(theta));
    return launched("theta_from_troubles");
}

int spdk_fallback_fluxes(const spdk_fv* w_old, const spdk_fv* theta, const spdk_vec* x_c, const spdk_vec* x_f,
                         const spdk_fv* fx, const spdk_vec* y_c, const spdk_vec* y_f, const spdk_fv* fy,
                         const spdk_vec* z_c, const spdk_vec* z_f, const spdk_fv* fz, int ader, const spdk_vec* w,
                         double dt, const spdk_proto_cfg* cfg, void* stream) {
    if (!cfg || !ok_fv(w_old) || !ok_fv(theta) || !ok_vec(w) || ader < 0 || ader >= w->n || w_old->ext[0] < kNV ||
        !cfg->active[0])
        return fail(SPDK_E_ARG, "fallback_fluxes: bad argument");
    const spdk_fv* F[3] = {fx, fy, fz};
    const spdk_vec* Cc[3] = {x_c, y_c, z_c};
    const spdk_vec* Xf[3] = {x_f, y_f, z_f};
    for (int d = 0; d < 3; d++)
        if (cfg->active[d] && (!ok_fv(F[d]) || !ok_vec(Cc[d]) || !ok_vec(Xf[d])))
            return fail(SPDK_E_ARG, "fallback_fluxes: missing flux, centres or faces of an active direction");
    cudaStream_t s = (cudaStream_t)stream;
    FVa Wo = fv(w_old);
    Geo G{x_c->data, x_f->data, cfg->active[1] ? y_c->data : nullptr, cfg->active[1] ? y_f->data : nullptr,
          cfg->active[2] ? z_c->data : nullptr, cfg->active[2] ? z_f->data : nullptr};
    k_fallback<<<blocks_for(Wo.cells()), kBlock, 0, s>>>(Wo, fv(theta), fv(fx), cfg->active[1] ? fv(fy) : Wo,
                                                         cfg->active[2] ? fv(fz) : Wo, G, w->data, ader, dt,
                                                         cfgof(cfg));
    return launched("fallback_fluxes");
}

}  // extern "C"
