/* CPU restatement of spd_K's spectral-difference hydro step.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker that the CUDA path is
 * compared against; nothing in the product links it. Every function restates
 * the reference routine cited beside it, with the same floating-point
 * operation order (the file is built with -ffp-contract=off), so results are
 * bit-identical to the reference's own CPU build. See spdk_oracle.h for the
 * layout and the slot-5 convention. */
#include "spdk_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define PI_REF 3.141592653589793
#define MIN_C2 1E-14
#define RHO_MIN 1E-10
#define RHO_MAX 1E10
#define P_MIN 1E-10
#define P_MAX 1E10
#define NGH 1
#define NGHFV 2
#define NV 5      /* rho, mx, my, mz, E */
#define NT 6      /* trouble slots: per-variable flags 0..4 + aggregate 5 */
#define VX 1
#define VY 2
#define VZ 3
#define VP 4

/* std::max / std::min semantics (first argument returned on ties/NaN) */
static inline double smax(double a, double b) { return (a < b) ? b : a; }
static inline double smin(double a, double b) { return (b < a) ? b : a; }

/* ------------------------------------------------------------------ */
/* arrays                                                              */
/* ------------------------------------------------------------------ */
typedef struct {
    double* v;
    int nt, nv, Nz, Ny, Nx, nz, ny, nx;
} sd_t;

typedef struct {
    double* v;
    int nv, Nz, Ny, Nx;
} fv_t;

static inline double* SD(const sd_t* a, int t, int var, int k, int j, int i, int kk, int jj, int ii) {
    long o = ((((((long)t * a->nv + var) * a->Nz + k) * a->Ny + j) * a->Nx + i) * a->nz + kk);
    o = (o * a->ny + jj) * a->nx + ii;
    return a->v + o;
}
static inline double* FV(const fv_t* a, int var, int k, int j, int i) {
    return a->v + ((((long)var * a->Nz + k) * a->Ny + j) * a->Nx + i);
}

static sd_t sd_alloc(int nt, int nv, int Nz, int Ny, int Nx, int nz, int ny, int nx) {
    sd_t a = {0, nt, nv, Nz, Ny, Nx, nz, ny, nx};
    a.v = (double*)calloc((size_t)nt * nv * Nz * Ny * Nx * nz * ny * nx, sizeof(double));
    return a;
}
static fv_t fv_alloc(int nv, int Nz, int Ny, int Nx) {
    fv_t a = {0, nv, Nz, Ny, Nx};
    a.v = (double*)calloc((size_t)nv * Nz * Ny * Nx, sizeof(double));
    return a;
}
static long sd_size(const sd_t* a) {
    return (long)a->nt * a->nv * a->Nz * a->Ny * a->Nx * a->nz * a->ny * a->nx;
}

/* ------------------------------------------------------------------ */
/* polynomials and quadrature: src/polynomials.cpp                     */
/* ------------------------------------------------------------------ */
/* src/polynomials.cpp:3-11 */
static double lagrange(const double* x, double y, int i, int n) {
    double lag = 1.;
    for (int j = 0; j < n; j++)
        if (j != i) lag *= (y - x[j]) / (x[i] - x[j]);
    return lag;
}
/* src/polynomials.cpp:21-35 */
static double lagrange_prime(const double* x, double y, int i, int n) {
    double lagp = 0;
    for (int k = 0; k < n; k++) {
        if (k == i) continue;
        double lag = 1;
        for (int j = 0; j < n; j++)
            if (j != i && j != k) lag *= (y - x[j]) / (x[i] - x[j]);
        lagp += lag / (x[i] - x[k]);
    }
    return lagp;
}
/* src/polynomials.cpp:46-79 (Newton iteration on P_n; note the 10-digit pi
 * of the starting guess, which is part of the result's rounding) */
static void gauss_legendre(double xi, double xf, int n, double* x, double* w) {
    double eps = 3E-14;
    int m = (n + 1) / 2;
    double xm = 0.5 * (xf + xi);
    double xl = 0.5 * (xf - xi);
    if (n > 0) {
        for (int i = 0; i < m; i++) {
            double z = cos(3.141592654 * (i + 0.75) / (n + 0.5));
            double z1 = 0.0, p1, p2, p3, pp = 0;
            while (fabs(z - z1) > eps) {
                p1 = 1.0;
                p2 = 0.0;
                for (int j = 0; j < n; j++) {
                    p3 = p2;
                    p2 = p1;
                    p1 = ((2.0 * j + 1) * z * p2 - j * p3) / (j + 1);
                }
                pp = n * (z * p1 - p2) / (z * z - 1.0);
                z1 = z;
                z = z1 - p1 / pp;
            }
            x[i] = xm - xl * z;
            x[n - i - 1] = xm + xl * z;
            w[i] = (2.0 * xl) / ((1.0 - z * z) * pp * pp);
            w[n - i - 1] = w[i];
        }
    } else {
        x[0] = 0.5;
        w[0] = 1;
    }
}
/* src/polynomials.cpp:81-93 */
static void flux_points(double* x_fp, const double* x, int n) {
    x_fp[0] = 0.0;
    for (int i = 1; i < n + 1; i++) x_fp[i] = x[i - 1];
    x_fp[n + 1] = 1.0;
}
static void solution_points(double* x_sp, int n) {
    for (int i = 0; i <= n; i++) x_sp[i] = 0.5 * (1.0 - cos((2 * i + 1) / (2.0 * (n + 1)) * PI_REF));
}
/* src/polynomials.cpp:13-19: M(j,i) = l_i(x_b[j]) over nodes x_a */
static void lagrange_matrix(double* M, const double* xa, const double* xb, int na, int nb) {
    for (int j = 0; j < nb; j++)
        for (int i = 0; i < na; i++) M[j * na + i] = lagrange(xa, xb[j], i, na);
}
static void lagrange_prime_matrix(double* M, const double* xa, const double* xb, int na, int nb) {
    for (int j = 0; j < nb; j++)
        for (int i = 0; i < na; i++) M[j * na + i] = lagrange_prime(xa, xb[j], i, na);
}
/* src/polynomials.cpp:95-101 */
static void ader_matrix(double* A, const double* xt, const double* wt, int n) {
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++)
            A[j * n + i] = lagrange(xt, 1, i, n) * lagrange(xt, 1, j, n) - lagrange_prime(xt, xt[i], j, n) * wt[i];
}
/* src/polynomials.cpp:103-124: cell averages of the sp interpolant over the
 * sub-cells [x_fp[k], x_fp[k+1]] by p-point GL quadrature */
static void integral_matrix(double* M, const double* x_fp, const double* x_sp, int n_cv, int n_sp) {
    int p = n_sp - 1;
    double x[32], w[32];
    gauss_legendre(0.0, 1.0, p, x, w);
    for (int k = 0; k < n_cv; k++) {
        if (p > 0) gauss_legendre(x_fp[k], x_fp[k + 1], p, x, w);
        for (int j = 0; j < n_sp; j++) {
            double integral;
            if (p > 0) {
                integral = 0.0;
                for (int i = 0; i < p; i++) integral += lagrange(x_sp, x[i], j, p + 1) * w[i];
            } else
                integral = 1.0;
            M[k * n_sp + j] = integral / (x_fp[k + 1] - x_fp[k]);
        }
    }
}
/* src/polynomials.cpp:126-198: Doolittle LU without pivoting, then one
 * forward/back substitution per unit vector */
static void inverse(const double* A, double* C, int n) {
    double B[64], Lm[64], U[64], b[8], d[8], x[8];
    for (int j = 0; j < n; j++) {
        b[j] = 0.0;
        for (int i = 0; i < n; i++) {
            B[i + j * n] = A[j * n + i];
            U[i + j * n] = 0;
            Lm[i + j * n] = 0;
        }
    }
    for (int k = 0; k < n - 1; k++)
        for (int i = k + 1; i < n; i++) {
            double coeff = B[k + i * n] / B[k + k * n];
            Lm[k + i * n] = coeff;
            for (int j = k + 1; j < n; j++) B[j + i * n] -= coeff * B[j + k * n];
        }
    for (int i = 0; i < n; i++) Lm[i + i * n] = 1.0;
    for (int j = 0; j < n; j++)
        for (int i = 0; i <= j; i++) U[j + i * n] = B[j + i * n];
    for (int k = 0; k < n; k++) {
        b[k] = 1.0;
        d[0] = b[0];
        for (int i = 1; i < n; i++) {
            d[i] = b[i];
            for (int j = 0; j < i; j++) d[i] -= Lm[j + i * n] * d[j];
        }
        x[n - 1] = d[n - 1] / U[n * n - 1];
        for (int i = n - 2; i >= 0; i--) {
            x[i] = d[i];
            for (int j = n - 1; j >= i + 1; j--) x[i] = x[i] - U[j + i * n] * x[j];
            x[i] = x[i] / U[i + i * n];
        }
        for (int i = 0; i < n; i++) C[i * n + k] = x[i];
        b[k] = 0.0;
    }
}

/* ------------------------------------------------------------------ */
/* geometry: src/structs.hpp:19-76                                     */
/* ------------------------------------------------------------------ */
typedef struct {
    int N, p, Ntot, nsp, nfp, fvn, idL, idR, active;
    double L, h;
    double* sd_faces;   /* Ntot x nfp */
    double* fv_faces;   /* fvn + 1 */
    double* fv_centers; /* fvn */
} dim_t;

static void dim_init(dim_t* D, int N, int p, double L, const double* x_fp, int active) {
    memset(D, 0, sizeof(*D));
    D->N = N;
    D->p = active ? p : 0;
    D->L = L;
    D->h = L / N;
    D->active = active;
    D->Ntot = 1; D->nsp = 1; D->nfp = 1; D->fvn = 1; D->idL = 0; D->idR = 1;
    if (active) {
        D->nsp = p + 1;
        D->nfp = p + 2;
        D->Ntot = N + 2 * NGH;
        D->fvn = N * D->nsp + 2 * NGHFV;
        D->idL = D->nsp - NGHFV;
        D->idR = D->fvn + D->idL;
    }
    /* one extra slot: the reference reads sd_faces(j, nsp) for inactive
     * directions (n_fp = 1) when forming centres; those centres are unused */
    D->sd_faces = (double*)calloc((size_t)D->Ntot * D->nfp + 1, sizeof(double));
    D->fv_faces = (double*)calloc((size_t)D->fvn + 1, sizeof(double));
    D->fv_centers = (double*)calloc((size_t)D->fvn, sizeof(double));
    for (int j = 0; j < D->Ntot; j++) {
        for (int i = 0; i < D->nfp; i++) {
            D->sd_faces[j * D->nfp + i] = (0 + j - NGH + x_fp[i]) * D->h;
            int g = i + j * D->nsp;
            if (g >= D->idL && g < D->idR) D->fv_faces[i - D->idL + j * D->nsp] = D->sd_faces[j * D->nfp + i];
        }
        for (int i = 0; i < D->nsp; i++) {
            double c = 0.5 * (D->sd_faces[j * D->nfp + i + 1] + D->sd_faces[j * D->nfp + i]);
            int g = i + j * D->nsp;
            if (g >= D->idL && g < D->idR) D->fv_centers[i - D->idL + j * D->nsp] = c;
        }
    }
}

/* ------------------------------------------------------------------ */
/* solver state                                                        */
/* ------------------------------------------------------------------ */
struct orc {
    orc_cfg c;
    int p, n, nf, nader, nstages, act[3], ghost[3], fvg[3];
    double rk_a[3];
    double xx[16], wx[16], xt[16], wt[16], x_gl[16], w_gl[16], x_sp[16], x_fp[16];
    double sp_to_fp[128], dfp_to_sp[128], sp_to_cv[64], cv_to_sp[64], ader[64], invader[64];
    dim_t d[3];
    sd_t W_sp, U_sp, W_cv, U_cv, T_sweep, U0_sp, U_ader_sp;
    sd_t U_ader_fp[3], F_ader_fp[3], T_fp[3];
    sd_t dU_sp[3];  /* viscous runs: gradients at the solution points (dUx/dUy/dUz_sp) */
    fv_t U_new, W_new, U_old, W_old, troubles, theta, theta_tmp, F[3], alpha[3];
};

static inline int choose(int dim, int i, int j, int k) { return dim == 0 ? i : (dim == 1 ? j : k); }

/* ------------------------------------------------------------------ */
/* pointwise physics: src/hydro.cpp                                    */
/* ------------------------------------------------------------------ */
/* src/hydro.cpp:27-32 */
static double sound_speed(double rho, double p, double gm) {
    double c2 = gm * p / rho;
    c2 = smax(c2, MIN_C2);
    return sqrt(c2);
}
/* src/hydro.cpp:34-45 */
static void conservatives(const double* w, double* u, double gm) {
    double E_kin = 0;
    u[0] = w[0];
    u[VX] = w[0] * w[VX];
    E_kin += w[VX] * u[VX];
    u[VY] = w[0] * w[VY];
    E_kin += w[VY] * u[VY];
    u[VZ] = w[0] * w[VZ];
    E_kin += w[VZ] * u[VZ];
    u[VP] = w[VP] / (gm - 1.) + 0.5 * E_kin;
}
/* src/hydro.cpp:95-106 */
static void primitives(const double* u, double* w, double gm) {
    double E_kin = 0;
    w[0] = u[0];
    w[VX] = u[VX] / u[0];
    E_kin += w[VX] * u[VX];
    w[VY] = u[VY] / u[0];
    E_kin += w[VY] * u[VY];
    w[VZ] = u[VZ] / u[0];
    E_kin += w[VZ] * u[VZ];
    w[VP] = (u[VP] - 0.5 * E_kin) * (gm - 1.);
}
/* src/hydro.cpp:155-161 */
static void fluxes(const double* u, const double* w, double* f, int v1, int v2, int v3) {
    f[0] = u[0] * w[v1];
    f[v1] = u[v1] * w[v1] + w[VP];
    f[v2] = u[v2] * w[v1];
    f[v3] = u[v3] * w[v1];
    f[VP] = (u[VP] + w[VP]) * w[v1];
}
/* src/hydro.cpp:270-289 */
static void riemann_llf(double* F, const double* UL, const double* UR, int v1, int v2, int v3, double gm) {
    double WL[NV] = {0}, WR[NV] = {0}, FL[NV] = {0}, FR[NV] = {0};
    primitives(UL, WL, gm);
    primitives(UR, WR, gm);
    fluxes(UL, WL, FL, v1, v2, v3);
    fluxes(UR, WR, FR, v1, v2, v3);
    double cL = sound_speed(WL[0], WL[VP], gm) + fabs(WL[v1]);
    double cR = sound_speed(WR[0], WR[VP], gm) + fabs(WR[v1]);
    double cmax = smax(cL, cR);
    for (int v = 0; v < NV; v++) F[v] = 0.5 * (FR[v] + FL[v]) - 0.5 * cmax * (UR[v] - UL[v]);
}
/* src/hydro.cpp:291-363 */
static void riemann_hllc(double* F, const double* UL, const double* UR, int v1, int v2, int v3, double gm) {
    double WL[NV], WR[NV];
    primitives(UL, WL, gm);
    primitives(UR, WR, gm);
    double cL = sound_speed(WL[0], WL[VP], gm) + fabs(WL[v1]);
    double cR = sound_speed(WR[0], WR[VP], gm) + fabs(WR[v1]);
    double cmax = smax(cL, cR);
    double vL = WL[v1], vR = WR[v1];
    double sL = smin(vL, vR) - cmax;
    double sR = smax(vL, vR) + cmax;
    double rcL = WL[0] * (vL - sL);
    double rcR = WR[0] * (sR - vR);
    double vs = (rcR * vR + rcL * vL + (WL[VP] - WR[VP])) / (rcR + rcL);
    double ps = (rcR * WL[VP] + rcL * WR[VP] + rcL * rcR * (vL - vR)) / (rcR + rcL);
    double rsL = WL[0] * (sL - vL) / (sL - vs);
    double esL = ((sL - vL) * UL[VP] - WL[VP] * vL + ps * vs) / (sL - vs);
    double rsR = WR[0] * (sR - vR) / (sR - vs);
    double esR = ((sR - vR) * UR[VP] - WR[VP] * vR + ps * vs) / (sR - vs);
    double r, v, pg, e;
    if (sL > 0) { r = WL[0]; v = WL[v1]; pg = WL[VP]; e = UL[VP]; }
    else if (vs > 0) { r = rsL; v = vs; pg = ps; e = esL; }
    else if (sR > 0) { r = rsR; v = vs; pg = ps; e = esR; }
    else { r = WR[0]; v = WR[v1]; pg = WR[VP]; e = UR[VP]; }
    F[0] = r * v;
    F[v1] = r * v * v + pg;
    F[v2] = r * v * (vs > 0 ? WL[v2] : WR[v2]);
    F[v3] = r * v * (vs > 0 ? WL[v3] : WR[v3]);
    F[VP] = v * (e + pg);
}

/* ------------------------------------------------------------------ */
/* transforms: src/transforms.cpp                                      */
/* ------------------------------------------------------------------ */
/* src/transforms.cpp:120-147: out(id) = sum_l in(l) M(id,l) along dim */
static void transform_1d(const sd_t* A, const sd_t* B, const double* M, int mcols, int dim) {
    int q = choose(dim, A->nx, A->ny, A->nz);
    for (int k = 0; k < B->Nz; k++) for (int j = 0; j < B->Ny; j++) for (int i = 0; i < B->Nx; i++)
    for (int kk = 0; kk < B->nz; kk++) for (int jj = 0; jj < B->ny; jj++) for (int ii = 0; ii < B->nx; ii++)
    for (int t = 0; t < A->nt; t++) for (int var = 0; var < A->nv; var++) {
        int id = choose(dim, ii, jj, kk);
        double u = 0;
        for (int ll = 0; ll < q; ll++) {
            int n0 = dim == 0 ? ll : ii, n1 = dim == 1 ? ll : jj, n2 = dim == 2 ? ll : kk;
            u += *SD(A, t, var, k, j, i, n2, n1, n0) * M[id * mcols + ll];
        }
        *SD(B, t, var, k, j, i, kk, jj, ii) = u;
    }
}
/* src/transforms.cpp:151-177: one slice t_src of A -> slice 0 of B */
static void transform_1d_slice(const sd_t* A, const sd_t* B, const double* M, int mcols, int dim, int tsrc) {
    int q = choose(dim, A->nx, A->ny, A->nz);
    for (int k = 0; k < B->Nz; k++) for (int j = 0; j < B->Ny; j++) for (int i = 0; i < B->Nx; i++)
    for (int kk = 0; kk < B->nz; kk++) for (int jj = 0; jj < B->ny; jj++) for (int ii = 0; ii < B->nx; ii++)
    for (int var = 0; var < A->nv; var++) {
        int id = choose(dim, ii, jj, kk);
        double u = 0;
        for (int ll = 0; ll < q; ll++) {
            int n0 = dim == 0 ? ll : ii, n1 = dim == 1 ? ll : jj, n2 = dim == 2 ? ll : kk;
            u += *SD(A, tsrc, var, k, j, i, n2, n1, n0) * M[id * mcols + ll];
        }
        *SD(B, 0, var, k, j, i, kk, jj, ii) = u;
    }
}
/* src/transforms.cpp:99-117: x, y, z sweeps ping-ponging through T so that
 * the last sweep lands in B */
static void transform_a_to_b(orc* s, const sd_t* A, const sd_t* B, const sd_t* T, const double* M) {
    int dims[3], nd = 0;
    for (int d = 0; d < 3; d++) if (s->act[d]) dims[nd++] = d;
    const sd_t* src = A;
    for (int q = 0; q < nd; q++) {
        const sd_t* dst = ((nd - 1 - q) % 2 == 0) ? B : T;
        transform_1d(src, dst, M, s->n, dims[q]);
        src = dst;
    }
}

/* src/transforms.cpp:16-27 (gravity source of one variable at one point) */
static double gravity_source(const sd_t* U, int var, int t, int k, int j, int i, int kk, int jj, int ii,
                             double gx, double gy, double gz) {
    if (var == VX) return *SD(U, t, 0, k, j, i, kk, jj, ii) * gx;
    if (var == VY) return *SD(U, t, 0, k, j, i, kk, jj, ii) * gy;
    if (var == VZ) return *SD(U, t, 0, k, j, i, kk, jj, ii) * gz;
    if (var == VP)
        return *SD(U, t, VX, k, j, i, kk, jj, ii) * gx + *SD(U, t, VY, k, j, i, kk, jj, ii) * gy +
               *SD(U, t, VZ, k, j, i, kk, jj, ii) * gz;
    return 0.0;
}

/* src/transforms.cpp:263-325. U_ader is updated variable by variable in
 * place, so the gravity source of a later variable sees the already updated
 * density/momentum of the same point: kept as in the reference. */
static void update_prediction(orc* s, double dt) {
    const sd_t *U = &s->U_sp, *Ua = &s->U_ader_sp;
    const sd_t *Fx = &s->F_ader_fp[0], *Fy = &s->F_ader_fp[1], *Fz = &s->F_ader_fp[2];
    int q = Fx->nx, nader = Fx->nt;
    double dx = s->d[0].h, dy = s->d[1].h, dz = s->d[2].h;
    double gx = s->c.g[0], gy = s->c.g[1], gz = s->c.g[2];
    int grav = (gx != 0.0 || gy != 0.0 || gz != 0.0);
    const double* D = s->dfp_to_sp;
    int nfc = s->nf;
    for (int k = 0; k < U->Nz; k++) for (int j = 0; j < U->Ny; j++) for (int i = 0; i < U->Nx; i++)
    for (int kk = 0; kk < U->nz; kk++) for (int jj = 0; jj < U->ny; jj++) for (int ii = 0; ii < U->nx; ii++)
    for (int var = 0; var < NV; var++) {
        double dudt[16];
        double u_old = *SD(U, 0, var, k, j, i, kk, jj, ii);
        for (int t = 0; t < nader; t++) {
            dudt[t] = 0;
            for (int ll = 0; ll < q; ll++) {
                if (s->act[0]) dudt[t] += *SD(Fx, t, var, k, j, i, kk, jj, ll) * D[ii * nfc + ll] / dx;
                if (s->act[1]) dudt[t] += *SD(Fy, t, var, k, j, i, kk, ll, ii) * D[jj * nfc + ll] / dy;
                if (s->act[2]) dudt[t] += *SD(Fz, t, var, k, j, i, ll, jj, ii) * D[kk * nfc + ll] / dz;
            }
            if (grav) dudt[t] -= gravity_source(Ua, var, t, k, j, i, kk, jj, ii, gx, gy, gz);
        }
        for (int t = 0; t < nader; t++) {
            double du = 0;
            for (int ll = 0; ll < nader; ll++) du += dudt[ll] * s->invader[t * nader + ll] * s->wt[ll] * dt;
            *SD(Ua, t, var, k, j, i, kk, jj, ii) = u_old - du;
        }
    }
}

/* src/transforms.cpp:327-374 */
static void update_solution(orc* s, double dt) {
    const sd_t *U = &s->U_sp, *Ua = &s->U_ader_sp;
    const sd_t *Fx = &s->F_ader_fp[0], *Fy = &s->F_ader_fp[1], *Fz = &s->F_ader_fp[2];
    int q = Fx->nx, nader = Fx->nt;
    double dx = s->d[0].h, dy = s->d[1].h, dz = s->d[2].h;
    double gx = s->c.g[0], gy = s->c.g[1], gz = s->c.g[2];
    int grav = (gx != 0.0 || gy != 0.0 || gz != 0.0);
    const double* D = s->dfp_to_sp;
    int nfc = s->nf;
    for (int k = 0; k < U->Nz; k++) for (int j = 0; j < U->Ny; j++) for (int i = 0; i < U->Nx; i++)
    for (int kk = 0; kk < U->nz; kk++) for (int jj = 0; jj < U->ny; jj++) for (int ii = 0; ii < U->nx; ii++)
    for (int var = 0; var < NV; var++) {
        double du = 0;
        for (int t = 0; t < nader; t++) {
            double dudt = 0;
            for (int ll = 0; ll < q; ll++) {
                if (s->act[0]) dudt += *SD(Fx, t, var, k, j, i, kk, jj, ll) * D[ii * nfc + ll] / dx;
                if (s->act[1]) dudt += *SD(Fy, t, var, k, j, i, kk, ll, ii) * D[jj * nfc + ll] / dy;
                if (s->act[2]) dudt += *SD(Fz, t, var, k, j, i, ll, jj, ii) * D[kk * nfc + ll] / dz;
            }
            if (grav) dudt -= gravity_source(Ua, var, t, k, j, i, kk, jj, ii, gx, gy, gz);
            du += dudt * s->wt[t] * dt;
        }
        *SD(U, 0, var, k, j, i, kk, jj, ii) -= du;
    }
}

/* src/transforms.cpp:252-261 */
static void combine_solution(const sd_t* U, const sd_t* U0, double a) {
    long n = (long)U->nv * U->Nz * U->Ny * U->Nx * U->nz * U->ny * U->nx;
    for (long o = 0; o < n; o++) U->v[o] = a * U0->v[o] + (1.0 - a) * U->v[o];
}

/* ------------------------------------------------------------------ */
/* SD primitives / conservatives / fluxes / dt: src/hydro.cpp          */
/* ------------------------------------------------------------------ */
/* src/hydro.cpp:47-70 and 108-132 (all elements, all slices) */
static void sd_conservatives(const sd_t* W, const sd_t* U, double gm) {
    long npts = (long)W->Nz * W->Ny * W->Nx * W->nz * W->ny * W->nx;
    for (int t = 0; t < W->nt; t++) for (long o = 0; o < npts; o++) {
        double w[NV], u[NV] = {0};
        for (int v = 0; v < NV; v++) w[v] = W->v[((long)t * W->nv + v) * npts + o];
        conservatives(w, u, gm);
        for (int v = 0; v < NV; v++) U->v[((long)t * U->nv + v) * npts + o] = u[v];
    }
}
static void sd_primitives(const sd_t* U, const sd_t* W, double gm) {
    long npts = (long)W->Nz * W->Ny * W->Nx * W->nz * W->ny * W->nx;
    for (int t = 0; t < W->nt; t++) for (long o = 0; o < npts; o++) {
        double u[NV], w[NV] = {0};
        for (int v = 0; v < NV; v++) u[v] = U->v[((long)t * U->nv + v) * npts + o];
        primitives(u, w, gm);
        for (int v = 0; v < NV; v++) W->v[((long)t * W->nv + v) * npts + o] = w[v];
    }
}
/* src/hydro.cpp:134-153 */
static void fv_primitives(const fv_t* U, const fv_t* W, double gm) {
    long npts = (long)W->Nz * W->Ny * W->Nx;
    for (long o = 0; o < npts; o++) {
        double u[NV], w[NV] = {0};
        for (int v = 0; v < NV; v++) u[v] = U->v[(long)v * npts + o];
        primitives(u, w, gm);
        for (int v = 0; v < NV; v++) W->v[(long)v * npts + o] = w[v];
    }
}
/* src/hydro.cpp:167-206: v1 is the normal velocity slot */
static void compute_fluxes(const sd_t* U, const sd_t* F, int v1, int v2, int v3, double gm) {
    long npts = (long)U->Nz * U->Ny * U->Nx * U->nz * U->ny * U->nx;
    for (int t = 0; t < U->nt; t++) for (long o = 0; o < npts; o++) {
        double u[NV], w[NV] = {0}, f[NV] = {0};
        for (int v = 0; v < NV; v++) u[v] = U->v[((long)t * U->nv + v) * npts + o];
        primitives(u, w, gm);
        fluxes(u, w, f, v1, v2, v3);
        for (int v = 0; v < NV; v++) F->v[((long)t * F->nv + v) * npts + o] = f[v];
    }
}
/* src/hydro.cpp:208-262 over active points; the reducer starts from the
 * largest double (Kokkos Min identity) */
static double compute_dt(orc* s, const sd_t* W) {
    double gm = s->c.gamma, cfl = s->c.cfl;
    double dx = s->d[0].h, dy = s->d[1].h, dz = s->d[2].h;
    int px = W->nx;
    double red = 1.7976931348623157e308;
    for (int k = s->ghost[2]; k < W->Nz - s->ghost[2]; k++)
    for (int j = s->ghost[1]; j < W->Ny - s->ghost[1]; j++)
    for (int i = s->ghost[0]; i < W->Nx - s->ghost[0]; i++)
    for (int kk = 0; kk < W->nz; kk++) for (int jj = 0; jj < W->ny; jj++) for (int ii = 0; ii < W->nx; ii++) {
        double cs = sound_speed(*SD(W, 0, 0, k, j, i, kk, jj, ii), *SD(W, 0, VP, k, j, i, kk, jj, ii), gm);
        double cmax = 0, dxmin = 1;
        if (s->act[0]) { cmax += (fabs(*SD(W, 0, VX, k, j, i, kk, jj, ii)) + cs); dxmin = smin(dxmin, dx); }
        if (s->act[1]) { cmax += (fabs(*SD(W, 0, VY, k, j, i, kk, jj, ii)) + cs); dxmin = smin(dxmin, dy); }
        if (s->act[2]) { cmax += (fabs(*SD(W, 0, VZ, k, j, i, kk, jj, ii)) + cs); dxmin = smin(dxmin, dz); }
        double dtm = cfl * dxmin / cmax / px;
        /* src/hydro.cpp:245-254: diffusion limit on the sub-cell grid */
        if (s->c.nu > 0.0) {
            double dx_sub = dxmin / px;
            double dt_visc = 0.25 * cfl * dx_sub * dx_sub / s->c.nu;
            dtm = dtm < dt_visc ? dtm : dt_visc;
        }
        red = red < dtm ? red : dtm;
    }
    return red;
}

/* ------------------------------------------------------------------ */
/* SD boundaries and Riemann solver                                    */
/* ------------------------------------------------------------------ */
/* src/boundary.cpp:48-113: fill the interface flux point of the ghost
 * elements of direction dim (pack, then unpack) */
static void sd_boundaries(orc* s, const sd_t* U, int dim) {
    int type = s->c.bc[dim];
    int N = s->d[dim].Ntot, n = s->d[dim].nfp;
    int Ez = dim == 2 ? 1 : U->Nz, Ey = dim == 1 ? 1 : U->Ny, Ex = dim == 0 ? 1 : U->Nx;
    int ez = dim == 2 ? 1 : U->nz, ey = dim == 1 ? 1 : U->ny, ex = dim == 0 ? 1 : U->nx;
    for (int k = 0; k < Ez; k++) for (int j = 0; j < Ey; j++) for (int i = 0; i < Ex; i++)
    for (int kk = 0; kk < ez; kk++) for (int jj = 0; jj < ey; jj++) for (int ii = 0; ii < ex; ii++)
    for (int t = 0; t < U->nt; t++) for (int var = 0; var < U->nv; var++) {
#define AT(E, P) SD(U, t, var, dim == 2 ? (E) : k, dim == 1 ? (E) : j, dim == 0 ? (E) : i, \
                    dim == 2 ? (P) : kk, dim == 1 ? (P) : jj, dim == 0 ? (P) : ii)
        double L, R;
        if (type == ORC_PERIODIC) { L = *AT(N - 2, n - 1); R = *AT(1, 0); }
        else if (type == ORC_GRADFREE) { L = *AT(1, 0); R = *AT(N - 2, n - 1); }
        else {
            double sgn = (var == 1 + dim) ? -1.0 : 1.0;
            L = sgn * *AT(1, 0);
            R = sgn * *AT(N - 2, n - 1);
        }
        *AT(0, n - 1) = L;
        *AT(N - 1, 0) = R;
#undef AT
    }
}

/* src/hydro.cpp:368-418: LLF at every element interface of direction D
 * (ghost rows included), written to both adjacent flux points */
/* src/hydro.cpp:265-268 */
static void riemann_wind(double* F, const double* UL, const double* UR, double wind) {
    for (int v = 0; v < NV; v++) F[v] = 0.5 * (UR[v] + UL[v]) + wind * (UR[v] - UL[v]);
}

static void sd_riemann(orc* s, const sd_t* U, const sd_t* F, int D) {
    static const int V1[3] = {VX, VY, VZ}, V2[3] = {VY, VZ, VX}, V3[3] = {VZ, VX, VY};
    int Nx = U->Nx - (D == 0), Ny = U->Ny - (D == 1), Nz = U->Nz - (D == 2);
    int px = D == 0 ? 1 : U->nx, py = D == 1 ? 1 : U->ny, pz = D == 2 ? 1 : U->nz;
    int n = choose(D, U->nx, U->ny, U->nz);
    double gm = s->c.gamma;
    for (int k = 0; k < Nz; k++) for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++)
    for (int kk = 0; kk < pz; kk++) for (int jj = 0; jj < py; jj++) for (int ii = 0; ii < px; ii++) {
        int l = choose(D, i, j, k);
        int kL = D == 2 ? l : k, jL = D == 1 ? l : j, iL = D == 0 ? l : i;
        int kR = D == 2 ? l + 1 : k, jR = D == 1 ? l + 1 : j, iR = D == 0 ? l + 1 : i;
        int kkL = D == 2 ? n - 1 : kk, jjL = D == 1 ? n - 1 : jj, iiL = D == 0 ? n - 1 : ii;
        int kkR = D == 2 ? 0 : kk, jjR = D == 1 ? 0 : jj, iiR = D == 0 ? 0 : ii;
        for (int t = 0; t < U->nt; t++) {
            double uL[NV], uR[NV], f[NV] = {0};
            for (int v = 0; v < NV; v++) {
                uL[v] = *SD(U, t, v, kL, jL, iL, kkL, jjL, iiL);
                uR[v] = *SD(U, t, v, kR, jR, iR, kkR, jjR, iiR);
            }
            riemann_llf(f, uL, uR, V1[D], V2[D], V3[D], gm);
            for (int v = 0; v < NV; v++) {
                *SD(F, t, v, kL, jL, iL, kkL, jjL, iiL) = f[v];
                *SD(F, t, v, kR, jR, iR, kkR, jjR, iiR) = f[v];
            }
            if (s->c.nu > 0.0) {
                /* viscous: the interface state the diffusive terms use */
                riemann_wind(f, uL, uR, 0.5);
                for (int v = 0; v < NV; v++) {
                    *SD(U, t, v, kL, jL, iL, kkL, jjL, iiL) = f[v];
                    *SD(U, t, v, kR, jR, iR, kkR, jjR, iiR) = f[v];
                }
            }
        }
    }
}

/* src/hydro.cpp:420-455: F += the wind-weighted interface value of the
 * viscous flux (arguments swapped as the reference passes them) */
static void sd_rusanov(orc* s, const sd_t* U, const sd_t* F, int D) {
    int Nx = U->Nx - (D == 0), Ny = U->Ny - (D == 1), Nz = U->Nz - (D == 2);
    int px = D == 0 ? 1 : U->nx, py = D == 1 ? 1 : U->ny, pz = D == 2 ? 1 : U->nz;
    int n = choose(D, U->nx, U->ny, U->nz);
    for (int k = 0; k < Nz; k++) for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++)
    for (int kk = 0; kk < pz; kk++) for (int jj = 0; jj < py; jj++) for (int ii = 0; ii < px; ii++) {
        int l = choose(D, i, j, k);
        int kL = D == 2 ? l : k, jL = D == 1 ? l : j, iL = D == 0 ? l : i;
        int kR = D == 2 ? l + 1 : k, jR = D == 1 ? l + 1 : j, iR = D == 0 ? l + 1 : i;
        int kkL = D == 2 ? n - 1 : kk, jjL = D == 1 ? n - 1 : jj, iiL = D == 0 ? n - 1 : ii;
        int kkR = D == 2 ? 0 : kk, jjR = D == 1 ? 0 : jj, iiR = D == 0 ? 0 : ii;
        for (int t = 0; t < U->nt; t++) {
            double uL[NV], uR[NV], f[NV];
            for (int v = 0; v < NV; v++) {
                uL[v] = *SD(U, t, v, kR, jR, iR, kkR, jjR, iiR);
                uR[v] = *SD(U, t, v, kL, jL, iL, kkL, jjL, iiL);
            }
            riemann_wind(f, uL, uR, -0.5);
            for (int v = 0; v < NV; v++) {
                *SD(F, t, v, kL, jL, iL, kkL, jjL, iiL) += f[v];
                *SD(F, t, v, kR, jR, iR, kkR, jjR, iiR) += f[v];
            }
        }
    }
}

/* src/hydro.cpp:457-490: dU = d/d(dim) of the flux-point values at the
 * solution points of the active elements */
static void compute_gradient(orc* s, const sd_t* U, const sd_t* dU, double h, int dim) {
    int q = choose(dim, dU->nx, dU->ny, dU->nz);
    int nfc = s->nf;
    for (int k = s->ghost[2]; k < dU->Nz - s->ghost[2]; k++)
    for (int j = s->ghost[1]; j < dU->Ny - s->ghost[1]; j++)
    for (int i = s->ghost[0]; i < dU->Nx - s->ghost[0]; i++)
    for (int kk = 0; kk < dU->nz; kk++) for (int jj = 0; jj < dU->ny; jj++) for (int ii = 0; ii < dU->nx; ii++)
    for (int t = 0; t < dU->nt; t++) for (int var = 0; var < NV; var++) {
        double du = 0;
        int id = choose(dim, ii, jj, kk);
        for (int ll = 0; ll < q + 1; ll++) {
            double u = dim == 0 ? *SD(U, t, var, k, j, i, kk, jj, ll)
                     : dim == 1 ? *SD(U, t, var, k, j, i, kk, ll, ii) : *SD(U, t, var, k, j, i, ll, jj, ii);
            du += u * s->dfp_to_sp[id * nfc + ll] / h;
        }
        *SD(dU, t, var, k, j, i, kk, jj, ii) = du;
    }
}

/* src/hydro.cpp:492-519 */
static void viscous_fluxes(double* f, const double* w, const double* du1, int v1, const double* du2, int v2,
                           const double* du3, int v3, double nu, double beta) {
    f[0] = 0;
    f[VP] = 0;
    f[v1] = 2 * nu * du1[v1] + beta * du1[v1];
    f[v1] += beta * du2[v2];
    f[v2] = nu * (du1[v2] + du2[v1]);
    f[VP] += w[v2] * f[v2];
    f[v1] += beta * du3[v3];
    f[v3] = nu * (du1[v3] + du3[v1]);
    f[VP] += w[v3] * f[v3];
    f[VP] += w[v1] * f[v1];
}

/* src/hydro.cpp:521-572: the viscous flux at every flux point of
 * direction dim (ghost elements included), written over U */
static void compute_viscous_flux(orc* s, const sd_t* U, const sd_t* dU1, int v1, const sd_t* dU2, int v2,
                                 const sd_t* dU3, int v3, int dim) {
    double nu = s->c.nu, beta = s->c.beta, gm = s->c.gamma;
    int q = choose(dim, U->nx, U->ny, U->nz);
    int n = s->n;
    for (int k = 0; k < U->Nz; k++) for (int j = 0; j < U->Ny; j++) for (int i = 0; i < U->Nx; i++)
    for (int kk = 0; kk < U->nz; kk++) for (int jj = 0; jj < U->ny; jj++) for (int ii = 0; ii < U->nx; ii++)
    for (int t = 0; t < U->nt; t++) {
        double f[NV] = {0}, u[NV], w[NV] = {0}, du1[NV], du2[NV], du3[NV];
        int id = choose(dim, ii, jj, kk);
        for (int var = 0; var < NV; var++) {
            du1[var] = 0;
            du2[var] = 0;
            du3[var] = 0;
            u[var] = *SD(U, t, var, k, j, i, kk, jj, ii);
            for (int ll = 0; ll < q - 1; ll++) {
                int nk = dim == 2 ? ll : kk, nj = dim == 1 ? ll : jj, ni = dim == 0 ? ll : ii;
                du1[var] += *SD(dU1, t, var, k, j, i, nk, nj, ni) * s->sp_to_fp[id * n + ll];
                du2[var] += *SD(dU2, t, var, k, j, i, nk, nj, ni) * s->sp_to_fp[id * n + ll];
                du3[var] += *SD(dU3, t, var, k, j, i, nk, nj, ni) * s->sp_to_fp[id * n + ll];
            }
        }
        primitives(u, w, gm);
        viscous_fluxes(f, w, du1, v1, du2, v2, du3, v3, nu, beta);
        for (int var = 0; var < NV; var++) *SD(U, t, var, k, j, i, kk, jj, ii) = f[var];
    }
}

/* src/hydro_ader.hpp:278-289: sp->fp, fluxes, ghost fill, LLF; with
 * hydro/nu > 0 the viscous terms (:380-405): gradients, viscous fluxes,
 * ghost fill, interface sums */
void orc_solve_fluxes(orc* s) {
    static const int V1[3] = {VX, VY, VZ}, V2[3] = {VY, VZ, VX}, V3[3] = {VZ, VX, VY};
    for (int d = 0; d < 3; d++)
        if (s->act[d]) transform_1d(&s->U_ader_sp, &s->U_ader_fp[d], s->sp_to_fp, s->n, d);
    for (int d = 0; d < 3; d++)
        if (s->act[d]) compute_fluxes(&s->U_ader_fp[d], &s->F_ader_fp[d], V1[d], V2[d], V3[d], s->c.gamma);
    for (int d = 0; d < 3; d++)
        if (s->act[d]) sd_boundaries(s, &s->U_ader_fp[d], d);
    for (int d = 0; d < 3; d++)
        if (s->act[d]) sd_riemann(s, &s->U_ader_fp[d], &s->F_ader_fp[d], d);
    if (s->c.nu > 0.0) {
        for (int d = 0; d < 3; d++)
            if (s->act[d]) compute_gradient(s, &s->U_ader_fp[d], &s->dU_sp[d], s->d[d].h, d);
        for (int d = 0; d < 3; d++)
            if (s->act[d])
                compute_viscous_flux(s, &s->U_ader_fp[d], &s->dU_sp[d], V1[d], &s->dU_sp[(d + 1) % 3], V2[d],
                                     &s->dU_sp[(d + 2) % 3], V3[d], d);
        for (int d = 0; d < 3; d++)
            if (s->act[d]) sd_boundaries(s, &s->U_ader_fp[d], d);
        for (int d = 0; d < 3; d++)
            if (s->act[d]) sd_rusanov(s, &s->U_ader_fp[d], &s->F_ader_fp[d], d);
    }
}

/* ------------------------------------------------------------------ */
/* FV sub-grid: face integral, update, boundaries                      */
/* ------------------------------------------------------------------ */
/* src/transforms.cpp:378-427 (one transverse direction active, 1D/2D) and
 * 435-481 (sweep form when both transverse directions are active) */
static void face_integral(orc* s, int dim, int tid) {
    const sd_t* Ff = &s->F_ader_fp[dim];
    const fv_t* F = &s->F[dim];
    int Nx = Ff->Nx + (dim == 0), Ny = Ff->Ny + (dim == 1), Nz = Ff->Nz + (dim == 2);
    int px = Ff->nx - (dim == 0), py = Ff->ny - (dim == 1), pz = Ff->nz - (dim == 2);
    int dim1 = choose(dim, 1, 2, 0), dim2 = choose(dim1, 1, 2, 0);
    int q1 = choose(dim1, px, py, pz), q2 = choose(dim2, px, py, pz);
    int a1 = s->act[dim1], a2 = s->act[dim2];
    const double* M = s->sp_to_cv;
    int n = s->n;
    int both = a1 && a2;
    if (both) transform_1d_slice(Ff, &s->T_fp[dim], M, n, dim1, tid);
    for (int k = s->ghost[2]; k < Nz - s->ghost[2]; k++)
    for (int j = s->ghost[1]; j < Ny - s->ghost[1]; j++)
    for (int i = s->ghost[0]; i < Nx - s->ghost[0]; i++)
    for (int kk = 0; kk < pz; kk++) for (int jj = 0; jj < py; jj++) for (int ii = 0; ii < px; ii++) {
        int I = ii + s->fvg[0] + (i - s->ghost[0]) * px;
        int J = jj + s->fvg[1] + (j - s->ghost[1]) * py;
        int K = kk + s->fvg[2] + (k - s->ghost[2]) * pz;
        int id1 = choose(dim1, ii, jj, kk), id2 = choose(dim2, ii, jj, kk);
        for (int var = 0; var < NV; var++) {
            double f = 0;
            int nid[3];
            if (!both) {
                for (int nn = 0; nn < q2; nn++) {
                    nid[0] = ii; nid[1] = jj; nid[2] = kk;
                    nid[dim2] = nn;
                    for (int ll = 0; ll < q1; ll++) {
                        nid[dim1] = ll;
                        double sv = *SD(Ff, tid, var, k, j, i, nid[2], nid[1], nid[0]);
                        if (a1) sv *= M[id1 * n + ll];
                        if (a2) sv *= M[id2 * n + nn];
                        f += sv;
                    }
                }
            } else {
                for (int nn = 0; nn < q2; nn++) {
                    nid[0] = ii; nid[1] = jj; nid[2] = kk;
                    nid[dim2] = nn;
                    f += *SD(&s->T_fp[dim], 0, var, k, j, i, nid[2], nid[1], nid[0]) * M[id2 * n + nn];
                }
            }
            if (K < F->Nz && J < F->Ny && I < F->Nx) *FV(F, var, K, J, I) = f;
        }
    }
}

/* src/transforms.cpp:483-543. With update set, U_cv is overwritten variable
 * by variable, so the gravity source of a later variable sees the updated
 * density/momentum of the same cell (as in the reference). */
static void fv_update_solution(orc* s, int tid, double dt, int update) {
    const sd_t* Ucv = &s->U_cv;
    double gx = s->c.g[0], gy = s->c.g[1], gz = s->c.g[2];
    int grav = (gx != 0.0 || gy != 0.0 || gz != 0.0);
    int px = Ucv->nx, py = Ucv->ny, pz = Ucv->nz;
    for (int k = s->ghost[2]; k < Ucv->Nz - s->ghost[2]; k++)
    for (int j = s->ghost[1]; j < Ucv->Ny - s->ghost[1]; j++)
    for (int i = s->ghost[0]; i < Ucv->Nx - s->ghost[0]; i++)
    for (int kk = 0; kk < pz; kk++) for (int jj = 0; jj < py; jj++) for (int ii = 0; ii < px; ii++) {
        int I = ii + s->fvg[0] + (i - s->ghost[0]) * px;
        int J = jj + s->fvg[1] + (j - s->ghost[1]) * py;
        int K = kk + s->fvg[2] + (k - s->ghost[2]) * pz;
        for (int var = 0; var < NV; var++) {
            double F = 0, h;
            *FV(&s->U_old, var, K, J, I) = *SD(Ucv, 0, var, k, j, i, kk, jj, ii);
            if (s->act[0]) {
                h = s->d[0].fv_faces[I + 1] - s->d[0].fv_faces[I];
                F += (*FV(&s->F[0], var, K, J, I + 1) - *FV(&s->F[0], var, K, J, I)) / h;
            }
            if (s->act[1]) {
                h = s->d[1].fv_faces[J + 1] - s->d[1].fv_faces[J];
                F += (*FV(&s->F[1], var, K, J + 1, I) - *FV(&s->F[1], var, K, J, I)) / h;
            }
            if (s->act[2]) {
                h = s->d[2].fv_faces[K + 1] - s->d[2].fv_faces[K];
                F += (*FV(&s->F[2], var, K + 1, J, I) - *FV(&s->F[2], var, K, J, I)) / h;
            }
            if (grav) F -= gravity_source(Ucv, var, 0, k, j, i, kk, jj, ii, gx, gy, gz);
            double u_new = *FV(&s->U_old, var, K, J, I) - s->wt[tid] * dt * F;
            *FV(&s->U_new, var, K, J, I) = u_new;
            if (update) *SD(Ucv, 0, var, k, j, i, kk, jj, ii) = u_new;
        }
    }
}

/* src/boundary.cpp:123-190 for cell-centred arrays: nGH ghost layers in
 * direction dim, over every transverse cell (ghost rows included) */
static void fv_boundaries_dim(orc* s, const fv_t* U, int dim) {
    int type = s->c.bc[dim];
    int N = s->d[dim].fvn;
    int Ez = dim == 2 ? NGHFV : U->Nz, Ey = dim == 1 ? NGHFV : U->Ny, Ex = dim == 0 ? NGHFV : U->Nx;
    for (int k = 0; k < Ez; k++) for (int j = 0; j < Ey; j++) for (int i = 0; i < Ex; i++)
    for (int var = 0; var < U->nv; var++) {
        int l = choose(dim, i, j, k);
#define AT(L) FV(U, var, dim == 2 ? (L) : k, dim == 1 ? (L) : j, dim == 0 ? (L) : i)
        double vL, vR;
        if (type == ORC_PERIODIC) { vL = *AT(N - 2 * NGHFV + l); vR = *AT(NGHFV + l); }
        else if (type == ORC_GRADFREE) { vL = *AT(NGHFV + l); vR = *AT(N - 2 * NGHFV + l); }
        else {
            double sgn = (var == 1 + dim) ? -1.0 : 1.0;
            vL = sgn * *AT(2 * NGHFV - 1 - l);
            vR = sgn * *AT(N - NGHFV - 1 - l);
        }
        *AT(l) = vL;
        *AT(N - NGHFV + l) = vR;
#undef AT
    }
}
static void fv_boundaries(orc* s, const fv_t* U) {
    for (int d = 0; d < 3; d++)
        if (s->act[d]) fv_boundaries_dim(s, U, d);
}

/* ------------------------------------------------------------------ */
/* trouble detection: src/trouble_detection.cpp                        */
/* ------------------------------------------------------------------ */
/* src/trouble_detection.cpp:12-31 */
static double Alpha(double dv, double dUm, double dU, double dUp) {
    double vL = dU - dUm;
    double ap = smin(1.0, smax(vL, 0.0) / dv);
    double am = smin(1.0, smin(vL, 0.0) / dv);
    double aL = (dv < 0.0 ? am : ap);
    aL = (dv == 0.0 ? 1.0 : aL);
    double vR = dUp - dU;
    ap = smin(1.0, smax(vR, 0.0) / dv);
    am = smin(1.0, smin(vR, 0.0) / dv);
    double aR = (dv < 0.0 ? am : ap);
    aR = (dv == 0.0 ? 1.0 : aR);
    return smin(aL, aR);
}

/* range of fv_for_cells_ngh / _2ngh (src/define.hpp:286-306) */
static void ngh_range(orc* s, const fv_t* U, int layers, int lo[3], int hi[3]) {
    int n[3] = {U->Nx, U->Ny, U->Nz};
    for (int d = 0; d < 3; d++) {
        int g = s->act[d] ? layers : 0;
        lo[d] = g;
        hi[d] = n[d] - g;
    }
}

/* src/trouble_detection.cpp:35-104 */
static void NAD(orc* s, const fv_t* Un, const fv_t* U, const fv_t* tr, double tol, int mask) {
    int lo[3], hi[3];
    ngh_range(s, U, 1, lo, hi);
    int ax = s->act[0], ay = s->act[1], az = s->act[2];
    for (int k = lo[2]; k < hi[2]; k++) for (int j = lo[1]; j < hi[1]; j++) for (int i = lo[0]; i < hi[0]; i++)
    for (int var = 0; var < NV; var++) {
        if (!((mask >> var) & 1)) continue;
        double un = *FV(Un, var, k, j, i);
        double mx = *FV(U, var, k, j, i), mn = mx;
        if (s->c.nad_moore) {
            for (int dk = -az; dk <= az; dk++) for (int dj = -ay; dj <= ay; dj++) for (int di = -ax; di <= ax; di++) {
                double u = *FV(U, var, k + dk, j + dj, i + di);
                mx = smax(mx, u);
                mn = smin(mn, u);
            }
        } else {
            for (int d = 0; d < 3; d++) {
                if (!s->act[d]) continue;
                double uL = *FV(U, var, k - (d == 2), j - (d == 1), i - (d == 0));
                double uR = *FV(U, var, k + (d == 2), j + (d == 1), i + (d == 0));
                mx = smax(smax(uL, mx), uR);
                mn = smin(smin(uL, mn), uR);
            }
        }
        if (s->c.nad_delta) {
            double eps = tol * (mx - mn);
            mn -= eps;
            mx += eps;
        } else {
            mn -= fabs(mn) * tol;
            mx += fabs(mx) * tol;
        }
        *FV(tr, var, k, j, i) = (un > mx || un < mn) ? 1 : 0;
    }
}

/* src/trouble_detection.cpp:107-148 (active cells only) */
static void smooth_extrema(orc* s, const fv_t* U, const fv_t* alpha, int dim, int mask) {
    int lo[3], hi[3];
    ngh_range(s, U, 2, lo, hi);
    const double* c = s->d[dim].fv_centers;
    const double* f = s->d[dim].fv_faces;
    for (int k = lo[2]; k < hi[2]; k++) for (int j = lo[1]; j < hi[1]; j++) for (int i = lo[0]; i < hi[0]; i++)
    for (int var = 0; var < NV; var++) {
        if (!((mask >> var) & 1)) continue;
        double u = *FV(U, var, k, j, i);
        int l = choose(dim, i, j, k);
        double h = (c[l + 1] - c[l - 1]);
        double hp = (c[l + 2] - c[l]);
        double hm = (c[l] - c[l - 2]);
        int ox = dim == 0, oy = dim == 1, oz = dim == 2;
        double du = (*FV(U, var, k + oz, j + oy, i + ox) - *FV(U, var, k - oz, j - oy, i - ox)) / h;
        double dup = (*FV(U, var, k + 2 * oz, j + 2 * oy, i + 2 * ox) - u) / hp;
        double dum = (u - *FV(U, var, k - 2 * oz, j - 2 * oy, i - 2 * ox)) / hm;
        double d2u = (dup - dum) / (c[l + 1] - c[l - 1]);
        double dv = 0.5 * d2u * (f[l + 1] - f[l]);
        *FV(alpha, var, k, j, i) = Alpha(dv, dum, du, dup);
    }
}

/* src/trouble_detection.cpp:152-183 */
static void relax_NAD(orc* s, const fv_t* tr, int mask, int use_sed) {
    int lo[3], hi[3];
    ngh_range(s, tr, 1, lo, hi);
    const fv_t *ax = &s->alpha[0], *ay = &s->alpha[1], *az = &s->alpha[2];
    for (int k = lo[2]; k < hi[2]; k++) for (int j = lo[1]; j < hi[1]; j++) for (int i = lo[0]; i < hi[0]; i++) {
        for (int var = 0; var < NV; var++) {
            if (!((mask >> var) & 1)) continue;
            double alpha = 1;
            if (s->act[0]) alpha = smin(smin(*FV(ax, var, k, j, i - 1), *FV(ax, var, k, j, i)), *FV(ax, var, k, j, i + 1));
            if (s->act[1]) alpha = smin(alpha, smin(smin(*FV(ay, var, k, j - 1, i), *FV(ay, var, k, j, i)), *FV(ay, var, k, j + 1, i)));
            if (s->act[2]) alpha = smin(alpha, smin(smin(*FV(az, var, k - 1, j, i), *FV(az, var, k, j, i)), *FV(az, var, k + 1, j, i)));
            double trouble = *FV(tr, var, k, j, i);
            if (use_sed) *FV(tr, var, k, j, i) = alpha < 1 ? trouble : 0;
        }
        double trouble = 0;
        for (int var = 0; var < NV; var++)
            if ((mask >> var) & 1) trouble = smax(trouble, *FV(tr, var, k, j, i));
        *FV(tr, NV, k, j, i) = trouble;
    }
}

/* src/trouble_detection.cpp:244-259 */
static void PAD(orc* s, const fv_t* W, const fv_t* tr) {
    int lo[3], hi[3];
    ngh_range(s, W, 1, lo, hi);
    for (int k = lo[2]; k < hi[2]; k++) for (int j = lo[1]; j < hi[1]; j++) for (int i = lo[0]; i < hi[0]; i++) {
        double rho = *FV(W, 0, k, j, i), p = *FV(W, VP, k, j, i);
        if (rho < RHO_MIN || rho > RHO_MAX) *FV(tr, NV, k, j, i) = 1;
        if (p < P_MIN || p > P_MAX) *FV(tr, NV, k, j, i) = 1;
    }
}

/* src/trouble_detection.cpp:191-210 */
static void apply_blending(orc* s, const fv_t* tr, const fv_t* th) {
    static const double w[4] = {1.0, 0.75, 0.5, 0.375};
    int lo[3], hi[3];
    ngh_range(s, tr, 1, lo, hi);
    int ax = s->act[0], ay = s->act[1], az = s->act[2];
    for (int k = lo[2]; k < hi[2]; k++) for (int j = lo[1]; j < hi[1]; j++) for (int i = lo[0]; i < hi[0]; i++) {
        double t = 0;
        for (int dk = -az; dk <= az; dk++) for (int dj = -ay; dj <= ay; dj++) for (int di = -ax; di <= ax; di++) {
            int n0 = (di != 0) + (dj != 0) + (dk != 0);
            t = smax(t, w[n0] * *FV(tr, NV, k + dk, j + dj, i + di));
        }
        *FV(th, 0, k, j, i) = t;
    }
}
/* src/trouble_detection.cpp:213-221 */
static void theta_from_troubles(orc* s, const fv_t* tr, const fv_t* th) {
    long n = (long)tr->Nz * tr->Ny * tr->Nx;
    for (long o = 0; o < n; o++) th->v[o] = tr->v[(long)NV * n + o];
}
/* src/trouble_detection.cpp:226-242 */
static void blending_ring(orc* s, const fv_t* ti, const fv_t* to) {
    int lo[3], hi[3];
    ngh_range(s, ti, 1, lo, hi);
    int ax = s->act[0], ay = s->act[1], az = s->act[2];
    for (int k = lo[2]; k < hi[2]; k++) for (int j = lo[1]; j < hi[1]; j++) for (int i = lo[0]; i < hi[0]; i++) {
        double t = *FV(ti, 0, k, j, i), ring = 0;
        for (int dk = -az; dk <= az; dk++) for (int dj = -ay; dj <= ay; dj++) for (int di = -ax; di <= ax; di++)
            if (*FV(ti, 0, k + dk, j + dj, i + di) > 0) ring = 0.25;
        *FV(to, 0, k, j, i) = smax(t, ring);
    }
}
/* src/trouble_detection.cpp:261-290 */
static void detect_troubles(orc* s, int mask) {
    double tol = s->c.nad_tolerance;
    int use_sed = s->c.sed && s->d[0].p > 1;
    NAD(s, &s->W_new, &s->W_old, &s->troubles, tol, mask);
    if (use_sed)
        for (int d = 0; d < 3; d++)
            if (s->act[d]) smooth_extrema(s, &s->W_new, &s->alpha[d], d, mask);
    relax_NAD(s, &s->troubles, mask, use_sed);
    PAD(s, &s->W_new, &s->troubles);
}

/* ------------------------------------------------------------------ */
/* MUSCL-Hancock fallback fluxes: src/hydro.cpp:591-788, src/muscl.hpp */
/* ------------------------------------------------------------------ */
/* src/muscl.hpp:2-12 */
static double minmod(double SL, double SR, double xL, double xR) {
    double ratio = SR / SL;
    ratio = smax(0.0, smin(ratio, 1.0));
    double slope = ratio * SL;
    return 0.5 * slope * (xR - xL);
}
/* src/hydro.cpp:591-615 (Hancock half step of the primitive variables) */
static void corrector(const double* W, double* dWt, const double* dWx, const double* dWy, const double* dWz,
                      double gm) {
    dWt[0] = 0;
    dWt[VP] = 0;
    dWt[0] -= W[VX] * dWx[0] + W[0] * dWx[VX];
    dWt[VX] = -W[VX] * dWx[VX] - dWx[VP] / W[0];
    dWt[VP] -= W[VX] * dWx[VP] + dWx[VX] * gm * W[VP];
    dWt[VX] -= W[VY] * dWy[VX];
    dWt[VX] -= W[VZ] * dWz[VX];

    dWt[0] -= W[VY] * dWy[0] + W[0] * dWy[VY];
    dWt[VY] = -W[VY] * dWy[VY] - dWy[VP] / W[0];
    dWt[VP] -= W[VY] * dWy[VP] + dWy[VY] * gm * W[VP];
    dWt[VY] -= W[VX] * dWx[VY];
    dWt[VY] -= W[VZ] * dWz[VY];

    dWt[0] -= W[VZ] * dWz[0] + W[0] * dWz[VZ];
    dWt[VZ] = -W[VZ] * dWz[VZ] - dWz[VP] / W[0];
    dWt[VP] -= W[VZ] * dWz[VP] + dWz[VZ] * gm * W[VP];
    dWt[VZ] -= W[VX] * dWx[VZ];
    dWt[VZ] -= W[VY] * dWy[VZ];
}
/* src/hydro.cpp:622-681: slopes in every active direction, Hancock step,
 * face values on the two faces of direction D */
static void slopes_d(orc* s, const fv_t* W, int D, int k, int j, int i, double* WL, double* WR, double dt) {
    const double *xc = s->d[0].fv_centers, *xf = s->d[0].fv_faces;
    const double *yc = s->d[1].fv_centers, *yf = s->d[1].fv_faces;
    const double *zc = s->d[2].fv_centers, *zf = s->d[2].fv_faces;
    double w[NV], dwx[NV], dwy[NV], dwz[NV], dwt[NV];
    for (int v = 0; v < NV; v++) {
        w[v] = *FV(W, v, k, j, i);
        double wL = *FV(W, v, k, j, i - 1), wR = *FV(W, v, k, j, i + 1);
        dwx[v] = minmod((wR - w[v]) / (xc[i + 1] - xc[i]), (w[v] - wL) / (xc[i] - xc[i - 1]), xf[i], xf[i + 1]);
        dwy[v] = 0;
        dwz[v] = 0;
        if (s->act[1]) {
            wL = *FV(W, v, k, j - 1, i);
            wR = *FV(W, v, k, j + 1, i);
            dwy[v] = minmod((wR - w[v]) / (yc[j + 1] - yc[j]), (w[v] - wL) / (yc[j] - yc[j - 1]), yf[j], yf[j + 1]);
        }
        if (s->act[2]) {
            wL = *FV(W, v, k - 1, j, i);
            wR = *FV(W, v, k + 1, j, i);
            dwz[v] = minmod((wR - w[v]) / (zc[k + 1] - zc[k]), (w[v] - wL) / (zc[k] - zc[k - 1]), zf[k], zf[k + 1]);
        }
    }
    corrector(w, dwt, dwx, dwy, dwz, s->c.gamma);
    for (int v = 0; v < NV; v++) {
        double h = (D == 0 ? xf[i + 1] - xf[i] : (D == 1 ? yf[j + 1] - yf[j] : zf[k + 1] - zf[k]));
        double dw = (D == 0 ? dwx[v] : (D == 1 ? dwy[v] : dwz[v]));
        WR[v] = w[v] - dw + dwt[v] * dt / h;
        WL[v] = w[v] + dw + dwt[v] * dt / h;
    }
}
/* src/hydro.cpp:683-751: HLLC flux of the MUSCL-Hancock face states,
 * blended into the SD face flux with theta_face = max of the two cells */
static void fallback_face(orc* s, const fv_t* W, const fv_t* F, int D, int k, int j, int i, double dt) {
    static const int V1[3] = {VX, VY, VZ}, V2[3] = {VY, VZ, VX}, V3[3] = {VZ, VX, VY};
    double wL[2][NV], wR[2][NV], uL[NV], uR[NV], fL[NV];
    for (int l = -1; l < 1; l++)
        slopes_d(s, W, D, k + (D == 2 ? l : 0), j + (D == 1 ? l : 0), i + (D == 0 ? l : 0), wL[l + 1], wR[l + 1], dt);
    conservatives(wL[0], uL, s->c.gamma);
    conservatives(wR[1], uR, s->c.gamma);
    riemann_hllc(fL, uL, uR, V1[D], V2[D], V3[D], s->c.gamma);
    double th = smax(*FV(&s->theta, 0, k, j, i), *FV(&s->theta, 0, k - (D == 2), j - (D == 1), i - (D == 0)));
    for (int v = 0; v < NV; v++) {
        double f = *FV(F, v, k, j, i);
        f = f + th * (fL[v] - f);
        *FV(F, v, k, j, i) = f;
    }
}
/* src/hydro.cpp:753-788 (fv_for_faces range: one cell past the active
 * region in every active direction) */
static void fallback_fluxes(orc* s, int tid, double dt) {
    const fv_t* W = &s->W_old;
    int lo[3], hi[3], n[3] = {W->Nx, W->Ny, W->Nz};
    for (int d = 0; d < 3; d++) {
        int g = s->act[d] ? NGHFV : 0;
        lo[d] = g;
        hi[d] = n[d] - 2 * g + (g > 0) + g;
    }
    double dtw = s->wt[tid] * dt;
    for (int k = lo[2]; k < hi[2]; k++) for (int j = lo[1]; j < hi[1]; j++) for (int i = lo[0]; i < hi[0]; i++) {
        fallback_face(s, W, &s->F[0], 0, k, j, i, dtw);
        if (s->act[1]) fallback_face(s, W, &s->F[1], 1, k, j, i, dtw);
        if (s->act[2]) fallback_face(s, W, &s->F[2], 2, k, j, i, dtw);
    }
}

/* src/hydro_ader.hpp:500-575 */
void orc_fv_update(orc* s, double dt) {
    const int mask = (1 << 0) | (1 << VP);
    transform_a_to_b(s, &s->U_sp, &s->U_cv, &s->T_sweep, s->sp_to_cv);
    for (int t = 0; t < s->nader; t++) {
        for (int d = 0; d < 3; d++)
            if (s->act[d]) face_integral(s, d, t);
        fv_update_solution(s, t, dt, 0);
        fv_boundaries(s, &s->U_old);
        fv_boundaries(s, &s->U_new);
        fv_primitives(&s->U_new, &s->W_new, s->c.gamma);
        fv_primitives(&s->U_old, &s->W_old, s->c.gamma);
        detect_troubles(s, mask);
        fv_boundaries(s, &s->troubles);
        if (s->c.blending) {
            apply_blending(s, &s->troubles, &s->theta_tmp);
            blending_ring(s, &s->theta_tmp, &s->theta);
        } else
            theta_from_troubles(s, &s->troubles, &s->theta);
        fv_boundaries(s, &s->theta);
        fallback_fluxes(s, t, dt);
        fv_update_solution(s, t, dt, 1);
    }
    transform_a_to_b(s, &s->U_cv, &s->U_sp, &s->T_sweep, s->cv_to_sp);
}

/* ------------------------------------------------------------------ */
/* initial conditions: src/initial_conditions.cpp:9-228                */
/* ------------------------------------------------------------------ */
static uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
/* uniform in [-1,1) from the bit patterns of the point coordinates: the
 * seeded noise of the project's Kelvin-Helmholtz problem */
static double coord_noise(uint64_t seed, double x, double y, double z) {
    uint64_t bx, by, bz;
    memcpy(&bx, &x, 8);
    memcpy(&by, &y, 8);
    memcpy(&bz, &z, 8);
    uint64_t h = splitmix64(seed ^ splitmix64(bx ^ splitmix64(by ^ splitmix64(bz))));
    return (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

static double ic_point(const orc_cfg* c, int var, double x, double y, double z, int ay, int az) {
    double gm = c->gamma;
    switch (c->problem) {
    case ORC_IC_SINE: /* src/initial_conditions.cpp:28-36 */
        if (var == 0) return c->d0 + c->amp * (sin(2 * PI_REF * (x + y)));
        if (var == VX) return c->v1;
        if (var == VY) return c->v2;
        if (var == VZ) return c->v3;
        if (var == VP) return c->p0;
        return 0;
    case ORC_IC_SEDOV: { /* :39-53 */
        double r = sqrt(pow(x - 0.5, 2.0) + pow(y - 0.5, 2.0) + (az ? pow(z - 0.5, 2.0) : 0.0));
        if (var == 0) return c->d0;
        if (var == VP) return r < c->radius ? 1E-6 + (gm - 1) : 1E-6;
        return 0;
    }
    case ORC_IC_BLAST: { /* :55-72 */
        double r = sqrt(pow(x - c->cx, 2) + pow(y - c->cy, 2) + (az ? pow(z - c->cz, 2) : 0.0));
        if (var == 0) return c->d0;
        if (var == VP) return r < c->radius ? c->p0 : c->p1;
        return 0;
    }
    case ORC_IC_SQUARE: { /* :9-26 */
        if (var == 0) {
            int in = fabs(x - 0.5) < c->radius;
            if (ay) in = in && fabs(y - 0.5) < c->radius;
            if (az) in = in && fabs(z - 0.5) < c->radius;
            return in ? c->d1 : c->d0;
        }
        if (var == VX) return c->v1;
        if (var == VY) return c->v2;
        if (var == VZ) return c->v3;
        if (var == VP) return c->p0;
        return 0;
    }
    case ORC_IC_SOD: { /* :74-84 */
        double sc = (c->dir == 0 ? x : (c->dir == 1 ? y : z));
        int left = sc < c->radius;
        if (var == 0) return left ? c->d0 : c->d1;
        if (var == VP) return left ? c->p0 : c->p1;
        return 0;
    }
    case ORC_IC_SHU_OSHER: { /* :86-99 */
        double xs = x - 1.0;
        int left = xs < -0.8;
        if (var == 0) return left ? 3.857143 : 1.0 + c->amp * sin(5 * PI_REF * xs);
        if (var == VX) return left ? 2.629369 : 0.0;
        if (var == VP) return left ? 10.33333 : 1.0;
        return 0;
    }
    case ORC_IC_KH: { /* :101-117 */
        int inner = (y > 0.25 && y < 0.75);
        if (var == 0) return inner ? c->d1 : c->d0;
        if (var == VX) return inner ? c->v1 : -c->v1;
        if (var == VY)
            return c->amp * sin(4 * PI_REF * x) *
                   (exp(-pow(y - 0.25, 2) / (2 * c->sigma * c->sigma)) + exp(-pow(y - 0.75, 2) / (2 * c->sigma * c->sigma)));
        if (var == VP) return c->p0;
        return 0;
    }
    case ORC_IC_IMPLOSION: { /* :119-129 */
        int inside = (x + y) < c->radius;
        if (var == 0) return inside ? c->d1 : c->d0;
        if (var == VP) return inside ? c->p1 : c->p0;
        return 0;
    }
    case ORC_IC_RTI: { /* :131-159 */
        double gy = c->g[1];
        double yc = c->radius, rho_hi = c->d0, rho_lo = c->d1, P0 = c->p0;
        int top = y > yc;
        if (var == 0) return top ? rho_lo : rho_hi;
        if (var == VY) {
            double dv = sqrt(gm * (rho_hi * yc + 1.0) / rho_hi);
            return -c->amp * dv * cos(8.0 * PI_REF * x);
        }
        if (var == VP) return top ? (P0 + rho_lo * gy * y + (rho_hi - rho_lo) * gy * yc) : (P0 + rho_hi * gy * y);
        return 0;
    }
    case ORC_IC_USER: { /* src/user_ic.hpp:40-51 */
        double dx = x - c->radius;
        double pulse = c->amp * exp(-dx * dx / (2 * c->sigma * c->sigma));
        if (var == 0) return c->d0;
        if (var == VX) return c->v1;
        if (var == VY) return pulse;
        if (var == VZ) return 0.0;
        if (var == VP) return c->p0;
        return 0;
    }
    case ORC_IC_KH_NOISE: {
        /* shear layer: rho=d1, vx=+v1 for |y-0.5|<0.25, else rho=d0, vx=-v1;
         * P=p0; vy = amp sin(4 pi x) + q[0] U(-1,1) */
        int inner = fabs(y - 0.5) < 0.25;
        if (var == 0) return inner ? c->d1 : c->d0;
        if (var == VX) return inner ? c->v1 : -c->v1;
        if (var == VY) return c->amp * sin(4 * PI_REF * x) + c->q[0] * coord_noise(c->seed, x, y, z);
        if (var == VP) return c->p0;
        return 0;
    }
    case ORC_IC_QUADRANT: {
        /* four-quadrant Riemann problem about (cx, cy); quadrant
         * q = (x>cx) + 2 (y>cy) holds rho=q[4q], P=q[4q+1], vx=q[4q+2], vy=q[4q+3] */
        int qd = (x > c->cx) + 2 * (y > c->cy);
        if (var == 0) return c->q[4 * qd];
        if (var == VP) return c->q[4 * qd + 1];
        if (var == VX) return c->q[4 * qd + 2];
        if (var == VY) return c->q[4 * qd + 3];
        return 0;
    }
    case ORC_IC_RTI_TOP: {
        /* heavy fluid d0 above y = radius, light d1 below, hydrostatic with
         * P = p0 at the interface; vy = amp (1+cos 4 pi x)(1+cos 3 pi (y-yc))/4 */
        double gy = c->g[1], yc = c->radius;
        int top = y > yc;
        double rho = top ? c->d0 : c->d1;
        if (var == 0) return rho;
        if (var == VY) return c->amp * (1 + cos(4 * PI_REF * x)) * (1 + cos(3 * PI_REF * (y - yc))) / 4;
        if (var == VP) return c->p0 + rho * gy * (y - yc);
        return 0;
    }
    }
    return 0;
}

/* src/initial_conditions.cpp:179-228: GL-quadrature averages of the point
 * ICs over every FV sub-cell (ghost elements included) */
static void initialize(orc* s, const sd_t* U) {
    const double *fx = s->d[0].sd_faces, *fy = s->d[1].sd_faces, *fz = s->d[2].sd_faces;
    int nfx = s->d[0].nfp, nfy = s->d[1].nfp, nfz = s->d[2].nfp;
    int ay = s->act[1], az = s->act[2];
    int px = U->nx, py = U->ny, pz = U->nz;
    for (int k = 0; k < U->Nz; k++) for (int j = 0; j < U->Ny; j++) for (int i = 0; i < U->Nx; i++)
    for (int kk = 0; kk < pz; kk++) for (int jj = 0; jj < py; jj++) for (int ii = 0; ii < px; ii++)
    for (int var = 0; var < NV; var++) {
        double value = 0, x, y = 0, z = 0;
        for (int nn = 0; nn < pz; nn++) {
            if (az) z = fz[k * nfz + kk] + s->xx[nn] * (fz[k * nfz + kk + 1] - fz[k * nfz + kk]);
            for (int mm = 0; mm < py; mm++) {
                if (ay) y = fy[j * nfy + jj] + s->xx[mm] * (fy[j * nfy + jj + 1] - fy[j * nfy + jj]);
                for (int ll = 0; ll < px; ll++) {
                    x = fx[i * nfx + ii] + s->xx[ll] * (fx[i * nfx + ii + 1] - fx[i * nfx + ii]);
                    double sv = ic_point(&s->c, var, x, y, z, ay, az);
                    sv *= s->wx[ll];
                    if (ay) sv *= s->wx[mm];
                    if (az) sv *= s->wx[nn];
                    value += sv;
                }
            }
        }
        *SD(U, 0, var, k, j, i, kk, jj, ii) = value;
    }
}

/* ------------------------------------------------------------------ */
/* construction and stepping: src/hydro_ader.hpp:76-213, 291-325       */
/* ------------------------------------------------------------------ */
orc* orc_create(const orc_cfg* cfg) {
    orc* s = (orc*)calloc(1, sizeof(orc));
    s->c = *cfg;
    int p = cfg->p;
    s->p = p;
    s->n = p + 1;
    s->nf = p + 2;
    for (int d = 0; d < 3; d++) {
        s->act[d] = cfg->N[d] > 1;
        s->ghost[d] = s->act[d] ? NGH : 0;
        s->fvg[d] = s->act[d] ? NGHFV : 0;
    }
    gauss_legendre(0.0, 1.0, p, s->x_gl, s->w_gl);
    flux_points(s->x_fp, s->x_gl, p);
    solution_points(s->x_sp, p);
    for (int d = 0; d < 3; d++) dim_init(&s->d[d], cfg->N[d], p, cfg->L[d], s->x_fp, s->act[d]);
    gauss_legendre(0.0, 1.0, p + 1, s->xx, s->wx);
    if (cfg->integrator == ORC_RK) {
        s->nader = 1;
        s->rk_a[0] = s->rk_a[1] = s->rk_a[2] = 0;
        s->nstages = cfg->rk_order == 1 ? 1 : cfg->rk_order == 2 ? 2 : 3;
        if (cfg->rk_order == 2) s->rk_a[1] = 0.5;
        if (cfg->rk_order == 3) { s->rk_a[1] = 0.75; s->rk_a[2] = 1.0 / 3.0; }
        s->xt[0] = 0.0;
        s->wt[0] = 1.0;
    } else {
        s->nader = p + 1;
        s->nstages = 1;
        memcpy(s->xt, s->xx, sizeof(s->xx));
        memcpy(s->wt, s->wx, sizeof(s->wx));
    }
    lagrange_matrix(s->sp_to_fp, s->x_sp, s->x_fp, p + 1, p + 2);
    lagrange_prime_matrix(s->dfp_to_sp, s->x_fp, s->x_sp, p + 2, p + 1);
    integral_matrix(s->sp_to_cv, s->x_fp, s->x_sp, p + 1, p + 1);
    inverse(s->sp_to_cv, s->cv_to_sp, p + 1);
    if (cfg->integrator == ORC_ADER) {
        ader_matrix(s->ader, s->xt, s->wt, p + 1);
        inverse(s->ader, s->invader, p + 1);
    }
    dim_t *X = &s->d[0], *Y = &s->d[1], *Z = &s->d[2];
    int Nz = Z->Ntot, Ny = Y->Ntot, Nx = X->Ntot, nz = Z->nsp, ny = Y->nsp, nx = X->nsp;
    s->W_sp = sd_alloc(1, NV, Nz, Ny, Nx, nz, ny, nx);
    s->U_sp = sd_alloc(1, NV, Nz, Ny, Nx, nz, ny, nx);
    s->W_cv = sd_alloc(1, NV, Nz, Ny, Nx, nz, ny, nx);
    s->U_cv = sd_alloc(1, NV, Nz, Ny, Nx, nz, ny, nx);
    s->T_sweep = sd_alloc(1, NV, Nz, Ny, Nx, nz, ny, nx);
    s->U0_sp = sd_alloc(1, NV, Nz, Ny, Nx, nz, ny, nx);
    s->U_ader_sp = sd_alloc(s->nader, NV, Nz, Ny, Nx, nz, ny, nx);
    if (cfg->nu > 0.0)
        for (int d = 0; d < 3; d++) s->dU_sp[d] = sd_alloc(s->nader, NV, Nz, Ny, Nx, nz, ny, nx);
    for (int d = 0; d < 3; d++) {
        int fx = d == 0 && s->act[0], fy = d == 1 && s->act[1], fz = d == 2 && s->act[2];
        int ex = fx ? X->nfp : nx, ey = fy ? Y->nfp : ny, ez = fz ? Z->nfp : nz;
        s->U_ader_fp[d] = sd_alloc(s->nader, NV, Nz, Ny, Nx, ez, ey, ex);
        s->F_ader_fp[d] = sd_alloc(s->nader, NV, Nz, Ny, Nx, ez, ey, ex);
        s->T_fp[d] = sd_alloc(1, NV, Nz, Ny, Nx, ez, ey, ex);
    }
    int Fz = Z->fvn, Fy = Y->fvn, Fx = X->fvn;
    s->U_new = fv_alloc(NV, Fz, Fy, Fx);
    s->W_new = fv_alloc(NV, Fz, Fy, Fx);
    s->U_old = fv_alloc(NV, Fz, Fy, Fx);
    s->W_old = fv_alloc(NV, Fz, Fy, Fx);
    s->troubles = fv_alloc(NT, Fz, Fy, Fx);
    s->theta = fv_alloc(1, Fz, Fy, Fx);
    s->theta_tmp = fv_alloc(1, Fz, Fy, Fx);
    for (int d = 0; d < 3; d++) {
        s->F[d] = fv_alloc(NV, Fz + (d == 2 && s->act[2]), Fy + (d == 1 && s->act[1]), Fx + (d == 0 && s->act[0]));
        s->alpha[d] = fv_alloc(NT, Fz, Fy, Fx);
    }
    initialize(s, &s->W_cv);
    transform_a_to_b(s, &s->W_cv, &s->W_sp, &s->T_sweep, s->cv_to_sp);
    sd_conservatives(&s->W_sp, &s->U_sp, s->c.gamma);
    return s;
}

void orc_destroy(orc* s) {
    if (!s) return;
    sd_t* sds[] = {&s->W_sp, &s->U_sp, &s->W_cv, &s->U_cv, &s->T_sweep, &s->U0_sp, &s->U_ader_sp,
                   &s->U_ader_fp[0], &s->U_ader_fp[1], &s->U_ader_fp[2], &s->F_ader_fp[0], &s->F_ader_fp[1],
                   &s->F_ader_fp[2], &s->T_fp[0], &s->T_fp[1], &s->T_fp[2], &s->dU_sp[0], &s->dU_sp[1],
                   &s->dU_sp[2]};
    for (unsigned q = 0; q < sizeof(sds) / sizeof(sds[0]); q++) free(sds[q]->v);
    fv_t* fvs[] = {&s->U_new, &s->W_new, &s->U_old, &s->W_old, &s->troubles, &s->theta, &s->theta_tmp,
                   &s->F[0], &s->F[1], &s->F[2], &s->alpha[0], &s->alpha[1], &s->alpha[2]};
    for (unsigned q = 0; q < sizeof(fvs) / sizeof(fvs[0]); q++) free(fvs[q]->v);
    for (int d = 0; d < 3; d++) {
        free(s->d[d].sd_faces);
        free(s->d[d].fv_faces);
        free(s->d[d].fv_centers);
    }
    free(s);
}

double orc_compute_dt(orc* s) { return compute_dt(s, &s->W_cv); }

/* src/hydro_ader.hpp:428-444 */
void orc_copy_ader(orc* s) {
    long n = sd_size(&s->U_sp);
    for (int t = 0; t < s->nader; t++) memcpy(s->U_ader_sp.v + t * n, s->U_sp.v, n * sizeof(double));
}
void orc_update_prediction(orc* s, double dt) { update_prediction(s, dt); }
void orc_update_solution(orc* s, double dt) { update_solution(s, dt); }
void orc_primitives_to_cv(orc* s) {
    sd_primitives(&s->U_sp, &s->W_sp, s->c.gamma);
    transform_a_to_b(s, &s->W_sp, &s->W_cv, &s->T_sweep, s->sp_to_cv);
}

void orc_step(orc* s, double dt) {
    if (s->c.integrator == ORC_RK) {
        /* src/hydro_ader.hpp:313-325 */
        memcpy(s->U0_sp.v, s->U_sp.v, sd_size(&s->U_sp) * sizeof(double));
        for (int st = 0; st < s->nstages; st++) {
            orc_copy_ader(s);
            orc_solve_fluxes(s);
            if (s->c.fallback) orc_fv_update(s, dt);
            else update_solution(s, dt);
            if (s->rk_a[st] > 0) combine_solution(&s->U_sp, &s->U0_sp, s->rk_a[st]);
        }
    } else {
        /* src/hydro_ader.hpp:291-305 */
        orc_copy_ader(s);
        for (int a = 0; a < s->nader; a++) {
            orc_solve_fluxes(s);
            if (a < s->nader - 1) update_prediction(s, dt);
        }
        if (s->c.fallback) orc_fv_update(s, dt);
        else update_solution(s, dt);
    }
    orc_primitives_to_cv(s);
}

static int fill_dims_sd(const sd_t* a, int* dims) {
    int v[8] = {a->nt, a->nv, a->Nz, a->Ny, a->Nx, a->nz, a->ny, a->nx};
    for (int q = 0; q < 8; q++) dims[q] = v[q];
    return 1;
}
static int fill_dims_fv(const fv_t* a, int* dims) {
    int v[8] = {a->nv, a->Nz, a->Ny, a->Nx, 1, 1, 1, 1};
    for (int q = 0; q < 8; q++) dims[q] = v[q];
    return 1;
}
static int fill_dims_1(int n0, int n1, int* dims) {
    for (int q = 0; q < 8; q++) dims[q] = 1;
    dims[0] = n0;
    dims[1] = n1;
    return 1;
}

double* orc_array(orc* s, const char* name, int* dims) {
#define SDN(str, arr) if (!strcmp(name, str)) { fill_dims_sd(&(arr), dims); return (arr).v; }
#define FVN(str, arr) if (!strcmp(name, str)) { fill_dims_fv(&(arr), dims); return (arr).v; }
    SDN("U_sp", s->U_sp) SDN("W_sp", s->W_sp) SDN("W_cv", s->W_cv) SDN("U_cv", s->U_cv)
    SDN("U_ader_sp", s->U_ader_sp)
    SDN("U_ader_fp_x", s->U_ader_fp[0]) SDN("U_ader_fp_y", s->U_ader_fp[1]) SDN("U_ader_fp_z", s->U_ader_fp[2])
    SDN("F_ader_fp_x", s->F_ader_fp[0]) SDN("F_ader_fp_y", s->F_ader_fp[1]) SDN("F_ader_fp_z", s->F_ader_fp[2])
    FVN("troubles", s->troubles) FVN("theta", s->theta) FVN("U_new", s->U_new) FVN("U_old", s->U_old)
    FVN("W_new", s->W_new) FVN("W_old", s->W_old) FVN("F_x", s->F[0]) FVN("F_y", s->F[1]) FVN("F_z", s->F[2])
    FVN("alpha_x", s->alpha[0]) FVN("alpha_y", s->alpha[1]) FVN("alpha_z", s->alpha[2])
    if (s->c.nu > 0.0) {
        SDN("dUx_sp", s->dU_sp[0]) SDN("dUy_sp", s->dU_sp[1]) SDN("dUz_sp", s->dU_sp[2])
    }
    int n = s->n, nf = s->nf;
    if (!strcmp(name, "sp_to_fp")) { fill_dims_1(nf, n, dims); return s->sp_to_fp; }
    if (!strcmp(name, "dfp_to_sp")) { fill_dims_1(n, nf, dims); return s->dfp_to_sp; }
    if (!strcmp(name, "sp_to_cv")) { fill_dims_1(n, n, dims); return s->sp_to_cv; }
    if (!strcmp(name, "cv_to_sp")) { fill_dims_1(n, n, dims); return s->cv_to_sp; }
    if (!strcmp(name, "invader")) { fill_dims_1(s->nader, s->nader, dims); return s->invader; }
    if (!strcmp(name, "ader")) { fill_dims_1(s->nader, s->nader, dims); return s->ader; }
    if (!strcmp(name, "x_sp")) { fill_dims_1(n, 1, dims); return s->x_sp; }
    if (!strcmp(name, "x_fp")) { fill_dims_1(nf, 1, dims); return s->x_fp; }
    if (!strcmp(name, "wt")) { fill_dims_1(s->nader, 1, dims); return s->wt; }
    if (!strcmp(name, "xt")) { fill_dims_1(s->nader, 1, dims); return s->xt; }
    if (!strcmp(name, "fv_faces_x")) { fill_dims_1(s->d[0].fvn + 1, 1, dims); return s->d[0].fv_faces; }
    if (!strcmp(name, "fv_faces_y")) { fill_dims_1(s->d[1].fvn + 1, 1, dims); return s->d[1].fv_faces; }
    if (!strcmp(name, "fv_faces_z")) { fill_dims_1(s->d[2].fvn + 1, 1, dims); return s->d[2].fv_faces; }
    if (!strcmp(name, "fv_centers_x")) { fill_dims_1(s->d[0].fvn, 1, dims); return s->d[0].fv_centers; }
    if (!strcmp(name, "fv_centers_y")) { fill_dims_1(s->d[1].fvn, 1, dims); return s->d[1].fv_centers; }
    if (!strcmp(name, "fv_centers_z")) { fill_dims_1(s->d[2].fvn, 1, dims); return s->d[2].fv_centers; }
    return 0;
#undef SDN
#undef FVN
}
