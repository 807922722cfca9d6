// Host-side setup: quadrature, transform matrices, FV sub-grid geometry and
// initial conditions. Compiled with -ffp-contract=off so every expression
// rounds exactly as the reference's CPU build does.
#include "spdk_setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace spdk {

namespace {

constexpr double kPi = 3.141592653589793;  // src/define.hpp:13

// src/polynomials.cpp:3-11
double lagrange(const double* x, double y, int i, int n) {
    double lag = 1.;
    for (int j = 0; j < n; j++)
        if (j != i) lag *= (y - x[j]) / (x[i] - x[j]);
    return lag;
}

// src/polynomials.cpp:21-35
double lagrange_prime(const double* x, double y, int i, int n) {
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

// src/polynomials.cpp:46-79: Newton iteration on P_n from the classic
// cosine guess (the guess uses a 10-digit pi, kept for identical rounding)
void gauss_legendre(double xi, double xf, int n, double* x, double* w) {
    const double eps = 3E-14;
    const int m = (n + 1) / 2;
    const double xm = 0.5 * (xf + xi);
    const double xl = 0.5 * (xf - xi);
    if (n <= 0) {
        x[0] = 0.5;
        w[0] = 1;
        return;
    }
    for (int i = 0; i < m; i++) {
        double z = std::cos(3.141592654 * (i + 0.75) / (n + 0.5));
        double z1 = 0.0, p1 = 0, p2 = 0, p3 = 0, pp = 0;
        while (std::fabs(z - z1) > eps) {
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
}

// src/polynomials.cpp:103-124
void integral_matrix(double* M, const double* x_fp, const double* x_sp, int n_cv, int n_sp) {
    const int p = n_sp - 1;
    double x[kMaxN + 1], w[kMaxN + 1];
    gauss_legendre(0.0, 1.0, p, x, w);
    for (int k = 0; k < n_cv; k++) {
        if (p > 0) gauss_legendre(x_fp[k], x_fp[k + 1], p, x, w);
        for (int j = 0; j < n_sp; j++) {
            double integral;
            if (p > 0) {
                integral = 0.0;
                for (int i = 0; i < p; i++) integral += lagrange(x_sp, x[i], j, p + 1) * w[i];
            } else {
                integral = 1.0;
            }
            M[k * n_sp + j] = integral / (x_fp[k + 1] - x_fp[k]);
        }
    }
}

// src/polynomials.cpp:126-198: LU without pivoting, column by column
void inverse(const double* A, double* C, int n) {
    double B[kMaxN * kMaxN], Lm[kMaxN * kMaxN], U[kMaxN * kMaxN], b[kMaxN], d[kMaxN], x[kMaxN];
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
            const double coeff = B[k + i * n] / B[k + k * n];
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

uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

// Seeded noise of the project's Kelvin-Helmholtz problem: uniform in
// [-1,1), a pure function of the point coordinates' bit patterns so every
// implementation that evaluates the same quadrature points agrees.
double coord_noise(uint64_t seed, double x, double y, double z) {
    uint64_t bx, by, bz;
    std::memcpy(&bx, &x, 8);
    std::memcpy(&by, &y, 8);
    std::memcpy(&bz, &z, 8);
    const uint64_t h = splitmix64(seed ^ splitmix64(bx ^ splitmix64(by ^ splitmix64(bz))));
    return (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// Point value of the primitive variable `var` (0 rho, 1..3 velocity,
// 4 pressure) of the configured problem. Reference problems follow
// src/initial_conditions.cpp:9-177 and src/user_ic.hpp:40-51.
double ic_point(const spdk_hydro_config& c, int var, double x, double y, double z, bool ay, bool az) {
    const double gm = c.gamma;
    switch (c.problem) {
    case SPDK_IC_SINE_WAVE:
        if (var == 0) return c.d0 + c.amp * (std::sin(2 * kPi * (x + y)));
        if (var == 1) return c.v1;
        if (var == 2) return c.v2;
        if (var == 3) return c.v3;
        if (var == 4) return c.p0;
        return 0;
    case SPDK_IC_SEDOV: {
        const double r = std::sqrt(std::pow(x - 0.5, 2.0) + std::pow(y - 0.5, 2.0) +
                                   (az ? std::pow(z - 0.5, 2.0) : 0.0));
        if (var == 0) return c.d0;
        if (var == 4) return r < c.radius ? 1E-6 + (gm - 1) : 1E-6;
        return 0;
    }
    case SPDK_IC_SPHERICAL_BLAST: {
        const double r = std::sqrt(std::pow(x - c.cx, 2.0) + std::pow(y - c.cy, 2.0) +
                                   (az ? std::pow(z - c.cz, 2.0) : 0.0));
        if (var == 0) return c.d0;
        if (var == 4) return r < c.radius ? c.p0 : c.p1;
        return 0;
    }
    case SPDK_IC_SQUARE: {
        if (var == 0) {
            bool in = std::fabs(x - 0.5) < c.radius;
            if (ay) in = in && std::fabs(y - 0.5) < c.radius;
            if (az) in = in && std::fabs(z - 0.5) < c.radius;
            return in ? c.d1 : c.d0;
        }
        if (var == 1) return c.v1;
        if (var == 2) return c.v2;
        if (var == 3) return c.v3;
        if (var == 4) return c.p0;
        return 0;
    }
    case SPDK_IC_SOD: {
        const double s = (c.dir == 0 ? x : (c.dir == 1 ? y : z));
        const bool left = s < c.radius;
        if (var == 0) return left ? c.d0 : c.d1;
        if (var == 4) return left ? c.p0 : c.p1;
        return 0;
    }
    case SPDK_IC_SHU_OSHER: {
        const double xs = x - 1.0;
        const bool left = xs < -0.8;
        if (var == 0) return left ? 3.857143 : 1.0 + c.amp * std::sin(5 * kPi * xs);
        if (var == 1) return left ? 2.629369 : 0.0;
        if (var == 4) return left ? 10.33333 : 1.0;
        return 0;
    }
    case SPDK_IC_KELVIN_HELMHOLTZ: {
        const bool inner = (y > 0.25 && y < 0.75);
        if (var == 0) return inner ? c.d1 : c.d0;
        if (var == 1) return inner ? c.v1 : -c.v1;
        if (var == 2)
            return c.amp * std::sin(4 * kPi * x) *
                   (std::exp(-std::pow(y - 0.25, 2.0) / (2 * c.sigma * c.sigma)) +
                    std::exp(-std::pow(y - 0.75, 2.0) / (2 * c.sigma * c.sigma)));
        if (var == 4) return c.p0;
        return 0;
    }
    case SPDK_IC_IMPLOSION: {
        const bool inside = (x + y) < c.radius;
        if (var == 0) return inside ? c.d1 : c.d0;
        if (var == 4) return inside ? c.p1 : c.p0;
        return 0;
    }
    case SPDK_IC_RTI: {
        const double gy = c.g[1], yc = c.radius, rho_hi = c.d0, rho_lo = c.d1, P0 = c.p0;
        const bool top = y > yc;
        if (var == 0) return top ? rho_lo : rho_hi;
        if (var == 2) {
            const double dv = std::sqrt(gm * (rho_hi * yc + 1.0) / rho_hi);
            return -c.amp * dv * std::cos(8.0 * kPi * x);
        }
        if (var == 4) return top ? (P0 + rho_lo * gy * y + (rho_hi - rho_lo) * gy * yc) : (P0 + rho_hi * gy * y);
        return 0;
    }
    case SPDK_IC_USER: {
        const double dx = x - c.radius;
        const double pulse = c.amp * std::exp(-dx * dx / (2 * c.sigma * c.sigma));
        if (var == 0) return c.d0;
        if (var == 1) return c.v1;
        if (var == 2) return pulse;
        if (var == 3) return 0.0;
        if (var == 4) return c.p0;
        return 0;
    }
    case SPDK_IC_KH_NOISE: {
        // shear layer rho=d1, vx=+v1 for |y-0.5|<0.25, else rho=d0, vx=-v1;
        // P=p0; vy = amp sin(4 pi x) + q[0] U(-1,1)
        const bool inner = std::fabs(y - 0.5) < 0.25;
        if (var == 0) return inner ? c.d1 : c.d0;
        if (var == 1) return inner ? c.v1 : -c.v1;
        if (var == 2) return c.amp * std::sin(4 * kPi * x) + c.q[0] * coord_noise(c.seed, x, y, z);
        if (var == 4) return c.p0;
        return 0;
    }
    case SPDK_IC_QUADRANT: {
        // four-quadrant Riemann problem about (cx, cy); quadrant
        // qd = (x>cx) + 2 (y>cy) holds rho=q[4qd], P=q[4qd+1], vx=q[4qd+2], vy=q[4qd+3]
        const int qd = (x > c.cx) + 2 * (y > c.cy);
        if (var == 0) return c.q[4 * qd];
        if (var == 4) return c.q[4 * qd + 1];
        if (var == 1) return c.q[4 * qd + 2];
        if (var == 2) return c.q[4 * qd + 3];
        return 0;
    }
    case SPDK_IC_RTI_TOP: {
        // heavy d0 above y = radius, light d1 below, hydrostatic with
        // P = p0 at the interface; vy = amp (1+cos 4 pi x)(1+cos 3 pi (y-yc))/4
        const double gy = c.g[1], yc = c.radius;
        const bool top = y > yc;
        const double rho = top ? c.d0 : c.d1;
        if (var == 0) return rho;
        if (var == 2) return c.amp * (1 + std::cos(4 * kPi * x)) * (1 + std::cos(3 * kPi * (y - yc))) / 4;
        if (var == 4) return c.p0 + rho * gy * (y - yc);
        return 0;
    }
    default:
        return 0;
    }
}

}  // namespace

void build_matrices(int p, bool ader, Matrices* m) {
    *m = Matrices{};
    m->p = p;
    m->n = p + 1;
    m->nf = p + 2;
    gauss_legendre(0.0, 1.0, p, m->x_gl, m->w_gl);
    // src/polynomials.cpp:81-93
    m->x_fp[0] = 0.0;
    for (int i = 1; i < p + 1; i++) m->x_fp[i] = m->x_gl[i - 1];
    m->x_fp[p + 1] = 1.0;
    for (int i = 0; i <= p; i++) m->x_sp[i] = 0.5 * (1.0 - std::cos((2 * i + 1) / (2.0 * (p + 1)) * kPi));
    gauss_legendre(0.0, 1.0, p + 1, m->xx, m->wx);
    const int n = p + 1, nf = p + 2;
    // src/hydro_ader.hpp:129-141
    for (int j = 0; j < nf; j++)
        for (int i = 0; i < n; i++) m->sp_to_fp[j * n + i] = lagrange(m->x_sp, m->x_fp[j], i, n);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < nf; i++) m->dfp_to_sp[j * nf + i] = lagrange_prime(m->x_fp, m->x_sp[j], i, nf);
    integral_matrix(m->sp_to_cv, m->x_fp, m->x_sp, n, n);
    inverse(m->sp_to_cv, m->cv_to_sp, n);
    integral_matrix(m->fp_to_cv, m->x_fp, m->x_fp, n, nf);
    if (ader) {
        m->nt = n;
        for (int i = 0; i < n; i++) {
            m->xt[i] = m->xx[i];
            m->wt[i] = m->wx[i];
        }
        // src/polynomials.cpp:95-101
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++)
                m->ader[j * n + i] = lagrange(m->xt, 1, i, n) * lagrange(m->xt, 1, j, n) -
                                     lagrange_prime(m->xt, m->xt[i], j, n) * m->wt[i];
        inverse(m->ader, m->invader, n);
    } else {
        m->nt = 1;
        m->xt[0] = 0.0;
        m->wt[0] = 1.0;
    }
}

void build_axis(int N, int p, double L, const double* x_fp, bool active, Axis* a, int lo, int N_all) {
    *a = Axis{};
    a->N = N;
    a->active = active;
    a->h = L / (N_all > 0 ? N_all : N);
    if (!active) return;
    const int nsp = p + 1, nfp = p + 2, Ntot = N + 2;
    a->n = nsp;
    a->nf = nfp;
    a->fvn = N * nsp + 4;
    const int idL = nsp - 2, idR = a->fvn + idL;
    a->sd_faces.assign((size_t)Ntot * nfp, 0.0);
    a->sd_centers.assign((size_t)Ntot * nsp, 0.0);
    a->fv_faces.assign(a->fvn + 1, 0.0);
    a->fv_centers.assign(a->fvn, 0.0);
    for (int j = 0; j < Ntot; j++) {
        for (int i = 0; i < nfp; i++) {
            const double f = (lo + j - 1 + x_fp[i]) * a->h;
            a->sd_faces[j * nfp + i] = f;
            const int g = i + j * nsp;
            if (g >= idL && g < idR) a->fv_faces[i - idL + j * nsp] = f;
        }
        for (int i = 0; i < nsp; i++) {
            const double c = 0.5 * (a->sd_faces[j * nfp + i + 1] + a->sd_faces[j * nfp + i]);
            a->sd_centers[j * nsp + i] = c;
            const int g = i + j * nsp;
            if (g >= idL && g < idR) a->fv_centers[i - idL + j * nsp] = c;
        }
    }
}

void initial_wcv(const spdk_hydro_config& c, const Matrices& m, const Axis ax[3], int D,
                 std::vector<double>* wcv) {
    const int n = m.n, nf = m.nf;
    const int V = D + 2;
    const int npt = D == 2 ? n * n : n * n * n;
    const int Nx = ax[0].N, Ny = ax[1].N, Nz = D == 3 ? ax[2].N : 1;
    const bool ay = true, az = D == 3;
    wcv->assign((size_t)Nx * Ny * Nz * V * npt, 0.0);
    // every element is independent (a pure function of its positions), so
    // the elements are split across host threads; the values do not depend
    // on the split
    const long long E = (long long)Nx * Ny * Nz;
    const long long work = E * npt * (long long)npt;  // point evaluations per variable
    unsigned nth = std::max(1u, std::thread::hardware_concurrency());
    if (work < (1LL << 22)) nth = 1;
    nth = (unsigned)std::min<long long>(nth, std::max<long long>(1, E));
    // slot of primitive var in the solver layout (rho, v_1..v_D, p)
    auto body = [&](long long e_begin, long long e_end) {
        for (long long e_it = e_begin; e_it < e_end; e_it++) {
            const int i = (int)(e_it % Nx), j = (int)((e_it / Nx) % Ny), k = (int)(e_it / ((long long)Nx * Ny));
            const size_t e = (size_t)e_it;
            // ghost-inclusive element indices of the reference geometry
            const int gi = i + 1, gj = j + 1, gk = az ? k + 1 : 0;
            const double* fx = &ax[0].sd_faces[(size_t)gi * nf];
            const double* fy = &ax[1].sd_faces[(size_t)gj * nf];
            const double* fz = az ? &ax[2].sd_faces[(size_t)gk * nf] : nullptr;
            const int pz = az ? n : 1;
            for (int kk = 0; kk < pz; kk++)
                for (int jj = 0; jj < n; jj++)
                    for (int ii = 0; ii < n; ii++) {
                        const int pt = (kk * n + jj) * n + ii;
                        for (int var = 0; var < 5; var++) {
                            int slot;
                            if (var == 0) slot = 0;
                            else if (var == 4) slot = D + 1;
                            else if (var <= D) slot = var;
                            else continue;  // z velocity of a 2D run: identically zero
                            double value = 0, x, y = 0, z = 0;
                            for (int nn = 0; nn < pz; nn++) {
                                if (az) z = fz[kk] + m.xx[nn] * (fz[kk + 1] - fz[kk]);
                                for (int mm = 0; mm < n; mm++) {
                                    if (ay) y = fy[jj] + m.xx[mm] * (fy[jj + 1] - fy[jj]);
                                    for (int ll = 0; ll < n; ll++) {
                                        x = fx[ii] + m.xx[ll] * (fx[ii + 1] - fx[ii]);
                                        double s = ic_point(c, var, x, y, z, ay, az);
                                        s *= m.wx[ll];
                                        if (ay) s *= m.wx[mm];
                                        if (az) s *= m.wx[nn];
                                        value += s;
                                    }
                                }
                            }
                            (*wcv)[(e * V + slot) * npt + pt] = value;
                        }
                    }
        }
    };
    if (nth == 1) {
        body(0, E);
        return;
    }
    std::vector<std::thread> pool;
    const long long chunk = (E + nth - 1) / nth;
    for (unsigned t = 0; t < nth; t++) {
        const long long b = (long long)t * chunk, en = std::min(E, b + chunk);
        if (b < en) pool.emplace_back(body, b, en);
    }
    for (std::thread& th : pool) th.join();
}

}  // namespace spdk
