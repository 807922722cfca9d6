// A-posteriori fallback of the spd_K B200 hydro step: NAD/SED/PAD trouble
// detection, theta blending and the MUSCL-Hancock/HLLC fallback flux on the
// FV sub-grid (the p+1 Gauss-point cells of every element), one time slice
// at a time (src/hydro_ader.hpp:500-575).
//
// The reference keeps the sub-grid in separate ghost-framed arrays; here the
// sub-cells stay inside their elements ([element][point] order) and the two
// ghost layers are evaluated through spdk::fv_image, which reproduces the
// reference's x-then-y-then-z ghost fill (corner ghosts included).
#pragma once
#include <cuda_runtime.h>

#include "spdk_kernels.cuh"

namespace spdk {

template <typename R>
struct FallbackArgsT {
    const R* ucv_in;        // U_cv at the start of slice t [E][V][NPT]
    R* ucv_out;             // U_cv after slice t
    R* ff0;                 // FV face fluxes of each direction, all slices
    R* ff1;
    R* ff2;
    const double2* rp_old;  // (rho, p) of U_old / U_new candidates of slice t
    const double2* rp_new;
    double2* rp_old_next;   // candidates of slice t+1
    double2* rp_new_next;
    uint8_t* trouble;       // [E][NPT]
    uint8_t* theta;         // [E][NPT], theta * 8
    int t;                  // slice
    int last;               // last slice of the stage: U_sp = cv_to_sp(U_cv)
    R* u;                   // U_sp (written on the last slice)
    const R* u0;            // RK step-start state
    double rk_a;
    int final_stage;        // compute W_cv and the next dt
    R* wcv;
    unsigned long long* dtmin;
    const double* dt;
    int* any_trouble;       // diagnostic counter of troubled sub-cells (nullable)
};
using FallbackArgs = FallbackArgsT<double>;

// active FV cell -> (element, point) index of a [E][NPT] array
template <int D, int P>
__device__ __forceinline__ long long cell_id(const DevGrid& G, const int a[3]) {
    constexpr int n = P + 1;
    int e[3] = {0, 0, 0}, c[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < D; d++) {
        e[d] = a[d] / n;
        c[d] = a[d] - e[d] * n;
    }
    const long long ge = ((long long)e[2] * G.N[1] + e[1]) * G.N[0] + e[0];
    return ge * Shape<D, P>::NPT + pt_index<n>(c);
}

// image of a possibly-ghost FV coordinate; flips[d] set for reflective images
template <int D, int P>
__device__ __forceinline__ long long cell_image(const DevGrid& G, const int a[3], bool flips[3]) {
    constexpr int n = P + 1;
    int m[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < D; d++) {
        flips[d] = false;
        m[d] = fv_image(a[d], G.N[d] * n, G.bc[d], &flips[d]);
    }
    return cell_id<D, P>(G, m);
}

__device__ __forceinline__ double rp_var(const double2 v, int k) { return k == 0 ? v.x : v.y; }

// ---------------------------------------------------------------------------
// Trouble detection of every active sub-cell (src/trouble_detection.cpp:35-290
// with limit mask rho|p, src/hydro_ader.hpp:522-524).
//
// The SED relaxation can only clear a flag NAD raised (relax_NAD keeps a
// flag iff alpha < 1), so the division-heavy smooth-extrema indicator is
// evaluated only at cells NAD flagged; the result is identical to computing
// it everywhere. W_old (rho, p) of the tile + 1 halo is staged in shared
// memory for the NAD box.
// ---------------------------------------------------------------------------
template <int D, int P>
__device__ __forceinline__ double sed_component(const DevGrid& G, const double2* __restrict__ rpn, const int a[3],
                                                int d, int k) {
    constexpr int n = P + 1;
    const int nd = G.N[d] * n;
    const double* C = G.fvc[d];
    const double* Fc = G.fvf[d];
    double al[3];
    bool fl[3];
#pragma unroll
    for (int s = -1; s <= 1; s++) {
        const int ad = a[d] + s;
        if (ad < 0 || ad >= nd) { al[s + 1] = 0.0; continue; }  // never computed outside the active cells
        int b[3] = {a[0], a[1], a[2]};
        double Wv[5];
#pragma unroll
        for (int off = -2; off <= 2; off++) {
            b[d] = ad + off;
            Wv[off + 2] = rp_var(rpn[cell_image<D, P>(G, b, fl)], k);
        }
        const int l = ad + 2;
        const double h = (C[l + 1] - C[l - 1]);
        const double hp = (C[l + 2] - C[l]);
        const double hm = (C[l] - C[l - 2]);
        const double u = Wv[2];
        const double du = (Wv[3] - Wv[1]) / h;
        const double dup = (Wv[4] - u) / hp;
        const double dum = (u - Wv[0]) / hm;
        const double d2u = (dup - dum) / (C[l + 1] - C[l - 1]);
        const double dv = 0.5 * d2u * (Fc[l + 1] - Fc[l]);
        al[s + 1] = sed_alpha(dv, dum, du, dup);
    }
    return smin(smin(al[0], al[1]), al[2]);
}

// R names the form (double: plain, float: precision) that launches the
// kernel; the detector computes in FP64 in both, and a separate
// instantiation per form keeps each form's compile flags on its own copy.
template <typename R, int D, int P, int TX, int TY, int TZ>
__device__ __forceinline__ void fv_detect_kernel_body(const DevGrid& G, const double2* __restrict__ rpo,
                                                            const double2* __restrict__ rpn,
                                                            uint8_t* __restrict__ T, int* any_trouble, long long bidx) {
    constexpr int n = P + 1;
    constexpr int NPT = Shape<D, P>::NPT;
    constexpr int Bx = TX * n, By = TY * n, Bz = D == 3 ? TZ * n : 1;
    constexpr int E1x = Bx + 2, E1y = By + 2, E1z = D == 3 ? Bz + 2 : 1;
    __shared__ double2 Ro[E1x * E1y * E1z];
    const int dz = D == 3 ? 1 : 0;
    int o[3];
    {
        int b = bidx;
        const int tx = G.N[0] / TX, ty = G.N[1] / TY;
        o[0] = (b % tx) * Bx;
        b /= tx;
        o[1] = (b % ty) * By;
        b /= ty;
        o[2] = D == 3 ? b * Bz : 0;
    }
    for (int q = threadIdx.x; q < E1x * E1y * E1z; q += blockDim.x) {
        int a[3] = {o[0] - 1 + q % E1x, o[1] - 1 + (q / E1x) % E1y, o[2] - dz + q / (E1x * E1y)};
        bool fl[3];
        Ro[q] = rpo[cell_image<D, P>(G, a, fl)];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < Bx * By * Bz; q += blockDim.x) {
        const int x = q % Bx, y = (q / Bx) % By, z = q / (Bx * By);
        int a[3] = {o[0] + x, o[1] + y, o[2] + z};
        const long long cid = cell_id<D, P>(G, a);
        const double2 here_new = rpn[cid];
        const int sc = (x + 1) + E1x * ((y + 1) + E1y * (z + dz));
        double flag[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const double un = rp_var(here_new, k);
            double mx = rp_var(Ro[sc], k), mn = mx;
            if (G.nad_moore) {
                for (int ok = -dz; ok <= dz; ok++)
#pragma unroll
                    for (int oj = -1; oj <= 1; oj++)
#pragma unroll
                        for (int oi = -1; oi <= 1; oi++) {
                            const double u = rp_var(Ro[sc + oi + E1x * (oj + E1y * ok)], k);
                            mx = smax(mx, u);
                            mn = smin(mn, u);
                        }
            } else {
#pragma unroll
                for (int d = 0; d < D; d++) {
                    const int st = d == 0 ? 1 : (d == 1 ? E1x : E1x * E1y);
                    const double uL = rp_var(Ro[sc - st], k);
                    const double uR = rp_var(Ro[sc + st], k);
                    mx = smax(smax(uL, mx), uR);
                    mn = smin(smin(uL, mn), uR);
                }
            }
            if (G.nad_delta) {
                const double eps = G.nad_tol * (mx - mn);
                mn -= eps;
                mx += eps;
            } else {
                mn -= fabs(mn) * G.nad_tol;
                mx += fabs(mx) * G.nad_tol;
            }
            flag[k] = (un > mx || un < mn) ? 1.0 : 0.0;
        }
        if (G.use_sed) {
#pragma unroll
            for (int k = 0; k < 2; k++) {
                if (flag[k] == 0.0) continue;  // relaxation cannot raise a flag
                double alpha = 1;
#pragma unroll
                for (int d = 0; d < D; d++) {
                    const double m3 = sed_component<D, P>(G, rpn, a, d, k);
                    alpha = d == 0 ? m3 : smin(alpha, m3);
                }
                flag[k] = alpha < 1 ? flag[k] : 0;
            }
        }
        double tr = 0;
        tr = smax(tr, flag[0]);
        tr = smax(tr, flag[1]);
        const double rho = here_new.x, p = here_new.y;
        if (rho < kRhoMin || rho > kRhoMax) tr = 1;
        if (p < kPMin || p > kPMax) tr = 1;
        const long long el = cid / NPT;
        if (G.elem_trouble && tr > 0) G.elem_trouble[el] = 1;  // a-posteriori label
        if (G.elem_pred && G.elem_pred[el]) tr = 1;            // a-priori prediction
        T[cid] = tr > 0 ? 1 : 0;
        if (any_trouble && tr > 0) atomicAdd(any_trouble, 1);
    }
}

template <typename R, int D, int P, int TX, int TY, int TZ>
__global__ void __launch_bounds__(kThreads) fv_detect_kernel(DevGrid G, const double2* __restrict__ rpo,
                                                            const double2* __restrict__ rpn,
                                                            uint8_t* __restrict__ T, int* any_trouble) {
    fv_detect_kernel_body<R, D, P, TX, TY, TZ>(G, rpo, rpn, T, any_trouble, blockIdx.x);
}

// cell box of an element tile with a halo of g cells per active side
template <int D, int P, int TX, int TY, int TZ>
struct CellBox {
    static constexpr int n = P + 1;
    __device__ static int ext(int d, int g) {
        return d >= D ? 1 : (d == 0 ? TX : (d == 1 ? TY : TZ)) * n + 2 * g;
    }
};

// ---------------------------------------------------------------------------
// theta = max over the Moore box of w(#offsets) * trouble, plus the 0.25 ring
// (src/trouble_detection.cpp:191-242); theta_from_troubles without blending
// ---------------------------------------------------------------------------
template <typename R, int D, int P, int TX, int TY, int TZ>
__device__ __forceinline__ void fv_theta_kernel_body(const DevGrid& G, const uint8_t* __restrict__ T,
                                                           uint8_t* __restrict__ theta, long long bidx) {
    constexpr int n = P + 1;
    using CB = CellBox<D, P, TX, TY, TZ>;
    constexpr int E2x = TX * n + 4, E2y = TY * n + 4, E2z = D == 3 ? TZ * n + 4 : 1;
    constexpr int E1x = TX * n + 2, E1y = TY * n + 2, E1z = D == 3 ? TZ * n + 2 : 1;
    __shared__ uint8_t Ts[E2x * E2y * E2z];
    __shared__ float Th[E1x * E1y * E1z];
    int o[3];
    {
        int b = bidx;
        const int tx = G.N[0] / TX, ty = G.N[1] / TY;
        o[0] = (b % tx) * TX * n;
        b /= tx;
        o[1] = (b % ty) * TY * n;
        b /= ty;
        o[2] = D == 3 ? b * TZ * n : 0;
    }
    (void)CB::ext;
    const int g2 = 2, gz2 = D == 3 ? 2 : 0;
    for (int q = threadIdx.x; q < E2x * E2y * E2z; q += blockDim.x) {
        int a[3] = {o[0] - g2 + q % E2x, o[1] - g2 + (q / E2x) % E2y, o[2] - gz2 + q / (E2x * E2y)};
        bool fl[3];
        Ts[q] = T[cell_image<D, P>(G, a, fl)];
    }
    __syncthreads();
    if (!G.blending) {
        for (int q = threadIdx.x; q < TX * n * TY * n * (D == 3 ? TZ * n : 1); q += blockDim.x) {
            const int bx = TX * n, by = TY * n;
            int a[3] = {q % bx, (q / bx) % by, q / (bx * by)};
            const int s = (a[0] + 2) + E2x * ((a[1] + 2) + E2y * (a[2] + gz2));
            int ga[3] = {o[0] + a[0], o[1] + a[1], o[2] + a[2]};
            theta[cell_id<D, P>(G, ga)] = Ts[s] ? 8 : 0;
        }
        return;
    }
    const float w4[4] = {1.0f, 0.75f, 0.5f, 0.375f};
    const int dz = D == 3 ? 1 : 0;
    for (int q = threadIdx.x; q < E1x * E1y * E1z; q += blockDim.x) {
        const int x = q % E1x + 1, y = (q / E1x) % E1y + 1, z = q / (E1x * E1y) + dz;
        float th = 0;
        for (int ok = -dz; ok <= dz; ok++)
            for (int oj = -1; oj <= 1; oj++)
                for (int oi = -1; oi <= 1; oi++) {
                    const int n0 = (oi != 0) + (oj != 0) + (ok != 0);
                    const float v = w4[n0] * (float)Ts[(x + oi) + E2x * ((y + oj) + E2y * (z + ok))];
                    th = th < v ? v : th;
                }
        Th[q] = th;
    }
    __syncthreads();
    const int bx = TX * n, by = TY * n, bz = D == 3 ? TZ * n : 1;
    for (int q = threadIdx.x; q < bx * by * bz; q += blockDim.x) {
        const int x = q % bx + 1, y = (q / bx) % by + 1, z = q / (bx * by) + dz;
        const float th = Th[x + E1x * (y + E1y * z)];
        float ring = 0;
        for (int ok = -dz; ok <= dz; ok++)
            for (int oj = -1; oj <= 1; oj++)
                for (int oi = -1; oi <= 1; oi++)
                    if (Th[(x + oi) + E1x * ((y + oj) + E1y * (z + ok))] > 0) ring = 0.25f;
        const float t = th < ring ? ring : th;
        int ga[3] = {o[0] + x - 1, o[1] + y - 1, o[2] + z - dz};
        theta[cell_id<D, P>(G, ga)] = (uint8_t)(t * 8.0f);
    }
}

template <typename R, int D, int P, int TX, int TY, int TZ>
__global__ void __launch_bounds__(kThreads) fv_theta_kernel(DevGrid G, const uint8_t* __restrict__ T,
                                                           uint8_t* __restrict__ theta) {
    fv_theta_kernel_body<R, D, P, TX, TY, TZ>(G, T, theta, blockIdx.x);
}

// MUSCL-Hancock face states of cell X for a face of direction Dn
// (src/hydro.cpp:622-681); returns the state on the cell's low face (wlo)
// and high face (whi). Wc(offset) gives W_old of neighbouring cells.
template <int D, typename R, typename WF>
__device__ __forceinline__ void muscl_cell(const DevGrid& G, const int fa[3], int Dn, R dtw, WF Wc,
                                           R* wlo, R* whi) {
    constexpr int V = D + 2;
    R w[V], dW[D][V], dwt[V];
    const R* wc = Wc(0, 0, 0);
#pragma unroll
    for (int v = 0; v < V; v++) w[v] = wc[v];
#pragma unroll
    for (int d = 0; d < D; d++) {
        const R* wm = Wc(d == 0 ? -1 : 0, d == 1 ? -1 : 0, d == 2 ? -1 : 0);
        const R* wp = Wc(d == 0 ? 1 : 0, d == 1 ? 1 : 0, d == 2 ? 1 : 0);
        const double* xc = G.fvc[d];
        const double* xf = G.fvf[d];
        const int i = fa[d];
#pragma unroll
        for (int v = 0; v < V; v++)
            dW[d][v] = minmod((wp[v] - w[v]) / (R)(xc[i + 1] - xc[i]), (w[v] - wm[v]) / (R)(xc[i] - xc[i - 1]),
                              (R)xf[i], (R)xf[i + 1]);
    }
    hancock<D>(w, dwt, dW, (R)G.gm);
    const double* xf = G.fvf[Dn];
    const int i = fa[Dn];
    const R h = (R)(xf[i + 1] - xf[i]);
#pragma unroll
    for (int v = 0; v < V; v++) {
        const R dw = dW[Dn][v];
        whi[v] = w[v] + dw + dwt[v] * dtw / h;  // reference "WL": left state of the high face
        wlo[v] = w[v] - dw + dwt[v] * dtw / h;  // reference "WR": right state of the low face
    }
}

template <typename R, int D, int P, int TX, int TY, int TZ>
struct UpdateSmem {
    static constexpr int n = P + 1, V = D + 2;
    static constexpr int NPT = Shape<D, P>::NPT;
    static constexpr int NE = TX * TY * TZ;
    static constexpr int Bx = TX * n, By = TY * n, Bz = D == 3 ? TZ * n : 1;
    static constexpr int NC = Bx * By * Bz;
    static constexpr int E1x = Bx + 2, E1y = By + 2, E1z = D == 3 ? Bz + 2 : 1;
    static constexpr int E2x = Bx + 4, E2y = By + 4, E2z = D == 3 ? Bz + 4 : 1;
    static constexpr int NF0 = (Bx + 1) * By * Bz;
    static constexpr int NF1 = Bx * (By + 1) * Bz;
    static constexpr int NF2 = D == 3 ? Bx * By * (Bz + 1) : 0;
    static constexpr size_t faces = (size_t)(NF0 + NF1 + NF2) * V;
    static constexpr size_t wold = (size_t)E2x * E2y * E2z * V;
    static constexpr size_t epi = 2 * (size_t)NE * V * NPT;
    static constexpr size_t reals = faces + (wold > epi ? wold : epi);
    static constexpr size_t bytes = reals * sizeof(R) + ((size_t)E1x * E1y * E1z + 15) / 16 * 16;
};

// ---------------------------------------------------------------------------
// Blended fluxes and the corrected sub-cell update of slice t
// (src/hydro.cpp:683-788, src/transforms.cpp:483-543 with update=1), then
// either the next slice's candidate or, after the last slice,
// U_sp = cv_to_sp(U_cv), the RK combination, W_cv and the next dt.
// ---------------------------------------------------------------------------
template <typename R, int D, int P, int TX, int TY, int TZ>
__device__ __forceinline__ void fv_update_kernel_body(const DevGrid& G, const DevMatsT<R>& M, const FallbackArgsT<R>& A, long long bidx) {
    using SM = UpdateSmem<R, D, P, TX, TY, TZ>;
    constexpr int n = P + 1, nf = P + 2, V = D + 2, NPT = SM::NPT, NFP = Shape<D, P>::NFP;
    constexpr int Bx = SM::Bx, By = SM::By, Bz = SM::Bz, NC = SM::NC;
    constexpr int E1x = SM::E1x, E1y = SM::E1y, E2x = SM::E2x, E2y = SM::E2y;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    R* smem = reinterpret_cast<R*>(smem_raw);
    R* Fs = smem;                                   // faces of the tile, [face][V]
    R* Wo = Fs + SM::faces;                         // W_old on the tile + 2 halo
    uint8_t* th = (uint8_t*)(Wo + (SM::wold > SM::epi ? SM::wold : SM::epi));
    __shared__ long long el_ge[SM::NE];
    const int dz = D == 3 ? 1 : 0;
    R* const ffd[3] = {A.ff0, A.ff1, A.ff2};

    int o[3], oe[3];
    {
        int b = bidx;
        const int tx = G.N[0] / TX, ty = G.N[1] / TY;
        oe[0] = (b % tx) * TX;
        b /= tx;
        oe[1] = (b % ty) * TY;
        b /= ty;
        oe[2] = D == 3 ? b * TZ : 0;
        o[0] = oe[0] * n;
        o[1] = oe[1] * n;
        o[2] = oe[2] * n;
    }
    for (int s = threadIdx.x; s < SM::NE; s += blockDim.x) {
        const int lx = s % TX, ly = (s / TX) % TY, lz = s / (TX * TY);
        el_ge[s] = ((long long)(oe[2] + lz) * G.N[1] + (oe[1] + ly)) * G.N[0] + (oe[0] + lx);
    }
    __syncthreads();  // el_ge is read by every thread below
    const R dt = (R)(*A.dt);
    const R wdt = M.wt[A.t] * dt;
    const long long E = G.E;
    // theta on the tile + 1 halo (ghost values are images)
    for (int q = threadIdx.x; q < E1x * E1y * SM::E1z; q += blockDim.x) {
        int a[3] = {o[0] - 1 + q % E1x, o[1] - 1 + (q / E1x) % E1y, o[2] - dz + q / (E1x * E1y)};
        bool fl[3];
        th[q] = A.theta[cell_image<D, P>(G, a, fl)];
    }
    // SD face fluxes of the tile
    const int nfaces[3] = {SM::NF0, SM::NF1, SM::NF2};
    int fbase[3] = {0, SM::NF0, SM::NF0 + SM::NF1};
    for (int d = 0; d < D; d++) {
        const int ex = Bx + (d == 0), ey = By + (d == 1);
        for (int q = threadIdx.x; q < nfaces[d]; q += blockDim.x) {
            int a[3] = {q % ex, (q / ex) % ey, q / (ex * ey)};  // tile-local: face a[d] is the low face of cell a
            int cl[3] = {a[0], a[1], a[2]};
            int llv;
            if (a[d] == (d == 0 ? Bx : (d == 1 ? By : Bz))) { cl[d] = a[d] - 1; llv = n; }
            else llv = -1;
            const int el = (cl[0] / n) + TX * ((cl[1] / n) + TY * (cl[2] / n));
            int c[3] = {cl[0] % n, cl[1] % n, cl[2] % n};
            if (llv < 0) llv = c[d];
            c[d] = llv;
            const int fi = fp_index<n, nf>(d, c);
            const R* src = ffd[d] + ((long long)A.t * E + el_ge[el]) * V * NFP;
            R* dst = Fs + (size_t)(fbase[d] + q) * V;
#pragma unroll
            for (int v = 0; v < V; v++) dst[v] = src[v * NFP + fi];
        }
    }
    __syncthreads();
    // faces that blend in the fallback flux
    int need = 0;
    for (int d = 0; d < D && !need; d++) {
        const int ex = Bx + (d == 0), ey = By + (d == 1);
        for (int q = threadIdx.x; q < nfaces[d]; q += blockDim.x) {
            int a[3] = {q % ex, (q / ex) % ey, q / (ex * ey)};
            const int sR = (a[0] + 1) + E1x * ((a[1] + 1) + E1y * (a[2] + dz));
            const int sL = sR - (d == 0 ? 1 : (d == 1 ? E1x : E1x * E1y));
            if (th[sR] | th[sL]) { need = 1; break; }
        }
    }
    need = __syncthreads_or(need);
    if (need) {
        // W_old = prim(U_cv) on the tile + 2 halo, reflective images flipped
        for (int q = threadIdx.x; q < E2x * E2y * SM::E2z; q += blockDim.x) {
            int a[3] = {o[0] - 2 + q % E2x, o[1] - 2 + (q / E2x) % E2y, o[2] - 2 * dz + q / (E2x * E2y)};
            bool fl[3] = {false, false, false};
            const long long cid = cell_image<D, P>(G, a, fl);
            const long long ge = cid / NPT;
            const int pt = (int)(cid - ge * NPT);
            R u[V], w[V];
#pragma unroll
            for (int v = 0; v < V; v++) u[v] = A.ucv_in[(ge * V + v) * NPT + pt];
            primitives<D>(u, w, (R)G.gm);
#pragma unroll
            for (int d = 0; d < D; d++)
                if (fl[d]) w[1 + d] = -w[1 + d];
#pragma unroll
            for (int v = 0; v < V; v++) Wo[(size_t)q * V + v] = w[v];
        }
        __syncthreads();
        for (int d = 0; d < D; d++) {
            const int ex = Bx + (d == 0), ey = By + (d == 1);
            for (int q = threadIdx.x; q < nfaces[d]; q += blockDim.x) {
                int a[3] = {q % ex, (q / ex) % ey, q / (ex * ey)};
                const int sR = (a[0] + 1) + E1x * ((a[1] + 1) + E1y * (a[2] + dz));
                const int sL = sR - (d == 0 ? 1 : (d == 1 ? E1x : E1x * E1y));
                const R tR = (R)(th[sR] * 0.125), tL = (R)(th[sL] * 0.125);
                const R tf = smax(tR, tL);
                if (!(tf > 0)) continue;
                // cells L (low) and R (high) of the face; W_old box index
                R wlo_R[V], whi_R[V], wlo_L[V], whi_L[V];
                for (int side = 0; side < 2; side++) {
                    int cb[3] = {a[0] + 2, a[1] + 2, a[2] + 2 * dz};
                    if (side == 0) cb[d] -= 1;
                    int fa[3];  // frame indices of the cell
                    fa[0] = o[0] + cb[0] - 2 + 2;
                    fa[1] = o[1] + cb[1] - 2 + 2;
                    fa[2] = o[2] + cb[2] - 2 * dz + 2;
                    auto Wc = [&](int oi, int oj, int ok) -> const R* {
                        return Wo + (size_t)((cb[0] + oi) + E2x * ((cb[1] + oj) + E2y * (cb[2] + ok))) * V;
                    };
                    if (side == 0) muscl_cell<D, R>(G, fa, d, wdt, Wc, wlo_L, whi_L);
                    else muscl_cell<D, R>(G, fa, d, wdt, Wc, wlo_R, whi_R);
                }
                R uL[V], uR[V], fL[V];
                conservatives<D>(whi_L, uL, (R)G.gm);
                conservatives<D>(wlo_R, uR, (R)G.gm);
                riemann_hllc<D>(fL, uL, uR, d, (R)G.gm);
                R* F = Fs + (size_t)(fbase[d] + q) * V;
#pragma unroll
                for (int v = 0; v < V; v++) {
                    R f = F[v];
                    f = f + tf * (fL[v] - f);
                    F[v] = f;
                }
            }
        }
        __syncthreads();
    }
    // corrected sub-cell update
    R* Ub = Wo;                   // [NE][V][NPT] new U_cv of the tile
    R* Tmp = Wo + SM::NE * V * NPT;
    for (int q = threadIdx.x; q < NC; q += blockDim.x) {
        int a[3] = {q % Bx, (q / Bx) % By, q / (Bx * By)};
        const int el = (a[0] / n) + TX * ((a[1] / n) + TY * (a[2] / n));
        int c[3] = {a[0] % n, a[1] % n, a[2] % n};
        const int pt = pt_index<n>(c);
        const long long ge = el_ge[el];
        R hd[3];
        int fl_[3], fr_[3];
#pragma unroll
        for (int d = 0; d < D; d++) {
            const long long I = (long long)o[d] + a[d] + 2;
            hd[d] = (R)(G.fvf[d][I + 1] - G.fvf[d][I]);
            const int ex = Bx + (d == 0), ey = By + (d == 1);
            int lo[3] = {a[0], a[1], a[2]}, hi[3] = {a[0], a[1], a[2]};
            hi[d] += 1;
            fl_[d] = fbase[d] + lo[0] + ex * (lo[1] + ey * lo[2]);
            fr_[d] = fbase[d] + hi[0] + ex * (hi[1] + ey * hi[2]);
        }
        R un[V];
#pragma unroll
        for (int v = 0; v < V; v++) {
            const R uold = A.ucv_in[(ge * V + v) * NPT + pt];
            R F = 0;
#pragma unroll
            for (int d = 0; d < D; d++) F += (Fs[(size_t)fr_[d] * V + v] - Fs[(size_t)fl_[d] * V + v]) / hd[d];
            if (G.grav && v != 0) {
                R s;
                if (v <= D) s = un[0] * (R)G.g[v - 1];
                else {
                    s = un[1] * (R)G.g[0] + un[2] * (R)G.g[1];
                    if (D == 3) s = s + un[3] * (R)G.g[2];
                }
                F -= s;
            }
            un[v] = uold - wdt * F;
        }
#pragma unroll
        for (int v = 0; v < V; v++) {
            A.ucv_out[(ge * V + v) * NPT + pt] = un[v];
            Ub[(el * V + v) * NPT + pt] = un[v];
        }
        if (!A.last) {
            // candidate of slice t+1 from the new U_cv
            R uc[V];
            fv_candidate<D, P, R>(G, ffd, A.t + 1, ge, pt, un, M.wt[A.t + 1] * dt, uc);
            A.rp_old_next[ge * NPT + pt] = rho_p_fp64<D>(un, G.gm);
            A.rp_new_next[ge * NPT + pt] = rho_p_fp64<D>(uc, G.gm);
        }
    }
    if (!A.last) return;
    __syncthreads();
    // U_sp = cv_to_sp(U_cv) (src/hydro_ader.hpp:570)
    {
        R* bufs[2] = {Tmp, Ub};
        const R* src = Ub;
        for (int d = 0; d < D; d++) {
            R* dst = bufs[d % 2];
            sweep_smem<D, P, R>(src, dst, M.cv_to_sp, d, SM::NE * V * NPT);
            __syncthreads();
            src = dst;
        }
        R* Wsp = (R*)(src == Ub ? Tmp : Ub);
        for (int q = threadIdx.x; q < SM::NE * NPT; q += blockDim.x) {
            const int el = q / NPT, pt = q % NPT;
            const long long ge = el_ge[el];
            R u[V];
#pragma unroll
            for (int v = 0; v < V; v++) {
                const long long gi = (ge * V + v) * NPT + pt;
                R val = src[(el * V + v) * NPT + pt];
                if (A.rk_a > 0) {
                    const R ra = (R)A.rk_a;
                    val = ra * A.u0[gi] + ((R)1.0 - ra) * val;
                }
                u[v] = val;
                A.u[gi] = val;
            }
            if (A.final_stage) {
                R w[V];
                primitives<D>(u, w, (R)G.gm);
#pragma unroll
                for (int v = 0; v < V; v++) Wsp[(el * V + v) * NPT + pt] = w[v];
            }
        }
        if (!A.final_stage) return;
        __syncthreads();
        R* bufs2[2] = {(R*)src, Wsp};
        const R* s2 = Wsp;
        for (int d = 0; d < D; d++) {
            R* dst = bufs2[d % 2];
            sweep_smem<D, P, R>(s2, dst, M.sp_to_cv, d, SM::NE * V * NPT);
            __syncthreads();
            s2 = dst;
        }
        double dtl = 1.7976931348623157e308;
        for (int q = threadIdx.x; q < SM::NE * NPT; q += blockDim.x) {
            const int el = q / NPT, pt = q % NPT;
            const long long ge = el_ge[el];
            R w[V];
#pragma unroll
            for (int v = 0; v < V; v++) w[v] = s2[(el * V + v) * NPT + pt];
            if (A.wcv)
#pragma unroll
                for (int v = 0; v < V; v++) A.wcv[(ge * V + v) * NPT + pt] = w[v];
            dtl = smin(dtl, point_dt<D>(G, w, n));
        }
        block_min_dt(dtl, A.dtmin);
    }
}

template <typename R, int D, int P, int TX, int TY, int TZ>
__global__ void __launch_bounds__(kThreads) fv_update_kernel(DevGrid G, DevMatsT<R> M, FallbackArgsT<R> A) {
    fv_update_kernel_body<R, D, P, TX, TY, TZ>(G, M, A, blockIdx.x);
}

}  // namespace spdk
