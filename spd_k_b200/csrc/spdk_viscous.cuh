// Viscous terms of the hydro step (hydro/nu > 0), solver layout.
//
// The reference evaluates them inside every flux evaluation
// (src/hydro_ader.hpp:278-289, :383-405; src/hydro.cpp:420-572):
//   1. the LLF pass also overwrites both interface flux points of U_fp with
//      the central state 0.5(uR+uL) + 0.5(uR-uL);
//   2. compute_gradient: dU_e at the solution points = d/de of the
//      flux-point values of direction e (interior points interpolated,
//      interface points the central state);
//   3. compute_viscous_flux: the gradients interpolated to the flux points of
//      direction d, the viscous flux from them and the interface velocity;
//   4. the ghost fill copies / mirrors those fluxes across the domain edge;
//   5. sd_rusanov_solver: the interface flux += the (-0.5)-wind mean of the
//      two sides' viscous fluxes.
// Only the interface values of step 3 reach the solution (the interior
// flux points' viscous fluxes are computed by the reference and never read),
// so this pre-pass writes, per element and slice, the viscous flux at the
// 2D faces' flux points: VG_d [slice][element][side][var][transverse point].
// The Picard pass then adds step 5 to its LLF interface flux. An element's
// faces need its own state and the face traces of its face neighbours
// (their extrapolation to the shared face): a one-element halo, read here
// from global memory.
#pragma once
#include <cuda_runtime.h>

#include "spdk_kernels.cuh"

namespace spdk {

constexpr int kViscThreads = 128;

template <typename R>
struct ViscArgsT {
    const R* ua_in;  // [slice][E][V][NPT], or U when in_slices == 1
    int in_slices;
    R* vg[3];        // [slice][E][2][V][NTP] per direction
};

// elements per block: a block owns EPB consecutive elements of one slice,
// so its threads share the few face, gradient and flux items of each
// element (one element per block left most of them idle at barriers); as
// many as fit in 40 KB of shared memory, at most 8
template <typename R, int D, int P>
struct ViscShape {
    using S = Shape<D, P>;
    static constexpr int n = S::n, nf = S::nf, NPT = S::NPT, NTP = S::NTP, NFP = S::NFP;
    static constexpr int SOWN = (D + 1) * NPT, UFP = D * D * NFP, WST = D * 2 * (D + 1) * NTP, DU = D * D * NPT;
    static constexpr size_t per_element = (size_t)(SOWN + UFP + WST + DU) * sizeof(R);
    static constexpr int fit = (int)(40960 / per_element);
    static constexpr int EPB = fit < 1 ? 1 : (fit > 8 ? 8 : fit);
};

// blockIdx.x = group of EPB elements, blockIdx.y = slice
template <typename R, int D, int P>
__global__ void __launch_bounds__(kViscThreads) visc_face_kernel(DevGrid G, DevMatsT<R> M, ViscArgsT<R> A) {
    using S = Shape<D, P>;
    using VS = ViscShape<R, D, P>;
    constexpr int n = S::n, nf = S::nf, V = S::V, NPT = S::NPT, NTP = S::NTP, NFP = S::NFP;
    constexpr int EPB = VS::EPB;
    __shared__ R Sown[EPB][VS::SOWN];   // rho and momenta of each element
    __shared__ R Ufp[EPB][VS::UFP];     // [d][momentum][flux point of d]
    __shared__ R Wst[EPB][VS::WST];     // [d][side][rho, momenta][tp] interface states
    __shared__ R dU[EPB][VS::DU];       // [e][momentum][point] gradients
    __shared__ R Msf[nf * n], Mdf[n * nf];

    pdl_wait();
    if (gate_closed(G)) return;
    const int tid = threadIdx.x;
    const long long E = G.E;
    const long long ge0 = (long long)blockIdx.x * EPB;
    const int ne = (int)(E - ge0 < EPB ? E - ge0 : EPB);  // elements of this block
    const int t = blockIdx.y;
    const R* src = A.ua_in + (A.in_slices > 1 ? (long long)t * E * V * NPT : 0);
    for (int i = tid; i < nf * n; i += kViscThreads) {
        Msf[i] = M.sp_to_fp[i];
        Mdf[i] = M.dfp_to_sp[i];
    }
    for (int q = tid; q < ne * VS::SOWN; q += kViscThreads) {
        const int el = q / VS::SOWN, r = q % VS::SOWN;
        Sown[el][r] = src[(ge0 + el) * V * NPT + r];
    }
    __syncthreads();

    // ---- interface states of the 2D faces and interior flux points ----
    constexpr int NFACE = D * 2 * NTP;
    constexpr int NINT = D * (nf - 2) * NTP;
    for (int qq = tid; qq < ne * (NFACE + NINT); qq += kViscThreads) {
        const int el = qq / (NFACE + NINT), q = qq % (NFACE + NINT);
        const long long ge = ge0 + el;
        int eg[3];
        eg[0] = (int)(ge % G.N[0]);
        eg[1] = (int)((ge / G.N[0]) % G.N[1]);
        eg[2] = (int)(ge / ((long long)G.N[0] * G.N[1]));
        int c[3] = {0, 0, 0};
        if (q < NFACE) {
            const int d = q / (2 * NTP), s = (q / NTP) % 2, tp = q % NTP;
            tp_coords<D, n>(d, tp, c);
            const int row = s ? nf - 1 : 0;
            R own[D + 1], nb[D + 1];
            for (int v = 0; v <= D; v++) {
                R a = 0;
                for (int l = 0; l < n; l++) {
                    c[d] = l;
                    a += Sown[el][v * NPT + pt_index<n>(c)] * Msf[row * n + l];
                }
                own[v] = a;
            }
            // face neighbour across side s, or the ghost image at a
            // non-periodic domain edge (src/boundary.cpp:48-113)
            int g[3] = {eg[0], eg[1], eg[2]};
            g[d] += s ? 1 : -1;
            bool ghost = false;
            if (g[d] < 0 || g[d] >= G.N[d]) {
                if (G.bc[d] != kPeriodic) ghost = true;
                else g[d] = g[d] < 0 ? g[d] + G.N[d] : g[d] - G.N[d];
            }
            if (ghost) {
                for (int v = 0; v <= D; v++) nb[v] = own[v];
                if (G.bc[d] == kReflective) nb[1 + d] = -nb[1 + d];
            } else {
                const long long gn = ((long long)g[2] * G.N[1] + g[1]) * G.N[0] + g[0];
                const int nrow = s ? 0 : nf - 1;
                for (int v = 0; v <= D; v++) {
                    R a = 0;
                    for (int l = 0; l < n; l++) {
                        c[d] = l;
                        a += src[(gn * V + v) * NPT + pt_index<n>(c)] * Msf[nrow * n + l];
                    }
                    nb[v] = a;
                }
            }
            // central state: left = the element on the lower side of the face
            c[d] = row;
            const int fi = fp_index<n, nf>(d, c);
            for (int v = 0; v <= D; v++) {
                const R uL = s ? own[v] : nb[v], uR = s ? nb[v] : own[v];
                const R m = wind_mix(uL, uR, R(0.5));
                Wst[el][((d * 2 + s) * (D + 1) + v) * NTP + tp] = m;
                if (v >= 1) Ufp[el][(d * D + v - 1) * NFP + fi] = m;
            }
        } else {
            const int r = q - NFACE;
            const int d = r / ((nf - 2) * NTP), rr = r % ((nf - 2) * NTP);
            const int ll = 1 + rr / NTP, tp = rr % NTP;
            tp_coords<D, n>(d, tp, c);
            R u[D];
            for (int m = 0; m < D; m++) {
                R a = 0;
                for (int l = 0; l < n; l++) {
                    c[d] = l;
                    a += Sown[el][(1 + m) * NPT + pt_index<n>(c)] * Msf[ll * n + l];
                }
                u[m] = a;
            }
            c[d] = ll;
            const int fi = fp_index<n, nf>(d, c);
            for (int m = 0; m < D; m++) Ufp[el][(d * D + m) * NFP + fi] = u[m];
        }
    }
    __syncthreads();

    // ---- momentum gradients at the solution points (compute_gradient) ----
    for (int qq = tid; qq < ne * D * D * NPT; qq += kViscThreads) {
        const int el = qq / (D * D * NPT), q = qq % (D * D * NPT);
        const int e = q / (D * NPT), m = (q / NPT) % D, pt = q % NPT;
        int c[3];
        pt_coords<n>(pt, c);
        const int id = c[e];
        R du = 0;
        for (int ll = 0; ll < nf; ll++) {
            c[e] = ll;
            du += div_h(Ufp[el][(e * D + m) * NFP + fp_index<n, nf>(e, c)] * Mdf[id * nf + ll], (R)G.h[e],
                        (R)G.rh[e], G.pow2[e] != 0);
        }
        dU[el][q] = du;
    }
    __syncthreads();

    // ---- viscous fluxes at the face flux points (compute_viscous_flux) ----
    for (int qq = tid; qq < ne * NFACE; qq += kViscThreads) {
        const int el = qq / NFACE, q = qq % NFACE;
        const long long ge = ge0 + el;
        const int d = q / (2 * NTP), s = (q / NTP) % 2, tp = q % NTP;
        int c[3] = {0, 0, 0};
        tp_coords<D, n>(d, tp, c);
        const int id = s ? nf - 1 : 0;
        const int d2 = (d + 1) % 3, d3 = (d + 2) % 3;
        R du1[3], du2[3], du3[3], w[3];
        for (int a = 0; a < 3; a++) {
            R g1 = 0, g2 = 0, g3 = 0;
            if (a < D) {
                for (int l = 0; l < n; l++) {
                    c[d] = l;
                    const int pt = pt_index<n>(c);
                    const R mm = Msf[id * n + l];
                    g1 += dU[el][(d * D + a) * NPT + pt] * mm;
                    if (d2 < D) g2 += dU[el][(d2 * D + a) * NPT + pt] * mm;
                    if (d3 < D) g3 += dU[el][(d3 * D + a) * NPT + pt] * mm;
                }
            }
            du1[a] = g1;
            du2[a] = g2;
            du3[a] = g3;
        }
        const R* ws = Wst[el] + (d * 2 + s) * (D + 1) * NTP + tp;
        for (int a = 0; a < 3; a++) w[a] = a < D ? ws[(1 + a) * NTP] / ws[0] : R(0);
        R fm[3], fe;
        viscous_flux(du1, du2, du3, w, d, d2, d3, (R)G.nu, (R)G.beta, fm, fe);
        R* dst = A.vg[d] + (((long long)t * E + ge) * 2 + s) * V * NTP + tp;
        dst[0] = 0;
        for (int m = 0; m < D; m++) dst[(1 + m) * NTP] = fm[m];
        dst[(D + 1) * NTP] = fe;
    }
}

}  // namespace spdk
