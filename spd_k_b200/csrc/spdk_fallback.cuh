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
    // learned indicator (nullable): after the final stage, the element means
    // of (rho, p) and the nodal part of each feature row (row length n_in)
    // of the new state, for the next step's a-priori flags
    uint16_t* feat;
    float2* means;
    int n_in;
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
// FV axes of the smooth-extrema indicator: active cells and the ghost-framed
// centre / face coordinates of each direction
struct SedGeom {
    int nd[3];
    const double* C[3];
    const double* Fc[3];
};

template <int D, int P>
__device__ __forceinline__ SedGeom sed_geom(const DevGrid& G) {
    SedGeom S;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        S.nd[d] = G.N[d] * (P + 1);
        S.C[d] = G.fvc[d];
        S.Fc[d] = G.fvf[d];
    }
    return S;
}

// rpv(b, k): variable k (rho, p) of the candidate at FV coordinate b, which
// lies at most two cells outside the active cells.
// The smooth-extrema alpha of position a in direction d (0 outside the
// active cells, where the reference never computes it).
template <typename RPV>
__device__ __forceinline__ double sed_al(const SedGeom& S, const RPV& rpv, const int a[3], int d, int k) {
    const int ad = a[d];
    if (ad < 0 || ad >= S.nd[d]) return 0.0;
    const double* C = S.C[d];
    const double* Fc = S.Fc[d];
    int b[3] = {a[0], a[1], a[2]};
    double Wv[5];
#pragma unroll
    for (int off = -2; off <= 2; off++) {
        b[d] = ad + off;
        Wv[off + 2] = rpv(b, k);
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
    return sed_alpha(dv, dum, du, dup);
}

// min of the alphas of the cell and its two neighbours in direction d
template <typename RPV>
__device__ __forceinline__ double sed_component(const SedGeom& S, const RPV& rpv, const int a[3], int d, int k) {
    double al[3];
#pragma unroll
    for (int s = -1; s <= 1; s++) {
        int b[3] = {a[0], a[1], a[2]};
        b[d] += s;
        al[s + 1] = sed_al(S, rpv, b, d, k);
    }
    return smin(smin(al[0], al[1]), al[2]);
}

// min over the directions of the SED alpha of 2D cell (ax, ay), variable k,
// from candidates staged on the tile + 3 halo (Rn, row length E3x, origin
// ox - 3, oy - 3). Not inlined: the rare flagged cells pay for its registers
// in its own frame, and the NAD pass of every cell keeps to its cap.
static __device__ __noinline__ double sed_alpha_staged_2d(const SedGeom S, const double2* Rn, int E3x, int ox, int oy,
                                                         int ax, int ay, int k) {
    auto staged = [&](const int b[3], int kk) { return rp_var(Rn[(b[0] - ox + 3) + E3x * (b[1] - oy + 3)], kk); };
    const int a[3] = {ax, ay, 0};
    const double m0 = sed_component(S, staged, a, 0, k);
    return smin(m0, sed_component(S, staged, a, 1, k));
}

// the same for a 3D cell, candidates staged on the tile + 3 halo (rows of
// E3x, planes of E3x * E3y, origin o - 3)
static __device__ __noinline__ double sed_alpha_staged_3d(const SedGeom S, const double2* Rn, int E3x, int E3y,
                                                         const int o[3], const int a[3], int k) {
    auto staged = [&](const int b[3], int kk) {
        return rp_var(Rn[(b[0] - o[0] + 3) + E3x * ((b[1] - o[1] + 3) + E3y * (b[2] - o[2] + 3))], kk);
    };
    const double m0 = sed_component(S, staged, a, 0, k);
    const double m1 = smin(m0, sed_component(S, staged, a, 1, k));
    return smin(m1, sed_component(S, staged, a, 2, k));
}

// every alpha of variable k that the cells of a 3D tile (Bx x By x Bz from
// o) take along each direction d: the tile extended by one cell along d
// only, Al = [d = 0: (Bx + 2) By Bz][d = 1: Bx (By + 2) Bz][d = 2: Bx By
// (Bz + 2)], each x-fastest; candidates staged on the tile + 3 halo
static __device__ __noinline__ void sed_al_tile_3d(const SedGeom S, const double2* Rn, int E3x, int E3y,
                                                   const int o[3], int Bx, int By, int Bz, int k, double* Al) {
    auto staged = [&](const int b[3], int kk) {
        return rp_var(Rn[(b[0] - o[0] + 3) + E3x * ((b[1] - o[1] + 3) + E3y * (b[2] - o[2] + 3))], kk);
    };
    const int n0 = (Bx + 2) * By * Bz, n1 = Bx * (By + 2) * Bz, n2 = Bx * By * (Bz + 2);
    for (int w = threadIdx.x; w < n0 + n1 + n2; w += blockDim.x) {
        const int d = w < n0 ? 0 : (w < n0 + n1 ? 1 : 2);
        const int r = w - (d == 0 ? 0 : (d == 1 ? n0 : n0 + n1));
        const int ex = Bx + 2 * (d == 0), ey = By + 2 * (d == 1);
        const int a[3] = {o[0] + r % ex - (d == 0), o[1] + (r / ex) % ey - (d == 1), o[2] + r / (ex * ey) - (d == 2)};
        Al[w] = sed_al(S, staged, a, d, k);
    }
}

// every alpha of the 2D tile + 1 halo (E1x x E1y positions from ox - 1,
// oy - 1) of the variables in kmask, by the whole block: Al[(k * 2 + d) *
// E1x * E1y + position]; for blocks with many flagged cells, whose
// neighbours would otherwise evaluate the same positions again
static __device__ __noinline__ void sed_al_tile_2d(const SedGeom S, const double2* Rn, int E3x, int E1x, int E1y,
                                                   int ox, int oy, unsigned kmask, double* Al) {
    auto staged = [&](const int b[3], int kk) { return rp_var(Rn[(b[0] - ox + 3) + E3x * (b[1] - oy + 3)], kk); };
    const int np = E1x * E1y;
    for (int w = threadIdx.x; w < 4 * np; w += blockDim.x) {
        const int pos = w % np, kd = w / np, k = kd >> 1, d = kd & 1;
        if (!((kmask >> k) & 1u)) continue;
        const int a[3] = {ox - 1 + pos % E1x, oy - 1 + pos / E1x, 0};
        Al[w] = sed_al(S, staged, a, d, k);
    }
}

// R names the form (double: plain, float: precision) that launches the
// kernel; the detector computes in FP64 in both, and a separate
// instantiation per form keeps each form's compile flags on its own copy.
//
// Each thread loads its cells' candidates before it stages the tile's W_old,
// so a block waits for one memory round trip, not two. In 2D the kernel is
// compiled for 4 resident blocks (64 registers, the NAD pass unspilled;
// measured on B200: 38.6 us against 43.2 us at 6 blocks with spills); in
// 3D for 3 (80 registers, 20-50 bytes of spills; 90 registers and 2
// blocks uncapped: KH 16^3 p=5 FP64 step 11.40 -> 11.28 ms at 3).
template <int D>
constexpr int kDetectBlocksPerSM = D == 2 ? 4 : 3;
// 3D tiles whose candidates on the tile + 3 halo fit the static shared
// memory beside W_old's tile + 1 halo stage them for the SED stencils
// (a flagged cell otherwise reads its 45 candidates per variable from
// global memory); the larger ones keep the global reads
template <int D, int P, int TX, int TY, int TZ>
constexpr bool kSedStage3 =
    D == 3 && ((size_t)(TX * (P + 1) + 6) * (TY * (P + 1) + 6) * (TZ * (P + 1) + 6) +
               (size_t)(TX * (P + 1) + 2) * (TY * (P + 1) + 2) * (TZ * (P + 1) + 2)) * sizeof(double2) <= 46 * 1024;
// flagged threads of a block above which it evaluates every alpha of its
// tile once instead of each flagged cell evaluating its own six
constexpr int kSedTileThreshold = 24;

template <typename R, int D, int P, int TX, int TY, int TZ>
__device__ __forceinline__ void fv_detect_kernel_body(const DevGrid& G, const double2* __restrict__ rpo,
                                                            const double2* __restrict__ rpn,
                                                            uint8_t* __restrict__ T, int* any_trouble, long long bidx) {
    constexpr int n = P + 1;
    constexpr int NPT = Shape<D, P>::NPT;
    constexpr int Bx = TX * n, By = TY * n, Bz = D == 3 ? TZ * n : 1;
    constexpr int E1x = Bx + 2, E1y = By + 2, E1z = D == 3 ? Bz + 2 : 1;
    constexpr int NC = Bx * By * Bz;
    constexpr int CPT = (NC + kThreads - 1) / kThreads;  // cells per thread
    static_assert(CPT <= 16, "NAD flag bits");
    constexpr int E3x = Bx + 6, E3y = By + 6, E3z = D == 3 ? Bz + 6 : 1;
    constexpr bool stage3 = kSedStage3<D, P, TX, TY, TZ>;
    __shared__ double2 Ro[E1x * E1y * E1z];
    __shared__ double2 Rn[D == 2 ? E3x * E3y : (stage3 ? E3x * E3y * E3z : 1)];
    __shared__ double Al[D == 2 ? 4 * E1x * E1y : 1];
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
    double2 here_new[CPT];
#pragma unroll
    for (int r = 0; r < CPT; r++) {
        const int q = threadIdx.x + r * kThreads;
        if (NC % kThreads == 0 || q < NC) {
            int a[3] = {o[0] + q % Bx, o[1] + (q / Bx) % By, o[2] + q / (Bx * By)};
            here_new[r] = rpn[cell_id<D, P>(G, a)];
        }
    }
    for (int q = threadIdx.x; q < E1x * E1y * E1z; q += blockDim.x) {
        int a[3] = {o[0] - 1 + q % E1x, o[1] - 1 + (q / E1x) % E1y, o[2] - dz + q / (E1x * E1y)};
        bool fl[3];
        Ro[q] = rpo[cell_image<D, P>(G, a, fl)];
    }
    __syncthreads();
    // NAD flags of this thread's cells: bit 2r + k for variable k of cell r
    unsigned nad = 0;
#pragma unroll
    for (int r = 0; r < CPT; r++) {
        const int q = threadIdx.x + r * kThreads;
        if (NC % kThreads != 0 && q >= NC) break;
        const int x = q % Bx, y = (q / Bx) % By, z = q / (Bx * By);
        const int sc = (x + 1) + E1x * ((y + 1) + E1y * (z + dz));
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const double un = rp_var(here_new[r], k);
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
            if (un > mx || un < mn) nad |= 1u << (2 * r + k);
        }
    }
    // SED relaxation of the NAD flags (it can only clear one). In 2D, and
    // in 3D where it fits, the block stages the candidates of the tile + 3
    // halo once when any of its cells needs it, so a flagged cell reads its
    // stencils from shared memory instead of a chain of global loads.
    const int nflag = G.use_sed ? __syncthreads_count(nad != 0) : 0;
    if (nflag) {
        if (D == 2 || stage3) {
            for (int q = threadIdx.x; q < E3x * E3y * E3z; q += blockDim.x) {
                int a[3] = {o[0] - 3 + q % E3x, o[1] - 3 + (q / E3x) % E3y, o[2] - 3 * dz + q / (E3x * E3y)};
                // three cells outside a non-periodic boundary: never read
                bool outside = false;
#pragma unroll
                for (int d = 0; d < D; d++)
                    outside |= G.bc[d] != kPeriodic && (a[d] < -2 || a[d] >= G.N[d] * n + 2);
                bool fl[3];
                Rn[q] = outside ? make_double2(0.0, 0.0) : rpn[cell_image<D, P>(G, a, fl)];
            }
            __syncthreads();
        }
        const SedGeom SG = sed_geom<D, P>(G);
        auto global = [&](const int b[3], int k) {
            bool fl[3];
            return rp_var(rpn[cell_image<D, P>(G, b, fl)], k);
        };
        const bool tile = D == 2 && nflag > kSedTileThreshold;
        const bool tile3 = stage3 && nflag > kSedTileThreshold;
        if (tile3) {
            if constexpr (stage3) {
                // many flagged cells: every alpha of the tile once per
                // variable, in the W_old tile's storage (free after NAD),
                // then each flagged cell takes the min of its own and its
                // neighbours' along each direction, in sed_component's order
                constexpr int n0 = (Bx + 2) * By * Bz, n1 = Bx * (By + 2) * Bz, n2 = Bx * By * (Bz + 2);
                static_assert((size_t)(n0 + n1 + n2) * sizeof(double) <= sizeof(Ro), "alphas fit the W_old tile");
                double* Al3 = reinterpret_cast<double*>(Ro);
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    if (!__syncthreads_or(nad & (k == 0 ? 0x55555555u : 0xAAAAAAAAu))) continue;
                    sed_al_tile_3d(SG, Rn, E3x, E3y, o, Bx, By, Bz, k, Al3);
                    __syncthreads();
#pragma unroll
                    for (int r = 0; r < CPT; r++) {
                        if (!(nad & (1u << (2 * r + k)))) continue;
                        const int q = threadIdx.x + r * kThreads;
                        const int x = q % Bx, y = (q / Bx) % By, z = q / (Bx * By);
                        double alpha = 1;
#pragma unroll
                        for (int d = 0; d < 3; d++) {
                            double al[3];
#pragma unroll
                            for (int sft = -1; sft <= 1; sft++) {
                                const int i = d == 0 ? (x + 1 + sft) + (Bx + 2) * (y + By * z)
                                                     : (d == 1 ? n0 + x + Bx * ((y + 1 + sft) + (By + 2) * z)
                                                               : n0 + n1 + x + Bx * (y + By * (z + 1 + sft)));
                                al[sft + 1] = Al3[i];
                            }
                            const double m3 = smin(smin(al[0], al[1]), al[2]);
                            alpha = d == 0 ? m3 : smin(alpha, m3);
                        }
                        if (!(alpha < 1)) nad &= ~(1u << (2 * r + k));
                    }
                    __syncthreads();
                }
            }
        } else {
            if (tile) {
                const unsigned kmask = (__syncthreads_or(nad & 0x55555555u) ? 1u : 0u) |
                                       (__syncthreads_or(nad & 0xAAAAAAAAu) ? 2u : 0u);
                sed_al_tile_2d(SG, Rn, E3x, E1x, E1y, o[0], o[1], kmask, Al);
                __syncthreads();
            }
#pragma unroll
            for (int r = 0; r < CPT; r++) {
                if (!(nad & (3u << (2 * r)))) continue;
                const int q = threadIdx.x + r * kThreads;
                int a[3] = {o[0] + q % Bx, o[1] + (q / Bx) % By, o[2] + q / (Bx * By)};
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    if (!(nad & (1u << (2 * r + k)))) continue;
                    double alpha = 1;
                    if (tile) {
                        // the alphas of the cell and its neighbours, in the
                        // order sed_component takes them
                        const int x = a[0] - o[0] + 1, y = a[1] - o[1] + 1;
                        const double* A0 = Al + (k * 2 + 0) * E1x * E1y;
                        const double* A1 = Al + (k * 2 + 1) * E1x * E1y;
                        const double m0 = smin(smin(A0[(x - 1) + E1x * y], A0[x + E1x * y]), A0[(x + 1) + E1x * y]);
                        const double m1 = smin(smin(A1[x + E1x * (y - 1)], A1[x + E1x * y]), A1[x + E1x * (y + 1)]);
                        alpha = smin(m0, m1);
                    } else if (D == 2) {
                        alpha = sed_alpha_staged_2d(SG, Rn, E3x, o[0], o[1], a[0], a[1], k);
                    } else if (stage3) {
                        alpha = sed_alpha_staged_3d(SG, Rn, E3x, E3y, o, a, k);
                    } else {
#pragma unroll
                        for (int d = 0; d < D; d++) {
                            const double m3 = sed_component(SG, global, a, d, k);
                            alpha = d == 0 ? m3 : smin(alpha, m3);
                        }
                    }
                    if (!(alpha < 1)) nad &= ~(1u << (2 * r + k));
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < CPT; r++) {
        const int q = threadIdx.x + r * kThreads;
        if (NC % kThreads != 0 && q >= NC) break;
        int a[3] = {o[0] + q % Bx, o[1] + (q / Bx) % By, o[2] + q / (Bx * By)};
        const long long cid = cell_id<D, P>(G, a);
        bool tr = (nad >> (2 * r)) & 3u;
        const double rho = here_new[r].x, p = here_new[r].y;
        if (rho < kRhoMin || rho > kRhoMax) tr = true;
        if (p < kPMin || p > kPMax) tr = true;
        const long long el = cid / NPT;
        if (G.elem_trouble && tr) G.elem_trouble[el] = 1;  // a-posteriori label
        if (G.elem_pred && G.elem_pred[el]) tr = true;     // a-priori prediction
        T[cid] = tr ? 1 : 0;
        if (any_trouble && tr) atomicAdd(any_trouble, 1);
    }
}

template <typename R, int D, int P, int TX, int TY, int TZ>
__global__ void __launch_bounds__(kThreads, kDetectBlocksPerSM<D>) fv_detect_kernel(DevGrid G, const double2* __restrict__ rpo,
                                                            const double2* __restrict__ rpn,
                                                            uint8_t* __restrict__ T, int* any_trouble) {
    pdl_wait();
    if (gate_closed(G)) return;
    fv_detect_kernel_body<R, D, P, TX, TY, TZ>(G, rpo, rpn, T, any_trouble, blockIdx.x);
}

// ---------------------------------------------------------------------------
// theta = max over the Moore box of w(#offsets) * trouble, plus the 0.25 ring
// (src/trouble_detection.cpp:191-242; theta_from_troubles without blending),
// evaluated by the update kernel on its tile + 1 halo from the troubles on
// the tile + 3 halo, in eighths: w * 8 = 8, 6, 4, 3 and the ring 2 (all
// exact, as is theta * 8 of the reference's float weights).
//
// A ghost cell's theta is the theta of its image (the reference fills the
// ghosts of theta after computing it on the active cells). Outside a
// periodic boundary that equals the theta evaluated in place, since the
// troubles around it are periodic images too; outside a reflective or
// zero-gradient boundary the image (one or two cells inside) lies in the
// same tile and its value is used. The tile's own cells are written to
// `theta_out` (the THETA field).
// ---------------------------------------------------------------------------
template <int D, int P, int TX, int TY, int TZ>
struct ThetaTile {
    static constexpr int n = P + 1;
    static constexpr int Bx = TX * n, By = TY * n, Bz = D == 3 ? TZ * n : 1;
    static constexpr int E3x = Bx + 6, E3y = By + 6, E3z = D == 3 ? Bz + 6 : 1;
    static constexpr int E2x = Bx + 4, E2y = By + 4, E2z = D == 3 ? Bz + 4 : 1;
    static constexpr int E1x = Bx + 2, E1y = By + 2, E1z = D == 3 ? Bz + 2 : 1;
    static constexpr int n3 = E3x * E3y * E3z, n2 = E2x * E2y * E2z, n1 = E1x * E1y * E1z;
    static constexpr size_t scratch = (size_t)n3 + n2;  // bytes of T3 + Th2
};

// called by every thread of the block; `scratch` holds ThetaTile::scratch
// bytes; th (tile + 1 halo) is complete after the caller's next barrier.
// Returns (to every thread) whether any trouble lies within reach of the
// tile: when none does, theta is zero on the tile + 1 halo and the blending
// passes are skipped.
template <int D, int P, int TX, int TY, int TZ>
__device__ __forceinline__ int theta_on_tile(const DevGrid& G, const uint8_t* __restrict__ T, const int o[3],
                                             uint8_t* scratch, uint8_t* th, uint8_t* __restrict__ theta_out) {
    using TT = ThetaTile<D, P, TX, TY, TZ>;
    constexpr int n = P + 1;
    const int dz = D == 3 ? 1 : 0;
    uint8_t* T3 = scratch;
    uint8_t* Th2 = scratch + TT::n3;
    int any = 0;
    for (int q = threadIdx.x; q < TT::n3; q += blockDim.x) {
        int a[3] = {o[0] - 3 + q % TT::E3x, o[1] - 3 + (q / TT::E3x) % TT::E3y, o[2] - 3 * dz + q / (TT::E3x * TT::E3y)};
        // a cell three layers outside a non-periodic boundary has no image
        // (the ghost frame is two layers deep) and feeds no theta below:
        // the theta of a ghost cell there is its image's
        bool outside = false;
#pragma unroll
        for (int d = 0; d < D; d++)
            outside |= G.bc[d] != kPeriodic && (a[d] < -2 || a[d] >= G.N[d] * n + 2);
        bool fl[3];
        const uint8_t tq = outside ? (uint8_t)0 : T[cell_image<D, P>(G, a, fl)];
        T3[q] = tq;
        any |= tq;
    }
    if (!__syncthreads_or(any)) {
        // no trouble within three cells of the tile: theta is zero on it
        for (int q = threadIdx.x; q < TT::n1; q += blockDim.x) {
            th[q] = 0;
            const int l0[3] = {q % TT::E1x, (q / TT::E1x) % TT::E1y, q / (TT::E1x * TT::E1y)};
            const bool inner = l0[0] >= 1 && l0[0] <= TT::Bx && l0[1] >= 1 && l0[1] <= TT::By &&
                               (D == 2 || (l0[2] >= 1 && l0[2] <= TT::Bz));
            if (inner) {
                int ga[3] = {o[0] + l0[0] - 1, o[1] + l0[1] - 1, o[2] + l0[2] - dz};
                theta_out[cell_id<D, P>(G, ga)] = 0;
            }
        }
        return 0;
    }
    if (G.blending) {
        for (int q = threadIdx.x; q < TT::n2; q += blockDim.x) {
            const int x = q % TT::E2x + 1, y = (q / TT::E2x) % TT::E2y + 1, z = q / (TT::E2x * TT::E2y) + dz;
            int m = 0;
            for (int ok = -dz; ok <= dz; ok++)
#pragma unroll
                for (int oj = -1; oj <= 1; oj++)
#pragma unroll
                    for (int oi = -1; oi <= 1; oi++) {
                        const int n0 = (oi != 0) + (oj != 0) + (ok != 0);
                        const int w8 = n0 == 0 ? 8 : (n0 == 1 ? 6 : (n0 == 2 ? 4 : 3));
                        if (T3[(x + oi) + TT::E3x * ((y + oj) + TT::E3y * (z + ok))]) m = m < w8 ? w8 : m;
                    }
            Th2[q] = (uint8_t)m;
        }
        __syncthreads();
    }
    for (int q = threadIdx.x; q < TT::n1; q += blockDim.x) {
        const int l0[3] = {q % TT::E1x, (q / TT::E1x) % TT::E1y, q / (TT::E1x * TT::E1y)};
        int l[3] = {l0[0], l0[1], l0[2]};
#pragma unroll
        for (int d = 0; d < D; d++) {
            const int a = o[d] - 1 + l[d], na = G.N[d] * n;
            if ((a < 0 || a >= na) && G.bc[d] != kPeriodic) {
                bool f = false;
                l[d] = fv_image(a, na, G.bc[d], &f) - o[d] + 1;
            }
        }
        int t8;
        if (G.blending) {
            const int x = l[0] + 1, y = l[1] + 1, z = l[2] + dz;
            const int c = Th2[x + TT::E2x * (y + TT::E2y * z)];
            int ring = 0;
            for (int ok = -dz; ok <= dz; ok++)
#pragma unroll
                for (int oj = -1; oj <= 1; oj++)
#pragma unroll
                    for (int oi = -1; oi <= 1; oi++)
                        if (Th2[(x + oi) + TT::E2x * ((y + oj) + TT::E2y * (z + ok))]) ring = 2;
            t8 = c < ring ? ring : c;
        } else {
            t8 = T3[(l[0] + 2) + TT::E3x * ((l[1] + 2) + TT::E3y * (l[2] + 2 * dz))] ? 8 : 0;
        }
        th[q] = (uint8_t)t8;
        const bool inner = l0[0] >= 1 && l0[0] <= TT::Bx && l0[1] >= 1 && l0[1] <= TT::By &&
                           (D == 2 || (l0[2] >= 1 && l0[2] <= TT::Bz));
        if (inner) {
            int ga[3] = {o[0] + l0[0] - 1, o[1] + l0[1] - 1, o[2] + l0[2] - dz};
            theta_out[cell_id<D, P>(G, ga)] = (uint8_t)t8;
        }
    }
    return 1;
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

// resident blocks the update kernel is compiled for: 5 (48 registers) in 2D,
// where the extra warps hide its gather latency (measured on B200 at 256^2,
// p = 3: 62.6 against 72.0 us in FP32, 139 against 176 us in FP64). In 3D
// (one element per block) the 140-register kernel ran one block per SM;
// measured per step of 4 updates, FP64: 32^3 p=3 6.15 / 3.47 / 2.52 ms at
// 2 / 3 / 4 blocks, 16^3 p=5 4.13 / 3.65 / 4.05 ms. The FP32 3D update
// above p = 3 fits 4 blocks without spills (64 registers) and takes them:
// KH 16^3 p=5 FP32 step 4.91 -> 4.68 ms together with the 3D detection's
// 3 blocks.
template <int D, int P>
constexpr int kUpdateBlocksPerSM = D == 2 ? 5 : (P <= 3 ? 4 : 3);

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
    static_assert(ThetaTile<D, P, TX, TY, TZ>::scratch <= (wold > epi ? wold : epi) * sizeof(R),
                  "theta scratch fits the W_old area");
    static_assert((size_t)NE * NPT * 16 + NE * 8 <= faces * sizeof(R), "indicator scratch fits the face area");
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
    // theta on the tile + 1 halo from the troubles (scratch: the W_old area,
    // written only after the barrier that follows)
    const int near = theta_on_tile<D, P, TX, TY, TZ>(G, A.trouble, o, reinterpret_cast<uint8_t*>(Wo), th, A.theta);
    // SD face fluxes of the tile
    const int nfaces[3] = {SM::NF0, SM::NF1, SM::NF2};
    int fbase[3] = {0, SM::NF0, SM::NF0 + SM::NF1};
    // direction loops unrolled: ffd, nfaces and fbase stay in registers
#pragma unroll
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
    // faces that blend in the fallback flux (none when no trouble is near)
    int need = 0;
#pragma unroll
    for (int d = 0; d < D; d++) {
        if (need || !near) break;
        const int ex = Bx + (d == 0), ey = By + (d == 1);
        for (int q = threadIdx.x; q < nfaces[d]; q += blockDim.x) {
            int a[3] = {q % ex, (q / ex) % ey, q / (ex * ey)};
            const int sR = (a[0] + 1) + E1x * ((a[1] + 1) + E1y * (a[2] + dz));
            const int sL = sR - (d == 0 ? 1 : (d == 1 ? E1x : E1x * E1y));
            if (th[sR] | th[sL]) { need = 1; break; }
        }
    }
    need = near ? __syncthreads_or(need) : 0;
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
            if (A.final_stage && A.feat) {
                // (rho, p) of the new state for the indicator's features;
                // the face-flux area is free now
                double r, pr;
                feature_rho_p(u, 1, V, G.gm, &r, &pr);
                reinterpret_cast<double2*>(Fs)[q] = make_double2(r, pr);
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
        if (A.feat) {
            // element means summed in point order, then the nodal features
            // rho / mean - 1 and p / mean - 1 as BF16 (the values of the
            // indicator's feature kernels)
            const double2* RPs = reinterpret_cast<const double2*>(Fs);
            float2* Mn = reinterpret_cast<float2*>(Fs) + 2 * SM::NE * NPT;
            for (int el = threadIdx.x; el < SM::NE; el += blockDim.x) {
                double sr = 0, sp = 0;
                for (int pt = 0; pt < NPT; pt++) {
                    sr = __dadd_rn(sr, RPs[el * NPT + pt].x);
                    sp = __dadd_rn(sp, RPs[el * NPT + pt].y);
                }
                const float2 mn = make_float2((float)__ddiv_rn(sr, (double)NPT), (float)__ddiv_rn(sp, (double)NPT));
                Mn[el] = mn;
                A.means[el_ge[el]] = mn;
            }
            __syncthreads();
            for (int q = threadIdx.x; q < SM::NE * NPT; q += blockDim.x) {
                const int el = q / NPT, pt = q % NPT;
                const double2 v = RPs[q];
                const float2 mn = Mn[el];
                uint16_t* row = A.feat + el_ge[el] * A.n_in;
                row[pt] = bf16_bits(feature_ratio(v.x, mn.x));
                row[NPT + pt] = bf16_bits(feature_ratio(v.y, mn.y));
            }
        }
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
__global__ void __launch_bounds__(kThreads, kUpdateBlocksPerSM<D, P> + (sizeof(R) == 4 && D == 3 && P > 3 ? 1 : 0)) fv_update_kernel(DevGrid G, DevMatsT<R> M, FallbackArgsT<R> A) {
    pdl_wait();
    if (gate_closed(G)) return;
    fv_update_kernel_body<R, D, P, TX, TY, TZ>(G, M, A, blockIdx.x);
}

}  // namespace spdk
