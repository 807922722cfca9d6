// Fused device kernels of the spd_K B200 hydro step.
//
// State layout (device, arithmetic type R = double or float, no ghost elements):
//   U, U_cv          [element][var][point]            V = D+2 slots
//   U_ader (A and B) [slice][element][var][point]     ping-pong per Picard pass
//   FF_d             [slice][element][var][face point] FV face fluxes of direction d,
//                                                      laid out like the element's
//                                                      d-flux points (n_f per line)
//   RP_old, RP_new   [element][point] double2          (rho, p) of the FV candidate
//   T, theta         [element][point] uint8            trouble flag / theta*8
// element = (k*Ny + j)*Nx + i, point = (kk*n + jj)*n + ii.
//
// Boundary conditions are applied by index mapping instead of ghost storage:
// an SD face on the domain edge pairs the element's own interface state with
// its periodic partner, a copy (gradfree) or a mirror (reflective); FV ghost
// cells are images of active cells (spdk::fv_image).
#pragma once
#include <cuda_runtime.h>

#include "spdk_physics.cuh"

namespace spdk {

constexpr int kThreads = 256;
constexpr int kMaxNd = 8;    // n = p+1 <= 8
constexpr int kMaxNfd = 9;

// Transform matrices in the arithmetic type R, passed by value (kernel
// parameter space). R = double is the plain form; R = float the precision form.
template <typename R>
struct DevMatsT {
    R sp_to_fp[kMaxNfd * kMaxNd];   // [nf][n]
    R dfp_to_sp[kMaxNd * kMaxNfd];  // [n][nf]
    R sp_to_cv[kMaxNd * kMaxNd];    // [n][n]
    R cv_to_sp[kMaxNd * kMaxNd];
    R invader[kMaxNd * kMaxNd];     // [nt][nt]
    R wt[kMaxNd];
};
using DevMats = DevMatsT<double>;

struct DevGrid {
    int N[3];
    int bc[3];
    double h[3], rh[3];
    int pow2[3];
    int uniform_pow2;  // all active h equal and a power of two
    double gm, cfl;
    double g[3];
    int grav;
    int nt;
    long long E;
    const double* fvf[3];  // FV faces in frame indexing (active cell a has faces a+2, a+3)
    const double* fvc[3];  // FV centres in frame indexing
    int* status;           // device-detected faults (kStatus* bits)
    // fallback settings
    double nad_tol;
    int nad_delta, nad_moore, use_sed, blending;
    // viscous terms (hydro/nu > 0; src/hydro.cpp:420-572)
    double nu, beta;
    // learned indicator: per element, set when NAD/SED/PAD flags any of its
    // sub-cells in any slice of the step (NULL: not recorded), and the
    // a-priori prediction that counts all its sub-cells troubled (NULL: off)
    uint8_t* elem_trouble;
    const uint8_t* elem_pred;
    // device-resident time loop (spdk_hydro_evolve): set once t reaches
    // t_end; every kernel of a step launched after that returns at once
    // (NULL: never)
    const int* gate;
};

__device__ __forceinline__ bool gate_closed(const DevGrid& G) { return G.gate && *G.gate; }

// Programmatic dependent launch: a step's kernels are launched with
// programmatic stream serialization, so a kernel may be scheduled while its
// predecessor drains; it waits here, before touching any memory, until the
// predecessor has completed and its writes are visible (a no-op for a
// normal launch)
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

enum { kPredict = 0, kCorrect = 1, kFlux = 2 };

template <typename R>
struct PicardArgsT {
    const R* ua_in;        // [slice][E][V][NPT], or U when in_slices == 1
    int in_slices;         // 1: every slice equals U (first Picard pass / RK stage)
    const R* u;            // U_sp
    R* ua_out;             // kPredict output
    R* u_out;              // kCorrect output (may alias u: element-local)
    const R* u0;           // RK step-start state
    double rk_a;           // RK convex weight (0: none)
    R* ff[3];              // kFlux: FV face fluxes, all slices
    R* ucv;                // kFlux: U_cv = sp_to_cv(U)
    double2* rp_old;       // kFlux: slice-0 candidate (rho, p) of U_old, FP64
    double2* rp_new;       // kFlux: slice-0 candidate (rho, p) of U_new, FP64
    R* wcv;                // kCorrect: W_cv output (nullable)
    unsigned long long* dtmin;  // kCorrect: next-dt reduction
    int final_stage;       // kCorrect: compute W_cv and dt
    const double* dt;      // device dt of this step
    const R* vg[3];        // viscous face fluxes of this pass's input (NULL: inviscid)
};
using PicardArgs = PicardArgsT<double>;

template <int D, int P>
struct Shape {
    static constexpr int n = P + 1;
    static constexpr int nf = P + 2;
    static constexpr int V = D + 2;
    static constexpr int NPT = D == 2 ? n * n : n * n * n;
    static constexpr int NTP = NPT / n;    // points across one direction
    static constexpr int NFP = NTP * nf;   // flux points per direction
};

// padded shared-memory strides of the Picard pass (bank spreading); an
// element block (SS) starts on a 16-byte boundary whenever its data is a
// whole number of 16-byte units, so it can be a bulk-copy destination
template <int D, int P, typename R = double>
struct PicardPad {
    static constexpr int V = D + 2;
    static constexpr int NPT = D == 2 ? (P + 1) * (P + 1) : (P + 1) * (P + 1) * (P + 1);
    static constexpr int NFP = NPT / (P + 1) * (P + 2);
    static constexpr int Q = 16 / (int)sizeof(R);                   // elements per 16 bytes
    static constexpr int WORDS = (int)sizeof(R) / 4;                 // 4-byte banks per element
    static constexpr int SS0 = (V * NPT + Q - 1) / Q * Q;
    static constexpr int SS = SS0 + ((SS0 * WORDS) % 32 == 0 ? Q : 0);
    static constexpr int FXS = NFP + ((NFP * V) % 16 == 0 ? 1 : 0);
};

// coordinates of a point index
template <int n>
__device__ __forceinline__ void pt_coords(int pt, int c[3]) {
    c[0] = pt % n;
    c[1] = (pt / n) % n;
    c[2] = pt / (n * n);
}
template <int n>
__device__ __forceinline__ int pt_index(const int c[3]) {
    return c[0] + n * (c[1] + n * c[2]);
}
// flux-point index of direction d: extent nf along d, n along the others
template <int n, int nf>
__device__ __forceinline__ int fp_index(int d, const int c[3]) {
    if (d == 0) return c[0] + nf * (c[1] + n * c[2]);
    if (d == 1) return c[0] + n * (c[1] + nf * c[2]);
    return c[0] + n * (c[1] + n * c[2]);
}
// transverse point tp of direction d -> coordinates (coordinate d untouched)
template <int D, int n>
__device__ __forceinline__ void tp_coords(int d, int tp, int c[3]) {
    const int a = tp % n, b = tp / n;
    if (d == 0) { c[1] = a; c[2] = D == 3 ? b : 0; }
    else if (d == 1) { c[0] = a; c[2] = D == 3 ? b : 0; }
    else { c[0] = a; c[1] = b; }
}

// Tile of TX x TY x TZ elements plus its face halo (no edges or corners).
template <int D, int TX, int TY, int TZ>
struct Tile {
    static constexpr int NE = TX * TY * TZ;
    static constexpr int HX = TY * TZ, HY = TX * TZ, HZ = TX * TY;
    static constexpr int NS = NE + 2 * HX + 2 * HY + (D == 3 ? 2 * HZ : 0);
    __device__ static int T(int d) { return d == 0 ? TX : (d == 1 ? TY : TZ); }
    // slot of tile-local element coordinates (at most one outside the tile)
    __device__ static int slot(int lx, int ly, int lz) {
        if (lx < 0 || lx >= TX) return NE + (lx < 0 ? 0 : HX) + ly + TY * lz;
        if (ly < 0 || ly >= TY) return NE + 2 * HX + (ly < 0 ? 0 : HY) + lx + TX * lz;
        if (lz < 0 || lz >= TZ) return NE + 2 * HX + 2 * HY + (lz < 0 ? 0 : HZ) + lx + TX * ly;
        return lx + TX * (ly + TY * lz);
    }
    // local coordinates of a slot
    __device__ static void coords(int s, int l[3]) {
        if (s < NE) {
            l[0] = s % TX; l[1] = (s / TX) % TY; l[2] = s / (TX * TY);
            return;
        }
        int r = s - NE;
        if (r < 2 * HX) {
            const int side = r / HX, q = r % HX;
            l[0] = side ? TX : -1; l[1] = q % TY; l[2] = q / TY;
            return;
        }
        r -= 2 * HX;
        if (r < 2 * HY) {
            const int side = r / HY, q = r % HY;
            l[1] = side ? TY : -1; l[0] = q % TX; l[2] = q / TX;
            return;
        }
        r -= 2 * HY;
        const int side = r / HZ, q = r % HZ;
        l[2] = side ? TZ : -1; l[0] = q % TX; l[1] = q / TX;
    }
};

// global element index of tile-local coordinates, or -1 when the element
// lies beyond a non-periodic domain edge
template <int D>
__device__ __forceinline__ long long elem_of(const DevGrid& G, const int o[3], const int l[3]) {
    int g[3];
    for (int d = 0; d < 3; d++) {
        g[d] = o[d] + l[d];
        if (d >= D) { g[d] = 0; continue; }
        if (g[d] < 0 || g[d] >= G.N[d]) {
            if (G.bc[d] != kPeriodic) return -1;
            g[d] = g[d] < 0 ? g[d] + G.N[d] : g[d] - G.N[d];
        }
    }
    return ((long long)g[2] * G.N[1] + g[1]) * G.N[0] + g[0];
}

// dt candidate of one W_cv point (src/hydro.cpp:222-254, inviscid), always
// evaluated in FP64
template <int D, typename R>
__device__ __forceinline__ double point_dt(const DevGrid& G, const R* wr, int n) {
    double w[D + 2];
#pragma unroll
    for (int v = 0; v < D + 2; v++) w[v] = (double)wr[v];
    const double cs = sound_speed(w[0], w[D + 1], G.gm);
    double cmax = 0, dxmin = 1;
#pragma unroll
    for (int d = 0; d < D; d++) {
        cmax += (fabs(w[1 + d]) + cs);
        dxmin = smin(dxmin, G.h[d]);
    }
    return G.cfl * dxmin / cmax / n;
}

// block-wide min of positive doubles, then one atomic per block (the order
// of a min never changes its value)
__device__ __forceinline__ void block_min_dt(double v, unsigned long long* out) {
    __shared__ double red[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) v = smin(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < (int)(blockDim.x >> 5) ? red[l] : 1.7976931348623157e308;
        for (int o = 16; o > 0; o >>= 1) v = smin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (l == 0) atomicMin(out, (unsigned long long)__double_as_longlong(v));
    }
}

// One directional sweep of element-local arrays in shared memory
// (src/transforms.cpp:120-147): out(c) = sum_l in(c with c_d = l) * M(c_d, l)
template <int D, int P, typename R>
__device__ __forceinline__ void sweep_smem(const R* in, R* out, const R* M, int d, int count) {
    using S = Shape<D, P>;
    constexpr int n = S::n;
    for (int q = threadIdx.x; q < count; q += blockDim.x) {
        const int pt = q % S::NPT, base = q - pt;
        int c[3];
        pt_coords<n>(pt, c);
        const int id = c[d];
        R u = 0;
#pragma unroll
        for (int l = 0; l < n; l++) {
            c[d] = l;
            u += in[base + pt_index<n>(c)] * M[id * n + l];
        }
        out[q] = u;
    }
}

// Sub-cell candidate of the FV update (src/transforms.cpp:483-543 with
// update=0): U_new = U_old - (w_t dt) sum_d (F_{+} - F_{-}) / h_d for the
// cell at point pt of element ge; F from FF_d of slice t.
template <int D, int P, typename R>
__device__ __forceinline__ void fv_candidate(const DevGrid& G, R* const* ff, int t, long long ge, int pt,
                                             const R* uold, R wdt, R* unew) {
    using S = Shape<D, P>;
    constexpr int n = S::n, nf = S::nf, V = S::V;
    int c[3];
    pt_coords<n>(pt, c);
    long long eg[3];
    eg[0] = ge % G.N[0];
    eg[1] = (ge / G.N[0]) % G.N[1];
    eg[2] = ge / ((long long)G.N[0] * G.N[1]);
    R hd[3];
    int fl[3], fr[3];
#pragma unroll
    for (int d = 0; d < D; d++) {
        const long long I = eg[d] * n + c[d] + 2;
        hd[d] = (R)(G.fvf[d][I + 1] - G.fvf[d][I]);
        int cc[3] = {c[0], c[1], c[2]};
        fl[d] = fp_index<n, nf>(d, cc);
        cc[d] = c[d] + 1;
        fr[d] = fp_index<n, nf>(d, cc);
    }
#pragma unroll
    for (int v = 0; v < V; v++) {
        R F = 0;
#pragma unroll
        for (int d = 0; d < D; d++) {
            const R* f = ff[d] + (((long long)t * G.E + ge) * V + v) * S::NFP;
            F += (f[fr[d]] - f[fl[d]]) / hd[d];
        }
        if (G.grav) {
            R s = 0;
            if (v >= 1 && v <= D) s = uold[0] * (R)G.g[v - 1];
            else if (v == D + 1) {
                s = uold[1] * (R)G.g[0] + uold[2] * (R)G.g[1];
                if (D == 3) s = s + uold[3] * (R)G.g[2];
            }
            if (v != 0) F -= s;
        }
        unew[v] = uold[v] - wdt * F;
    }
}

// (rho, p) of a conserved state with the pressure recovered in FP64
// (src/hydro.cpp:95-106); for R = double these are primitives()'s operations
template <int D, typename R>
__device__ __forceinline__ double2 rho_p_fp64(const R* u, double gm) {
    const double r = (double)u[0];
    if constexpr (sizeof(R) == 4) {
        double m2 = 0;
#pragma unroll
        for (int d = 1; d <= D; d++) m2 += (double)u[d] * (double)u[d];
        return make_double2(r, ((double)u[D + 1] - 0.5 * m2 * rcp_fp64(u[0])) * (gm - 1.));
    }
    double ek = 0;
#pragma unroll
    for (int d = 1; d <= D; d++) {
        const double v = (double)u[d] / r;
        ek += v * (double)u[d];
    }
    return make_double2(r, ((double)u[D + 1] - 0.5 * ek) * (gm - 1.));
}

// ---------------------------------------------------------------------------
// Bulk asynchronous copies (TMA engine, 1-D cp.async.bulk) into shared memory
// completing on an mbarrier. Every wait is bounded: on time-out the kernel
// records kStatusStagingTimeout in *status and carries on, so a lost copy
// can never hang the device; the host turns the flag into an error.
// ---------------------------------------------------------------------------
constexpr int kStatusStagingTimeout = 1;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait on one mbarrier phase; false (and the status flag) on time-out
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* status) {
    for (int i = 0; i < (1 << 20); i++)
        if (mbar_try_wait(bar, parity)) return true;
    if (status) atomicOr(status, kStatusStagingTimeout);
    return false;
}

// interior flux point of direction d: interpolation, primitives, Euler flux
template <typename R, int D, int P, int TX, int TY, int TZ, int d>
__device__ __forceinline__ void picard_interior_item(const DevGrid& G, const R* sp_to_fp, const R* Ss, R* FX, int q) {
    using S = Shape<D, P>;
    constexpr int n = S::n, nf = S::nf, V = S::V, NPT = S::NPT, NTP = S::NTP;
    constexpr int NE = TX * TY * TZ;
    constexpr int SS = PicardPad<D, P, R>::SS, FXS = PicardPad<D, P, R>::FXS;
    const int el = q / ((nf - 2) * NTP);
    const int rr = q % ((nf - 2) * NTP);
    const int ll = 1 + rr / NTP, tp = rr % NTP;
    int c[3] = {0, 0, 0};
    tp_coords<D, n>(d, tp, c);
    R u[V], w[V], f[V];
    const R* src = Ss + el * SS;
#pragma unroll
    for (int v = 0; v < V; v++) {
        R a = 0;
#pragma unroll
        for (int l = 0; l < n; l++) {
            c[d] = l;
            a += src[v * NPT + pt_index<n>(c)] * sp_to_fp[ll * n + l];
        }
        u[v] = a;
    }
    primitives<D>(u, w, (R)G.gm);
    euler_flux<D>(u, w, f, d);
    c[d] = ll;
    const int fi = fp_index<n, nf>(d, c);
    R* dst = FX + (d * NE + el) * V * FXS;
#pragma unroll
    for (int v = 0; v < V; v++) dst[v * FXS + fi] = f[v];
}

// element interface of direction d: both interface states, ghost image at a
// non-periodic domain edge (src/boundary.cpp:48-113), LLF flux written to
// the adjacent flux points of the tile's elements
template <typename R, int D, int P, int TX, int TY, int TZ, int d, bool VISC>
__device__ __forceinline__ void picard_face_item(const DevGrid& G, const DevMatsT<R>& M, const R* Ss, R* FX,
                                                 const int o[3], int q, const R* vg, const long long* sl_elem,
                                                 int vt) {
    using S = Shape<D, P>;
    using TL = Tile<D, TX, TY, TZ>;
    constexpr int n = S::n, nf = S::nf, V = S::V, NPT = S::NPT, NTP = S::NTP;
    constexpr int NE = TL::NE;
    constexpr int SS = PicardPad<D, P, R>::SS, FXS = PicardPad<D, P, R>::FXS;
    constexpr int Td = d == 0 ? TX : (d == 1 ? TY : TZ);
    constexpr int per = (NE / Td) * NTP;
    const int fidx = q / per;
    const int rr = q % per;
    const int qq = rr / NTP, tp = rr % NTP;
    int c[3] = {0, 0, 0};
    tp_coords<D, n>(d, tp, c);
    int lL[3] = {0, 0, 0};
    if (d == 0) { lL[1] = qq % TY; lL[2] = qq / TY; }
    else if (d == 1) { lL[0] = qq % TX; lL[2] = qq / TX; }
    else { lL[0] = qq % TX; lL[1] = qq / TX; }
    int lR[3] = {lL[0], lL[1], lL[2]};
    lL[d] = fidx - 1;
    lR[d] = fidx;
    const int gface = o[d] + fidx;
    const bool ghostL = gface == 0 && G.bc[d] != kPeriodic;
    const bool ghostR = gface == G.N[d] && G.bc[d] != kPeriodic;
    R uL[V], uR[V];
    if (!ghostL) {
        const R* src = Ss + TL::slot(lL[0], lL[1], lL[2]) * SS;
#pragma unroll
        for (int v = 0; v < V; v++) {
            R a = 0;
#pragma unroll
            for (int l = 0; l < n; l++) {
                c[d] = l;
                a += src[v * NPT + pt_index<n>(c)] * M.sp_to_fp[(nf - 1) * n + l];
            }
            uL[v] = a;
        }
    }
    if (!ghostR) {
        const R* src = Ss + TL::slot(lR[0], lR[1], lR[2]) * SS;
#pragma unroll
        for (int v = 0; v < V; v++) {
            R a = 0;
#pragma unroll
            for (int l = 0; l < n; l++) {
                c[d] = l;
                a += src[v * NPT + pt_index<n>(c)] * M.sp_to_fp[l];
            }
            uR[v] = a;
        }
    }
    if (ghostL) {
#pragma unroll
        for (int v = 0; v < V; v++) uL[v] = uR[v];
        if (G.bc[d] == kReflective) uL[1 + d] = -uL[1 + d];
    }
    if (ghostR) {
#pragma unroll
        for (int v = 0; v < V; v++) uR[v] = uL[v];
        if (G.bc[d] == kReflective) uR[1 + d] = -uR[1 + d];
    }
    R F[V];
    riemann_llf<D>(F, uL, uR, d, (R)G.gm);
    if constexpr (VISC) {
        // viscous interface flux (src/hydro.cpp:420-455): the two sides'
        // viscous fluxes from the pre-pass, the ghost side an image of the
        // active side, combined with wind -0.5 and the sides swapped
        R gL[V], gR[V];
        if (!ghostL) {
            const long long eL = sl_elem[TL::slot(lL[0], lL[1], lL[2])];
            const R* g = vg + ((((long long)vt * G.E + eL) * 2 + 1) * V) * NTP + tp;
#pragma unroll
            for (int v = 0; v < V; v++) gL[v] = g[v * NTP];
        }
        if (!ghostR) {
            const long long eR = sl_elem[TL::slot(lR[0], lR[1], lR[2])];
            const R* g = vg + ((((long long)vt * G.E + eR) * 2 + 0) * V) * NTP + tp;
#pragma unroll
            for (int v = 0; v < V; v++) gR[v] = g[v * NTP];
        }
        if (ghostL) {
#pragma unroll
            for (int v = 0; v < V; v++) gL[v] = gR[v];
            if (G.bc[d] == kReflective) gL[1 + d] = -gL[1 + d];
        }
        if (ghostR) {
#pragma unroll
            for (int v = 0; v < V; v++) gR[v] = gL[v];
            if (G.bc[d] == kReflective) gR[1 + d] = -gR[1 + d];
        }
#pragma unroll
        for (int v = 0; v < V; v++) F[v] += wind_mix(gR[v], gL[v], R(-0.5));
    }
    if (fidx >= 1) {
        c[d] = nf - 1;
        const int fi = fp_index<n, nf>(d, c);
        R* dst = FX + (d * NE + TL::slot(lL[0], lL[1], lL[2])) * V * FXS;
#pragma unroll
        for (int v = 0; v < V; v++) dst[v * FXS + fi] = F[v];
    }
    if (fidx < Td) {
        c[d] = 0;
        const int fi = fp_index<n, nf>(d, c);
        R* dst = FX + (d * NE + TL::slot(lR[0], lR[1], lR[2])) * V * FXS;
#pragma unroll
        for (int v = 0; v < V; v++) dst[v * FXS + fi] = F[v];
    }
}

// resident blocks per SM the register allocation is sized for: 2 (128
// registers a thread); for the FP32 form in 2D, whose per-point slices take
// half the registers of FP64, 4 (64) at p <= 2, 5 (48) at p = 3 and 3 (80)
// above, where
// the extra resident warps outweigh a few spilled registers (measured on
// B200: 159 us against 178 us per predictor pass at 256^2 going from 2 to
// 4 blocks; from 4 to 5 blocks, 16 / 8 bytes of spills in the predictor /
// corrector, 0.798 against 0.812 ms per FP32 blast step at 256^2; p = 2 at
// 4 blocks and p = 5 at 3, without spills: blast steps 0.328 -> 0.285 ms
// at 192^2 p=2, 1.635 -> 1.340 ms at 128^2 p=5, the first 16 problems of
// the batched ensemble 43.6 -> 37.6 ms). The
// flux pass keeps no per-slice registers (FP32 5 blocks: 159 against 167
// us; FP64 3 blocks: 338 against 376 us). The FP64 2D predictor and
// corrector at p = 3 take 3 blocks too (80 registers, 184 / 88 bytes of
// spills): 1.704 against 1.717 ms per plain FP64 step at 256^2. The FP32
// 3D passes at p <= 3 (2x1x1 tiles, 23-52 KB of shared memory) take 3
// blocks (80 registers, at most 52 bytes of spills): steps 7.30 -> 6.42 ms
// (40^3 p=2 blast), 3.58 -> 3.43 ms (24^3 p=3 KH), 4.63 -> 4.60 ms (32^3
// p=3 blast).
// In 3D at p = 5 the FP64 passes' 161 KB of shared memory admit one block
// per SM anyway, so they take the whole register file instead of spilling
// at 128 registers.
// The FP64 3D passes on 2x2x1-element tiles (p = 2, 3) are compiled for one
// block per SM as well: at p = 3 their 154 KB of shared memory admit only
// one; at p = 2, compiled for two blocks (128 registers, 300-450 bytes of
// spills per thread) they gave results that differ from the oracle in every
// value after one ADER step, while the same source compiled without spills
// (one block, 188-211 registers) is bit-identical. Extra barriers around the
// staging and disabling the first-pass shortcut did not change the spilled
// build's results; the tile index arithmetic was checked against the
// oracle at p = 1 and p = 3 on the same tiles.
template <typename R, int D, int P, int MODE, int NE = 1>
constexpr int kPicardBlocksPerSM = (sizeof(R) == 4 && D == 2)
                                       ? (P == 3 ? 5 : (P == 2 ? 4 : 3))
                                       : (sizeof(R) == 8 && D == 3 && (P >= 5 || (NE >= 4 && P >= 2)))
                                             ? 1
                                             : (D == 2 && P == 3 ? 3 : ((sizeof(R) == 4 && D == 3 && P <= 3) ? 3 : 2));

// flux-point buffers of a Picard pass (alternated between slices when 2)
template <typename R>
constexpr int kFxBuffers = sizeof(R) == 4 ? 2 : 1;

// ---------------------------------------------------------------------------
// Picard pass: interpolation to flux points, Euler fluxes, LLF at element
// interfaces, flux divergence and the ADER predictor / corrector update,
// fused so that only U_ader crosses HBM.
// ---------------------------------------------------------------------------
template <typename R, int D, int P, int TX, int TY, int TZ, int MODE, bool VISC = false>
__device__ __forceinline__ void picard_kernel_body(const DevGrid& G, const DevMatsT<R>& M, const PicardArgsT<R>& A, long long bidx) {
    using S = Shape<D, P>;
    using TL = Tile<D, TX, TY, TZ>;
    constexpr int n = S::n, nf = S::nf, V = S::V, NPT = S::NPT, NTP = S::NTP, NFP = S::NFP;
    constexpr int NE = TL::NE, NS = TL::NS;
    constexpr int PPT = (NE * NPT + kThreads - 1) / kThreads;
    constexpr int NT = MODE == kFlux ? 1 : (P + 1);  // register slices kept per point

    // padded strides: an element block of the staged state (SS) and a
    // variable row of the flux-point arrays (FXS) start on different banks
    constexpr int SS = PicardPad<D, P, R>::SS;
    constexpr int FXS = PicardPad<D, P, R>::FXS;
    // element-slice chunks are copied by the TMA engine when they are whole
    // 16-byte units (V*NPT even); otherwise by plain loads
    constexpr bool kBulk = (V * NPT * sizeof(R)) % 16 == 0;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    R* smem = reinterpret_cast<R*>(smem_raw);
    R* Sbuf = smem;                     // 2 x [NS][SS >= V*NPT] (R buffer)
    // [kFxBuffers][D][NE][V][FXS >= NFP]: with two buffers (FP32) every
    // pass alternates them between slices, so a slice's flux points can be
    // written while slow threads still read the previous slice's (no
    // end-of-slice barrier). FP64 keeps one buffer: its occupancy is bound
    // by shared memory, and the larger footprint cost more than the barrier
    // saved.
    constexpr int NFX = kFxBuffers<R>;
    R* FX0 = Sbuf + 2 * NS * SS;
    R* TT = FX0 + NFX * D * NE * V * FXS;  // [NE][V][NFP] face-integral scratch (3D)
    __shared__ long long sl_elem[NS];
    __shared__ uint64_t bar[2];
    // the transform matrices in shared memory: the per-point coefficient
    // lookups differ across a warp's lanes, which the constant bank (where
    // the kernel parameters live) serves one address at a time
    __shared__ R Msf[S::nf * S::n];   // sp_to_fp [nf][n]
    __shared__ R Mdf[S::n * S::nf];   // dfp_to_sp [n][nf]
    __shared__ R Mcv[S::n * S::n];    // sp_to_cv [n][n]

    const int tid = threadIdx.x;
    for (int i = tid; i < S::nf * S::n; i += kThreads) {
        Msf[i] = M.sp_to_fp[i];
        Mdf[i] = M.dfp_to_sp[i];
    }
    for (int i = tid; i < S::n * S::n; i += kThreads) Mcv[i] = M.sp_to_cv[i];
    int o[3];
    {
        int b = bidx;
        const int tx = G.N[0] / TX, ty = G.N[1] / TY;
        o[0] = (b % tx) * TX;
        b /= tx;
        o[1] = (b % ty) * TY;
        b /= ty;
        o[2] = D == 3 ? b * TZ : 0;
    }
    for (int s = tid; s < NS; s += kThreads) {
        int l[3];
        TL::coords(s, l);
        sl_elem[s] = elem_of<D>(G, o, l);
    }
    if (kBulk && tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    const R dt = (R)(*A.dt);
    const int nt = G.nt;
    const long long E = G.E;

    R dreg[PPT][V][NT];   // kPredict: dudt per slice; kCorrect: du in [..][..][0]
#pragma unroll
    for (int r = 0; r < PPT; r++)
#pragma unroll
        for (int v = 0; v < V; v++)
#pragma unroll
            for (int t = 0; t < NT; t++) dreg[r][v][t] = 0;

    __syncthreads();
    // one elected thread issues the bulk copies of slice t into buffer b
    auto issue = [&](int t, int b) {
        const R* src = A.in_slices > 1 ? A.ua_in + (long long)t * E * V * NPT : A.ua_in;
        R* dst = Sbuf + b * NS * SS;
        if (kBulk) {
            if (tid == 0) {
                uint32_t bytes = 0;
                for (int s = 0; s < NS; s++)
                    if (sl_elem[s] >= 0) bytes += V * NPT * sizeof(R);
                fence_proxy_async_smem();
                mbar_expect_tx(&bar[b], bytes);
                for (int s = 0; s < NS; s++)
                    if (sl_elem[s] >= 0)
                        bulk_g2s(dst + s * SS, src + sl_elem[s] * V * NPT, V * NPT * sizeof(R), &bar[b]);
            }
        } else {
            for (int q = tid; q < NS * V * NPT; q += kThreads) {
                const int s = q / (V * NPT), off = q - s * (V * NPT);
                const long long ge = sl_elem[s];
                if (ge >= 0) dst[s * SS + off] = src[ge * V * NPT + off];
            }
        }
    };
    const bool multi = A.in_slices > 1;
    // a predictor pass whose slices all equal U (the first Picard pass:
    // copy_ader) has the same flux divergence in every slice: it is
    // evaluated once and stored for every slice
    const int nt_eval = (MODE == kPredict && !multi) ? 1 : nt;
    issue(0, 0);
    for (int t = 0; t < nt_eval; t++) {
        // ---- stage slice t (prefetch t+1 into the other buffer) ----
        const int b = multi ? (t & 1) : 0;
        R* Ss = Sbuf + b * NS * SS;
        R* FX = FX0 + (NFX == 1 ? 0 : (t & 1)) * (D * NE * V * FXS);
        if (multi && t + 1 < nt) issue(t + 1, b ^ 1);
        if (t == 0 || multi) {
            if (kBulk) mbar_wait_bounded(&bar[b], multi ? ((t >> 1) & 1) : 0, G.status);
            else if (!multi || t == 0) __syncthreads();
        }
        if (!kBulk && multi && t > 0) __syncthreads();
        // ---- phase A: flux-point fluxes of every direction ----
        // one list: interfaces (about three times the work of an interior
        // point: two extrapolations and an LLF solve) first, then interior
        // flux points; every item runs with a compile-time direction. When
        // the interfaces fit in one pass of the block, each of the first NFT
        // threads takes one interface and the remaining threads share the
        // interior points, which evens out the work before the barrier.
        {
            constexpr int NINT = NE * (nf - 2) * NTP;
            constexpr int NF0 = (TX + 1) * (NE / TX) * NTP;
            constexpr int NF1 = (TY + 1) * (NE / TY) * NTP;
            constexpr int NF2 = D == 3 ? (TZ + 1) * (NE / TZ) * NTP : 0;
            constexpr int NFT = NF0 + NF1 + NF2;
            constexpr int total = NFT + D * NINT;
            auto item = [&](int q) {
                const int vt = A.in_slices > 1 ? t : 0;
                if (q < NF0) picard_face_item<R, D, P, TX, TY, TZ, 0, VISC>(G, M, Ss, FX, o, q, A.vg[0], sl_elem, vt);
                else if (q < NF0 + NF1)
                    picard_face_item<R, D, P, TX, TY, TZ, 1, VISC>(G, M, Ss, FX, o, q - NF0, A.vg[1], sl_elem, vt);
                else if (D == 3 && q < NFT)
                    picard_face_item<R, D, P, TX, TY, TZ, (D == 3 ? 2 : 1), VISC>(G, M, Ss, FX, o, q - NF0 - NF1,
                                                                                   A.vg[D == 3 ? 2 : 1], sl_elem, vt);
                else {
                    const int r = q - NFT;
                    if (r < NINT) picard_interior_item<R, D, P, TX, TY, TZ, 0>(G, Msf, Ss, FX, r);
                    else if (r < 2 * NINT) picard_interior_item<R, D, P, TX, TY, TZ, 1>(G, Msf, Ss, FX, r - NINT);
                    else picard_interior_item<R, D, P, TX, TY, TZ, (D == 3 ? 2 : 1)>(G, Msf, Ss, FX, r - 2 * NINT);
                }
            };
            constexpr int TI = kThreads - NFT;  // threads left for the interior points
            // (measured on B200 at 2D p=3: faster for every FP32 pass and the
            // FP64 flux pass, slower for the FP64 predictor and corrector)
            constexpr bool kBalanced = sizeof(R) == 4 || MODE == kFlux;
            if constexpr (kBalanced && NFT > 0 && TI >= kThreads / 4) {
                if (tid < NFT) item(tid);
                else
                    for (int r = tid - NFT; r < D * NINT; r += TI) item(NFT + r);
            } else {
                for (int q = tid; q < total; q += kThreads) item(q);
            }
        }
        __syncthreads();
        if (MODE != kFlux) {
            // ---- phase B: flux divergence at the solution points ----
#pragma unroll
            for (int r = 0; r < PPT; r++) {
                const int q = tid + r * kThreads;
                if (q < NE * NPT) {
                    const int el = q / NPT, pt = q % NPT;
                    int c[3];
                    pt_coords<n>(pt, c);
                    int fpi[3][kMaxNfd];
#pragma unroll
                    for (int d = 0; d < D; d++) {
                        int cc[3] = {c[0], c[1], c[2]};
#pragma unroll
                        for (int ll = 0; ll < nf; ll++) {
                            cc[d] = ll;
                            fpi[d][ll] = fp_index<n, nf>(d, cc);
                        }
                    }
#pragma unroll
                    for (int v = 0; v < V; v++) {
                        R dudt = 0;
                        if (G.uniform_pow2) {
                            // every active h is the same power of two: the
                            // scaling of each term by 1/h is exact and
                            // commutes with the rounding of the sum
#pragma unroll
                            for (int ll = 0; ll < nf; ll++)
#pragma unroll
                                for (int d = 0; d < D; d++)
                                    dudt += FX[((d * NE + el) * V + v) * FXS + fpi[d][ll]] * Mdf[c[d] * nf + ll];
                            dudt *= (R)G.rh[0];
                        } else {
#pragma unroll
                            for (int ll = 0; ll < nf; ll++) {
#pragma unroll
                                for (int d = 0; d < D; d++) {
                                    const R Fv = FX[((d * NE + el) * V + v) * FXS + fpi[d][ll]];
                                    dudt += div_h(Fv * Mdf[c[d] * nf + ll], (R)G.h[d], (R)G.rh[d], G.pow2[d] != 0);
                                }
                            }
                        }
                        if (MODE == kPredict) {
#pragma unroll
                            for (int tt = 0; tt < NT; tt++)
                                if (tt == t || (!multi && tt < nt)) dreg[r][v][tt] = dudt;
                        } else {
                            if (G.grav && v != 0) {
                                const R* uv = Ss + el * SS;
                                R s;
                                if (v <= D) s = uv[pt] * (R)G.g[v - 1];
                                else {
                                    s = uv[NPT + pt] * (R)G.g[0] + uv[2 * NPT + pt] * (R)G.g[1];
                                    if (D == 3) s = s + uv[3 * NPT + pt] * (R)G.g[2];
                                }
                                dudt -= s;
                            }
                            dreg[r][v][0] += dudt * M.wt[t] * dt;
                        }
                    }
                }
            }
        } else {
            // ---- FV face fluxes of slice t (src/transforms.cpp:378-481) ----
            const R* Mc = Mcv;
#pragma unroll
            for (int d = 0; d < D; d++) {
                R* out = A.ff[d];
                const R* Fd = FX + d * NE * V * FXS;
                if (D == 2) {
                    for (int q = tid; q < NE * NFP; q += kThreads) {
                        const int el = q / NFP, fi = q % NFP;
                        // fi = (face ll along d, transverse cell cc)
                        int ll, cc;
                        if (d == 0) { ll = fi % nf; cc = fi / nf; }
                        else { cc = fi % n; ll = fi / n; }
                        R* dst = out + (((long long)t * E + sl_elem[el]) * V) * NFP + fi;
                        const R* srcb = Fd + el * V * FXS + (d == 0 ? ll : n * ll);
#pragma unroll
                        for (int v = 0; v < V; v++) {
                            R f = 0;
#pragma unroll
                            for (int m = 0; m < n; m++)
                                f += srcb[v * FXS + (d == 0 ? nf * m : m)] * Mc[cc * n + m];
                            dst[v * NFP] = f;
                        }
                    }
                } else {
                    // two transverse sweeps: dim1 = next(d), dim2 = next(dim1)
                    const int d1 = d == 0 ? 1 : (d == 1 ? 2 : 0);
                    const int d2 = d1 == 0 ? 1 : (d1 == 1 ? 2 : 0);
                    for (int q = tid; q < NE * V * NFP; q += kThreads) {
                        const int base = (q / NFP) * FXS;
                        const int fi = q % NFP;
                        int c[3];
                        // decode face index of direction d
                        if (d == 0) { c[0] = fi % nf; c[1] = (fi / nf) % n; c[2] = fi / (nf * n); }
                        else if (d == 1) { c[0] = fi % n; c[1] = (fi / n) % nf; c[2] = fi / (n * nf); }
                        else { c[0] = fi % n; c[1] = (fi / n) % n; c[2] = fi / (n * n); }
                        const int id = c[d1];
                        R u = 0;
#pragma unroll
                        for (int m = 0; m < n; m++) {
                            c[d1] = m;
                            u += Fd[base + fp_index<n, nf>(d, c)] * Mc[id * n + m];
                        }
                        TT[q] = u;
                    }
                    __syncthreads();
                    for (int q = tid; q < NE * V * NFP; q += kThreads) {
                        const int base = q - q % NFP;
                        const int fi = q % NFP;
                        const int el = q / (V * NFP), v = (q / NFP) % V;
                        int c[3];
                        if (d == 0) { c[0] = fi % nf; c[1] = (fi / nf) % n; c[2] = fi / (nf * n); }
                        else if (d == 1) { c[0] = fi % n; c[1] = (fi / n) % nf; c[2] = fi / (n * nf); }
                        else { c[0] = fi % n; c[1] = (fi / n) % n; c[2] = fi / (n * n); }
                        const int id = c[d2];
                        R f = 0;
#pragma unroll
                        for (int m = 0; m < n; m++) {
                            c[d2] = m;
                            f += TT[base + fp_index<n, nf>(d, c)] * Mc[id * n + m];
                        }
                        out[(((long long)t * E + sl_elem[el]) * V + v) * NFP + fi] = f;
                    }
                    __syncthreads();
                }
            }
        }
        // one FX buffer is reused by the next slice; the next slice's staging
        // overwrites this slice's buffer, which the corrector's gravity
        // source still reads (with two FX buffers the flux pass's face
        // integral reads only this slice's FX, which the next slice leaves)
        if (NFX == 1 || (MODE == kCorrect && G.grav)) __syncthreads();
    }
    __syncthreads();

    if (MODE == kPredict) {
        // ---- ADER predictor (src/transforms.cpp:309-323) ----
        __shared__ R Cw[NT * NT];
        if constexpr (sizeof(R) == 4) {
            for (int i = tid; i < NT * NT; i += kThreads) {
                const int tt = i / NT, ll = i % NT;
                Cw[i] = (tt < nt && ll < nt) ? M.invader[tt * nt + ll] * M.wt[ll] * dt : R(0);
            }
            __syncthreads();
        }
#pragma unroll
        for (int r = 0; r < PPT; r++) {
            const int q = tid + r * kThreads;
            if (q < NE * NPT) {
                const int el = q / NPT, pt = q % NPT;
                const long long ge = sl_elem[el];
                R nw[D + 1][NT];  // updated rho and momenta (gravity of later slots)
#pragma unroll
                for (int v = 0; v < V; v++) {
                    const R u_old = A.u[(ge * V + v) * NPT + pt];
                    R dudt[NT];
#pragma unroll
                    for (int tt = 0; tt < NT; tt++) {
                        dudt[tt] = dreg[r][v][tt];
                        if (G.grav && v != 0 && tt < nt) {
                            R s;
                            if (v <= D) s = nw[0][tt] * (R)G.g[v - 1];
                            else {
                                s = nw[1][tt] * (R)G.g[0] + nw[2][tt] * (R)G.g[1];
                                if (D == 3) s = s + nw[3][tt] * (R)G.g[2];
                            }
                            dudt[tt] -= s;
                        }
                    }
#pragma unroll
                    for (int tt = 0; tt < NT; tt++) {
                        if (tt >= nt) break;
                        R du = 0;
                        if constexpr (sizeof(R) == 4) {
                            // precision form: one product per term with the
                            // coefficients invader(t,l) w_l dt formed once
#pragma unroll
                            for (int ll = 0; ll < NT; ll++)
                                if (ll < nt) du += dudt[ll] * Cw[tt * NT + ll];
                        } else {
#pragma unroll
                            for (int ll = 0; ll < NT; ll++)
                                if (ll < nt) du += dudt[ll] * M.invader[tt * nt + ll] * M.wt[ll] * dt;
                        }
                        const R val = u_old - du;
                        if (v <= D) nw[v][tt] = val;
                        A.ua_out[(((long long)tt * E + ge) * V + v) * NPT + pt] = val;
                    }
                }
            }
        }
    } else if (MODE == kCorrect) {
        // ---- corrector / RK stage (src/transforms.cpp:327-374, 252-261) ----
        R* Wsp = Sbuf;                // reuse staging memory: [NE][V][NPT]
        R* Tmp = Sbuf + NE * V * NPT;
#pragma unroll
        for (int r = 0; r < PPT; r++) {
            const int q = tid + r * kThreads;
            if (q < NE * NPT) {
                const int el = q / NPT, pt = q % NPT;
                const long long ge = sl_elem[el];
                R un[V];
#pragma unroll
                for (int v = 0; v < V; v++) {
                    const long long gi = (ge * V + v) * NPT + pt;
                    R val = A.u[gi] - dreg[r][v][0];
                    if (A.rk_a > 0) {
                        const R ra = (R)A.rk_a;
                        val = ra * A.u0[gi] + ((R)1.0 - ra) * val;
                    }
                    un[v] = val;
                    A.u_out[gi] = val;
                }
                if (A.final_stage) {
                    R w[V];
                    primitives<D>(un, w, (R)G.gm);
#pragma unroll
                    for (int v = 0; v < V; v++) Wsp[(el * V + v) * NPT + pt] = w[v];
                }
            }
        }
        if (A.final_stage) {
            __syncthreads();
            // W_cv = sp_to_cv(W_sp): x, y(, z) sweeps (src/transforms.cpp:99-117)
            R* bufs[2] = {Tmp, Wsp};
            const R* src = Wsp;
            for (int d = 0; d < D; d++) {
                R* dst = bufs[d % 2];
                sweep_smem<D, P, R>(src, dst, Mcv, d, NE * V * NPT);
                __syncthreads();
                src = dst;
            }
            double dtl = 1.7976931348623157e308;
#pragma unroll
            for (int r = 0; r < PPT; r++) {
                const int q = tid + r * kThreads;
                if (q < NE * NPT) {
                    const int el = q / NPT, pt = q % NPT;
                    const long long ge = sl_elem[el];
                    R w[V];
#pragma unroll
                    for (int v = 0; v < V; v++) w[v] = src[(el * V + v) * NPT + pt];
                    if (A.wcv)
#pragma unroll
                        for (int v = 0; v < V; v++) A.wcv[(ge * V + v) * NPT + pt] = w[v];
                    dtl = smin(dtl, point_dt<D>(G, w, n));
                }
            }
            block_min_dt(dtl, A.dtmin);
        }
    } else {
        // ---- U_cv = sp_to_cv(U) and the slice-0 FV candidate ----
        R* Ut = Sbuf;
        R* Tmp = Sbuf + NE * V * NPT;
        for (int q = tid; q < NE * V * NPT; q += kThreads) {
            const int el = q / (V * NPT), off = q % (V * NPT);
            Ut[q] = A.u[sl_elem[el] * V * NPT + off];
        }
        __syncthreads();
        R* bufs[2] = {Tmp, Ut};
        const R* src = Ut;
        for (int d = 0; d < D; d++) {
            R* dst = bufs[d % 2];
            sweep_smem<D, P, R>(src, dst, Mcv, d, NE * V * NPT);
            __syncthreads();
            src = dst;
        }
        for (int q = tid; q < NE * V * NPT; q += kThreads) {
            const int el = q / (V * NPT), off = q % (V * NPT);
            A.ucv[sl_elem[el] * V * NPT + off] = src[q];
        }
        for (int q = tid; q < NE * NPT; q += kThreads) {
            const int el = q / NPT, pt = q % NPT;
            const long long ge = sl_elem[el];
            R uo[V], un[V];
#pragma unroll
            for (int v = 0; v < V; v++) uo[v] = src[(el * V + v) * NPT + pt];
            fv_candidate<D, P, R>(G, A.ff, 0, ge, pt, uo, M.wt[0] * dt, un);
            A.rp_old[ge * NPT + pt] = rho_p_fp64<D>(uo, G.gm);
            A.rp_new[ge * NPT + pt] = rho_p_fp64<D>(un, G.gm);
        }
    }
}

}  // namespace spdk

#include "spdk_picard2d.cuh"

namespace spdk {

// VISC: instantiation that adds the viscous interface fluxes (hydro/nu > 0);
// the inviscid kernels carry none of that code. 2D runs take the
// line-organised pass of spdk_picard2d.cuh.
template <typename R, int D, int P, int TX, int TY, int TZ, int MODE, bool VISC = false>
__global__ void __launch_bounds__(kThreads, kPicardBlocksPerSM<R, D, P, MODE, TX * TY * TZ>) picard_kernel(DevGrid G, DevMatsT<R> M, PicardArgsT<R> A) {
    pdl_wait();
    if (gate_closed(G)) return;
    if constexpr (D == 2) picard2d_body<R, P, TX, TY, MODE, VISC>(G, M, A, blockIdx.x);
    else picard_kernel_body<R, D, P, TX, TY, TZ, MODE, VISC>(G, M, A, blockIdx.x);
}

template <typename R, int D, int P, int TX, int TY, int TZ>
constexpr size_t picard_smem_bytes() {
    if constexpr (D == 2) {
        return Smem2<R, P, TX, TY>::bytes;
    } else {
        using S = Shape<D, P>;
        using TL = Tile<D, TX, TY, TZ>;
        size_t a = 2 * (size_t)TL::NS * PicardPad<D, P, R>::SS;
        size_t b = (size_t)kFxBuffers<R> * D * TL::NE * S::V * PicardPad<D, P, R>::FXS;
        size_t c = (size_t)TL::NE * S::V * S::NFP;
        size_t need_epi = 2 * (size_t)TL::NE * S::V * S::NPT;  // W_sp + sweep scratch reuse
        size_t total = a + b + c;
        if (need_epi > total) total = need_epi;
        return total * sizeof(R);
    }
}

}  // namespace spdk
