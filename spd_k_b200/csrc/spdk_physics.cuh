// Pointwise Euler physics shared by the spd_K B200 kernels.
//
// Every routine evaluates the same floating-point operations in the same
// order as the reference routine cited beside it. For R = double (the plain
// form) the build compiles with -fmad=false, so no product is fused into a
// sum and FP64 results are bit-identical to the reference's x86-64 CPU build;
// R = float is the precision form (FMA allowed, FP64 islands where noted). Conserved slots are
// rho, m_1..m_D, E (V = D+2): in 2D the reference also carries m_z = 0,
// whose terms only ever add or multiply signed zeros, so they are dropped.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

namespace spdk {

// std::max / std::min semantics (first operand kept on ties and NaN)
template <typename R> __device__ __forceinline__ R smax(R a, R b) { return (a < b) ? b : a; }
template <typename R> __device__ __forceinline__ R smin(R a, R b) { return (b < a) ? b : a; }

constexpr double kMinC2 = 1E-14;    // src/define.hpp:15
constexpr double kRhoMin = 1E-10;   // src/define.hpp:16-19
constexpr double kRhoMax = 1E10;
constexpr double kPMin = 1E-10;
constexpr double kPMax = 1E10;

// src/hydro.cpp:27-32
template <typename R> __device__ __forceinline__ R sound_speed(R rho, R p, R gm) {
    R c2 = gm * p / rho;
    c2 = smax(c2, R(kMinC2));
    return sqrt(c2);
}

// 1/x in FP64 for an FP32 x: an FP32 seed refined by two Newton-Raphson
// steps r <- r + r(1 - x r) (each squares the relative error: 1e-7 -> 1e-14
// -> below FP64 rounding), without a double-precision division
__device__ __forceinline__ double rcp_fp64(float x) {
    const double xd = x;
    double r = (double)(1.0f / x);
    r = r + r * (1.0 - xd * r);
    r = r + r * (1.0 - xd * r);
    return r;
}

// src/hydro.cpp:95-106: w = (rho, v_1..v_D, p). In the FP32 precision form
// the pressure is recovered in FP64: E - |m|^2/(2 rho) cancels badly where
// the kinetic energy nearly equals the total energy, so |m|^2 is formed from
// exact FP64 products of the FP32 momenta and divided by rho in FP64.
template <int D, typename R> __device__ __forceinline__ void primitives(const R* u, R* w, R gm) {
    if constexpr (sizeof(R) == 4) {
        const float rf = 1.0f / u[0];
        double m2 = 0;
        w[0] = u[0];
#pragma unroll
        for (int d = 1; d <= D; d++) {
            w[d] = u[d] * rf;
            m2 += (double)u[d] * (double)u[d];
        }
        w[D + 1] = (R)(((double)u[D + 1] - 0.5 * m2 * rcp_fp64(u[0])) * ((double)gm - 1.0));
    } else {
        R ek = 0;
        w[0] = u[0];
#pragma unroll
        for (int d = 1; d <= D; d++) {
            w[d] = u[d] / u[0];
            ek += w[d] * u[d];
        }
        w[D + 1] = (u[D + 1] - R(0.5) * ek) * (gm - R(1.));
    }
}

// src/hydro.cpp:34-45
template <int D, typename R> __device__ __forceinline__ void conservatives(const R* w, R* u, R gm) {
    R ek = 0;
    u[0] = w[0];
#pragma unroll
    for (int d = 1; d <= D; d++) {
        u[d] = w[0] * w[d];
        ek += w[d] * u[d];
    }
    u[D + 1] = w[D + 1] / (gm - R(1.)) + R(0.5) * ek;
}

// src/hydro.cpp:155-161, normal direction n (0-based): flux of every slot
template <int D, typename R> __device__ __forceinline__ void euler_flux(const R* u, const R* w, R* f, int n) {
    const R vn = w[1 + n];
    f[0] = u[0] * vn;
#pragma unroll
    for (int d = 1; d <= D; d++) f[d] = (d == 1 + n) ? (u[d] * vn + w[D + 1]) : (u[d] * vn);
    f[D + 1] = (u[D + 1] + w[D + 1]) * vn;
}

// src/hydro.cpp:270-289: local Lax-Friedrichs flux
template <int D, typename R>
__device__ __forceinline__ void riemann_llf(R* F, const R* uL, const R* uR, int n, R gm) {
    constexpr int V = D + 2;
    R wL[V], wR[V], fL[V], fR[V];
    primitives<D>(uL, wL, gm);
    primitives<D>(uR, wR, gm);
    euler_flux<D>(uL, wL, fL, n);
    euler_flux<D>(uR, wR, fR, n);
    R cL = sound_speed(wL[0], wL[D + 1], gm) + fabs(wL[1 + n]);
    R cR = sound_speed(wR[0], wR[D + 1], gm) + fabs(wR[1 + n]);
    R cmax = smax(cL, cR);
#pragma unroll
    for (int v = 0; v < V; v++) F[v] = R(0.5) * (fR[v] + fL[v]) - R(0.5) * cmax * (uR[v] - uL[v]);
}

// src/hydro.cpp:291-363: HLLC with HLL wave speeds and acoustic star state
template <int D, typename R>
__device__ __forceinline__ void riemann_hllc(R* F, const R* UL, const R* UR, int n, R gm) {
    constexpr int V = D + 2;
    const int v1 = 1 + n;
    R WL[V], WR[V];
    primitives<D>(UL, WL, gm);
    primitives<D>(UR, WR, gm);
    R cL = sound_speed(WL[0], WL[D + 1], gm) + fabs(WL[v1]);
    R cR = sound_speed(WR[0], WR[D + 1], gm) + fabs(WR[v1]);
    R cmax = smax(cL, cR);
    R vL = WL[v1], vR = WR[v1];
    R sL = smin(vL, vR) - cmax;
    R sR = smax(vL, vR) + cmax;
    R rcL = WL[0] * (vL - sL);
    R rcR = WR[0] * (sR - vR);
    R vs = (rcR * vR + rcL * vL + (WL[D + 1] - WR[D + 1])) / (rcR + rcL);
    R ps = (rcR * WL[D + 1] + rcL * WR[D + 1] + rcL * rcR * (vL - vR)) / (rcR + rcL);
    R rsL = WL[0] * (sL - vL) / (sL - vs);
    R esL = ((sL - vL) * UL[D + 1] - WL[D + 1] * vL + ps * vs) / (sL - vs);
    R rsR = WR[0] * (sR - vR) / (sR - vs);
    R esR = ((sR - vR) * UR[D + 1] - WR[D + 1] * vR + ps * vs) / (sR - vs);
    R r, v, pg, e;
    if (sL > 0) { r = WL[0]; v = WL[v1]; pg = WL[D + 1]; e = UL[D + 1]; }
    else if (vs > 0) { r = rsL; v = vs; pg = ps; e = esL; }
    else if (sR > 0) { r = rsR; v = vs; pg = ps; e = esR; }
    else { r = WR[0]; v = WR[v1]; pg = WR[D + 1]; e = UR[D + 1]; }
    F[0] = r * v;
#pragma unroll
    for (int d = 1; d <= D; d++) {
        if (d == v1) F[d] = r * v * v + pg;
        else F[d] = r * v * (vs > 0 ? WL[d] : WR[d]);
    }
    F[D + 1] = v * (e + pg);
}

// src/muscl.hpp:2-12
template <typename R> __device__ __forceinline__ R minmod(R SL, R SR, R xL, R xR) {
    R ratio = SR / SL;
    ratio = smax(R(0.0), smin(ratio, R(1.0)));
    R slope = ratio * SL;
    return R(0.5) * slope * (xR - xL);
}

// src/hydro.cpp:591-615: Hancock time derivative of the primitives from the
// limited slopes dW[d][*] of every active direction (terms of inactive
// directions vanish and are not formed)
template <int D, typename R>
__device__ __forceinline__ void hancock(const R* W, R* dWt, const R (*dW)[D + 2], R gm) {
    constexpr int P = D + 1;
    dWt[0] = 0;
    dWt[P] = 0;
#pragma unroll
    for (int a = 0; a < D; a++) {
        const int va = 1 + a;
        dWt[0] -= W[va] * dW[a][0] + W[0] * dW[a][va];
        dWt[va] = -W[va] * dW[a][va] - dW[a][P] / W[0];
        dWt[P] -= W[va] * dW[a][P] + dW[a][va] * gm * W[P];
#pragma unroll
        for (int b = 0; b < D; b++)
            if (b != a) dWt[va] -= W[1 + b] * dW[b][va];
    }
}

// src/trouble_detection.cpp:12-31 (smooth-extrema indicator)
// (the reference divides both one-sided limits and then selects one; only
// the selected quotient is formed here, which gives the same value)
__device__ __forceinline__ double sed_alpha(double dv, double dUm, double dU, double dUp) {
    const double vL = dU - dUm;
    double aL = smin(1.0, (dv < 0.0 ? smin(vL, 0.0) : smax(vL, 0.0)) / dv);
    aL = (dv == 0.0 ? 1.0 : aL);
    const double vR = dUp - dU;
    double aR = smin(1.0, (dv < 0.0 ? smin(vR, 0.0) : smax(vR, 0.0)) / dv);
    aR = (dv == 0.0 ? 1.0 : aR);
    return smin(aL, aR);
}

// Boundary kinds (src/define.hpp:57)
enum BcKind : int { kPeriodic = 0, kGradfree = 1, kReflective = 2 };

// Ghost-cell image of an FV sub-grid coordinate a in [-2, n+1] of one
// direction (src/boundary.cpp:142-189 with nGH = 2): the active cell whose
// value the ghost holds; *flip is set for a reflective image (normal
// momentum / velocity negated).
__device__ __forceinline__ int fv_image(int a, int n, int bc, bool* flip) {
    if (a >= 0 && a < n) return a;
    if (bc == kPeriodic) return a < 0 ? a + n : a - n;
    if (bc == kGradfree) return a < 0 ? a + 2 : a - 2;
    *flip = !*flip;
    return a < 0 ? -1 - a : 2 * n - 1 - a;
}

// x / h with an exact reciprocal multiply when h is a power of two (same
// correctly rounded result as the division)
template <typename R> __device__ __forceinline__ R div_h(R x, R h, R rh, bool pow2) {
    return pow2 ? x * rh : x / h;
}

// ---------------------------------------------------------------------------
// Viscous terms (hydro/nu > 0)
// ---------------------------------------------------------------------------
// src/hydro.cpp:265-268: upwind-weighted mean of two interface values; the
// interface state of the diffusive terms takes wind = +0.5, the interface
// viscous flux wind = -0.5 with the two sides swapped
template <typename R> __device__ __forceinline__ R wind_mix(R uL, R uR, R wind) {
    return R(0.5) * (uR + uL) + wind * (uR - uL);
}

// src/hydro.cpp:492-519: viscous flux along momentum component a1 (0-based
// x, y, z; a2, a3 the cyclic others) from the momentum gradients along a1
// (du1), a2 (du2), a3 (du3) and the velocity w, all indexed by component
// (a component of an inactive direction is zero). fm: momentum fluxes, fe:
// energy flux; the density flux is zero. Operation order of the reference.
template <typename R>
__device__ __forceinline__ void viscous_flux(const R* du1, const R* du2, const R* du3, const R* w, int a1, int a2,
                                             int a3, R nu, R beta, R* fm, R& fe) {
    fe = 0;
    fm[a1] = R(2) * nu * du1[a1] + beta * du1[a1];
    fm[a1] += beta * du2[a2];
    fm[a2] = nu * (du1[a2] + du2[a1]);
    fe += w[a2] * fm[a2];
    fm[a1] += beta * du3[a3];
    fm[a3] = nu * (du1[a3] + du3[a1]);
    fe += w[a3] * fm[a3];
    fe += w[a1] * fm[a1];
}

// ---------------------------------------------------------------------------
// Feature values of the learned indicator, shared by the feature kernels and
// the solver's update epilogue. Every FP64 operation is an explicitly
// rounded intrinsic, so the values do not depend on the translation unit's
// contraction flags (the FP32 form's units allow FMA).
// ---------------------------------------------------------------------------
// density and pressure of the state u[0], u[stride], ..., u[(V-1) stride]
template <typename R>
__device__ __forceinline__ void feature_rho_p(const R* u, int stride, int V, double gm, double* rho, double* p) {
    const double r = (double)u[0];
    double m2 = 0;
    for (int d = 1; d < V - 1; d++) {
        const double m = (double)u[d * stride];
        m2 = __dadd_rn(m2, __dmul_rn(m, m));
    }
    *rho = r;
    *p = __dmul_rn(__dsub_rn((double)u[(V - 1) * stride], __ddiv_rn(__dmul_rn(0.5, m2), r)), gm - 1.0);
}

// BF16 bit pattern of x, rounded to nearest even
__device__ __forceinline__ uint16_t bf16_bits(float x) {
    const __nv_bfloat16 b = __float2bfloat16_rn(x);
    return *reinterpret_cast<const uint16_t*>(&b);
}

// a / b - 1 (0 where b is not a positive finite number or the result is
// not finite)
__device__ __forceinline__ float feature_ratio(double a, double b) {
    const double r = (b > 0 && isfinite(b)) ? __dsub_rn(__ddiv_rn(a, b), 1.0) : 0.0;
    return isfinite(r) ? (float)r : 0.0f;
}

}  // namespace spdk
