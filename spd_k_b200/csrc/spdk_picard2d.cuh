// Fused Picard pass of 2D runs: balanced interface / interior flux points
// and a register-blocked flux divergence.
//
// Same inputs, outputs and arithmetic as picard_kernel_body (spdk_kernels.cuh),
// reorganised so that operands are read once:
//
// * Phase A (fluxes at the flux points of one slice). Interfaces (both
//   sides extrapolated, ghost image at a non-periodic edge, LLF) take one
//   thread each; interior flux points are shared by the remaining threads,
//   ordered by (direction, flux point) so that a warp's points read the same
//   interpolation coefficients (one broadcast shared-memory word); x lines
//   are loaded as 16-byte vectors.
// * Phase B (divergence at the solution points). A thread owns a BX x BY block
//   of solution points of one variable of one element, for the whole pass:
//   every x-flux value it reads serves BX points, every y-flux value BY
//   points; items are ordered block-major, so a warp's derivative
//   coefficients are broadcast words too. Each point's sum keeps the
//   reference's order (flux points outer, directions inner:
//   src/transforms.cpp:296-303), so the FP64 plain form is unchanged bit for
//   bit.
// * Epilogues. The step-start state of the tile is staged point-major by
//   coalesced loads while slice 0 arrives; results are assembled in shared
//   memory and written back with coalesced 16-byte stores.
#pragma once
#include <type_traits>

namespace spdk {

// point block of the 2D divergence: BX x BY points of one variable per thread
template <int n>
struct DivBlock2 {
    static constexpr int BX = n == 2 ? 2 : n == 3 ? 3 : n == 4 ? 2 : n == 5 ? 5 : n == 6 ? 3 : n == 7 ? 1 : 2;
    static constexpr int BY = (n == 4 || n == 8) ? 2 : 1;
    static constexpr int NBX = n / BX, NBY = n / BY;
    static constexpr int NB = NBX * NBY;
};

// interfaces of a TX x TY tile per direction: (faces along d) x (rows or columns) x n
template <int P, int TX, int TY>
struct Lines2 {
    static constexpr int n = P + 1;
    static constexpr int L0 = (TX + 1) * TY * n;
    static constexpr int L1 = (TY + 1) * TX * n;
};

// shared-memory layout of the 2D pass (in elements of R): staging buffers,
// flux-point buffers; the epilogues' buffers reuse that space. Values that
// phase-B threads read or write (their lanes run over element x variable at
// a common point) sit point-major, [point][element x variable + pad], so
// that those lanes hit distinct banks, and so do the copy-out lanes running
// over points. The step-start state of the tile follows at the end.
template <typename R, int P, int TX, int TY>
struct Smem2 {
    static constexpr int n = P + 1, NPT = n * n, V = 4, NE = TX * TY;
    static constexpr int NS = Tile<2, TX, TY, 1>::NS;
    static constexpr int nt = P + 1;
    static constexpr int KS = NE * V + (sizeof(R) == 4 ? 2 : 1);  // point stride of a point-major tile
    static constexpr size_t tsz = (size_t)NPT * KS;                // one point-major tile
    static constexpr size_t stage = 2 * (size_t)NS * PicardPad<2, P, R>::SS;
    static constexpr size_t fx = (size_t)kFxBuffers<R> * 2 * NE * V * PicardPad<2, P, R>::FXS;
    static constexpr size_t out = (size_t)nt * tsz;                           // predictor slices
    static constexpr size_t epi = 2 * (size_t)NE * V * NPT + tsz;             // corrector W_sp, scratch, U - du
    static constexpr size_t main0 = stage + fx > out ? stage + fx : out;
    static constexpr size_t main1 = main0 > epi ? main0 : epi;
    static constexpr size_t ubuf = main1;                                     // point-major U of the tile
    static constexpr size_t total = ubuf + tsz;
    static constexpr size_t bytes = total * sizeof(R);
};

// the n values of one line of one variable's point block into registers:
// x lines are contiguous (16-byte vectors when they are whole vectors), y
// lines strided by n
template <typename R, int n, int d>
__device__ __forceinline__ void load_line(const R* src, int tp, R (&u)[n]) {
    constexpr int VW = 16 / (int)sizeof(R);
    if constexpr (d == 0 && n % VW == 0) {
        using VT = typename std::conditional<sizeof(R) == 4, float4, double2>::type;
        const VT* p = reinterpret_cast<const VT*>(src + n * tp);
#pragma unroll
        for (int c = 0; c < n / VW; c++) {
            __align__(16) R t[VW];
            *reinterpret_cast<VT*>(t) = p[c];
#pragma unroll
            for (int w = 0; w < VW; w++) u[c * VW + w] = t[w];
        }
    } else {
#pragma unroll
        for (int l = 0; l < n; l++) u[l] = src[d == 0 ? l + n * tp : tp + n * l];
    }
}

// one element interface of direction d (phase A): the face between the
// elements at positions f-1 and f of row/column r, at transverse point tp;
// both sides extrapolated to the face, the ghost image at a non-periodic
// domain edge (src/boundary.cpp:48-113), the LLF flux written to the
// adjacent flux points of the tile's elements
template <typename R, int P, int TX, int TY, int d, bool VISC>
__device__ __forceinline__ void face_item2(const DevGrid& G, const DevMatsT<R>& M, const R* Ss, R* FX, const int o[3],
                                           int q, const R* vg, const long long* sl_elem, int vt) {
    using TL = Tile<2, TX, TY, 1>;
    constexpr int n = P + 1, nf = P + 2, V = 4, NPT = n * n, NE = TL::NE;
    constexpr int SS = PicardPad<2, P, R>::SS, FXS = PicardPad<2, P, R>::FXS;
    constexpr int Td = d == 0 ? TX : TY, Tt = d == 0 ? TY : TX;
    constexpr int NTP = n;
    const int tp = q % n;
    const int r = (q / n) % Tt;
    const int f = q / (n * Tt);
    int lL[2], lR[2];
    lL[d] = f - 1;
    lR[d] = f;
    lL[1 - d] = r;
    lR[1 - d] = r;
    const int sL = TL::slot(lL[0], lL[1], 0), sR = TL::slot(lR[0], lR[1], 0);
    const int gface = o[d] + f;
    const bool ghostL = gface == 0 && G.bc[d] != kPeriodic;
    const bool ghostR = gface == G.N[d] && G.bc[d] != kPeriodic;
    // offset of flux point ll of the line inside a variable's flux-point block
    auto fpo = [&](int ll) { return d == 0 ? ll + nf * tp : tp + n * ll; };
    R uL[V], uR[V];
    if (!ghostR) {
        const R* src = Ss + sR * SS;
#pragma unroll
        for (int v = 0; v < V; v++) {
            R ul[n];
            load_line<R, n, d>(src + v * NPT, tp, ul);
            R a = 0;
#pragma unroll
            for (int l = 0; l < n; l++) a += ul[l] * M.sp_to_fp[l];
            uR[v] = a;
        }
    }
    if (!ghostL) {
        const R* src = Ss + sL * SS;
#pragma unroll
        for (int v = 0; v < V; v++) {
            R ul[n];
            load_line<R, n, d>(src + v * NPT, tp, ul);
            R a = 0;
#pragma unroll
            for (int l = 0; l < n; l++) a += ul[l] * M.sp_to_fp[(nf - 1) * n + l];
            uL[v] = a;
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
    riemann_llf<2>(F, uL, uR, d, (R)G.gm);
    if constexpr (VISC) {
        // viscous interface flux (src/hydro.cpp:420-455), as in picard_face_item
        R gL[V], gR[V];
        if (!ghostL) {
            const R* g = vg + ((((long long)vt * G.E + sl_elem[sL]) * 2 + 1) * V) * NTP + tp;
#pragma unroll
            for (int v = 0; v < V; v++) gL[v] = g[v * NTP];
        }
        if (!ghostR) {
            const R* g = vg + ((((long long)vt * G.E + sl_elem[sR]) * 2 + 0) * V) * NTP + tp;
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
    if (f >= 1) {
        R* dst = FX + (d * NE + sL) * V * FXS + fpo(nf - 1);
#pragma unroll
        for (int v = 0; v < V; v++) dst[v * FXS] = F[v];
    }
    if (f < Td) {
        R* dst = FX + (d * NE + sR) * V * FXS + fpo(0);
#pragma unroll
        for (int v = 0; v < V; v++) dst[v * FXS] = F[v];
    }
}

// interior flux point ll (1..nf-2) of direction d at transverse point tp of
// tile element el (phase A): interpolation, primitives, Euler flux. The
// coefficients come from the shared copy of sp_to_fp; a warp's items share
// ll, so every lane reads the same word.
template <typename R, int P, int TX, int TY, int d>
__device__ __forceinline__ void interior_item2(const DevGrid& G, const R* Msf, const R* Ss, R* FX, int el, int ll,
                                               int tp) {
    constexpr int n = P + 1, nf = P + 2, V = 4, NPT = n * n, NE = TX * TY;
    constexpr int SS = PicardPad<2, P, R>::SS, FXS = PicardPad<2, P, R>::FXS;
    const R* src = Ss + el * SS;
    R m[n];
#pragma unroll
    for (int l = 0; l < n; l++) m[l] = Msf[ll * n + l];
    R u[V], w[V], fl[V];
#pragma unroll
    for (int v = 0; v < V; v++) {
        R ul[n];
        load_line<R, n, d>(src + v * NPT, tp, ul);
        R a = 0;
#pragma unroll
        for (int l = 0; l < n; l++) a += ul[l] * m[l];
        u[v] = a;
    }
    primitives<2>(u, w, (R)G.gm);
    euler_flux<2>(u, w, fl, d);
    R* dst = FX + (d * NE + el) * V * FXS + (d == 0 ? ll + nf * tp : tp + n * ll);
#pragma unroll
    for (int v = 0; v < V; v++) dst[v * FXS] = fl[v];
}

// divergence of one BX x BY point block of one variable (phase B): dd[j][i]
// at point (bx0 + i, by0 + j). The sum over the flux points ll takes the
// x term, then the y term, at each ll (the reference's order). The
// derivative coefficients come from the shared copy of dfp_to_sp; a warp's
// items share their block, so every lane reads the same word.
template <typename R, int P>
__device__ __forceinline__ void div_block2(const DevGrid& G, const R* Mdf, const R* Fx, const R* Fy, int bx0, int by0,
                                           R (&dd)[DivBlock2<P + 1>::BY][DivBlock2<P + 1>::BX]) {
    using DB = DivBlock2<P + 1>;
    constexpr int n = P + 1, nf = P + 2, BX = DB::BX, BY = DB::BY;
#pragma unroll
    for (int j = 0; j < BY; j++)
#pragma unroll
        for (int i = 0; i < BX; i++) dd[j][i] = 0;
    const bool uni = G.uniform_pow2 != 0;
    const bool p2x = G.pow2[0] != 0, p2y = G.pow2[1] != 0;
    const R hx = (R)G.h[0], hy = (R)G.h[1], rhx = (R)G.rh[0], rhy = (R)G.rh[1];
#pragma unroll
    for (int ll = 0; ll < nf; ll++) {
        R fx[BY], fy[BX], cx[BX], cy[BY];
#pragma unroll
        for (int j = 0; j < BY; j++) {
            fx[j] = Fx[ll + nf * (by0 + j)];
            cy[j] = Mdf[(by0 + j) * nf + ll];
        }
#pragma unroll
        for (int i = 0; i < BX; i++) {
            fy[i] = Fy[(bx0 + i) + n * ll];
            cx[i] = Mdf[(bx0 + i) * nf + ll];
        }
        if (uni) {
            // every active h is the same power of two: the scaling of each
            // term by 1/h is exact and commutes with the rounding of the sum
#pragma unroll
            for (int j = 0; j < BY; j++)
#pragma unroll
                for (int i = 0; i < BX; i++) {
                    dd[j][i] += fx[j] * cx[i];
                    dd[j][i] += fy[i] * cy[j];
                }
        } else {
#pragma unroll
            for (int j = 0; j < BY; j++)
#pragma unroll
                for (int i = 0; i < BX; i++) {
                    dd[j][i] += div_h(fx[j] * cx[i], hx, rhx, p2x);
                    dd[j][i] += div_h(fy[i] * cy[j], hy, rhy, p2y);
                }
        }
    }
    if (uni)
#pragma unroll
        for (int j = 0; j < BY; j++)
#pragma unroll
            for (int i = 0; i < BX; i++) dd[j][i] *= rhx;
}

// 16-byte vector of R
template <typename R> struct Vec16;
template <> struct Vec16<float> { using T = float4; };
template <> struct Vec16<double> { using T = double2; };

// W consecutive values (W = 1 or a 16-byte vector) between memory and registers
template <typename R, int W>
__device__ __forceinline__ void vload(const R* p, R* out) {
    if constexpr (W == 1) {
        out[0] = p[0];
    } else {
        using VT = typename Vec16<R>::T;
        static_assert(W * sizeof(R) == 16, "W is one 16-byte vector");
        __align__(16) R t[W];
        *reinterpret_cast<VT*>(t) = *reinterpret_cast<const VT*>(p);
#pragma unroll
        for (int w = 0; w < W; w++) out[w] = t[w];
    }
}
template <typename R, int W>
__device__ __forceinline__ void vstore(R* p, const R* in) {
    if constexpr (W == 1) {
        p[0] = in[0];
    } else {
        using VT = typename Vec16<R>::T;
        __align__(16) R t[W];
#pragma unroll
        for (int w = 0; w < W; w++) t[w] = in[w];
        *reinterpret_cast<VT*>(p) = *reinterpret_cast<const VT*>(t);
    }
}

template <typename R, int P, int TX, int TY, int MODE, bool VISC>
__device__ __forceinline__ void picard2d_body(const DevGrid& G, const DevMatsT<R>& M, const PicardArgsT<R>& A,
                                              long long bidx) {
    constexpr int D = 2;
    using S = Shape<2, P>;
    using TL = Tile<2, TX, TY, 1>;
    using DB = DivBlock2<P + 1>;
    using LN = Lines2<P, TX, TY>;
    using SM = Smem2<R, P, TX, TY>;
    using VT = typename Vec16<R>::T;
    constexpr int n = S::n, nf = S::nf, V = S::V, NPT = S::NPT, NFP = S::NFP;
    constexpr int NE = TL::NE, NS = TL::NS;
    constexpr int NT = MODE == kFlux ? 1 : (P + 1);
    constexpr int SS = PicardPad<2, P, R>::SS;
    constexpr int FXS = PicardPad<2, P, R>::FXS;
    constexpr int NFX = kFxBuffers<R>;
    constexpr int BX = DB::BX, BY = DB::BY, BXY = BX * BY;
    constexpr int ITEMS = NE * V * DB::NB;                 // phase-B items
    constexpr int IPT = (ITEMS + kThreads - 1) / kThreads;  // items per thread
    constexpr int VW = 16 / (int)sizeof(R);                  // values per 16-byte vector
    constexpr int CH = V * NPT / VW;                         // vectors per element chunk
    constexpr int PW = NPT % VW == 0 ? VW : 1;               // values per transfer of a variable's points
    static_assert((V * NPT * sizeof(R)) % 16 == 0, "2D element chunks are whole 16-byte units");
    static_assert(SM::out <= SM::ubuf && SM::epi <= SM::ubuf, "epilogue buffers overlap the step-start state");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    R* smem = reinterpret_cast<R*>(smem_raw);
    R* Sbuf = smem;                       // 2 x [NS][SS]
    R* FX0 = Sbuf + 2 * NS * SS;          // [NFX][2][NE][V][FXS]
    R* Ubuf = smem + SM::ubuf;            // [NPT][KS]: U of the tile's elements, point-major
    constexpr int KS = SM::KS;
    __shared__ long long sl_elem[NS];
    __shared__ uint64_t bar[2];
    __shared__ R Mcv[S::n * S::n];
    __shared__ R Msf[S::nf * S::n];   // sp_to_fp [nf][n]
    __shared__ R Mdf[S::n * S::nf];   // dfp_to_sp [n][nf]

    const int tid = threadIdx.x;
    for (int i = tid; i < S::n * S::n; i += kThreads) Mcv[i] = M.sp_to_cv[i];
    for (int i = tid; i < S::nf * S::n; i += kThreads) {
        Msf[i] = M.sp_to_fp[i];
        Mdf[i] = M.dfp_to_sp[i];
    }
    int o[3];
    {
        int b = (int)bidx;
        const int tx = G.N[0] / TX;
        o[0] = (b % tx) * TX;
        o[1] = (b / tx) * TY;
        o[2] = 0;
    }
    for (int s = tid; s < NS; s += kThreads) {
        int l[3];
        TL::coords(s, l);
        sl_elem[s] = elem_of<2>(G, o, l);
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    const R dt = (R)(*A.dt);
    const int nt = G.nt;
    const long long E = G.E;

    // phase-B items of this thread: element, variable and point block
    // (items ordered block-major, so a warp's items share their block)
    int it_el[IPT], it_v[IPT], it_b[IPT], it_bx[IPT], it_by[IPT];
    bool it_ok[IPT];
#pragma unroll
    for (int k = 0; k < IPT; k++) {
        const int it = tid + k * kThreads;
        it_ok[k] = it < ITEMS;
        const int itc = it_ok[k] ? it : 0;
        const int b = itc / (NE * V), rem = itc % (NE * V);
        it_el[k] = rem / V;
        it_v[k] = rem % V;
        it_b[k] = b;
        it_bx[k] = (b % DB::NBX) * BX;
        it_by[k] = (b / DB::NBX) * BY;
    }
    R dreg[IPT][BXY][NT];  // kPredict: dudt per slice; kCorrect: du in [..][..][0]
#pragma unroll
    for (int k = 0; k < IPT; k++)
#pragma unroll
        for (int p = 0; p < BXY; p++)
#pragma unroll
            for (int t = 0; t < NT; t++) dreg[k][p][t] = 0;

    __syncthreads();
    // one elected thread issues the bulk copies of slice t into buffer b
    auto issue = [&](int t, int b) {
        const R* src = A.in_slices > 1 ? A.ua_in + (long long)t * E * V * NPT : A.ua_in;
        R* dst = Sbuf + b * NS * SS;
        if (tid == 0) {
            uint32_t bytes = 0;
            for (int s = 0; s < NS; s++)
                if (sl_elem[s] >= 0) bytes += V * NPT * sizeof(R);
            fence_proxy_async_smem();
            mbar_expect_tx(&bar[b], bytes);
            for (int s = 0; s < NS; s++)
                if (sl_elem[s] >= 0) bulk_g2s(dst + s * SS, src + sl_elem[s] * V * NPT, V * NPT * sizeof(R), &bar[b]);
        }
    };
    const bool multi = A.in_slices > 1;
    const int nt_eval = (MODE == kPredict && !multi) ? 1 : nt;
    issue(0, 0);
    // the step-start state of the tile's elements (predictor and corrector
    // epilogues), point-major, by coalesced loads while slice 0 is staged
    if (MODE != kFlux) {
        for (int q = tid; q < NE * V * (NPT / PW); q += kThreads) {
            const int c = q % (NPT / PW), k = q / (NPT / PW);
            R w4[PW];
            vload<R, PW>(A.u + sl_elem[k / V] * V * NPT + (k % V) * NPT + c * PW, w4);
#pragma unroll
            for (int w = 0; w < PW; w++) Ubuf[(c * PW + w) * KS + k] = w4[w];
        }
    }
    for (int t = 0; t < nt_eval; t++) {
        const int b = multi ? (t & 1) : 0;
        R* Ss = Sbuf + b * NS * SS;
        R* FX = FX0 + (NFX == 1 ? 0 : (t & 1)) * (2 * NE * V * FXS);
        if (multi && t + 1 < nt) issue(t + 1, b ^ 1);
        if (t == 0 || multi) mbar_wait_bounded(&bar[b], multi ? ((t >> 1) & 1) : 0, G.status);
        // ---- phase A: fluxes at every flux point of the slice ----
        // interfaces (two extrapolations and an LLF solve, about twice an
        // interior point's work) on the first NFT threads, one each; the
        // interior points on the rest, ordered by (direction, flux point)
        // so that a warp's points share both and take their coefficients
        // from constant offsets
        {
            constexpr int NF0 = LN::L0, NF1 = LN::L1, NFT = NF0 + NF1;
            constexpr int NPL = NE * n;                 // interior items per (direction, flux point)
            constexpr int NINT = 2 * (nf - 2) * NPL;
            constexpr int TI = kThreads - NFT;
            const int vt = A.in_slices > 1 ? t : 0;
            auto face = [&](int q) {
                if (q < NF0) face_item2<R, P, TX, TY, 0, VISC>(G, M, Ss, FX, o, q, A.vg[0], sl_elem, vt);
                else face_item2<R, P, TX, TY, 1, VISC>(G, M, Ss, FX, o, q - NF0, A.vg[1], sl_elem, vt);
            };
            auto interior = [&](int r) {
                const int g = r / NPL, el = (r % NPL) / n, tp = r % n;
                if (g < nf - 2) interior_item2<R, P, TX, TY, 0>(G, Msf, Ss, FX, el, 1 + g, tp);
                else interior_item2<R, P, TX, TY, 1>(G, Msf, Ss, FX, el, 1 + g - (nf - 2), tp);
            };
            if constexpr (TI >= kThreads / 4) {
                if (tid < NFT) face(tid);
                else
                    for (int r = tid - NFT; r < NINT; r += TI) interior(r);
            } else {
                for (int q = tid; q < NFT + NINT; q += kThreads) {
                    if (q < NFT) face(q);
                    else interior(q - NFT);
                }
            }
        }
        __syncthreads();
        if (MODE != kFlux) {
            // ---- phase B: divergence of the thread's point blocks ----
#pragma unroll
            for (int k = 0; k < IPT; k++) {
                if (!it_ok[k]) continue;
                const int el = it_el[k], v = it_v[k], bx0 = it_bx[k], by0 = it_by[k];
                const R* Fx = FX + ((0 * NE + el) * V + v) * FXS;
                const R* Fy = FX + ((1 * NE + el) * V + v) * FXS;
                R dd[BY][BX];
                div_block2<R, P>(G, Mdf, Fx, Fy, bx0, by0, dd);
#pragma unroll
                for (int j = 0; j < BY; j++)
#pragma unroll
                    for (int i = 0; i < BX; i++) {
                        const int p = j * BX + i;
                        if (MODE == kPredict) {
#pragma unroll
                            for (int tt = 0; tt < NT; tt++)
                                if (tt == t || (!multi && tt < nt)) dreg[k][p][tt] = dd[j][i];
                        } else {
                            R dudt = dd[j][i];
                            if (G.grav && v != 0) {
                                const int pt = (bx0 + i) + n * (by0 + j);
                                const R* uv = Ss + el * SS;
                                R s;
                                if (v <= D) s = uv[pt] * (R)G.g[v - 1];
                                else s = uv[NPT + pt] * (R)G.g[0] + uv[2 * NPT + pt] * (R)G.g[1];
                                dudt -= s;
                            }
                            dreg[k][p][0] += dudt * M.wt[t] * dt;
                        }
                    }
            }
        } else {
            // ---- FV face fluxes of slice t (src/transforms.cpp:378-481) ----
#pragma unroll
            for (int d = 0; d < D; d++) {
                R* out = A.ff[d];
                const R* Fd = FX + d * NE * V * FXS;
                for (int q = tid; q < NE * NFP; q += kThreads) {
                    const int el = q / NFP, fi = q % NFP;
                    int ll, cc;
                    if (d == 0) { ll = fi % nf; cc = fi / nf; }
                    else { cc = fi % n; ll = fi / n; }
                    R* dst = out + (((long long)t * E + sl_elem[el]) * V) * NFP + fi;
                    const R* srcb = Fd + el * V * FXS + (d == 0 ? ll : n * ll);
#pragma unroll
                    for (int v = 0; v < V; v++) {
                        R f = 0;
#pragma unroll
                        for (int m = 0; m < n; m++) f += srcb[v * FXS + (d == 0 ? nf * m : m)] * Mcv[cc * n + m];
                        dst[v * NFP] = f;
                    }
                }
            }
        }
        // with one FX buffer the next slice's phase A overwrites this
        // slice's fluxes; the corrector's gravity source reads this slice's
        // staging buffer, which the next slice's prefetch overwrites
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
        }
        __syncthreads();
        R* O = smem;  // [slice][point][KS], point-major
        // with gravity the source of a momentum (energy) slot uses the
        // updated density (momenta) of the same point and slice
        // (src/transforms.cpp:16-27 on U_ader being written): variables are
        // finished in three rounds that read the earlier rounds' results
        const int rounds = G.grav ? 3 : 1;
        for (int round = 0; round < rounds; round++) {
#pragma unroll
            for (int k = 0; k < IPT; k++) {
                if (!it_ok[k]) continue;
                const int el = it_el[k], v = it_v[k], kk = el * V + v;
                if (G.grav && (v == 0 ? 0 : (v <= D ? 1 : 2)) != round) continue;
#pragma unroll
                for (int j = 0; j < BY; j++)
#pragma unroll
                    for (int i = 0; i < BX; i++) {
                        const int p = j * BX + i;
                        const int pt = (it_bx[k] + i) + n * (it_by[k] + j);
                        const R u_old = Ubuf[pt * KS + kk];
                        R dudt[NT];
#pragma unroll
                        for (int tt = 0; tt < NT; tt++) {
                            dudt[tt] = dreg[k][p][tt];
                            if (G.grav && v != 0 && tt < nt) {
                                const R* nw = O + (tt * NPT + pt) * KS + el * V;
                                R s;
                                if (v <= D) s = nw[0] * (R)G.g[v - 1];
                                else s = nw[1] * (R)G.g[0] + nw[2] * (R)G.g[1];
                                dudt[tt] -= s;
                            }
                        }
#pragma unroll
                        for (int tt = 0; tt < NT; tt++) {
                            if (tt >= nt) break;
                            R du = 0;
                            if constexpr (sizeof(R) == 4) {
#pragma unroll
                                for (int ll = 0; ll < NT; ll++)
                                    if (ll < nt) du += dudt[ll] * Cw[tt * NT + ll];
                            } else {
#pragma unroll
                                for (int ll = 0; ll < NT; ll++)
                                    if (ll < nt) du += dudt[ll] * M.invader[tt * nt + ll] * M.wt[ll] * dt;
                            }
                            O[(tt * NPT + pt) * KS + kk] = u_old - du;
                        }
                    }
            }
            if (G.grav) __syncthreads();
        }
        __syncthreads();
        // coalesced write-back of every slice: consecutive threads take
        // consecutive points of an element's variable rows
        for (int q = tid; q < NE * V * (NPT / PW); q += kThreads) {
            const int c = q % (NPT / PW), k = q / (NPT / PW);
            R* dst = A.ua_out + sl_elem[k / V] * V * NPT + (k % V) * NPT + c * PW;
            const R* src = O + c * PW * KS + k;
            for (int tt = 0; tt < nt; tt++) {
                R w4[PW];
#pragma unroll
                for (int w = 0; w < PW; w++) w4[w] = src[w * KS];
                vstore<R, PW>(dst, w4);
                dst += E * V * NPT;
                src += NPT * KS;
            }
        }
    } else if (MODE == kCorrect) {
        // ---- corrector / RK stage (src/transforms.cpp:327-374, 252-261) ----
        R* Wsp = smem;                     // [NE][V][NPT]
        R* Tmp = smem + NE * V * NPT;
        R* Tu = smem + 2 * NE * V * NPT;   // [NPT][KS]: U - du, point-major
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            if (!it_ok[k]) continue;
            const int kk = it_el[k] * V + it_v[k];
#pragma unroll
            for (int j = 0; j < BY; j++)
#pragma unroll
                for (int i = 0; i < BX; i++) {
                    const int pt = (it_bx[k] + i) + n * (it_by[k] + j);
                    Tu[pt * KS + kk] = Ubuf[pt * KS + kk] - dreg[k][j * BX + i][0];
                }
        }
        __syncthreads();
        // RK convex combination and the write of U, coalesced; W_sp's
        // element-major copy for the final stage's primitives and sweeps
        for (int q = tid; q < NE * V * (NPT / PW); q += kThreads) {
            const int c = q % (NPT / PW), k = q / (NPT / PW);
            const long long g = sl_elem[k / V] * V * NPT + (k % V) * NPT + c * PW;
            R val[PW];
#pragma unroll
            for (int w = 0; w < PW; w++) val[w] = Tu[(c * PW + w) * KS + k];
            if (A.rk_a > 0) {
                const R ra = (R)A.rk_a;
                R u0[PW];
                vload<R, PW>(A.u0 + g, u0);
#pragma unroll
                for (int w = 0; w < PW; w++) val[w] = ra * u0[w] + ((R)1.0 - ra) * val[w];
            }
            vstore<R, PW>(A.u_out + g, val);
            vstore<R, PW>(Wsp + k * NPT + c * PW, val);
        }
        if (A.final_stage) {
            __syncthreads();
            for (int q = tid; q < NE * NPT; q += kThreads) {
                const int el = q / NPT, pt = q % NPT;
                R un[V], w[V];
#pragma unroll
                for (int v = 0; v < V; v++) un[v] = Wsp[(el * V + v) * NPT + pt];
                primitives<D>(un, w, (R)G.gm);
#pragma unroll
                for (int v = 0; v < V; v++) Wsp[(el * V + v) * NPT + pt] = w[v];
            }
            __syncthreads();
            // W_cv = sp_to_cv(W_sp): x, y sweeps (src/transforms.cpp:99-117)
            sweep_smem<D, P, R>(Wsp, Tmp, Mcv, 0, NE * V * NPT);
            __syncthreads();
            sweep_smem<D, P, R>(Tmp, Wsp, Mcv, 1, NE * V * NPT);
            __syncthreads();
            double dtl = 1.7976931348623157e308;
            for (int q = tid; q < NE * NPT; q += kThreads) {
                const int el = q / NPT, pt = q % NPT;
                const long long ge = sl_elem[el];
                R w[V];
#pragma unroll
                for (int v = 0; v < V; v++) w[v] = Wsp[(el * V + v) * NPT + pt];
                if (A.wcv)
#pragma unroll
                    for (int v = 0; v < V; v++) A.wcv[(ge * V + v) * NPT + pt] = w[v];
                dtl = smin(dtl, point_dt<D>(G, w, n));
            }
            block_min_dt(dtl, A.dtmin);
        }
    } else {
        // ---- U_cv = sp_to_cv(U) and the slice-0 FV candidate ----
        R* Ut = Sbuf;
        R* Tmp = Sbuf + NE * V * NPT;
        for (int q = tid; q < NE * CH; q += kThreads) {
            const int el = q / CH, c = q % CH;
            reinterpret_cast<VT*>(Ut + el * V * NPT)[c] = reinterpret_cast<const VT*>(A.u + sl_elem[el] * V * NPT)[c];
        }
        __syncthreads();
        sweep_smem<D, P, R>(Ut, Tmp, Mcv, 0, NE * V * NPT);
        __syncthreads();
        sweep_smem<D, P, R>(Tmp, Ut, Mcv, 1, NE * V * NPT);
        __syncthreads();
        const R* src = Ut;
        for (int q = tid; q < NE * CH; q += kThreads) {
            const int el = q / CH, c = q % CH;
            reinterpret_cast<VT*>(A.ucv + sl_elem[el] * V * NPT)[c] = reinterpret_cast<const VT*>(src + el * V * NPT)[c];
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
