// Native 2D induction solver: the reference's Induction_ader restricted to a
// field in the x-y plane (B = (B_x, B_y, 0), v = (v_x, v_y, 0)), where only the
// edge EMF E_z is nonzero (src/induction_ader.hpp:332-483,
// src/induction.cpp:123-200, 330-420, 487-560). No counterpart in the
// reference as a 2D code: the reference needs three active directions, and a
// quasi-2D reference run (nx3 = 2, periodic z, B_z = 0, v_z = 0) is what this
// solver reproduces.
//
// Device layout (R = double: plain form, reference operation order; R = float:
// precision form), no ghost elements, element = j*Nx + i:
//   B_x  [element][jj][ix]    n  x nf   (y solution points x x flux points)
//   B_y  [element][jy][ii]    nf x n    (y flux points x x solution points)
// One fused kernel per Picard pass (ind2_pass): E_z, its interface sweeps
// and the curl update stay in shared memory and registers; the predictor's
// slices are the only intermediate in HBM. Periodic boundaries.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "spdk.h"
#include "spdk_induction.h"
#include "spdk_setup.h"

namespace spdk {
int fail(int code, const std::string& msg);
}

namespace {

using namespace spdk;

template <typename R>
struct Ind2Mats {
    R sp_to_fp[kMaxNF * kMaxN];   // [nf][n]
    R dfp_to_sp[kMaxN * kMaxNF];  // [n][nf]
    R invader[kMaxN * kMaxN];     // [nt][nt]
    R wt[kMaxN];
};

struct Ind2Geo {
    int N[2];
    double h[2];
    double rh[2];   // 1/h when h is a power of two (the division is then an exact scaling), else 0
    double v[2];
    int nt;
    long long E;
};

// src/induction.cpp:487-491
template <typename R>
__device__ __forceinline__ R upwind(R left, R right, R vel) {
    if (vel == 0) return R(0.5) * (left + right);
    return vel > 0 ? left : right;
}

// One Picard pass (predictor) or the corrector over a tile of TX x TY
// elements, everything on chip: per slice the face fields of the tile and of
// a one-element ring around it (periodic images) are staged in shared
// memory; E_z = v_x b_y - v_y b_x is formed at every staged element's edge
// points (compute_E, src/induction.cpp:123-200: b_x interpolated in y to the
// y flux points, b_y in x); the unique EMF of each tile edge point follows
// the reference's interface sweeps (E_riemann_solver, src/induction.cpp:
// 494-558, as called at src/induction_ader.hpp:401-412: x interfaces first,
// then y, each upwinded with its face-normal velocity, so a corner takes the
// y sweep of the two rows' x-swept values); dB/dt = curl E through
// dfp_to_sp at the face points (src/induction.cpp:310-400, dim = x, y; the
// E_x, E_y terms there are signed zeros of a plane field) accumulates per
// slice in shared memory; the epilogue writes the predictor's slices
// (update_B_prediction) or the corrected field (update_B_solution, with the
// SSP-RK combination). Only B crosses HBM.
enum { kInd2Predict = 0, kInd2Correct = 1 };

template <typename R, int P, int TX, int TY>
struct Ind2Tile {
    static constexpr int n = P + 1, nf = P + 2;
    static constexpr int SX = TX + 2, SY = TY + 2, NS = SX * SY;  // staged elements (tile + ring)
    static constexpr int NE = TX * TY;
    static constexpr int FB = n * nf;                             // B_x (or B_y) values per element
    static constexpr int ITEMS = NE * 2 * FB;                     // face points of the tile
    static constexpr int IPT = (ITEMS + 255) / 256;
    // shared memory (elements of R): B_x, B_y of the staged elements, raw E
    // of the staged elements, unique E of the tile's elements, dB/dt of
    // every face point and slice
    static constexpr int OFF_BY = NS * FB, OFF_ER = 2 * NS * FB, OFF_EU = OFF_ER + NS * nf * nf;
    static constexpr int OFF_DD = OFF_EU + NE * nf * nf;
    static constexpr int TOTAL = OFF_DD + ITEMS * n;
};

struct Ind2Pass {
    const void* bx_in;   // [slice][E][n][nf] (in_slices == 1: B itself)
    const void* by_in;
    int in_slices;
    const void* bx_old;  // B at the step (stage) start
    const void* by_old;
    const void* bx0;     // RK step-start state
    const void* by0;
    void* bx_out;        // predictor: [slice][E][..]; corrector: B (may alias bx_old: element-local)
    void* by_out;
    double dt;
    double rk_a;
};

template <typename R, int P, int TX, int TY, int MODE>
__global__ void __launch_bounds__(256, 3) ind2_pass(Ind2Geo G, Ind2Mats<R> M, Ind2Pass A) {
    using T = Ind2Tile<R, P, TX, TY>;
    constexpr int n = T::n, nf = T::nf, FB = T::FB, NS = T::NS, SX = T::SX, NE = T::NE, IPT = T::IPT;
    static_assert(T::TOTAL * sizeof(R) <= 72 * 1024, "three blocks per SM");
    constexpr int nt_max = P + 1;
    extern __shared__ __align__(16) unsigned char ind2_smem[];
    R* sm = reinterpret_cast<R*>(ind2_smem);
    R* Sbx = sm;
    R* Sby = sm + T::OFF_BY;
    R* Er = sm + T::OFF_ER;
    R* Eu = sm + T::OFF_EU;
    R* Dd = sm + T::OFF_DD;  // [slice][item]
    __shared__ int sl_el[NS];
    // the coefficients are read at lane-dependent offsets, which the kernel
    // parameter space would serve one address at a time
    __shared__ R Msf[nf * n], Mdf[n * nf];
    const int tid = threadIdx.x;
    for (int i = tid; i < nf * n; i += 256) {
        Msf[i] = M.sp_to_fp[i];
        Mdf[i] = M.dfp_to_sp[i];
    }
    const int tiles_x = G.N[0] / TX;
    const int i0 = (int)(blockIdx.x % tiles_x) * TX, j0 = (int)(blockIdx.x / tiles_x) * TY;
    for (int s = tid; s < NS; s += 256) {
        int i = i0 + s % SX - 1, j = j0 + s / SX - 1;
        if (i < 0) i += G.N[0];
        if (i >= G.N[0]) i -= G.N[0];
        if (j < 0) j += G.N[1];
        if (j >= G.N[1]) j -= G.N[1];
        sl_el[s] = j * G.N[0] + i;
    }
    const R vx = (R)G.v[0], vy = (R)G.v[1];
    const int nt = G.nt;
    const int nt_eval = A.in_slices > 1 ? nt : 1;
    // (E D) / h: a product by 1/h where h is a power of two (exact, so the
    // FP64 bits are the division's) and always in the FP32 form
    const R hx = (R)G.h[0], hy = (R)G.h[1];
    const bool px = sizeof(R) == 4 || G.rh[0] != 0, py = sizeof(R) == 4 || G.rh[1] != 0;
    const R rhx = G.rh[0] != 0 ? (R)G.rh[0] : (R)(1.0 / G.h[0]);
    const R rhy = G.rh[1] != 0 ? (R)G.rh[1] : (R)(1.0 / G.h[1]);
    __syncthreads();
    for (int t = 0; t < nt_eval; t++) {
        // ---- stage B_x, B_y of slice t (tile and ring) ----
        const R* bxs = (const R*)A.bx_in + (A.in_slices > 1 ? (long long)t * G.E * FB : 0);
        const R* bys = (const R*)A.by_in + (A.in_slices > 1 ? (long long)t * G.E * FB : 0);
        for (int q = tid; q < NS * FB; q += 256) {
            const int sl = q / FB, r = q % FB;
            const long long g = (long long)sl_el[sl] * FB + r;
            Sbx[q] = bxs[g];
            Sby[q] = bys[g];
        }
        __syncthreads();
        // ---- raw E_z at the edge points the tile's sweeps read: every point
        // of the tile elements; of the ring, the column (row) next to the
        // tile and the corner point next to it ----
        constexpr int TXn = TX * nf, TYn = TY * nf;
        constexpr int NRAW = NE * nf * nf + 2 * TYn + 2 * TXn + 4;
        for (int q = tid; q < NRAW; q += 256) {
            int sl, ix, jy;
            if (q < NE * nf * nf) {
                const int el = q / (nf * nf);
                sl = (el / TX + 1) * SX + el % TX + 1;
                ix = q % nf;
                jy = (q / nf) % nf;
            } else {
                int r = q - NE * nf * nf;
                if (r < 2 * TYn) {          // left / right ring: the column next to the tile
                    const int side = r / TYn;
                    r %= TYn;
                    sl = (r / nf + 1) * SX + (side ? TX + 1 : 0);
                    jy = r % nf;
                    ix = side ? 0 : nf - 1;
                } else if ((r -= 2 * TYn) < 2 * TXn) {  // bottom / top ring: the row next to the tile
                    const int side = r / TXn;
                    r %= TXn;
                    sl = (side ? TY + 1 : 0) * SX + r / nf + 1;
                    ix = r % nf;
                    jy = side ? 0 : nf - 1;
                } else {                    // the four ring corners: the point next to the tile
                    r -= 2 * TXn;
                    const int cx = r & 1, cy = r >> 1;
                    sl = (cy ? TY + 1 : 0) * SX + (cx ? TX + 1 : 0);
                    ix = cx ? 0 : nf - 1;
                    jy = cy ? 0 : nf - 1;
                }
            }
            const int qo = (sl * nf + jy) * nf + ix;
            const R* X = Sbx + sl * FB;  // [jj][ix]
            const R* Y = Sby + sl * FB;  // [jy][ii]
            R b1 = 0, b2 = 0;
#pragma unroll
            for (int l = 0; l < n; l++) {
                b1 += X[l * nf + ix] * Msf[jy * n + l];
                b2 += Y[jy * n + l] * Msf[ix * n + l];
            }
            Er[qo] = vx * b2 - vy * b1;
        }
        __syncthreads();
        // ---- unique E_z at the tile elements' edge points ----
        for (int q = tid; q < NE * nf * nf; q += 256) {
            const int el = q / (nf * nf), ix = q % nf, jy = (q / nf) % nf;
            const int lx = el % TX + 1, ly = el / TX + 1;  // staged coordinates
            auto raw = [&](int sx, int sy, int j, int i) { return Er[((sy * SX + sx) * nf + j) * nf + i]; };
            const bool xf = ix == 0 || ix == nf - 1, yf = jy == 0 || jy == nf - 1;
            R e;
            if (!xf && !yf) {
                e = raw(lx, ly, jy, ix);
            } else {
                const int xl = ix == 0 ? lx - 1 : lx, xr = ix == 0 ? lx : lx + 1;
                auto xswept = [&](int sy, int j) { return upwind(raw(xl, sy, j, nf - 1), raw(xr, sy, j, 0), vx); };
                if (!yf) {
                    e = xswept(ly, jy);
                } else {
                    const int yb = jy == 0 ? ly - 1 : ly, yt = jy == 0 ? ly : ly + 1;
                    if (!xf) e = upwind(raw(lx, yb, nf - 1, ix), raw(lx, yt, 0, ix), vy);
                    else e = upwind(xswept(yb, nf - 1), xswept(yt, 0), vy);
                }
            }
            Eu[q] = e;
        }
        __syncthreads();
        // ---- dB/dt of slice t at the tile's face points ----
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const int it = tid + k * 256;
            if (it >= T::ITEMS) continue;
            const int el = it / (2 * FB), r = it % (2 * FB);
            const R* E = Eu + el * nf * nf;
            R s = 0;
            if (r < FB) {
                // B_x at (jj, ix): dBx/dt = -dEz/dy
                const int jj = r / nf, ix = r % nf;
#pragma unroll
                for (int ll = 0; ll < nf; ll++) {
                    const R v = E[ll * nf + ix] * Mdf[jj * nf + ll];
                    s -= py ? v * rhy : v / hy;
                }
            } else {
                // B_y at (jy, ii): dBy/dt = +dEz/dx
                const int jy = (r - FB) / n, ii = (r - FB) % n;
#pragma unroll
                for (int ll = 0; ll < nf; ll++) {
                    const R v = E[jy * nf + ll] * Mdf[ii * nf + ll];
                    s += px ? v * rhx : v / hx;
                }
            }
            Dd[t * T::ITEMS + it] = s;
        }
        __syncthreads();
    }
    // ---- predictor / corrector ----
    const R dt = (R)A.dt;
#pragma unroll
    for (int k = 0; k < IPT; k++) {
        const int it = tid + k * 256;
        if (it >= T::ITEMS) continue;
        const int el = it / (2 * FB), r = it % (2 * FB);
        const bool isx = r < FB;
        const long long q = (long long)sl_el[(el / TX + 1) * SX + el % TX + 1] * FB + (isx ? r : r - FB);
        const R b_old = isx ? ((const R*)A.bx_old)[q] : ((const R*)A.by_old)[q];
        R* out = (R*)(isx ? A.bx_out : A.by_out);
        if (MODE == kInd2Predict) {
#pragma unroll
            for (int tt = 0; tt < nt_max; tt++) {
                if (tt >= nt) break;
                R dB = 0;
#pragma unroll
                for (int ll = 0; ll < nt_max; ll++)
                    if (ll < nt) dB += Dd[(ll < nt_eval ? ll : 0) * T::ITEMS + it] * M.invader[tt * nt + ll] * M.wt[ll] * dt;
                out[(long long)tt * G.E * FB + q] = b_old - dB;
            }
        } else {
            R dB = 0;
#pragma unroll
            for (int tt = 0; tt < nt_max; tt++)
                if (tt < nt) dB += Dd[(tt < nt_eval ? tt : 0) * T::ITEMS + it] * M.wt[tt] * dt;
            R b = b_old - dB;
            if (A.rk_a > 0) {
                const R ra = (R)A.rk_a;
                b = ra * (isx ? ((const R*)A.bx0)[q] : ((const R*)A.by0)[q]) + ((R)1.0 - ra) * b;
            }
            out[q] = b;
        }
    }
}

// B2_cv of the quasi-2D reference run at sub-cell row kk = 0 of its z
// direction (src/induction.cpp:420-452): the x (y) sub-cell averages of B_x
// (B_y) times the z average of a z-independent field, in the reference's
// loop and product order, so the FP64 values are its bytes. Output
// [element][var][jj][ii], var = B_x, B_y, B_z (zero), |B|^2.
template <typename R, int P>
__global__ void __launch_bounds__(256) ind2_b2cv(long long E, const R* __restrict__ bx, const R* __restrict__ by,
                                                 const double* __restrict__ cv, const double* __restrict__ fcv,
                                                 double* __restrict__ out) {
    constexpr int n = P + 1, nf = P + 2;
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < E * n * n;
         o += (long long)gridDim.x * blockDim.x) {
        const long long e = o / (n * n);
        const int jj = (int)((o / n) % n), ii = (int)(o % n);
        const R* X = bx + e * n * nf;
        const R* Y = by + e * nf * n;
        double bxv = 0, byv = 0;
        for (int nn = 0; nn < n; nn++)
            for (int mm = 0; mm < n; mm++)
                for (int ll = 0; ll < nf; ll++)
                    bxv += (double)X[mm * nf + ll] * cv[0 * n + nn] * cv[jj * n + mm] * fcv[ii * nf + ll];
        for (int nn = 0; nn < n; nn++)
            for (int mm = 0; mm < nf; mm++)
                for (int ll = 0; ll < n; ll++)
                    byv += (double)Y[mm * n + ll] * cv[0 * n + nn] * fcv[jj * nf + mm] * cv[ii * n + ll];
        const double bzv = 0.0;
        double* dst = out + e * 4 * n * n + jj * n + ii;
        dst[0] = bxv;
        dst[n * n] = byv;
        dst[2 * n * n] = bzv;
        dst[3 * n * n] = bxv * bxv + byv * byv + bzv * bzv;
    }
}

}  // namespace

struct spdk_induction2d {
    spdk_induction2d_config cfg{};
    int n = 0, nf = 0, nt = 0, nstages = 1, esz = 8;
    long long E = 0;
    double rk_a[3] = {0, 0, 0};
    double Dt = 0, dt = 0;
    Ind2Geo G{};
    Matrices m;
    void *bx = nullptr, *by = nullptr, *bxa[2] = {nullptr, nullptr}, *bya[2] = {nullptr, nullptr};
    void *bx0 = nullptr, *by0 = nullptr;
    double *b2 = nullptr, *cv = nullptr, *fcv = nullptr;
    cudaStream_t stream = nullptr;
    int launches = 0;
};

namespace {

int dalloc2(void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess)
        return fail(SPDK_E_NOMEM, "cudaMalloc(" + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    return 0;
}

unsigned blocks_for(long long items) {
    long long b = (items + 255) / 256;
    return (unsigned)std::max<long long>(1, std::min<long long>(b, 148LL * 64));
}

template <typename R>
void fill_mats(const Matrices& m, int nt, Ind2Mats<R>* M) {
    std::memset(M, 0, sizeof(*M));
    for (int q = 0; q < m.nf * m.n; q++) {
        M->sp_to_fp[q] = (R)m.sp_to_fp[q];
        M->dfp_to_sp[q] = (R)m.dfp_to_sp[q];
    }
    for (int q = 0; q < nt * nt; q++) M->invader[q] = (R)m.invader[q];
    for (int q = 0; q < nt; q++) M->wt[q] = (R)m.wt[q];
}

// one step's launches (src/induction_ader.hpp:351-385): per stage, the
// Picard passes (ADER: nt - 1 predictor passes, then the corrector; SSP-RK:
// the corrector of a single slice) on tiles of TX x TY elements
template <typename R, int P, int TX, int TY>
int enqueue_t(spdk_induction2d* s) {
    using T = Ind2Tile<R, P, TX, TY>;
    Ind2Mats<R> M;
    fill_mats<R>(s->m, s->nt, &M);
    const long long E = s->E;
    const int nt = s->nt;
    const size_t state = (size_t)E * T::FB;
    const size_t smem = (size_t)T::TOTAL * sizeof(R);
    cudaStream_t st = s->stream;
    auto kp = ind2_pass<R, P, TX, TY, kInd2Predict>;
    auto kc = ind2_pass<R, P, TX, TY, kInd2Correct>;
    if (cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(kc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return fail(SPDK_E_CUDA, "induction2d: shared memory request of " + std::to_string(smem) + " bytes");
    const unsigned blocks = (unsigned)(E / (TX * TY));
    int launches = 0;
    R* bx = (R*)s->bx;
    R* by = (R*)s->by;
    if (s->nstages > 1) {
        if (cudaMemcpyAsync(s->bx0, bx, state * sizeof(R), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(s->by0, by, state * sizeof(R), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return fail(SPDK_E_CUDA, "induction2d: step-start copy");
    }
    for (int stg = 0; stg < s->nstages; stg++) {
        Ind2Pass A{};
        A.bx_in = bx;
        A.by_in = by;
        A.in_slices = 1;
        A.bx_old = bx;
        A.by_old = by;
        A.dt = s->dt;
        if (nt == 1) {
            // an SSP-RK stage updates B in place while neighbouring tiles
            // stage their ring from it: the stage reads a copy (the
            // reference's copy_ader into B_ader)
            if (cudaMemcpyAsync(s->bxa[0], bx, state * sizeof(R), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
                cudaMemcpyAsync(s->bya[0], by, state * sizeof(R), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
                return fail(SPDK_E_CUDA, "induction2d: stage copy");
            A.bx_in = s->bxa[0];
            A.by_in = s->bya[0];
        }
        for (int it = 0; it + 1 < nt; it++) {
            A.bx_out = s->bxa[it % 2];
            A.by_out = s->bya[it % 2];
            kp<<<blocks, 256, smem, st>>>(s->G, M, A);
            launches++;
            A.bx_in = A.bx_out;
            A.by_in = A.by_out;
            A.in_slices = nt;
        }
        // the corrector updates B in place: element-local reads and writes,
        // its E from the last predictor slices (or the stage copy)
        A.bx0 = s->bx0;
        A.by0 = s->by0;
        A.bx_out = bx;
        A.by_out = by;
        A.rk_a = s->rk_a[stg];
        kc<<<blocks, 256, smem, st>>>(s->G, M, A);
        launches++;
    }
    s->launches = launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("induction2d launch: ") + cudaGetErrorString(e));
    return 0;
}

// tiles of 4 x 4 elements up to p = 4, 2 x 2 above (their per-thread
// predictor slices stay in registers), whichever divides the element counts
template <typename R, int P>
int enqueue2(spdk_induction2d* s) {
    const int Nx = s->cfg.N[0], Ny = s->cfg.N[1];
    if constexpr (P <= 4) {
        if (Nx % 4 == 0 && Ny % 4 == 0) return enqueue_t<R, P, 4, 4>(s);
    }
    if (Nx % 2 == 0 && Ny % 2 == 0) return enqueue_t<R, P, 2, 2>(s);
    return enqueue_t<R, P, 1, 1>(s);
}

template <typename R>
int enqueue_r(spdk_induction2d* s) {
    switch (s->cfg.p) {
    case 1: return enqueue2<R, 1>(s);
    case 2: return enqueue2<R, 2>(s);
    case 3: return enqueue2<R, 3>(s);
    case 4: return enqueue2<R, 4>(s);
    case 5: return enqueue2<R, 5>(s);
    case 6: return enqueue2<R, 6>(s);
    case 7: return enqueue2<R, 7>(s);
    }
    return fail(SPDK_E_ARG, "p must be in 1..7");
}

template <typename R>
int b2cv_r(spdk_induction2d* s) {
    const long long items = s->E * s->n * s->n;
    switch (s->cfg.p) {
#define CASE(P)                                                                                                   \
    case P:                                                                                                       \
        ind2_b2cv<R, P><<<blocks_for(items), 256, 0, s->stream>>>(s->E, (const R*)s->bx, (const R*)s->by, s->cv, \
                                                                 s->fcv, s->b2);                                  \
        break;
        CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7)
#undef CASE
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("induction2d B2_cv: ") + cudaGetErrorString(e));
    return 0;
}

void release2(spdk_induction2d* s) {
    void* ptrs[] = {s->bx, s->by, s->bxa[0], s->bxa[1], s->bya[0], s->bya[1], s->bx0, s->by0,
                    s->b2, s->cv, s->fcv};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s->stream) cudaStreamDestroy(s->stream);
}

// A_z of the magnetic loop (src/initial_conditions.cpp:235-249, centre and
// radius as parameters): A0 (R - r) inside r <= R
double loop_az(const spdk_induction2d_config& c, double x, double y) {
    x = x - c.loop_center[0];
    y = y - c.loop_center[1];
    const double r = std::sqrt(x * x + y * y);
    if (r <= c.loop_R) return c.loop_A0 * (c.loop_R - r);
    return 0;
}

}  // namespace

extern "C" {

int spdk_induction2d_create(const spdk_induction2d_config* cfg, spdk_induction2d** out) {
    if (!cfg || !out) return fail(SPDK_E_ARG, "null argument");
    *out = nullptr;
    const spdk_induction2d_config& c = *cfg;
    if (c.p < 1 || c.p > kMaxP) return fail(SPDK_E_ARG, "p must be in 1..7");
    for (int d = 0; d < 2; d++) {
        if (c.N[d] < 2) return fail(SPDK_E_ARG, "nx1 and nx2 must be at least 2");
        if (!(c.L[d] > 0)) return fail(SPDK_E_ARG, "box lengths must be positive");
    }
    if (!(std::isfinite(c.velocity[0]) && std::isfinite(c.velocity[1])))
        return fail(SPDK_E_ARG, "velocity must be finite");
    if (c.velocity[0] == 0.0 && c.velocity[1] == 0.0) return fail(SPDK_E_ARG, "velocity must not vanish");
    const bool ader = c.integrator == SPDK_INTEGRATOR_ADER;
    if (!ader && c.integrator != SPDK_INTEGRATOR_RK) return fail(SPDK_E_ARG, "unknown integrator");
    if (!ader && (c.rk_order < 1 || c.rk_order > 3)) return fail(SPDK_E_ARG, "rk_order must be 1, 2 or 3");
    if (c.precision != SPDK_PRECISION_FP64 && c.precision != SPDK_PRECISION_FP32)
        return fail(SPDK_E_ARG, "unsupported precision");
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(SPDK_E_CUDA, "cudaSetDevice failed");

    spdk_induction2d* s = new spdk_induction2d;
    s->cfg = c;
    build_matrices(c.p, ader, &s->m);
    s->n = c.p + 1;
    s->nf = c.p + 2;
    s->nt = ader ? s->n : 1;
    s->nstages = ader ? 1 : c.rk_order;
    if (c.rk_order == 2 && !ader) s->rk_a[1] = 0.5;
    if (c.rk_order == 3 && !ader) { s->rk_a[1] = 0.75; s->rk_a[2] = 1.0 / 3.0; }
    s->esz = c.precision == SPDK_PRECISION_FP32 ? 4 : 8;
    s->E = (long long)c.N[0] * c.N[1];
    const int n = s->n, nf = s->nf, nt = s->nt;
    Axis X, Y;
    build_axis(c.N[0], c.p, c.L[0], s->m.x_fp, true, &X);
    build_axis(c.N[1], c.p, c.L[1], s->m.x_fp, true, &Y);
    s->G.N[0] = c.N[0];
    s->G.N[1] = c.N[1];
    s->G.h[0] = X.h;
    s->G.h[1] = Y.h;
    for (int d = 0; d < 2; d++) {
        int ex = 0;
        const double mant = std::frexp(s->G.h[d], &ex);
        s->G.rh[d] = mant == 0.5 ? std::ldexp(1.0, 1 - ex) : 0.0;
    }
    s->G.v[0] = c.velocity[0];
    s->G.v[1] = c.velocity[1];
    s->G.nt = nt;
    s->G.E = s->E;

    int rc = 0;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
        rc = fail(SPDK_E_CUDA, "stream creation failed");
    const size_t state = (size_t)s->E * n * nf;
    if (!rc) rc = dalloc2(&s->bx, state * s->esz);
    if (!rc) rc = dalloc2(&s->by, state * s->esz);
    // predictor slices (ADER, ping-pong) or the stage copy (SSP-RK)
    for (int b = 0; b < (nt > 1 ? 2 : 1) && !rc; b++) {
        rc = dalloc2(&s->bxa[b], (size_t)nt * state * s->esz);
        if (!rc) rc = dalloc2(&s->bya[b], (size_t)nt * state * s->esz);
    }
    if (!rc && s->nstages > 1) {
        rc = dalloc2(&s->bx0, state * s->esz);
        if (!rc) rc = dalloc2(&s->by0, state * s->esz);
    }
    if (!rc) rc = dalloc2((void**)&s->b2, (size_t)4 * s->E * n * n * sizeof(double));
    if (!rc) rc = dalloc2((void**)&s->cv, (size_t)n * n * sizeof(double));
    if (!rc) rc = dalloc2((void**)&s->fcv, (size_t)n * nf * sizeof(double));
    if (!rc && (cudaMemcpy(s->cv, s->m.sp_to_cv, (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice) !=
                    cudaSuccess ||
                cudaMemcpy(s->fcv, s->m.fp_to_cv, (size_t)n * nf * sizeof(double), cudaMemcpyHostToDevice) !=
                    cudaSuccess))
        rc = fail(SPDK_E_CUDA, "induction2d: matrix upload");
    if (!rc) {
        // initial condition (src/induction_ader.hpp:176-187): A_z at the edge
        // points (x and y flux points), B = curl A (rotational_a_to_b); the
        // A_x, A_y terms of the reference are signed zeros and drop out
        const double* D = s->m.dfp_to_sp;  // [n][nf]
        std::vector<double> Bx(state), By(state), Az((size_t)nf * nf);
        for (int j = 0; j < c.N[1]; j++)
            for (int i = 0; i < c.N[0]; i++) {
                const long long e = (long long)j * c.N[0] + i;
                for (int jy = 0; jy < nf; jy++)
                    for (int ix = 0; ix < nf; ix++)
                        Az[jy * nf + ix] = loop_az(c, X.sd_faces[(size_t)(i + 1) * nf + ix],
                                                   Y.sd_faces[(size_t)(j + 1) * nf + jy]);
                for (int jj = 0; jj < n; jj++)
                    for (int ix = 0; ix < nf; ix++) {
                        double d1a2 = 0;
                        for (int ll = 0; ll < nf; ll++) d1a2 += Az[ll * nf + ix] * D[jj * nf + ll];
                        Bx[(size_t)e * n * nf + jj * nf + ix] = d1a2 / Y.h - 0.0;
                    }
                for (int jy = 0; jy < nf; jy++)
                    for (int ii = 0; ii < n; ii++) {
                        double d2a1 = 0;
                        for (int ll = 0; ll < nf; ll++) d2a1 += Az[jy * nf + ll] * D[ii * nf + ll];
                        By[(size_t)e * nf * n + jy * n + ii] = 0.0 - d2a1 / X.h;
                    }
            }
        if (s->esz == 8) {
            if (cudaMemcpy(s->bx, Bx.data(), state * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(s->by, By.data(), state * 8, cudaMemcpyHostToDevice) != cudaSuccess)
                rc = fail(SPDK_E_CUDA, "induction2d: upload B");
        } else {
            std::vector<float> fx(Bx.begin(), Bx.end()), fy(By.begin(), By.end());
            if (cudaMemcpy(s->bx, fx.data(), state * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(s->by, fy.data(), state * 4, cudaMemcpyHostToDevice) != cudaSuccess)
                rc = fail(SPDK_E_CUDA, "induction2d: upload B");
        }
        // Induction_compute_dt (src/induction.cpp:52-91) for v_z = 0: every
        // point gives cfl min(1, h_x, h_y) / (|v_x| + |v_y| + 0) / n; no
        // resistive cap (nu = 0)
        double v_max = 0, dx_min = 1;
        v_max += std::fabs(c.velocity[0]);
        dx_min = std::min(dx_min, X.h);
        v_max += std::fabs(c.velocity[1]);
        dx_min = std::min(dx_min, Y.h);
        v_max += std::fabs(0.0);
        const double dt_v = c.cfl * dx_min / v_max / n;
        s->Dt = std::min(dt_v, 1E6);
        s->dt = s->Dt;
    }
    if (rc) {
        release2(s);
        delete s;
        return rc;
    }
    *out = s;
    return 0;
}

int spdk_induction2d_destroy(spdk_induction2d* s) {
    if (!s) return 0;
    cudaStreamSynchronize(s->stream);
    release2(s);
    delete s;
    return 0;
}

int spdk_induction2d_get_dt(spdk_induction2d* s, double* dt) {
    if (!s || !dt) return fail(SPDK_E_ARG, "null argument");
    *dt = s->dt;
    return 0;
}

int spdk_induction2d_set_dt(spdk_induction2d* s, double dt) {
    if (!s) return fail(SPDK_E_ARG, "null argument");
    if (!(dt > 0) || !std::isfinite(dt)) return fail(SPDK_E_ARG, "dt must be positive and finite");
    s->dt = dt;
    return 0;
}

int spdk_induction2d_step(spdk_induction2d* s) {
    if (!s) return fail(SPDK_E_ARG, "null argument");
    return s->esz == 8 ? enqueue_r<double>(s) : enqueue_r<float>(s);
}

int spdk_induction2d_get_stream(spdk_induction2d* s, void** stream) {
    if (!s || !stream) return fail(SPDK_E_ARG, "null argument");
    *stream = (void*)s->stream;
    return 0;
}

int spdk_induction2d_sync(spdk_induction2d* s) {
    if (!s) return fail(SPDK_E_ARG, "null argument");
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("induction2d sync: ") + cudaGetErrorString(e));
    return 0;
}

int spdk_induction2d_evolve(spdk_induction2d* s, double t_end, double dt_output, long long* steps, double* t_out) {
    if (!s) return fail(SPDK_E_ARG, "null argument");
    // Induction_ader::time_evolution (src/induction_ader.hpp:273-330): dt = Dt
    // each step, clamped to the next output time
    double t = 0, t_output = dt_output;
    long long k = 0;
    s->dt = s->Dt;
    while (t < t_end) {
        if (int rc = spdk_induction2d_step(s)) return rc;
        t += s->dt;
        k++;
        s->dt = s->Dt;
        if (dt_output > 0) {
            if (t >= t_output) t_output = t + dt_output;
            if (t + s->dt > t_output) s->dt = t_output - t;
        }
    }
    if (steps) *steps = k;
    if (t_out) *t_out = t;
    return spdk_induction2d_sync(s);
}

int spdk_induction2d_get_info(const spdk_induction2d* s, spdk_induction2d_info* info) {
    if (!s || !info) return fail(SPDK_E_ARG, "null argument");
    info->p = s->cfg.p;
    info->N[0] = s->cfg.N[0];
    info->N[1] = s->cfg.N[1];
    info->n_elements = s->E;
    info->n_face_values = 2 * s->E * s->n * s->nf;
    info->n_time_slices = s->nt;
    info->launches_per_step = s->nstages * s->nt;
    return 0;
}

int spdk_induction2d_read(spdk_induction2d* s, int field, double* host, size_t count) {
    if (!s || !host) return fail(SPDK_E_ARG, "null argument");
    const size_t state = (size_t)s->E * s->n * s->nf;
    if (field == SPDK_IND2_FIELD_BX || field == SPDK_IND2_FIELD_BY) {
        if (count != state) return fail(SPDK_E_ARG, "count must be E*n*(n+1) = " + std::to_string(state));
        const void* src = field == SPDK_IND2_FIELD_BX ? s->bx : s->by;
        if (s->esz == 8) {
            if (cudaMemcpyAsync(host, src, state * 8, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess)
                return fail(SPDK_E_CUDA, "induction2d read");
            return spdk_induction2d_sync(s);
        }
        std::vector<float> f(state);
        if (cudaMemcpyAsync(f.data(), src, state * 4, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess)
            return fail(SPDK_E_CUDA, "induction2d read");
        if (int rc = spdk_induction2d_sync(s)) return rc;
        for (size_t q = 0; q < state; q++) host[q] = f[q];
        return 0;
    }
    if (field == SPDK_IND2_FIELD_B2_CV) {
        const size_t cnt = (size_t)4 * s->E * s->n * s->n;
        if (count != cnt) return fail(SPDK_E_ARG, "count must be 4*E*n*n = " + std::to_string(cnt));
        const int rc = s->esz == 8 ? b2cv_r<double>(s) : b2cv_r<float>(s);
        if (rc) return rc;
        if (cudaMemcpyAsync(host, s->b2, cnt * sizeof(double), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess)
            return fail(SPDK_E_CUDA, "induction2d read");
        return spdk_induction2d_sync(s);
    }
    return fail(SPDK_E_ARG, "unknown field");
}

}  // extern "C"
