// Kernel table of one (ndim, p, tile) instantiation and the element-local
// set-up kernels. Instantiated in spdk_select_*.cu so the (ndim, p) variants
// compile in parallel.
#pragma once
#include <cuda_runtime.h>

#include "spdk_fallback.cuh"
#include "spdk_kernels.cuh"
#include "spdk_viscous.cuh"

namespace spdk {

// ---------------------------------------------------------------------------
// element-local set-up kernels
// ---------------------------------------------------------------------------
// U_sp = conservatives(cv_to_sp(W_cv)) and dt(W_cv): the constructor tail
// (src/hydro_ader.hpp:205-208)
template <typename R, int D, int P>
__global__ void __launch_bounds__(kThreads) init_state_kernel(DevGrid G, DevMatsT<R> M, const R* __restrict__ wcv,
                                                             R* __restrict__ u,
                                                             unsigned long long* dtmin) {
    using S = Shape<D, P>;
    constexpr int V = S::V, NPT = S::NPT;
    __shared__ R b0[V * NPT], b1[V * NPT];
    const long long ge = blockIdx.x;
    for (int q = threadIdx.x; q < V * NPT; q += blockDim.x) b0[q] = wcv[ge * V * NPT + q];
    __syncthreads();
    double dtl = 1.7976931348623157e308;
    for (int q = threadIdx.x; q < NPT; q += blockDim.x) {
        R w[V];
        for (int v = 0; v < V; v++) w[v] = b0[v * NPT + q];
        dtl = smin(dtl, point_dt<D>(G, w, S::n));
    }
    R* bufs[2] = {b1, b0};
    const R* src = b0;
    for (int d = 0; d < D; d++) {
        R* dst = bufs[d % 2];
        sweep_smem<D, P, R>(src, dst, M.cv_to_sp, d, V * NPT);
        __syncthreads();
        src = dst;
    }
    for (int q = threadIdx.x; q < NPT; q += blockDim.x) {
        R w[V], uu[V];
        for (int v = 0; v < V; v++) w[v] = src[v * NPT + q];
        conservatives<D>(w, uu, (R)G.gm);
        for (int v = 0; v < V; v++) u[ge * V * NPT + v * NPT + q] = uu[v];
    }
    block_min_dt(dtl, dtmin);
}

// W_cv = sp_to_cv(primitives(U_sp)) and dt, for a state written by the host
template <typename R, int D, int P>
__global__ void __launch_bounds__(kThreads) derive_kernel(DevGrid G, DevMatsT<R> M, const R* __restrict__ u,
                                                         R* __restrict__ wcv, unsigned long long* dtmin) {
    using S = Shape<D, P>;
    constexpr int V = S::V, NPT = S::NPT;
    __shared__ R b0[V * NPT], b1[V * NPT];
    const long long ge = blockIdx.x;
    for (int q = threadIdx.x; q < NPT; q += blockDim.x) {
        R uu[V], w[V];
        for (int v = 0; v < V; v++) uu[v] = u[ge * V * NPT + v * NPT + q];
        primitives<D>(uu, w, (R)G.gm);
        for (int v = 0; v < V; v++) b0[v * NPT + q] = w[v];
    }
    __syncthreads();
    R* bufs[2] = {b1, b0};
    const R* src = b0;
    for (int d = 0; d < D; d++) {
        R* dst = bufs[d % 2];
        sweep_smem<D, P, R>(src, dst, M.sp_to_cv, d, V * NPT);
        __syncthreads();
        src = dst;
    }
    double dtl = 1.7976931348623157e308;
    for (int q = threadIdx.x; q < NPT; q += blockDim.x) {
        R w[V];
        for (int v = 0; v < V; v++) {
            w[v] = src[v * NPT + q];
            wcv[ge * V * NPT + v * NPT + q] = w[v];
        }
        dtl = smin(dtl, point_dt<D>(G, w, S::n));
    }
    block_min_dt(dtl, dtmin);
}

// next dt <- reduced minimum, capped by the viscous diffusion limit when
// cap > 0 (src/hydro.cpp:245-254: every point's candidate is min(dt, cap),
// so the minimum over points is min(reduced, cap)); re-arm the reduction
static __global__ void advance_dt_kernel(double* dt, unsigned long long* dtmin, double cap) {
    pdl_wait();
    const double v = __longlong_as_double((long long)*dtmin);
    *dt = (cap > 0.0 && !(v < cap)) ? cap : v;
    *dtmin = 0x7FEFFFFFFFFFFFFFULL;
}

// The device-resident time loop's step end (src/hydro_ader.hpp:234-261):
// t += dt of the step, next dt from the reduction (viscous cap as above),
// dt clamped to the next output time, and the gate closed once t >= t_end.
// tb = {t, t_output, steps, t_end, dt_output (<= 0: no outputs)}; the same
// FP64 operations as the host loop, so the dt sequence is identical.
static __global__ void evolve_advance_kernel(double* dt, unsigned long long* dtmin, double cap, double* tb,
                                             int* gate) {
    pdl_wait();
    if (*gate) return;
    const double used = *dt;
    const double v = __longlong_as_double((long long)*dtmin);
    double next = (cap > 0.0 && !(v < cap)) ? cap : v;
    *dtmin = 0x7FEFFFFFFFFFFFFFULL;
    const double t = tb[0] + used;
    double t_output = tb[1];
    if (tb[4] > 0) {
        if (t >= t_output) t_output = t + tb[4];
        if (t + next > t_output) next = t_output - t;
    }
    *dt = next;
    tb[0] = t;
    tb[1] = t_output;
    tb[2] += 1.0;
    if (!(t < tb[3])) *gate = 1;
}

// per-element trouble labels of a step <- 0 (skipped once the gate is closed)
static __global__ void clear_labels_kernel(DevGrid G, uint8_t* labels, long long n) {
    pdl_wait();
    if (gate_closed(G)) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        labels[i] = 0;
}

// ---------------------------------------------------------------------------
// kernel table of one (R, D, P, tile) instantiation
// ---------------------------------------------------------------------------
template <typename R>
struct KernelSetT {
    void (*predict)(DevGrid, DevMatsT<R>, PicardArgsT<R>) = nullptr;
    void (*correct)(DevGrid, DevMatsT<R>, PicardArgsT<R>) = nullptr;
    void (*flux)(DevGrid, DevMatsT<R>, PicardArgsT<R>) = nullptr;
    void (*detect)(DevGrid, const double2*, const double2*, uint8_t*, int*) = nullptr;
    void (*update)(DevGrid, DevMatsT<R>, FallbackArgsT<R>) = nullptr;
    void (*init)(DevGrid, DevMatsT<R>, const R*, R*, unsigned long long*) = nullptr;
    void (*derive)(DevGrid, DevMatsT<R>, const R*, R*, unsigned long long*) = nullptr;
    void (*visc)(DevGrid, DevMatsT<R>, ViscArgsT<R>) = nullptr;
    size_t picard_smem = 0, update_smem = 0;
    int tile[3] = {1, 1, 1};
    int visc_epb = 1;  // elements per block of the viscous face kernel
};
using KernelSet = KernelSetT<double>;

template <typename R, int D, int P, int TX, int TY, int TZ, bool VISC = false>
KernelSetT<R> make_set() {
    KernelSetT<R> k;
    k.predict = picard_kernel<R, D, P, TX, TY, TZ, kPredict, VISC>;
    k.correct = picard_kernel<R, D, P, TX, TY, TZ, kCorrect, VISC>;
    k.flux = picard_kernel<R, D, P, TX, TY, TZ, kFlux, VISC>;
    k.detect = fv_detect_kernel<R, D, P, TX, TY, TZ>;
    k.update = fv_update_kernel<R, D, P, TX, TY, TZ>;
    k.init = init_state_kernel<R, D, P>;
    k.derive = derive_kernel<R, D, P>;
    k.visc = visc_face_kernel<R, D, P>;
    k.visc_epb = ViscShape<R, D, P>::EPB;
    k.picard_smem = picard_smem_bytes<R, D, P, TX, TY, TZ>();
    k.update_smem = UpdateSmem<R, D, P, TX, TY, TZ>::bytes;
    k.tile[0] = TX;
    k.tile[1] = TY;
    k.tile[2] = TZ;
    return k;
}

// Tile choice: the largest instantiated tile that divides the element counts.
// Viscous runs (VISC) take the same tiles with the viscous Picard passes.
template <typename R, int P, bool VISC>
bool pick2_t(int Nx, int Ny, KernelSetT<R>* k) {
    if constexpr (P <= 4) {
        if (Nx % 4 == 0 && Ny % 4 == 0) { *k = make_set<R, 2, P, 4, 4, 1, VISC>(); return true; }
    }
    if (Nx % 2 == 0 && Ny % 2 == 0) { *k = make_set<R, 2, P, 2, 2, 1, VISC>(); return true; }
    *k = make_set<R, 2, P, 1, 1, 1, VISC>();
    return true;
}
template <typename R, int P>
bool pick2(int Nx, int Ny, KernelSetT<R>* k, bool visc) {
    return visc ? pick2_t<R, P, true>(Nx, Ny, k) : pick2_t<R, P, false>(Nx, Ny, k);
}
// 3D: one element per tile, or 2x1x1 elements at p <= 3, where one
// element's (p+1)^3 points would leave most of the block idle in the
// per-point phases; the FP64 form takes 2x2x1 elements at p = 2, 3 when
// nx1 and nx2 are even
template <typename R, int P>
bool pick3(int Nx, int Ny, int, KernelSetT<R>* k, bool visc) {
    if (visc) {
        *k = make_set<R, 3, P, 1, 1, 1, true>();
        return true;
    }
    if constexpr (sizeof(R) == 8 && (P == 2 || P == 3)) {
        if (Nx % 2 == 0 && Ny % 2 == 0) {
            *k = make_set<R, 3, P, 2, 2, 1>();
            return true;
        }
    }
    if constexpr (P <= 3) {
        if (Nx % 2 == 0) {
            *k = make_set<R, 3, P, 2, 1, 1>();
            return true;
        }
    }
    *k = make_set<R, 3, P, 1, 1, 1>();
    return true;
}

// per-translation-unit selectors (spdk_select_*.cu): the FP64 units are
// compiled without FMA contraction (reference rounding), the FP32 units with it
bool select_2d_low(int p, const int N[3], KernelSetT<double>* k, bool visc);   // p = 1..3
bool select_2d_high(int p, const int N[3], KernelSetT<double>* k, bool visc);  // p = 4..7
bool select_3d(int p, const int N[3], KernelSetT<double>* k, bool visc);       // p = 1..5
bool select_f32_2d(int p, const int N[3], KernelSetT<float>* k, bool visc);    // p = 1..7
bool select_f32_3d(int p, const int N[3], KernelSetT<float>* k, bool visc);    // p = 1..5

inline bool select_kernels(int D, int p, const int N[3], KernelSetT<double>* k, bool visc = false) {
    if (D == 2) return p <= 3 ? select_2d_low(p, N, k, visc) : select_2d_high(p, N, k, visc);
    if (D == 3) return select_3d(p, N, k, visc);
    return false;
}
inline bool select_kernels(int D, int p, const int N[3], KernelSetT<float>* k, bool visc = false) {
    if (D == 2) return select_f32_2d(p, N, k, visc);
    if (D == 3) return select_f32_3d(p, N, k, visc);
    return false;
}

}  // namespace spdk
