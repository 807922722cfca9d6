// spd_K B200 hydro solver: device state, step orchestration and the C ABI
// declared in include/spdk.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "spdk.h"
#include "spdk_learned.h"
#include "spdk_learned_impl.h"
#include "spdk_kernelset.cuh"
#include "spdk_setup.h"

namespace spdk {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define SPDK_CUDA(call)                                                                  \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(SPDK_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

}  // namespace spdk

using namespace spdk;

#include "spdk_hydro_impl.h"

namespace {

// device-detected faults: a bounded wait that ran out sets a status bit
int check_status(spdk_hydro* h) {
    int st = 0;
    cudaError_t e = cudaMemcpyAsync(&st, h->status, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("status read: ") + cudaGetErrorString(e));
    if (st & kStatusStagingTimeout) return fail(1, "a shared-memory staging wait timed out on the device");
    return 0;
}

int dalloc(spdk_hydro* h, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess)
        return fail(SPDK_E_NOMEM, "cudaMalloc(" + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    h->bytes += bytes;
    return 0;
}

// open / close an event bracket around one launch when profiling
void prof_begin(spdk_hydro* h) {
    if (!h->profiling) return;
    if (h->ev_used + 2 > h->ev.size()) {
        for (int q = 0; q < 64; q++) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            h->ev.push_back(e);
        }
    }
    cudaEventRecord(h->ev[h->ev_used], h->stream);
}
void prof_end(spdk_hydro* h, int kind) {
    if (!h->profiling) return;
    cudaEventRecord(h->ev[h->ev_used + 1], h->stream);
    h->ev_kind.push_back(kind);
    h->ev_used += 2;
}

// a launch of one of the step's kernels with programmatic stream
// serialization: it may be scheduled while the previous kernel on the stream
// drains, and waits (pdl_wait) before it reads anything
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

unsigned grid_blocks(const spdk_hydro* h) {
    long long b = 1;
    for (int d = 0; d < h->D; d++) b *= h->G.N[d] / h->tile[d];
    return (unsigned)b;
}

// launches of one step, recorded on h->stream (also used for capture)
template <typename R>
int enqueue_step_t(spdk_hydro* h, const KernelSetT<R>& k, const DevMatsT<R>& dm) {
    const unsigned blocks = grid_blocks(h);
    int launches = 0;
    // viscous face fluxes of a pass's input, written just before the pass
    auto viscous = [&](PicardArgsT<R>& A) -> int {
        if (!h->vg[0]) return 0;
        ViscArgsT<R> V{};
        V.ua_in = A.ua_in;
        V.in_slices = A.in_slices;
        for (int d = 0; d < 3; d++) {
            V.vg[d] = (R*)h->vg[d];
            A.vg[d] = (const R*)h->vg[d];
        }
        const dim3 grid((unsigned)((h->E + k.visc_epb - 1) / k.visc_epb), (unsigned)(A.in_slices > 1 ? h->nt : 1));
        prof_begin(h);
        SPDK_CUDA(launch_pdl(k.visc, grid, dim3(kViscThreads), 0, h->stream, h->G, dm, V));
        prof_end(h, SPDK_KERNEL_OTHER);
        launches++;
        return 0;
    };
    R* const ua[2] = {(R*)h->ua[0], (R*)h->ua[1]};
    R* const ucv[2] = {(R*)h->ucv[0], (R*)h->ucv[1]};
    if (h->nstages > 1)
        SPDK_CUDA(cudaMemcpyAsync(h->u0, h->u, (size_t)h->E * h->V * h->NPT * sizeof(R),
                                  cudaMemcpyDeviceToDevice, h->stream));
    for (int s = 0; s < h->nstages; s++) {
        const bool final_stage = s == h->nstages - 1;
        PicardArgsT<R> A{};
        A.u = (const R*)h->u;
        A.dt = h->dt;
        const R* in = (const R*)h->u;
        int in_slices = 1;
        if (h->nt == 1 && !h->cfg.fallback) {
            // an RK stage updates U in place, so the stage reads its halo
            // from a copy (the reference's copy_ader into U_ader_sp)
            SPDK_CUDA(cudaMemcpyAsync(h->ua[0], h->u, (size_t)h->E * h->V * h->NPT * sizeof(R),
                                      cudaMemcpyDeviceToDevice, h->stream));
            in = ua[0];
        }
        // Picard predictor passes (ADER only: nt = p+1)
        for (int it = 0; it + 1 < h->nt; it++) {
            A.ua_in = in;
            A.in_slices = in_slices;
            A.ua_out = ua[it % 2];
            if (int rc = viscous(A)) return rc;
            prof_begin(h);
            SPDK_CUDA(launch_pdl(k.predict, dim3(blocks), dim3(kThreads), k.picard_smem, h->stream, h->G, dm, A));
            prof_end(h, SPDK_KERNEL_PREDICT);
            launches++;
            in = ua[it % 2];
            in_slices = h->nt;
        }
        A.ua_in = in;
        A.in_slices = in_slices;
        if (int rc = viscous(A)) return rc;
        if (!h->cfg.fallback) {
            A.u_out = (R*)h->u;
            A.u0 = (const R*)h->u0;
            A.rk_a = h->rk_a[s];
            A.final_stage = final_stage;
            A.wcv = (R*)h->wcv;
            A.dtmin = h->dtmin;
            prof_begin(h);
            SPDK_CUDA(launch_pdl(k.correct, dim3(blocks), dim3(kThreads), k.picard_smem, h->stream, h->G, dm, A));
            prof_end(h, SPDK_KERNEL_CORRECT);
            launches++;
        } else {
            for (int d = 0; d < 3; d++) A.ff[d] = (R*)h->ff[d];
            A.ucv = ucv[0];
            A.rp_old = h->rpo;
            A.rp_new = h->rpn;
            prof_begin(h);
            SPDK_CUDA(launch_pdl(k.flux, dim3(blocks), dim3(kThreads), k.picard_smem, h->stream, h->G, dm, A));
            prof_end(h, SPDK_KERNEL_FLUX);
            launches++;
            if (h->join_pending) {
                SPDK_CUDA(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
                h->join_pending = false;
            }
            for (int t = 0; t < h->nt; t++) {
                prof_begin(h);
                SPDK_CUDA(launch_pdl(k.detect, dim3(blocks), dim3(kThreads), 0, h->stream, h->G,
                                     (const double2*)h->rpo, (const double2*)h->rpn, h->trouble, (int*)nullptr));
                prof_end(h, SPDK_KERNEL_DETECT);
                FallbackArgsT<R> F{};
                F.ucv_in = ucv[t % 2];
                F.ucv_out = ucv[(t + 1) % 2];
                F.ff0 = (R*)h->ff[0];
                F.ff1 = (R*)h->ff[1];
                F.ff2 = (R*)h->ff[2];
                F.rp_old = h->rpo;
                F.rp_new = h->rpn;
                F.rp_old_next = h->rpo;
                F.rp_new_next = h->rpn;
                F.trouble = h->trouble;
                F.theta = h->theta;
                F.t = t;
                F.last = t == h->nt - 1;
                F.u = (R*)h->u;
                F.u0 = (const R*)h->u0;
                F.rk_a = h->rk_a[s];
                F.final_stage = final_stage;
                F.wcv = (R*)h->wcv;
                F.dtmin = h->dtmin;
                F.dt = h->dt;
                if (h->mlp && final_stage && t == h->nt - 1) {
                    F.feat = h->feat;
                    F.means = h->means;
                    F.n_in = 2 * h->NPT + 4 * h->D;
                }
                prof_begin(h);
                SPDK_CUDA(launch_pdl(k.update, dim3(blocks), dim3(kThreads), k.update_smem, h->stream, h->G, dm, F));
                prof_end(h, SPDK_KERNEL_UPDATE);
                launches += 2;
            }
        }
    }
    prof_begin(h);
    if (h->evolve_mode)
        SPDK_CUDA(launch_pdl(evolve_advance_kernel, dim3(1), dim3(1), 0, h->stream, h->dt, h->dtmin, h->dt_cap, h->tb,
                             h->gate));
    else SPDK_CUDA(launch_pdl(advance_dt_kernel, dim3(1), dim3(1), 0, h->stream, h->dt, h->dtmin, h->dt_cap));
    prof_end(h, SPDK_KERNEL_OTHER);
    launches++;
    h->launches = launches;
    SPDK_CUDA(cudaGetLastError());
    return 0;
}

// the indicator's nodal features and element means of the current U, when
// no step has left them (after creation, a write of U, or steps without the
// indicator)
int refresh_features(spdk_hydro* h) {
    if (!h->mlp || h->feat_valid) return 0;
    const int N[3] = {h->G.N[0], h->G.N[1], h->G.N[2]};
    const int rc = feature_rows(h->u, h->prec == SPDK_PRECISION_FP32, h->D, h->p, N, h->G.bc, h->G.gm, h->E,
                                h->means, h->feat, h->stream);
    if (!rc) h->feat_valid = true;
    return rc;
}

int enqueue_step(spdk_hydro* h) {
    if (h->elem_trouble) {
        clear_labels_kernel<<<(unsigned)std::min<long long>((h->E + 255) / 256, 1024), 256, 0, h->stream>>>(
            h->G, h->elem_trouble, h->E);
        SPDK_CUDA(cudaGetLastError());
    }
    if (h->mlp) {
        if (int rc = refresh_features(h)) return rc;
        // a-priori flags of the state at the start of the step, on the side
        // stream, from the features the previous step's last update stored
        // (they are not written again before the step's last update)
        SPDK_CUDA(cudaEventRecord(h->ev_fork, h->stream));
        SPDK_CUDA(cudaStreamWaitEvent(h->side, h->ev_fork, 0));
        const int N[3] = {h->G.N[0], h->G.N[1], h->G.N[2]};
        const int rc = indicator_flags(h->mlp, h->feat, h->means, h->D, h->p, N, h->G.bc, h->E, h->elem_pred, h->thr,
                                       h->side, h->G.gate);
        if (rc) return rc;
        SPDK_CUDA(cudaEventRecord(h->ev_join, h->side));
        h->join_pending = true;
    }
    const int rc = h->prec == SPDK_PRECISION_FP32 ? enqueue_step_t<float>(h, h->ks32, h->dm32)
                                                  : enqueue_step_t<double>(h, h->ks64, h->dm64);
    h->feat_valid = !rc && h->mlp != nullptr;
    return rc;
}

// dt candidates of the W_cv points of elements [e_lo, e_hi) (a slab's owned
// rows), the same per-point formula as the step's epilogues
template <typename R, int D>
__global__ void __launch_bounds__(kThreads) slab_dt_kernel(DevGrid G, const R* __restrict__ wcv, long long e_lo,
                                                          long long e_hi, int n, int NPT,
                                                          unsigned long long* dtmin) {
    constexpr int V = D + 2;
    double dtl = 1.7976931348623157e308;
    const long long cnt = (e_hi - e_lo) * NPT;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < cnt;
         q += (long long)gridDim.x * blockDim.x) {
        const long long e = e_lo + q / NPT;
        const int pt = (int)(q % NPT);
        R w[V];
#pragma unroll
        for (int v = 0; v < V; v++) w[v] = wcv[(e * V + v) * NPT + pt];
        dtl = smin(dtl, point_dt<D>(G, w, n));
    }
    block_min_dt(dtl, dtmin);
}

__global__ void widen_kernel(const float* __restrict__ a, double* __restrict__ b, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

// the precision form's host exchange buffer: doubles, converted on the
// device (allocated on the first read or write of a state field)
int ensure_stage(spdk_hydro* h) {
    if (h->stage) return 0;
    return dalloc(h, &h->stage, (size_t)h->E * h->V * h->NPT * sizeof(double));
}

__global__ void narrow_kernel(const double* __restrict__ a, float* __restrict__ b, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// per-kernel attributes: dynamic shared memory and the full carveout
template <typename R>
int set_attributes(const KernelSetT<R>& ks) {
    const void* fns[] = {(const void*)ks.predict, (const void*)ks.correct, (const void*)ks.flux};
    for (const void* f : fns) {
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ks.picard_smem) != cudaSuccess)
            return fail(SPDK_E_CUDA, "shared memory request of " + std::to_string(ks.picard_smem) + " bytes");
        // the whole unified L1/shared array as shared memory: residency is
        // limited by shared memory, not by L1 (staging goes through TMA)
        cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    }
    cudaFuncSetAttribute((const void*)ks.update, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (cudaFuncSetAttribute((const void*)ks.update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ks.update_smem) != cudaSuccess)
        return fail(SPDK_E_CUDA, "shared memory request of " + std::to_string(ks.update_smem) + " bytes");
    return 0;
}

void release(spdk_hydro* h) {
    checkpoint_release(h);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    if (h->graph_evolve) cudaGraphExecDestroy(h->graph_evolve);
    for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
    void* ptrs[] = {h->u, h->ua[0], h->ua[1], h->u0, h->ucv[0], h->ucv[1], h->ff[0], h->ff[1], h->ff[2],
                    h->wcv, h->dt, h->fvf[0], h->fvf[1], h->fvf[2], h->fvc[0], h->fvc[1], h->fvc[2],
                    h->rpo, h->rpn, h->trouble, h->theta, h->dtmin, h->status, h->elem_trouble, h->elem_pred,
                    h->feat, h->means, h->vg[0], h->vg[1], h->vg[2], h->gate, h->tb, h->stage};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->stream) cudaStreamDestroy(h->stream);
}

}  // namespace

extern "C" {

const char* spdk_last_error(void) { return spdk::g_last_error.c_str(); }
int spdk_abi_version(void) { return SPDK_ABI_VERSION; }

int spdk_hydro_create(const spdk_hydro_config* cfg, spdk_hydro** out) {
    if (!cfg || !out) return fail(SPDK_E_ARG, "null argument");
    *out = nullptr;
    const spdk_hydro_config& c = *cfg;
    if (c.p < 1 || c.p > kMaxP) return fail(SPDK_E_ARG, "p must be in 1..7");
    if (c.N[0] < 2 || c.N[1] < 2) return fail(SPDK_E_ARG, "x and y must be active (nx1, nx2 > 1)");
    const int D = c.N[2] > 1 ? 3 : 2;
    if (D == 3 && c.p > 5) return fail(SPDK_E_ARG, "3D runs support p <= 5");
    if (D == 2 && (c.g[2] != 0.0 || ((c.problem == SPDK_IC_SINE_WAVE || c.problem == SPDK_IC_SQUARE) && c.v3 != 0.0)))
        return fail(SPDK_E_ARG, "a 2D run cannot carry z momentum or z gravity");
    if (c.precision != SPDK_PRECISION_FP64 && c.precision != SPDK_PRECISION_FP32)
        return fail(SPDK_E_ARG, "unsupported precision");
    for (int d = 0; d < D; d++)
        if (c.bc[d] < 0 || c.bc[d] > 2) return fail(SPDK_E_ARG, "bad boundary type");
    if (c.integrator == SPDK_INTEGRATOR_RK && (c.rk_order < 1 || c.rk_order > 3))
        return fail(SPDK_E_ARG, "rk_order must be 1, 2 or 3");
    if (!(c.nu >= 0.0) || !std::isfinite(c.nu) || !std::isfinite(c.beta))
        return fail(SPDK_E_ARG, "nu must be >= 0 and nu, beta finite");
    if (c.slab_n != 0 || c.slab_lo != 0) {
        const int rows = c.N[D - 1];
        if (c.slab_lo < 0 || c.slab_n < rows || c.slab_lo + rows > c.slab_n)
            return fail(SPDK_E_ARG, "slab rows [slab_lo, slab_lo + N) must lie inside the slab_n rows of the domain");
        if (c.bc[D - 1] == SPDK_BC_PERIODIC)
            return fail(SPDK_E_ARG, "the slab axis (y in 2D, z in 3D) needs a non-periodic boundary");
    }

    spdk_hydro* h = new spdk_hydro();
    h->cfg = c;
    h->D = D;
    h->p = c.p;
    h->n = c.p + 1;
    h->nf = c.p + 2;
    h->V = D + 2;
    h->NPT = D == 2 ? h->n * h->n : h->n * h->n * h->n;
    const bool ader = c.integrator == SPDK_INTEGRATOR_ADER;
    h->nt = ader ? c.p + 1 : 1;
    h->nstages = 1;
    if (!ader) {
        h->nstages = c.rk_order;
        if (c.rk_order == 2) h->rk_a[1] = 0.5;
        if (c.rk_order == 3) { h->rk_a[1] = 0.75; h->rk_a[2] = 1.0 / 3.0; }
    }
    int N[3] = {c.N[0], c.N[1], D == 3 ? c.N[2] : 1};
    h->prec = c.precision;
    h->esz = h->prec == SPDK_PRECISION_FP32 ? sizeof(float) : sizeof(double);
    const bool visc = c.nu > 0.0;
    if (!select_kernels(D, c.p, N, &h->ks64, visc) ||
        (h->prec == SPDK_PRECISION_FP32 && !select_kernels(D, c.p, N, &h->ks32, visc))) {
        delete h;
        return fail(SPDK_E_ARG, "no kernel instantiation for this ndim/p");
    }
    // the step kernels' tile (their launch grid): the kernel set of the run's
    // arithmetic; the FP64 set of an FP32 run only serves the element-local
    // set-up kernels, and the two sets may choose different tiles
    for (int d = 0; d < 3; d++)
        h->tile[d] = h->prec == SPDK_PRECISION_FP32 ? h->ks32.tile[d] : h->ks64.tile[d];
    int rc = cudaSetDevice(c.device) == cudaSuccess ? 0 : fail(SPDK_E_CUDA, "cudaSetDevice failed");
    if (rc) { delete h; return rc; }
    build_matrices(c.p, ader, &h->mats);
    for (int d = 0; d < 3; d++) {
        const bool slab = d == D - 1 && c.slab_n > 0;
        build_axis(N[d], c.p, c.L[d], h->mats.x_fp, d < D, &h->ax[d], slab ? c.slab_lo : 0, slab ? c.slab_n : 0);
    }
    // device matrices (same values as the host setup)
    const int n = h->n, nf = h->nf;
    std::memset(&h->dm64, 0, sizeof(h->dm64));
    for (int j = 0; j < nf; j++)
        for (int i = 0; i < n; i++) h->dm64.sp_to_fp[j * n + i] = h->mats.sp_to_fp[j * n + i];
    for (int j = 0; j < n; j++)
        for (int i = 0; i < nf; i++) h->dm64.dfp_to_sp[j * nf + i] = h->mats.dfp_to_sp[j * nf + i];
    for (int q = 0; q < n * n; q++) {
        h->dm64.sp_to_cv[q] = h->mats.sp_to_cv[q];
        h->dm64.cv_to_sp[q] = h->mats.cv_to_sp[q];
    }
    for (int q = 0; q < h->nt * h->nt; q++) h->dm64.invader[q] = h->mats.invader[q];
    for (int q = 0; q < h->nt; q++) h->dm64.wt[q] = h->mats.wt[q];
    {
        // the precision form's matrices: the FP64 values rounded once
        const double* src = (const double*)&h->dm64;
        float* dst = (float*)&h->dm32;
        for (size_t q = 0; q < sizeof(h->dm64) / sizeof(double); q++) dst[q] = (float)src[q];
    }
    // grid
    DevGrid& G = h->G;
    h->E = (long long)N[0] * N[1] * N[2];
    for (int d = 0; d < 3; d++) {
        G.N[d] = N[d];
        G.bc[d] = c.bc[d];
        G.h[d] = h->ax[d].h;
        int ex = 0;
        const double m = std::frexp(G.h[d], &ex);
        G.pow2[d] = (m == 0.5) ? 1 : 0;
        G.rh[d] = G.pow2[d] ? std::ldexp(1.0, 1 - ex) : 0.0;
        G.g[d] = c.g[d];
    }
    G.uniform_pow2 = 1;
    for (int d = 0; d < D; d++)
        if (!G.pow2[d] || G.h[d] != G.h[0]) G.uniform_pow2 = 0;
    G.gm = c.gamma;
    G.cfl = c.cfl;
    G.grav = (c.g[0] != 0.0 || c.g[1] != 0.0 || c.g[2] != 0.0) ? 1 : 0;
    G.nt = h->nt;
    G.E = h->E;
    G.nad_tol = c.nad_tolerance;
    G.nad_delta = c.nad_delta;
    G.nad_moore = c.nad_moore;
    G.use_sed = (c.sed && c.p > 1) ? 1 : 0;
    G.blending = c.blending;
    G.nu = c.nu;
    G.beta = c.beta;
    if (c.nu > 0.0) {
        // src/hydro.cpp:230-254: dx_min over the active directions (from 1),
        // the diffusion limit 0.25 cfl (dx_min/(p+1))^2 / nu
        double dxmin = 1;
        for (int d = 0; d < D; d++) dxmin = G.h[d] < dxmin ? G.h[d] : dxmin;
        const double dx_sub = dxmin / h->n;
        h->dt_cap = 0.25 * c.cfl * dx_sub * dx_sub / c.nu;
    }

    const size_t state = (size_t)h->E * h->V * h->NPT * h->esz;
    const size_t state64 = (size_t)h->E * h->V * h->NPT * sizeof(double);
    rc = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess
             ? 0 : fail(SPDK_E_CUDA, "cudaStreamCreate failed");
    if (!rc) rc = dalloc(h, (void**)&h->u, state);
    if (!rc && h->nt > 1) {
        rc = dalloc(h, (void**)&h->ua[0], state * h->nt);
        if (!rc) rc = dalloc(h, (void**)&h->ua[1], state * h->nt);
    } else if (!rc && !c.fallback) {
        rc = dalloc(h, (void**)&h->ua[0], state);  // RK stage input copy
    }
    if (!rc && h->nstages > 1) rc = dalloc(h, (void**)&h->u0, state);
    if (!rc) rc = dalloc(h, (void**)&h->wcv, state);
    if (!rc) rc = dalloc(h, (void**)&h->dt, sizeof(double) * 2);
    if (!rc) rc = dalloc(h, (void**)&h->dtmin, sizeof(unsigned long long));
    if (!rc) rc = dalloc(h, (void**)&h->status, sizeof(int));
    if (!rc) rc = dalloc(h, (void**)&h->gate, sizeof(int));
    if (!rc) rc = dalloc(h, (void**)&h->tb, 8 * sizeof(double));
    if (!rc && cudaMemset(h->gate, 0, sizeof(int)) != cudaSuccess) rc = fail(SPDK_E_CUDA, "memset gate");
    if (!rc && cudaMemset(h->status, 0, sizeof(int)) != cudaSuccess) rc = fail(SPDK_E_CUDA, "memset status");
    G.status = h->status;
    if (!rc && c.fallback) {
        const size_t ffb = (size_t)h->nt * h->E * h->V * (h->NPT / h->n) * h->nf * h->esz;
        for (int d = 0; d < D && !rc; d++) rc = dalloc(h, (void**)&h->ff[d], ffb);
        if (!rc) rc = dalloc(h, (void**)&h->ucv[0], state);
        if (!rc) rc = dalloc(h, (void**)&h->ucv[1], state);
        if (!rc) rc = dalloc(h, (void**)&h->rpo, (size_t)h->E * h->NPT * sizeof(double2));
        if (!rc) rc = dalloc(h, (void**)&h->rpn, (size_t)h->E * h->NPT * sizeof(double2));
        if (!rc) rc = dalloc(h, (void**)&h->trouble, (size_t)h->E * h->NPT);
        if (!rc) rc = dalloc(h, (void**)&h->theta, (size_t)h->E * h->NPT);
        if (!rc) rc = dalloc(h, (void**)&h->elem_trouble, (size_t)h->E);
        if (!rc && cudaMemset(h->elem_trouble, 0, (size_t)h->E) != cudaSuccess) rc = fail(SPDK_E_CUDA, "memset");
        G.elem_trouble = h->elem_trouble;
        for (int d = 0; d < D && !rc; d++) {
            rc = dalloc(h, (void**)&h->fvf[d], h->ax[d].fv_faces.size() * sizeof(double));
            if (!rc) rc = dalloc(h, (void**)&h->fvc[d], h->ax[d].fv_centers.size() * sizeof(double));
            if (!rc && cudaMemcpy(h->fvf[d], h->ax[d].fv_faces.data(), h->ax[d].fv_faces.size() * sizeof(double),
                                  cudaMemcpyHostToDevice) != cudaSuccess)
                rc = fail(SPDK_E_CUDA, "upload fv_faces");
            if (!rc && cudaMemcpy(h->fvc[d], h->ax[d].fv_centers.data(),
                                  h->ax[d].fv_centers.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
                rc = fail(SPDK_E_CUDA, "upload fv_centers");
            G.fvf[d] = h->fvf[d];
            G.fvc[d] = h->fvc[d];
        }
        if (!rc && cudaMemset(h->trouble, 0, (size_t)h->E * h->NPT) != cudaSuccess)
            rc = fail(SPDK_E_CUDA, "memset");
        if (!rc && cudaMemset(h->theta, 0, (size_t)h->E * h->NPT) != cudaSuccess) rc = fail(SPDK_E_CUDA, "memset");
    }
    if (!rc && c.nu > 0.0) {
        const size_t vgb = (size_t)h->nt * h->E * 2 * h->V * (h->NPT / h->n) * h->esz;
        for (int d = 0; d < D && !rc; d++) rc = dalloc(h, &h->vg[d], vgb);
    }
    if (!rc) rc = h->prec == SPDK_PRECISION_FP32 ? set_attributes(h->ks32) : set_attributes(h->ks64);
    if (!rc) {
        // initial condition on the host (transcendentals through the same
        // libm as the reference), U_sp and dt on the device in FP64; the
        // precision form starts from that state rounded once to FP32
        std::vector<double> w0;
        initial_wcv(c, h->mats, h->ax, D, &w0);
        double *w64 = nullptr, *u64 = nullptr;
        if (cudaMalloc((void**)&w64, state64) != cudaSuccess || cudaMalloc((void**)&u64, state64) != cudaSuccess)
            rc = fail(SPDK_E_NOMEM, "set-up buffers");
        if (!rc && cudaMemcpy(w64, w0.data(), state64, cudaMemcpyHostToDevice) != cudaSuccess)
            rc = fail(SPDK_E_CUDA, "upload W_cv");
        if (!rc) {
            const unsigned long long maxbits = 0x7FEFFFFFFFFFFFFFULL;
            cudaMemcpy(h->dtmin, &maxbits, sizeof(maxbits), cudaMemcpyHostToDevice);
            h->ks64.init<<<(unsigned)h->E, kThreads, 0, h->stream>>>(h->G, h->dm64, w64, u64, h->dtmin);
            advance_dt_kernel<<<1, 1, 0, h->stream>>>(h->dt, h->dtmin, h->dt_cap);
            const long long nv = h->E * h->V * h->NPT;
            if (h->prec == SPDK_PRECISION_FP32) {
                narrow_kernel<<<1024, 256, 0, h->stream>>>(u64, (float*)h->u, nv);
                narrow_kernel<<<1024, 256, 0, h->stream>>>(w64, (float*)h->wcv, nv);
            } else {
                cudaMemcpyAsync(h->u, u64, state64, cudaMemcpyDeviceToDevice, h->stream);
                cudaMemcpyAsync(h->wcv, w64, state64, cudaMemcpyDeviceToDevice, h->stream);
            }
            cudaError_t e = cudaStreamSynchronize(h->stream);
            if (e != cudaSuccess) rc = fail(SPDK_E_CUDA, std::string("init: ") + cudaGetErrorString(e));
        }
        if (w64) cudaFree(w64);
        if (u64) cudaFree(u64);
    }
    if (rc) {
        release(h);
        delete h;
        return rc;
    }
    *out = h;
    return 0;
}

int spdk_hydro_destroy(spdk_hydro* h) {
    if (!h) return 0;
    cudaStreamSynchronize(h->stream);
    release(h);
    delete h;
    return 0;
}

int spdk_hydro_get_info(const spdk_hydro* h, spdk_hydro_info* info) {
    if (!h || !info) return fail(SPDK_E_ARG, "null argument");
    info->ndim = h->D;
    info->p = h->p;
    info->n_points = h->NPT;
    info->nvar = h->V;
    for (int d = 0; d < 3; d++) info->N[d] = h->G.N[d];
    info->n_elements = h->E;
    info->n_dof = h->E * h->NPT;
    info->n_time_slices = h->nt;
    int l = 0;
    for (int s = 0; s < h->nstages; s++) l += (h->nt - 1) + (h->cfg.fallback ? 1 + 2 * h->nt : 1);
    if (h->vg[0]) l += h->nstages * h->nt;  // a viscous pre-pass before every Picard pass
    info->launches_per_step = l + 1 + (h->mlp ? 2 : 0) + (h->elem_trouble ? 1 : 0);
    info->device_bytes = h->bytes;
    return 0;
}

int spdk_hydro_get_dt(spdk_hydro* h, double* dt) {
    if (!h || !dt) return fail(SPDK_E_ARG, "null argument");
    SPDK_CUDA(cudaMemcpyAsync(dt, h->dt, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    SPDK_CUDA(cudaStreamSynchronize(h->stream));
    return check_status(h);
}

int spdk_hydro_set_dt(spdk_hydro* h, double dt) {
    if (!h) return fail(SPDK_E_ARG, "null argument");
    SPDK_CUDA(cudaMemcpyAsync(h->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    SPDK_CUDA(cudaStreamSynchronize(h->stream));
    return 0;
}

int spdk_hydro_step(spdk_hydro* h) {
    if (!h) return fail(SPDK_E_ARG, "null argument");
    return enqueue_step(h);
}

int spdk_hydro_steps(spdk_hydro* h, int nsteps) {
    if (!h || nsteps < 0) return fail(SPDK_E_ARG, "bad argument");
    if (nsteps == 0) return 0;
    if (!h->graph) {
        // features the captured step does not compute itself are formed
        // before the capture, so every replay finds them current
        if (int rc = refresh_features(h)) return rc;
        // capture one step; replays reuse the same device pointers
        cudaGraph_t g;
        SPDK_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_step(h);
        cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&h->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
    }
    if (int rc = refresh_features(h)) return rc;
    for (int s = 0; s < nsteps; s++) SPDK_CUDA(cudaGraphLaunch(h->graph, h->stream));
    return 0;
}

int spdk_hydro_get_stream(spdk_hydro* h, void** stream) {
    if (!h || !stream) return fail(SPDK_E_ARG, "null argument");
    *stream = (void*)h->stream;
    return 0;
}

int spdk_hydro_profile(spdk_hydro* h, int nsteps, double* ms, long long* launches) {
    if (!h || !ms || !launches || nsteps < 0) return fail(SPDK_E_ARG, "bad argument");
    h->profiling = true;
    h->ev_used = 0;
    h->ev_kind.clear();
    int rc = 0;
    for (int s = 0; s < nsteps && !rc; s++) {
        rc = enqueue_step(h);
        if (!rc && cudaStreamSynchronize(h->stream) != cudaSuccess) rc = fail(SPDK_E_CUDA, "profile sync");
        for (size_t q = 0; q < h->ev_kind.size() && !rc; q++) {
            float t = 0;
            if (cudaEventElapsedTime(&t, h->ev[2 * q], h->ev[2 * q + 1]) != cudaSuccess)
                rc = fail(SPDK_E_CUDA, "event timing");
            ms[h->ev_kind[q]] += t;
            launches[h->ev_kind[q]] += 1;
        }
        h->ev_used = 0;
        h->ev_kind.clear();
    }
    h->profiling = false;
    return rc;
}

int spdk_hydro_sync(spdk_hydro* h) {
    if (!h) return fail(SPDK_E_ARG, "null argument");
    SPDK_CUDA(cudaStreamSynchronize(h->stream));
    return check_status(h);
}

int spdk_hydro_evolve(spdk_hydro* h, double t_end, double dt_output, long long* steps, double* t_out) {
    return spdk_hydro_evolve_from(h, 0.0, dt_output, t_end, dt_output, steps, t_out);
}

int spdk_hydro_evolve_from(spdk_hydro* h, double t0, double t_output0, double t_end, double dt_output,
                           long long* steps, double* t_out) {
    if (!h) return fail(SPDK_E_ARG, "null argument");
    // src/hydro_ader.hpp:215-273 as a device-resident loop: the step's dt,
    // t, the output clamping and the stop test live on the device
    // (evolve_advance_kernel, the host loop's operations), so the host
    // launches captured steps in batches and reads the loop state once per
    // batch instead of once per step. Steps launched after t reaches t_end
    // find the gate closed and do nothing.
    if (steps) *steps = 0;
    if (t_out) *t_out = t0;
    if (!(t0 < t_end)) return 0;
    if (int rc = refresh_features(h)) return rc;
    if (!h->graph_evolve) {
        cudaGraph_t g;
        DevGrid keep = h->G;
        h->G.gate = h->gate;
        h->evolve_mode = true;
        SPDK_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_step(h);
        cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        h->evolve_mode = false;
        h->G = keep;
        if (rc) return rc;
        if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&h->graph_evolve, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
    }
    const double tb0[5] = {t0, t_output0, 0.0, t_end, dt_output > 0 ? dt_output : -1.0};
    SPDK_CUDA(cudaMemcpyAsync(h->tb, tb0, sizeof(tb0), cudaMemcpyHostToDevice, h->stream));
    SPDK_CUDA(cudaMemsetAsync(h->gate, 0, sizeof(int), h->stream));
    // loop state read back after every batch: t, t_output, steps, and the
    // next dt, from which the next batch's length is estimated as the steps
    // the remaining time takes at that dt (a shrinking dt needs another
    // batch; a growing one leaves a few gated no-op replays)
    double st[3] = {t0, t_output0, 0};
    double dt_now = 0;
    SPDK_CUDA(cudaMemcpyAsync(&dt_now, h->dt, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    SPDK_CUDA(cudaStreamSynchronize(h->stream));
    int closed = 0;
    while (!closed) {
        double est = dt_now > 0 ? std::ceil((t_end - st[0]) / dt_now) : 1.0;
        if (!(est >= 1.0)) est = 1.0;
        const int batch = (int)std::min(est, 256.0);
        for (int q = 0; q < batch; q++) SPDK_CUDA(cudaGraphLaunch(h->graph_evolve, h->stream));
        SPDK_CUDA(cudaMemcpyAsync(st, h->tb, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
        SPDK_CUDA(cudaMemcpyAsync(&dt_now, h->dt, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        SPDK_CUDA(cudaMemcpyAsync(&closed, h->gate, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        SPDK_CUDA(cudaStreamSynchronize(h->stream));
        if (int rc = check_status(h)) return rc;
    }
    // the stream now only holds no-op launches; reopen the gate for later steps
    SPDK_CUDA(cudaMemsetAsync(h->gate, 0, sizeof(int), h->stream));
    if (steps) *steps = (long long)st[2];
    if (t_out) *t_out = st[0];
    return 0;
}

int spdk_hydro_read(spdk_hydro* h, int field, double* host, size_t count) {
    if (!h || !host) return fail(SPDK_E_ARG, "null argument");
    const size_t state = (size_t)h->E * h->V * h->NPT;
    const size_t cells = (size_t)h->E * h->NPT;
    if (field == SPDK_FIELD_U_SP || field == SPDK_FIELD_W_CV) {
        if (count != state) return fail(SPDK_E_ARG, "count must be E*V*NPT = " + std::to_string(state));
        const void* src = field == SPDK_FIELD_U_SP ? h->u : h->wcv;
        if (h->prec == SPDK_PRECISION_FP32) {
            // FP32 values widened exactly to doubles on the device
            if (int rc = ensure_stage(h)) return rc;
            widen_kernel<<<1024, 256, 0, h->stream>>>((const float*)src, (double*)h->stage, (long long)state);
            SPDK_CUDA(cudaGetLastError());
            SPDK_CUDA(cudaMemcpyAsync(host, h->stage, state * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            SPDK_CUDA(cudaStreamSynchronize(h->stream));
            return 0;
        }
        SPDK_CUDA(cudaMemcpyAsync(host, src, state * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        SPDK_CUDA(cudaStreamSynchronize(h->stream));
        return 0;
    }
    if (field == SPDK_FIELD_ELEMENT_TROUBLES || field == SPDK_FIELD_ELEMENT_PREDICTED) {
        if (!h->cfg.fallback) return fail(SPDK_E_STATE, "fallback is off");
        const uint8_t* src = field == SPDK_FIELD_ELEMENT_TROUBLES ? h->elem_trouble : h->elem_pred;
        if (!src) return fail(SPDK_E_STATE, "no indicator set");
        if (count != (size_t)h->E) return fail(SPDK_E_ARG, "count must be the number of elements");
        std::vector<uint8_t> b(h->E);
        SPDK_CUDA(cudaMemcpyAsync(b.data(), src, h->E, cudaMemcpyDeviceToHost, h->stream));
        SPDK_CUDA(cudaStreamSynchronize(h->stream));
        for (long long q = 0; q < h->E; q++) host[q] = b[q];
        return 0;
    }
    if (field == SPDK_FIELD_TROUBLES || field == SPDK_FIELD_THETA) {
        if (!h->cfg.fallback) return fail(SPDK_E_STATE, "fallback is off");
        if (count != cells) return fail(SPDK_E_ARG, "count must be E*NPT = " + std::to_string(cells));
        std::vector<uint8_t> b(cells);
        SPDK_CUDA(cudaMemcpyAsync(b.data(), field == SPDK_FIELD_TROUBLES ? h->trouble : h->theta, cells,
                                  cudaMemcpyDeviceToHost, h->stream));
        SPDK_CUDA(cudaStreamSynchronize(h->stream));
        for (size_t q = 0; q < cells; q++) host[q] = field == SPDK_FIELD_TROUBLES ? b[q] : b[q] * 0.125;
        return 0;
    }
    return fail(SPDK_E_ARG, "unknown field");
}

int spdk_hydro_write(spdk_hydro* h, int field, const double* host, size_t count) {
    if (!h || !host) return fail(SPDK_E_ARG, "null argument");
    const size_t state = (size_t)h->E * h->V * h->NPT;
    if (field != SPDK_FIELD_U_SP) return fail(SPDK_E_ARG, "only U_sp can be written");
    if (count != state) return fail(SPDK_E_ARG, "count must be E*V*NPT = " + std::to_string(state));
    const unsigned long long maxbits = 0x7FEFFFFFFFFFFFFFULL;
    h->feat_valid = false;
    if (h->prec == SPDK_PRECISION_FP32) {
        // doubles rounded once to FP32, on the device
        if (int rc = ensure_stage(h)) return rc;
        SPDK_CUDA(cudaMemcpyAsync(h->stage, host, state * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        narrow_kernel<<<1024, 256, 0, h->stream>>>((const double*)h->stage, (float*)h->u, (long long)state);
        SPDK_CUDA(cudaMemcpyAsync(h->dtmin, &maxbits, sizeof(maxbits), cudaMemcpyHostToDevice, h->stream));
        h->ks32.derive<<<(unsigned)h->E, kThreads, 0, h->stream>>>(h->G, h->dm32, (const float*)h->u,
                                                                    (float*)h->wcv, h->dtmin);
        advance_dt_kernel<<<1, 1, 0, h->stream>>>(h->dt, h->dtmin, h->dt_cap);
        SPDK_CUDA(cudaGetLastError());
        // the caller's buffer must outlive the copy
        SPDK_CUDA(cudaStreamSynchronize(h->stream));
        return 0;
    }
    SPDK_CUDA(cudaMemcpyAsync(h->u, host, state * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    SPDK_CUDA(cudaMemcpyAsync(h->dtmin, &maxbits, sizeof(maxbits), cudaMemcpyHostToDevice, h->stream));
    h->ks64.derive<<<(unsigned)h->E, kThreads, 0, h->stream>>>(h->G, h->dm64, (const double*)h->u,
                                                                (double*)h->wcv, h->dtmin);
    advance_dt_kernel<<<1, 1, 0, h->stream>>>(h->dt, h->dtmin, h->dt_cap);
    SPDK_CUDA(cudaGetLastError());
    SPDK_CUDA(cudaStreamSynchronize(h->stream));
    return 0;
}

int spdk_hydro_rows(spdk_hydro* h, int to_solver, int lo, int hi, void* device_buffer) {
    if (!h || !device_buffer) return fail(SPDK_E_ARG, "null argument");
    const int nrows = h->G.N[h->D - 1];
    if (lo < 0 || hi > nrows || lo >= hi) return fail(SPDK_E_ARG, "rows out of range");
    const size_t row = (size_t)(h->E / nrows) * h->V * h->NPT * h->esz;
    char* u = (char*)h->u + (size_t)lo * row;
    const size_t bytes = (size_t)(hi - lo) * row;
    if (to_solver) {
        SPDK_CUDA(cudaMemcpyAsync(u, device_buffer, bytes, cudaMemcpyDeviceToDevice, h->stream));
        h->feat_valid = false;
    } else {
        SPDK_CUDA(cudaMemcpyAsync(device_buffer, u, bytes, cudaMemcpyDeviceToDevice, h->stream));
    }
    return 0;
}

int spdk_hydro_slab_dt(spdk_hydro* h, int lo, int hi) {
    if (!h) return fail(SPDK_E_ARG, "null argument");
    const int nrows = h->G.N[h->D - 1];
    if (lo < 0 || hi > nrows || lo >= hi) return fail(SPDK_E_ARG, "rows out of range");
    const long long per = h->E / nrows;
    const long long cnt = (long long)(hi - lo) * per * h->NPT;
    long long blocks = (cnt + kThreads - 1) / kThreads;
    if (blocks > 148 * 8) blocks = 148 * 8;
    const unsigned long long maxbits = 0x7FEFFFFFFFFFFFFFULL;
    SPDK_CUDA(cudaMemcpyAsync(h->dtmin, &maxbits, sizeof(maxbits), cudaMemcpyHostToDevice, h->stream));
    const long long e_lo = lo * per, e_hi = hi * per;
    if (h->prec == SPDK_PRECISION_FP32) {
        if (h->D == 2) slab_dt_kernel<float, 2><<<(unsigned)blocks, kThreads, 0, h->stream>>>(h->G, (const float*)h->wcv, e_lo, e_hi, h->n, h->NPT, h->dtmin);
        else slab_dt_kernel<float, 3><<<(unsigned)blocks, kThreads, 0, h->stream>>>(h->G, (const float*)h->wcv, e_lo, e_hi, h->n, h->NPT, h->dtmin);
    } else {
        if (h->D == 2) slab_dt_kernel<double, 2><<<(unsigned)blocks, kThreads, 0, h->stream>>>(h->G, (const double*)h->wcv, e_lo, e_hi, h->n, h->NPT, h->dtmin);
        else slab_dt_kernel<double, 3><<<(unsigned)blocks, kThreads, 0, h->stream>>>(h->G, (const double*)h->wcv, e_lo, e_hi, h->n, h->NPT, h->dtmin);
    }
    advance_dt_kernel<<<1, 1, 0, h->stream>>>(h->dt, h->dtmin, h->dt_cap);
    SPDK_CUDA(cudaGetLastError());
    return 0;
}

}  // extern "C"

extern "C" {

int spdk_hydro_feature_size(spdk_hydro* h, int* n_in) {
    if (!h || !n_in) return fail(SPDK_E_ARG, "null argument");
    *n_in = 2 * h->NPT + 4 * h->D;
    return 0;
}

int spdk_hydro_features(spdk_hydro* h, uint16_t* x, size_t count) {
    if (!h || !x) return fail(SPDK_E_ARG, "null argument");
    const size_t need = (size_t)h->E * (2 * h->NPT + 4 * h->D);
    if (count != need) return fail(SPDK_E_ARG, "count must be " + std::to_string(need));
    if (!h->means && dalloc(h, (void**)&h->means, (size_t)h->E * sizeof(float2))) return fail(SPDK_E_NOMEM, "means");
    const int N[3] = {h->G.N[0], h->G.N[1], h->G.N[2]};
    return feature_rows(h->u, h->prec == SPDK_PRECISION_FP32, h->D, h->p, N, h->G.bc, h->G.gm, h->E, h->means, x,
                        h->stream);
}

int spdk_hydro_set_indicator(spdk_hydro* h, spdk_mlp* m, float threshold) {
    if (!h) return fail(SPDK_E_ARG, "null argument");
    if (m && !h->cfg.fallback) return fail(SPDK_E_STATE, "the indicator feeds the fallback: set fallback = 1");
    if (m && mlp_n_in(m) != 2 * h->NPT + 4 * h->D)
        return fail(SPDK_E_ARG, "the network's input size does not match this solver's feature rows");
    SPDK_CUDA(cudaStreamSynchronize(h->stream));
    if (m) {
        if (!h->side) {
            SPDK_CUDA(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
            SPDK_CUDA(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
            SPDK_CUDA(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
        }
        if (!h->feat && dalloc(h, (void**)&h->feat, (size_t)h->E * (2 * h->NPT + 4 * h->D) * sizeof(uint16_t)))
            return fail(SPDK_E_NOMEM, "features");
        if (!h->means && dalloc(h, (void**)&h->means, (size_t)h->E * sizeof(float2))) return fail(SPDK_E_NOMEM, "means");
        if (!h->elem_pred) {
            if (dalloc(h, (void**)&h->elem_pred, (size_t)h->E)) return fail(SPDK_E_NOMEM, "predictions");
            SPDK_CUDA(cudaMemset(h->elem_pred, 0, (size_t)h->E));
        }
    }
    h->mlp = m;
    h->thr = threshold;
    h->feat_valid = false;
    h->G.elem_pred = m ? h->elem_pred : nullptr;
    // the captured steps hold the old kernel arguments
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    if (h->graph_evolve) {
        cudaGraphExecDestroy(h->graph_evolve);
        h->graph_evolve = nullptr;
    }
    return 0;
}

}  // extern "C"
