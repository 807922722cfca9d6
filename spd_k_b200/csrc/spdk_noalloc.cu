// Allocation-free step entry point.
//
// Some hosts cannot call cudaMalloc at the point where they want to advance
// the solution: an application that owns every byte of device memory through
// its own pool and forbids libraries from allocating behind its back, a
// plugin running inside a stream capture it does not own (an allocation
// there breaks the capture), or a real-time loop that cannot absorb the
// device synchronisation an allocation may cause. For them,
// spdk_hydro_step_noalloc advances one ADER or SSP-RK step (no fallback) on
// buffers the caller owns, and keeps its working storage in one fixed
// device array that is part of the library image.
//
// The working storage is the file-scope array g_scratch below, 16 MiB, held
// on every GPU that loads the library until the process exits. Its first
// 256 bytes hold the dt reduction word and the status word; the rest holds
// the Picard slices (ADER) or the stage copies (RK). Every call uses the
// same array and leaves its contents behind, so two calls whose work
// overlaps on the GPU (different streams, or different host threads on the
// same device) race and corrupt each other: order them on one stream.
//
// In host code g_scratch names a host-side shadow, not a device address.
// The first call on each device, with that device current, resolves the
// real address with cudaGetSymbolAddress and sets the kernels' shared-memory
// attributes; make that first call before any stream capture. After that a
// call only enqueues kernels and device-to-device copies on the caller's
// stream; no call allocates.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "spdk.h"
#include "spdk_kernelset.cuh"
#include "spdk_setup.h"

namespace spdk {
int fail(int code, const std::string& msg);
}

namespace {

using namespace spdk;

constexpr size_t kScratchBytes = (size_t)SPDK_NOALLOC_SCRATCH_BYTES;
constexpr size_t kHeaderBytes = 256;  // dt reduction word, status word

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_setup_mutex;

// start of every call: dt reduction word <- largest double, status word <- 0
__global__ void noalloc_arm(unsigned long long* dtmin, int* status) {
    *dtmin = 0x7FEFFFFFFFFFFFFFULL;
    *status = 0;
}

// end of every call: the next dt, or NaN when a bounded staging wait ran
// out during the call (the state it leaves is then not to be trusted; the
// status word keeps the bit for spdk_hydro_noalloc_status)
__global__ void noalloc_finish(double* dt, unsigned long long* dtmin, const int* status) {
    *dt = (*status & kStatusStagingTimeout) ? __longlong_as_double(0x7FF8000000000000LL)
                                            : __longlong_as_double((long long)*dtmin);
    *dtmin = 0x7FEFFFFFFFFFFFFFULL;
}

// once per device, with the device current: the device address of
// g_scratch (its host-side name is only a shadow) and a zero status word
int setup_device(int dev, const KernelSet& ks, void** base) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (dev < 0 || dev >= kMaxDevices) return fail(SPDK_E_ARG, "device ordinal out of range");
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p)
            return fail(SPDK_E_CUDA, std::string("cudaGetSymbolAddress(g_scratch): ") + cudaGetErrorString(e));
        e = cudaMemset((char*)p + sizeof(unsigned long long), 0, sizeof(int));
        if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("scratch status reset: ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    // per-kernel attributes (idempotent, not an allocation)
    const void* fns[] = {(const void*)ks.predict, (const void*)ks.correct};
    for (const void* f : fns) {
        cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ks.picard_smem);
        if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
        cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    }
    *base = g_scratch_ptr[dev];
    return 0;
}

}  // namespace

extern "C" int spdk_hydro_step_noalloc(const spdk_hydro_config* cfg, const double* u_in, double* u_out,
                                       double* wcv_out, double* dt_inout, void* stream) {
    if (!cfg || !u_in || !u_out || !dt_inout) return fail(SPDK_E_ARG, "null argument");
    const spdk_hydro_config& c = *cfg;
    if (c.fallback) return fail(SPDK_E_ARG, "the allocation-free step has no fallback: set fallback = 0");
    if (c.nu != 0.0) return fail(SPDK_E_ARG, "the allocation-free step has no viscous terms: set nu = 0");
    if (c.p < 1 || c.p > kMaxP) return fail(SPDK_E_ARG, "p must be in 1..7");
    if (c.N[0] < 2 || c.N[1] < 2) return fail(SPDK_E_ARG, "x and y must be active (nx1, nx2 > 1)");
    if (c.precision != SPDK_PRECISION_FP64) return fail(SPDK_E_ARG, "unsupported precision");
    if (c.slab_n != 0 || c.slab_lo != 0)
        return fail(SPDK_E_ARG, "the allocation-free step steps whole domains: set slab_lo = slab_n = 0");
    const int D = c.N[2] > 1 ? 3 : 2;
    if (D == 3 && c.p > 5) return fail(SPDK_E_ARG, "3D runs support p <= 5");
    if (D == 2 && (c.g[2] != 0.0 || ((c.problem == SPDK_IC_SINE_WAVE || c.problem == SPDK_IC_SQUARE) && c.v3 != 0.0)))
        return fail(SPDK_E_ARG, "a 2D run cannot carry z momentum or z gravity");
    const bool ader = c.integrator == SPDK_INTEGRATOR_ADER;
    if (!ader && (c.rk_order < 1 || c.rk_order > 3)) return fail(SPDK_E_ARG, "rk_order must be 1, 2 or 3");
    const int n = c.p + 1, V = D + 2;
    const int NPT = D == 2 ? n * n : n * n * n;
    const int nt = ader ? n : 1;
    const int nstages = ader ? 1 : c.rk_order;
    const int N[3] = {c.N[0], c.N[1], D == 3 ? c.N[2] : 1};
    const long long E = (long long)N[0] * N[1] * N[2];
    const size_t state = (size_t)E * V * NPT * sizeof(double);
    // working storage: two Picard buffers of nt slices (ADER), or the stage
    // input copy plus the step-start state (RK)
    const size_t need = ader ? 2 * (size_t)nt * state : 2 * state;
    if (need > kScratchBytes - kHeaderBytes)
        return fail(SPDK_E_ARG, "problem needs " + std::to_string(need) + " bytes of working storage; the "
                                "allocation-free step has " + std::to_string(kScratchBytes - kHeaderBytes));

    KernelSet ks;
    if (!select_kernels(D, c.p, N, &ks)) return fail(SPDK_E_ARG, "no kernel instantiation for this ndim/p");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(SPDK_E_CUDA, "cudaGetDevice failed");
    void* base = nullptr;
    int rc = setup_device(dev, ks, &base);
    if (rc) return rc;
    unsigned long long* dtmin = (unsigned long long*)base;
    int* status = (int*)((char*)base + sizeof(unsigned long long));
    double* work = (double*)((char*)base + kHeaderBytes);

    Matrices mats;
    build_matrices(c.p, ader, &mats);
    DevMats dm;
    std::memset(&dm, 0, sizeof(dm));
    const int nf = n + 1;
    for (int j = 0; j < nf; j++)
        for (int i = 0; i < n; i++) dm.sp_to_fp[j * n + i] = mats.sp_to_fp[j * n + i];
    for (int j = 0; j < n; j++)
        for (int i = 0; i < nf; i++) dm.dfp_to_sp[j * nf + i] = mats.dfp_to_sp[j * nf + i];
    for (int q = 0; q < n * n; q++) {
        dm.sp_to_cv[q] = mats.sp_to_cv[q];
        dm.cv_to_sp[q] = mats.cv_to_sp[q];
    }
    for (int q = 0; q < nt * nt; q++) dm.invader[q] = mats.invader[q];
    for (int q = 0; q < nt; q++) dm.wt[q] = mats.wt[q];

    DevGrid G;
    std::memset(&G, 0, sizeof(G));
    for (int d = 0; d < 3; d++) {
        G.N[d] = N[d];
        G.bc[d] = c.bc[d];
        G.h[d] = c.L[d] / N[d];
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
    G.nt = nt;
    G.E = E;
    G.status = status;

    cudaStream_t s = (cudaStream_t)stream;
    long long blocks = 1;
    for (int d = 0; d < D; d++) blocks *= N[d] / ks.tile[d];
    noalloc_arm<<<1, 1, 0, s>>>(dtmin, status);
    double rk_a[3] = {0, 0, 0};
    if (c.rk_order == 2) rk_a[1] = 0.5;
    if (c.rk_order == 3) { rk_a[1] = 0.75; rk_a[2] = 1.0 / 3.0; }
    if (ader) {
        double* ua[2] = {work, work + (size_t)nt * E * V * NPT};
        PicardArgs A{};
        A.u = u_in;
        A.dt = dt_inout;
        const double* in = u_in;
        int in_slices = 1;
        for (int it = 0; it + 1 < nt; it++) {
            A.ua_in = in;
            A.in_slices = in_slices;
            A.ua_out = ua[it % 2];
            ks.predict<<<(unsigned)blocks, kThreads, ks.picard_smem, s>>>(G, dm, A);
            in = ua[it % 2];
            in_slices = nt;
        }
        A.ua_in = in;
        A.in_slices = in_slices;
        A.u_out = u_out;
        A.final_stage = 1;
        A.wcv = wcv_out;
        A.dtmin = dtmin;
        ks.correct<<<(unsigned)blocks, kThreads, ks.picard_smem, s>>>(G, dm, A);
    } else {
        double* stage_in = work;
        double* u0 = work + (size_t)E * V * NPT;
        if (nstages > 1 && cudaMemcpyAsync(u0, u_in, state, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            return fail(SPDK_E_CUDA, "step-start copy failed");
        const double* cur = u_in;
        for (int st = 0; st < nstages; st++) {
            // a stage updates the state in place, so its halo is read from a copy
            if (cudaMemcpyAsync(stage_in, cur, state, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
                return fail(SPDK_E_CUDA, "stage copy failed");
            PicardArgs A{};
            A.ua_in = stage_in;
            A.in_slices = 1;
            A.u = cur;
            A.u_out = u_out;
            A.u0 = u0;
            A.rk_a = rk_a[st];
            A.final_stage = st == nstages - 1;
            A.wcv = wcv_out;
            A.dtmin = dtmin;
            A.dt = dt_inout;
            ks.correct<<<(unsigned)blocks, kThreads, ks.picard_smem, s>>>(G, dm, A);
            cur = u_out;
        }
    }
    noalloc_finish<<<1, 1, 0, s>>>(dt_inout, dtmin, status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return 0;
}

extern "C" int spdk_hydro_noalloc_status(int* status_out, void* stream) {
    if (!status_out) return fail(SPDK_E_ARG, "null argument");
    *status_out = 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(SPDK_E_CUDA, "cudaGetDevice failed");
    if (dev < 0 || dev >= kMaxDevices) return fail(SPDK_E_ARG, "device ordinal out of range");
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        base = g_scratch_ptr[dev];
    }
    if (!base) return 0;  // no step on this device yet: nothing to report
    cudaStream_t s = (cudaStream_t)stream;
    int st = 0;
    cudaError_t e = cudaMemcpyAsync(&st, (char*)base + sizeof(unsigned long long), sizeof(int),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("status read: ") + cudaGetErrorString(e));
    *status_out = st;
    return 0;
}
