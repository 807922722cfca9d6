// The hydro solver object behind the C ABI (spdk_hydro.cu), shared with the
// batched form (spdk_batch_host.cu), which drives the member solvers'
// device buffers with its own launches.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <thread>
#include <vector>

#include "spdk.h"
#include "spdk_kernelset.cuh"
#include "spdk_learned.h"
#include "spdk_setup.h"

using namespace spdk;

struct spdk_hydro {
    spdk_hydro_config cfg{};

    int D = 2, p = 3, n = 4, nf = 5, V = 4, NPT = 16, nt = 4, nstages = 1;
    double rk_a[3] = {0, 0, 0};
    long long E = 0;
    Matrices mats;
    Axis ax[3];
    int prec = SPDK_PRECISION_FP64;
    size_t esz = sizeof(double);       // bytes per state value
    DevMatsT<double> dm64{};
    DevMatsT<float> dm32{};
    DevGrid G{};
    KernelSetT<double> ks64;           // FP64 kernels (also the FP32 form's set-up)
    KernelSetT<float> ks32;
    int tile[3] = {1, 1, 1};
    cudaStream_t stream = nullptr;
    // state buffers hold doubles (plain form) or floats (precision form)
    void *u = nullptr, *ua[2] = {nullptr, nullptr}, *u0 = nullptr, *ucv[2] = {nullptr, nullptr};
    void *ff[3] = {nullptr, nullptr, nullptr}, *wcv = nullptr;
    double* dt = nullptr;
    double *fvf[3] = {nullptr, nullptr, nullptr}, *fvc[3] = {nullptr, nullptr, nullptr};
    double2 *rpo = nullptr, *rpn = nullptr;
    uint8_t *trouble = nullptr, *theta = nullptr;
    unsigned long long* dtmin = nullptr;
    // viscous runs: face viscous fluxes of the pass being evaluated, per
    // direction, and the diffusion limit on dt (0: inviscid)
    void* vg[3] = {nullptr, nullptr, nullptr};
    double dt_cap = 0.0;
    int* status = nullptr;  // device-detected faults (kStatus* bits)
    // learned indicator: per-element labels, predictions, feature rows
    uint8_t *elem_trouble = nullptr, *elem_pred = nullptr;
    uint16_t* feat = nullptr;
    float2* means = nullptr;
    spdk_mlp* mlp = nullptr;
    float thr = 0.5f;
    // the indicator runs on a side stream, forked at the start of a step and
    // joined before the first detection, so it overlaps the Picard passes
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool join_pending = false;
    // feat / means hold the nodal features and element means of the current
    // U (the last update of a step with the indicator writes them)
    bool feat_valid = false;
    size_t bytes = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    // device-resident time loop (spdk_hydro_evolve): a step graph whose
    // kernels return once `gate` is set, ending in evolve_advance_kernel on
    // tb = {t, t_output, steps, t_end, dt_output}
    cudaGraphExec_t graph_evolve = nullptr;
    bool evolve_mode = false;  // enqueue_step records the device loop's step end
    int* gate = nullptr;
    double* tb = nullptr;
    void* stage = nullptr;  // precision form: doubles exchanged with the host
    int launches = 0;
    // per-launch event timing (spdk_hydro_profile)
    bool profiling = false;
    std::vector<cudaEvent_t> ev;
    std::vector<int> ev_kind;
    size_t ev_used = 0;
    // asynchronous checkpoint (spdk_checkpoint.cu): a device snapshot of U
    // and dt, its pinned host copy, the copy stream and the writer thread
    unsigned char* ck_dev = nullptr;
    unsigned char* ck_host = nullptr;
    size_t ck_bytes = 0;
    cudaStream_t ck_stream = nullptr;
    cudaEvent_t ck_snap = nullptr, ck_done = nullptr;
    std::thread* ck_thread = nullptr;
    int ck_status = 0;
    std::string ck_error;
};

// joins a pending checkpoint write and frees its buffers (spdk_checkpoint.cu)
void checkpoint_release(spdk_hydro* h);
