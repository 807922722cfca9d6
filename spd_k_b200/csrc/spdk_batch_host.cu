// Batched form: host orchestration (declarations in include/spdk_batch.h).
//
// The member problems are ordinary solvers (spdk_hydro_create builds their
// buffers, matrices, initial state and first dt); the batch plans, per order
// group, the same pass sequence spdk_hydro_step launches -- p Picard passes,
// the flux pass and p+1 fallback slices (or the corrector) -- with one
// table item per member and pass, and launches each pass once for the whole
// group. A final kernel hands every member its next dt.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "spdk.h"
#include "spdk_batch.cuh"
#include "spdk_batch.h"
#include "spdk_hydro_impl.h"

namespace spdk {
int fail(int code, const std::string& msg);

__global__ void dt_batched(const DtArgs* __restrict__ a, int n) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) {
        *a[q].dt = __longlong_as_double((long long)*a[q].dtmin);
        *a[q].dtmin = 0x7FEFFFFFFFFFFFFFULL;
    }
}

}  // namespace spdk

namespace {

enum { kPassPredict, kPassCorrect, kPassFlux, kPassDetect, kPassUpdate };

struct Pass {
    int kind;
    unsigned blocks;
    void* items;  // device table
    int n;
};

struct Group {
    int p = 0;
    std::vector<int> members;
    int tile = 2;
    BatchSetT<double> k64;
    BatchSetT<float> k32;
    std::vector<Pass> passes;
    cudaStream_t st = nullptr;
    cudaEvent_t join = nullptr;
};

}  // namespace

struct spdk_batch {
    std::vector<spdk_hydro*> probs;
    int prec = SPDK_PRECISION_FP64;
    bool fallback = false;
    std::vector<Group> groups;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
    DtArgs* dt_items = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool labels = false;  // per-step element trouble labels (spdk_batch_record_labels)
};

namespace {

#define BCUDA(call)                                                                      \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(SPDK_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void free_tables(Group& g) {
    for (Pass& p : g.passes) cudaFree(p.items);
    g.passes.clear();
}

template <typename Item>
int upload_pass(Group& g, int kind, unsigned blocks, const std::vector<Item>& items) {
    void* d = nullptr;
    BCUDA(cudaMalloc(&d, items.size() * sizeof(Item)));
    BCUDA(cudaMemcpy(d, items.data(), items.size() * sizeof(Item), cudaMemcpyHostToDevice));
    g.passes.push_back(Pass{kind, blocks, d, (int)items.size()});
    return 0;
}

template <typename R>
const BatchSetT<R>& set_of(const Group& g);
template <>
const BatchSetT<double>& set_of<double>(const Group& g) { return g.k64; }
template <>
const BatchSetT<float>& set_of<float>(const Group& g) { return g.k32; }

// the pass sequence of enqueue_step_t (ADER, one stage) for every member
template <typename R>
int plan_group(spdk_batch* b, Group& g) {
    free_tables(g);
    const int n = (int)g.members.size();
    std::vector<long long> first(n);
    long long total = 0;
    for (int q = 0; q < n; q++) {
        const spdk_hydro* h = b->probs[g.members[q]];
        first[q] = total;
        total += (long long)(h->G.N[0] / g.tile) * (h->G.N[1] / g.tile);
    }
    const unsigned blocks = (unsigned)total;
    const int nt = b->probs[g.members[0]]->nt;
    std::vector<const R*> in(n);
    std::vector<int> in_slices(n, 1);
    for (int q = 0; q < n; q++) in[q] = (const R*)b->probs[g.members[q]]->u;
    auto base = [&](int q) {
        const spdk_hydro* h = b->probs[g.members[q]];
        BatchItem<PicardArgsT<R>> it{};
        it.G = h->G;
        it.G.elem_trouble = nullptr;  // no per-step labels in the batch
        it.G.elem_pred = nullptr;
        it.first = first[q];
        it.A.u = (const R*)h->u;
        it.A.dt = h->dt;
        return it;
    };
    int rc = 0;
    for (int i = 0; i + 1 < nt && !rc; i++) {
        std::vector<BatchItem<PicardArgsT<R>>> items(n);
        for (int q = 0; q < n; q++) {
            const spdk_hydro* h = b->probs[g.members[q]];
            items[q] = base(q);
            items[q].A.ua_in = in[q];
            items[q].A.in_slices = in_slices[q];
            items[q].A.ua_out = (R*)h->ua[i % 2];
            in[q] = (const R*)h->ua[i % 2];
            in_slices[q] = nt;
        }
        rc = upload_pass(g, kPassPredict, blocks, items);
    }
    if (rc) return rc;
    if (!b->fallback) {
        std::vector<BatchItem<PicardArgsT<R>>> items(n);
        for (int q = 0; q < n; q++) {
            spdk_hydro* h = b->probs[g.members[q]];
            items[q] = base(q);
            items[q].A.ua_in = in[q];
            items[q].A.in_slices = in_slices[q];
            items[q].A.u_out = (R*)h->u;
            items[q].A.u0 = (const R*)h->u0;
            items[q].A.rk_a = 0;
            items[q].A.final_stage = 1;
            items[q].A.wcv = (R*)h->wcv;
            items[q].A.dtmin = h->dtmin;
        }
        return upload_pass(g, kPassCorrect, blocks, items);
    }
    {
        std::vector<BatchItem<PicardArgsT<R>>> items(n);
        for (int q = 0; q < n; q++) {
            spdk_hydro* h = b->probs[g.members[q]];
            items[q] = base(q);
            items[q].A.ua_in = in[q];
            items[q].A.in_slices = in_slices[q];
            for (int d = 0; d < 3; d++) items[q].A.ff[d] = (R*)h->ff[d];
            items[q].A.ucv = (R*)h->ucv[0];
            items[q].A.rp_old = h->rpo;
            items[q].A.rp_new = h->rpn;
        }
        if ((rc = upload_pass(g, kPassFlux, blocks, items))) return rc;
    }
    for (int t = 0; t < nt && !rc; t++) {
        std::vector<BatchItem<DetectArgs>> det(n);
        std::vector<BatchItem<FallbackArgsT<R>>> up(n);
        for (int q = 0; q < n; q++) {
            spdk_hydro* h = b->probs[g.members[q]];
            const BatchItem<PicardArgsT<R>> bq = base(q);
            det[q].G = bq.G;
            if (b->labels) det[q].G.elem_trouble = h->elem_trouble;
            det[q].first = bq.first;
            det[q].A = DetectArgs{h->rpo, h->rpn, h->trouble};
            up[q].G = bq.G;
            up[q].first = bq.first;
            FallbackArgsT<R>& F = up[q].A;
            F = FallbackArgsT<R>{};
            F.ucv_in = (R*)h->ucv[t % 2];
            F.ucv_out = (R*)h->ucv[(t + 1) % 2];
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
            F.last = t == nt - 1;
            F.u = (R*)h->u;
            F.u0 = (const R*)h->u0;
            F.rk_a = 0;
            F.final_stage = 1;
            F.wcv = (R*)h->wcv;
            F.dtmin = h->dtmin;
            F.dt = h->dt;
        }
        rc = upload_pass(g, kPassDetect, blocks, det);
        if (!rc) rc = upload_pass(g, kPassUpdate, blocks, up);
    }
    return rc;
}

template <typename R>
int set_batch_attributes(const BatchSetT<R>& k) {
    const void* fns[] = {(const void*)k.predict, (const void*)k.correct, (const void*)k.flux};
    for (const void* f : fns) {
        BCUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.picard_smem));
        cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    }
    BCUDA(cudaFuncSetAttribute((const void*)k.update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.update_smem));
    cudaFuncSetAttribute((const void*)k.update, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return 0;
}

int select_group(spdk_batch* b, Group& g, int tile) {
    for (int q : g.members) {
        const spdk_hydro* h = b->probs[q];
        if (h->G.N[0] % tile || h->G.N[1] % tile) return fail(SPDK_E_ARG, "tile does not divide an element count");
    }
    const bool ok = b->prec == SPDK_PRECISION_FP32 ? batch_set(g.p, tile, &g.k32) : batch_set(g.p, tile, &g.k64);
    if (!ok) return fail(SPDK_E_ARG, "no batched kernels for this order / tile");
    g.tile = tile;
    int rc = b->prec == SPDK_PRECISION_FP32 ? set_batch_attributes(g.k32) : set_batch_attributes(g.k64);
    if (!rc) rc = b->prec == SPDK_PRECISION_FP32 ? plan_group<float>(b, g) : plan_group<double>(b, g);
    return rc;
}

template <typename R>
int launch_group_t(spdk_batch* b, const Group& g, cudaStream_t st) {
    const BatchSetT<R>& k = set_of<R>(g);
    const spdk_hydro* h0 = b->probs[g.members[0]];
    const DevMatsT<R>& dm = *reinterpret_cast<const DevMatsT<R>*>(
        b->prec == SPDK_PRECISION_FP32 ? (const void*)&h0->dm32 : (const void*)&h0->dm64);
    using PI = BatchItem<PicardArgsT<R>>;
    using DI = BatchItem<DetectArgs>;
    using UI = BatchItem<FallbackArgsT<R>>;
    for (const Pass& p : g.passes) {
        const PI* pi = static_cast<const PI*>(p.items);
        const DI* di = static_cast<const DI*>(p.items);
        const UI* ui = static_cast<const UI*>(p.items);
        switch (p.kind) {
        case kPassPredict: k.predict<<<p.blocks, kThreads, k.picard_smem, st>>>(pi, p.n, dm); break;
        case kPassCorrect: k.correct<<<p.blocks, kThreads, k.picard_smem, st>>>(pi, p.n, dm); break;
        case kPassFlux: k.flux<<<p.blocks, kThreads, k.picard_smem, st>>>(pi, p.n, dm); break;
        case kPassDetect: k.detect<<<p.blocks, kThreads, 0, st>>>(di, p.n); break;
        case kPassUpdate: k.update<<<p.blocks, kThreads, k.update_smem, st>>>(ui, p.n, dm); break;
        }
    }
    BCUDA(cudaGetLastError());
    return 0;
}

int launch_group(spdk_batch* b, const Group& g, cudaStream_t st) {
    return b->prec == SPDK_PRECISION_FP32 ? launch_group_t<float>(b, g, st) : launch_group_t<double>(b, g, st);
}

// one step: the groups concurrently on their streams, then every dt
int enqueue_batch_step(spdk_batch* b) {
    if (b->labels)
        for (spdk_hydro* h : b->probs) BCUDA(cudaMemsetAsync(h->elem_trouble, 0, (size_t)h->E, b->stream));
    BCUDA(cudaEventRecord(b->fork, b->stream));
    for (Group& g : b->groups) {
        BCUDA(cudaStreamWaitEvent(g.st, b->fork, 0));
        int rc = launch_group(b, g, g.st);
        if (rc) return rc;
        BCUDA(cudaEventRecord(g.join, g.st));
        BCUDA(cudaStreamWaitEvent(b->stream, g.join, 0));
    }
    const int n = (int)b->probs.size();
    dt_batched<<<(n + 127) / 128, 128, 0, b->stream>>>(b->dt_items, n);
    BCUDA(cudaGetLastError());
    return 0;
}

void drop_graph(spdk_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

void release(spdk_batch* b) {
    drop_graph(b);
    for (Group& g : b->groups) {
        free_tables(g);
        if (g.st) cudaStreamDestroy(g.st);
        if (g.join) cudaEventDestroy(g.join);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->dt_items) cudaFree(b->dt_items);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (spdk_hydro* h : b->probs) spdk_hydro_destroy(h);
}

}  // namespace

extern "C" {

int spdk_batch_create(const spdk_hydro_config* cfgs, int count, spdk_batch** out) {
    if (!cfgs || !out || count < 1) return fail(SPDK_E_ARG, "bad argument");
    *out = nullptr;
    for (int i = 0; i < count; i++) {
        const spdk_hydro_config& c = cfgs[i];
        if (c.N[2] > 1) return fail(SPDK_E_ARG, "the batched form is 2D");
        if (c.integrator != SPDK_INTEGRATOR_ADER) return fail(SPDK_E_ARG, "the batched form runs ADER");
        if (c.p != 2 && c.p != 3 && c.p != 5) return fail(SPDK_E_ARG, "batched orders are 2, 3 and 5");
        if (c.precision != cfgs[0].precision || (c.fallback != 0) != (cfgs[0].fallback != 0) ||
            c.device != cfgs[0].device)
            return fail(SPDK_E_ARG, "all problems of a batch share precision, fallback and device");
        if (c.N[0] % 2 || c.N[1] % 2) return fail(SPDK_E_ARG, "element counts must be even");
        if (c.nu != 0.0) return fail(SPDK_E_ARG, "the batched form is inviscid: set nu = 0");
    }
    spdk_batch* b = new spdk_batch;
    b->prec = cfgs[0].precision;
    b->fallback = cfgs[0].fallback != 0;
    int rc = 0;
    for (int i = 0; i < count && !rc; i++) {
        spdk_hydro* h = nullptr;
        rc = spdk_hydro_create(&cfgs[i], &h);
        if (!rc) b->probs.push_back(h);
    }
    if (!rc) {
        BCUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        BCUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        std::map<int, int> gi;
        for (int i = 0; i < count; i++) {
            const int p = cfgs[i].p;
            if (!gi.count(p)) {
                gi[p] = (int)b->groups.size();
                b->groups.emplace_back();
                b->groups.back().p = p;
            }
            b->groups[gi[p]].members.push_back(i);
        }
        for (Group& g : b->groups) {
            BCUDA(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
            BCUDA(cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming));
            if (!rc) rc = select_group(b, g, 2);
        }
        std::vector<DtArgs> dts(count);
        for (int i = 0; i < count; i++) dts[i] = DtArgs{b->probs[i]->dt, b->probs[i]->dtmin};
        if (!rc && cudaMalloc((void**)&b->dt_items, count * sizeof(DtArgs)) != cudaSuccess)
            rc = fail(SPDK_E_NOMEM, "batch dt table");
        if (!rc && cudaMemcpy(b->dt_items, dts.data(), count * sizeof(DtArgs), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = fail(SPDK_E_CUDA, "batch dt table");
    }
    if (rc) {
        release(b);
        delete b;
        return rc;
    }
    *out = b;
    return 0;
}

int spdk_batch_destroy(spdk_batch* b) {
    if (!b) return 0;
    if (b->stream) cudaStreamSynchronize(b->stream);
    release(b);
    delete b;
    return 0;
}

int spdk_batch_steps(spdk_batch* b, int nsteps) {
    if (!b || nsteps < 0) return fail(SPDK_E_ARG, "bad argument");
    if (nsteps == 0) return 0;
    if (!b->graph) {
        cudaGraph_t g;
        BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_batch_step(b);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("batch capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("batch instantiate: ") + cudaGetErrorString(e));
    }
    for (int s = 0; s < nsteps; s++) BCUDA(cudaGraphLaunch(b->graph, b->stream));
    return 0;
}

int spdk_batch_record_labels(spdk_batch* b, int on) {
    if (!b) return fail(SPDK_E_ARG, "null argument");
    if (on && !b->fallback) return fail(SPDK_E_STATE, "labels come from the fallback's detection: set fallback = 1");
    BCUDA(cudaStreamSynchronize(b->stream));
    b->labels = on != 0;
    for (Group& g : b->groups) {
        const int rc = b->prec == SPDK_PRECISION_FP32 ? plan_group<float>(b, g) : plan_group<double>(b, g);
        if (rc) return rc;
    }
    drop_graph(b);
    return 0;
}

int spdk_batch_sync(spdk_batch* b) {
    if (!b) return fail(SPDK_E_ARG, "null argument");
    BCUDA(cudaStreamSynchronize(b->stream));
    for (spdk_hydro* h : b->probs) {
        int st = 0;
        BCUDA(cudaMemcpy(&st, h->status, sizeof(int), cudaMemcpyDeviceToHost));
        if (st) return fail(st, "device-detected fault in a batch member (status " + std::to_string(st) + ")");
    }
    return 0;
}

int spdk_batch_autotune(spdk_batch* b, int steps) {
    if (!b || steps < 1) return fail(SPDK_E_ARG, "bad argument");
    BCUDA(cudaStreamSynchronize(b->stream));
    // save every member's state (U, W_cv, dt) so that tuning changes nothing
    std::vector<void*> saved;
    for (spdk_hydro* h : b->probs) {
        const size_t state = (size_t)h->E * h->V * h->NPT * h->esz;
        void* s = nullptr;
        BCUDA(cudaMalloc(&s, 2 * state + sizeof(double)));
        BCUDA(cudaMemcpy(s, h->u, state, cudaMemcpyDeviceToDevice));
        BCUDA(cudaMemcpy((char*)s + state, h->wcv, state, cudaMemcpyDeviceToDevice));
        BCUDA(cudaMemcpy((char*)s + 2 * state, h->dt, sizeof(double), cudaMemcpyDeviceToDevice));
        saved.push_back(s);
    }
    auto restore = [&]() {
        for (size_t i = 0; i < b->probs.size(); i++) {
            spdk_hydro* h = b->probs[i];
            const size_t state = (size_t)h->E * h->V * h->NPT * h->esz;
            cudaMemcpy(h->u, saved[i], state, cudaMemcpyDeviceToDevice);
            cudaMemcpy(h->wcv, (char*)saved[i] + state, state, cudaMemcpyDeviceToDevice);
            cudaMemcpy(h->dt, (char*)saved[i] + 2 * state, sizeof(double), cudaMemcpyDeviceToDevice);
        }
    };
    int rc = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int n = (int)b->probs.size();
    for (Group& g : b->groups) {
        float best = 1e30f;
        int best_tile = g.tile;
        for (int tile : {1, 2, 4}) {
            if (select_group(b, g, tile)) continue;  // not instantiated / does not divide
            restore();
            // one untimed step, then `steps` timed steps of this group
            for (int s = 0; s <= steps && !rc; s++) {
                if (s == 1) cudaEventRecord(e0, b->stream);
                rc = launch_group(b, g, b->stream);
                dt_batched<<<(n + 127) / 128, 128, 0, b->stream>>>(b->dt_items, n);
            }
            cudaEventRecord(e1, b->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail(SPDK_E_CUDA, "autotune run");
            if (rc) break;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) {
                best = ms;
                best_tile = tile;
            }
        }
        if (!rc) rc = select_group(b, g, best_tile);
        if (rc) break;
    }
    restore();
    cudaDeviceSynchronize();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (void* s : saved) cudaFree(s);
    drop_graph(b);
    return rc;
}

int spdk_batch_get_info(spdk_batch* b, spdk_batch_info* info) {
    if (!b || !info) return fail(SPDK_E_ARG, "null argument");
    std::memset(info, 0, sizeof(*info));
    info->n_problems = (int)b->probs.size();
    info->n_groups = (int)b->groups.size();
    int launches = 1;
    for (size_t i = 0; i < b->groups.size(); i++) {
        const Group& g = b->groups[i];
        launches += (int)g.passes.size();
        if (i < 8) {
            info->group_p[i] = g.p;
            info->group_tile[i] = g.tile;
            info->group_size[i] = (int)g.members.size();
        }
    }
    info->launches_per_step = launches;
    for (spdk_hydro* h : b->probs) {
        info->n_dof += h->E * h->NPT;
        info->device_bytes += h->bytes;
    }
    return 0;
}

int spdk_batch_get_stream(spdk_batch* b, void** stream) {
    if (!b || !stream) return fail(SPDK_E_ARG, "null argument");
    *stream = (void*)b->stream;
    return 0;
}

int spdk_batch_member(spdk_batch* b, int i, spdk_hydro** h) {
    if (!b || !h || i < 0 || i >= (int)b->probs.size()) return fail(SPDK_E_ARG, "bad argument");
    *h = b->probs[i];
    return 0;
}

}  // extern "C"
