// Checkpoint / restart of a hydro solver (include/spdk.h). No counterpart in
// the reference, whose runs always start from the initial condition.
//
// The file holds U_sp in the solver's own arithmetic and the next step's dt
// as the device holds it, so a restored solver continues bit for bit: every
// other buffer is either rebuilt from U at the start of a step (U_ader, the
// RK stage state, U_cv and the FV candidates, the indicator's features) or
// recomputed by spdk_hydro_write (W_cv).
//
// The asynchronous form copies U and dt to a device snapshot on the solver
// stream (ordered after the steps already enqueued, and before any later
// step overwrites U), then a copy stream moves the snapshot to pinned host
// memory and a writer thread waits for that copy and writes the file, while
// the caller keeps stepping.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "spdk.h"
#include "spdk_hydro_impl.h"

namespace spdk {
int fail(int code, const std::string& msg);
}

namespace {

constexpr char kMagic[8] = {'S', 'P', 'D', 'K', 'C', 'K', 'P', '1'};
// version 2 adds the geometry and physics fields after cfl; version 1 files
// (those fields zero) are still read, with the version-1 checks only
constexpr uint32_t kVersion = 2;

// 256 bytes, little-endian, naturally aligned
struct CkptHeader {
    char magic[8];
    uint32_t version, precision, D, p, N[3], V, NPT, integrator, rk_order, fallback, bc[3], esz, reserved0, reserved1;
    uint64_t count;  // values of U
    double t, dt, t_output;
    int64_t steps, outputs;
    double gamma, cfl;
    // version 2: box lengths, gravity, viscosity, fallback settings, slab
    double L[3], g[3], nu, beta, nad_tolerance;
    int32_t nad_delta, nad_moore, sed, blending, slab_lo, slab_n;
    uint8_t reserved[16];
};
static_assert(sizeof(CkptHeader) == 256, "checkpoint header layout");

CkptHeader make_header(const spdk_hydro* h, const spdk_checkpoint_info& info) {
    CkptHeader hd;
    std::memset(&hd, 0, sizeof(hd));
    std::memcpy(hd.magic, kMagic, 8);
    hd.version = kVersion;
    hd.precision = (uint32_t)h->prec;
    hd.D = (uint32_t)h->D;
    hd.p = (uint32_t)h->p;
    for (int d = 0; d < 3; d++) {
        hd.N[d] = (uint32_t)h->cfg.N[d];
        hd.bc[d] = (uint32_t)h->cfg.bc[d];
    }
    hd.V = (uint32_t)h->V;
    hd.NPT = (uint32_t)h->NPT;
    hd.integrator = (uint32_t)h->cfg.integrator;
    hd.rk_order = (uint32_t)h->cfg.rk_order;
    hd.fallback = (uint32_t)(h->cfg.fallback != 0);
    hd.esz = (uint32_t)h->esz;
    hd.count = (uint64_t)h->E * h->V * h->NPT;
    hd.t = info.t;
    hd.t_output = info.t_output;
    hd.steps = info.steps;
    hd.outputs = info.outputs;
    hd.gamma = h->cfg.gamma;
    hd.cfl = h->cfg.cfl;
    for (int d = 0; d < 3; d++) {
        hd.L[d] = h->cfg.L[d];
        hd.g[d] = h->cfg.g[d];
    }
    hd.nu = h->cfg.nu;
    hd.beta = h->cfg.beta;
    hd.nad_tolerance = h->cfg.nad_tolerance;
    hd.nad_delta = h->cfg.nad_delta;
    hd.nad_moore = h->cfg.nad_moore;
    hd.sed = h->cfg.sed;
    hd.blending = h->cfg.blending;
    hd.slab_lo = h->cfg.slab_lo;
    hd.slab_n = h->cfg.slab_n;
    return hd;
}

// header + state into path (through a temporary name, so a reader never
// sees a partial file); returns false with *err set on failure
bool write_ckpt(const std::string& path, const CkptHeader& hd, const void* data, size_t bytes, std::string* err) {
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) {
        *err = "cannot open " + tmp + " for writing";
        return false;
    }
    const bool ok = std::fwrite(&hd, sizeof(hd), 1, f) == 1 && std::fwrite(data, 1, bytes, f) == bytes;
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) {
        std::remove(tmp.c_str());
        *err = "write to " + tmp + " failed";
        return false;
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
        std::remove(tmp.c_str());
        *err = "cannot rename " + tmp + " to " + path;
        return false;
    }
    return true;
}

int read_header(FILE* f, const char* path, CkptHeader* hd) {
    if (std::fread(hd, sizeof(*hd), 1, f) != 1) return fail(SPDK_E_IO, std::string("short checkpoint header in ") + path);
    if (std::memcmp(hd->magic, kMagic, 8) != 0) return fail(SPDK_E_ARG, std::string(path) + " is not a checkpoint");
    if (hd->version != 1 && hd->version != kVersion)
        return fail(SPDK_E_ARG, "checkpoint version " + std::to_string(hd->version) + " is not supported");
    return 0;
}

// offset of dt in the snapshot: after U, 8-byte aligned
size_t dt_offset(size_t ubytes) { return (ubytes + 7) / 8 * 8; }

}  // namespace

void checkpoint_release(spdk_hydro* h) {
    if (h->ck_thread) {
        h->ck_thread->join();
        delete h->ck_thread;
        h->ck_thread = nullptr;
    }
    if (h->ck_dev) cudaFree(h->ck_dev);
    if (h->ck_host) cudaFreeHost(h->ck_host);
    if (h->ck_snap) cudaEventDestroy(h->ck_snap);
    if (h->ck_done) cudaEventDestroy(h->ck_done);
    if (h->ck_stream) cudaStreamDestroy(h->ck_stream);
    h->ck_dev = h->ck_host = nullptr;
    h->ck_snap = h->ck_done = nullptr;
    h->ck_stream = nullptr;
    h->ck_bytes = 0;
}

extern "C" {

int spdk_hydro_checkpoint(spdk_hydro* h, const char* path, const spdk_checkpoint_info* info) {
    if (!h || !path || !info) return fail(SPDK_E_ARG, "null argument");
    if (int rc = spdk_hydro_checkpoint_wait(h)) return rc;
    const size_t ubytes = (size_t)h->E * h->V * h->NPT * h->esz;
    std::vector<unsigned char> buf(ubytes);
    double dt = 0;
    if (cudaMemcpyAsync(buf.data(), h->u, ubytes, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(&dt, h->dt, sizeof(double), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
        return fail(SPDK_E_CUDA, std::string("checkpoint copy: ") + cudaGetErrorString(cudaGetLastError()));
    CkptHeader hd = make_header(h, *info);
    hd.dt = dt;
    std::string err;
    if (!write_ckpt(path, hd, buf.data(), ubytes, &err)) return fail(SPDK_E_IO, err);
    return 0;
}

int spdk_hydro_checkpoint_async(spdk_hydro* h, const char* path, const spdk_checkpoint_info* info) {
    if (!h || !path || !info) return fail(SPDK_E_ARG, "null argument");
    if (int rc = spdk_hydro_checkpoint_wait(h)) return rc;
    const size_t ubytes = (size_t)h->E * h->V * h->NPT * h->esz;
    const size_t total = dt_offset(ubytes) + sizeof(double);
    if (!h->ck_dev) {
        // snapshot buffers, made once per solver (outside any step)
        if (cudaMalloc((void**)&h->ck_dev, total) != cudaSuccess)
            return fail(SPDK_E_NOMEM, "checkpoint snapshot");
        if (cudaMallocHost((void**)&h->ck_host, total) != cudaSuccess ||
            cudaStreamCreateWithFlags(&h->ck_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->ck_snap, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->ck_done, cudaEventDisableTiming) != cudaSuccess) {
            checkpoint_release(h);
            return fail(SPDK_E_CUDA, "checkpoint buffers");
        }
        h->ck_bytes = total;
    }
    if (cudaMemcpyAsync(h->ck_dev, h->u, ubytes, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(h->ck_dev + dt_offset(ubytes), h->dt, sizeof(double), cudaMemcpyDeviceToDevice, h->stream) !=
            cudaSuccess ||
        cudaEventRecord(h->ck_snap, h->stream) != cudaSuccess ||
        cudaStreamWaitEvent(h->ck_stream, h->ck_snap, 0) != cudaSuccess ||
        cudaMemcpyAsync(h->ck_host, h->ck_dev, total, cudaMemcpyDeviceToHost, h->ck_stream) != cudaSuccess ||
        cudaEventRecord(h->ck_done, h->ck_stream) != cudaSuccess)
        return fail(SPDK_E_CUDA, std::string("checkpoint snapshot: ") + cudaGetErrorString(cudaGetLastError()));
    const CkptHeader hd0 = make_header(h, *info);
    const std::string file(path);
    const int device = h->cfg.device;
    h->ck_status = 0;
    h->ck_error.clear();
    h->ck_thread = new std::thread([h, hd0, file, ubytes, device]() {
        cudaSetDevice(device);
        if (cudaEventSynchronize(h->ck_done) != cudaSuccess) {
            h->ck_status = SPDK_E_CUDA;
            h->ck_error = "checkpoint copy failed";
            return;
        }
        CkptHeader hd = hd0;
        std::memcpy(&hd.dt, h->ck_host + dt_offset(ubytes), sizeof(double));
        std::string err;
        if (!write_ckpt(file, hd, h->ck_host, ubytes, &err)) {
            h->ck_status = SPDK_E_IO;
            h->ck_error = err;
        }
    });
    return 0;
}

int spdk_hydro_checkpoint_wait(spdk_hydro* h) {
    if (!h) return fail(SPDK_E_ARG, "null argument");
    if (!h->ck_thread) return 0;
    h->ck_thread->join();
    delete h->ck_thread;
    h->ck_thread = nullptr;
    if (h->ck_status) return fail(h->ck_status, h->ck_error);
    return 0;
}

int spdk_hydro_restore(spdk_hydro* h, const char* path, spdk_checkpoint_info* info) {
    if (!h || !path) return fail(SPDK_E_ARG, "null argument");
    if (int rc = spdk_hydro_checkpoint_wait(h)) return rc;
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(SPDK_E_IO, std::string("cannot open ") + path);
    CkptHeader hd;
    int rc = read_header(f, path, &hd);
    const CkptHeader mine = make_header(h, spdk_checkpoint_info{});
    if (!rc) {
        bool same = hd.precision == mine.precision && hd.D == mine.D && hd.p == mine.p && hd.V == mine.V &&
                    hd.NPT == mine.NPT && hd.integrator == mine.integrator && hd.rk_order == mine.rk_order &&
                    hd.fallback == mine.fallback && hd.esz == mine.esz && hd.count == mine.count &&
                    hd.gamma == mine.gamma && hd.cfl == mine.cfl;
        for (int d = 0; d < 3; d++) same = same && hd.N[d] == mine.N[d] && hd.bc[d] == mine.bc[d];
        if (hd.version >= 2) {
            // geometry and physics: a state of another box, gravity, viscosity,
            // fallback setting or slab would restore silently and diverge
            for (int d = 0; d < 3; d++) same = same && hd.L[d] == mine.L[d] && hd.g[d] == mine.g[d];
            same = same && hd.nu == mine.nu && hd.beta == mine.beta && hd.nad_tolerance == mine.nad_tolerance &&
                   hd.nad_delta == mine.nad_delta && hd.nad_moore == mine.nad_moore && hd.sed == mine.sed &&
                   hd.blending == mine.blending && hd.slab_lo == mine.slab_lo && hd.slab_n == mine.slab_n;
        }
        if (!same) rc = fail(SPDK_E_ARG, std::string(path) + " was written by a solver of another configuration");
    }
    std::vector<unsigned char> buf;
    if (!rc) {
        buf.resize(hd.count * hd.esz);
        if (std::fread(buf.data(), 1, buf.size(), f) != buf.size())
            rc = fail(SPDK_E_IO, std::string("short checkpoint state in ") + path);
    }
    std::fclose(f);
    if (rc) return rc;
    // U through the write path (which also recomputes W_cv); FP32 values
    // widen to doubles and round back to themselves
    if (h->prec == SPDK_PRECISION_FP32) {
        std::vector<double> w(hd.count);
        const float* v = reinterpret_cast<const float*>(buf.data());
        for (size_t q = 0; q < hd.count; q++) w[q] = v[q];
        rc = spdk_hydro_write(h, SPDK_FIELD_U_SP, w.data(), w.size());
    } else {
        rc = spdk_hydro_write(h, SPDK_FIELD_U_SP, reinterpret_cast<const double*>(buf.data()), hd.count);
    }
    if (!rc) rc = spdk_hydro_set_dt(h, hd.dt);
    if (rc) return rc;
    if (info) {
        info->t = hd.t;
        info->t_output = hd.t_output;
        info->steps = hd.steps;
        info->outputs = hd.outputs;
    }
    return 0;
}

int spdk_checkpoint_peek(const char* path, spdk_checkpoint_info* info, int* precision, int* p, int N[3],
                         int* integrator, int* rk_order) {
    if (!path) return fail(SPDK_E_ARG, "null argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(SPDK_E_IO, std::string("cannot open ") + path);
    CkptHeader hd;
    const int rc = read_header(f, path, &hd);
    std::fclose(f);
    if (rc) return rc;
    if (info) {
        info->t = hd.t;
        info->t_output = hd.t_output;
        info->steps = hd.steps;
        info->outputs = hd.outputs;
    }
    if (precision) *precision = (int)hd.precision;
    if (p) *p = (int)hd.p;
    if (N)
        for (int d = 0; d < 3; d++) N[d] = (int)hd.N[d];
    if (integrator) *integrator = (int)hd.integrator;
    if (rk_order) *rk_order = (int)hd.rk_order;
    return 0;
}

}  // extern "C"
