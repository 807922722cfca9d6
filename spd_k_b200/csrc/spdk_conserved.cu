// Domain integrals of the conserved variables in FP64 with compensated
// summation, for both forms (the precision form's FP32 state is widened
// exactly). The reference's mass diagnostic (src/hydro_ader.hpp:464-498,
// fv_mass) sums the sub-cell averages U_cv of the density times the
// sub-cell volumes over the active cells; this does the same for every
// conserved variable: U_cv from U_sp by sp_to_cv along each direction, each
// product U_cv * volume added with Neumaier's compensated summation in a
// fixed order (per thread, then per block, then over the blocks), so the
// result is reproducible and carries no accumulated rounding of the sum.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "spdk.h"
#include "spdk_hydro_impl.h"

namespace spdk {
int fail(int code, const std::string& msg);
}

namespace {

constexpr int kThreadsC = 256;
constexpr int kMaxV = 5;

struct ConservedArgs {
    const void* u;       // [E][V][NPT] of double or float
    int fp32;
    int D, n, V, NPT;
    int N[3];
    long long E;
    const double* w[3];  // active sub-cell widths per direction (N[d] * n)
    double C[64];        // sp_to_cv [n][n]
    double2* part;       // [gridDim.x][V] (sum, compensation)
};

// Neumaier's compensated addition: s + c carries the sum of the addends
// with the rounding of each addition kept in c
__device__ __forceinline__ void nadd(double& s, double& c, double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

__global__ void __launch_bounds__(kThreadsC) conserved_partials(ConservedArgs A) {
    extern __shared__ double sbuf[];
    double* a = sbuf;                      // [V][NPT]
    double* b = sbuf + A.V * A.NPT;        // [V][NPT]
    __shared__ double2 red[kThreadsC];
    double s[kMaxV], c[kMaxV];
    for (int v = 0; v < kMaxV; v++) s[v] = c[v] = 0;
    const int n = A.n, NPT = A.NPT, VN = A.V * A.NPT;
    for (long long e = blockIdx.x; e < A.E; e += gridDim.x) {
        for (int q = threadIdx.x; q < VN; q += blockDim.x)
            a[q] = A.fp32 ? (double)((const float*)A.u)[e * VN + q] : ((const double*)A.u)[e * VN + q];
        __syncthreads();
        // sp -> cv along each direction: out[c_d = i] = sum_m C[i][m] in[c_d = m]
        double* src = a;
        double* dst = b;
        for (int d = 0; d < A.D; d++) {
            const int st = d == 0 ? 1 : (d == 1 ? n : n * n);
            for (int q = threadIdx.x; q < VN; q += blockDim.x) {
                const int pt = q % NPT;
                const int id = (pt / st) % n;
                const int base = q - id * st;
                double u = 0;
                for (int m = 0; m < n; m++) u += A.C[id * n + m] * src[base + m * st];
                dst[q] = u;
            }
            __syncthreads();
            double* t = src;
            src = dst;
            dst = t;
        }
        const long long ex = e % A.N[0], ey = (e / A.N[0]) % A.N[1], ez = e / ((long long)A.N[0] * A.N[1]);
        for (int q = threadIdx.x; q < VN; q += blockDim.x) {
            const int v = q / NPT, pt = q % NPT;
            const int ii = pt % n, jj = (pt / n) % n, kk = pt / (n * n);
            double vol = A.w[0][ex * n + ii];
            if (A.D >= 2) vol *= A.w[1][ey * n + jj];
            if (A.D == 3) vol *= A.w[2][ez * n + kk];
            const double x = src[q] * vol;
            for (int k = 0; k < kMaxV; k++)
                if (k == v) nadd(s[k], c[k], x);
        }
        __syncthreads();
    }
    // the block's pairs, variable by variable, in thread order
    for (int v = 0; v < A.V; v++) {
        red[threadIdx.x] = make_double2(s[v], c[v]);
        __syncthreads();
        if (threadIdx.x == 0) {
            double bs = 0, bc = 0;
            for (int t = 0; t < blockDim.x; t++) {
                nadd(bs, bc, red[t].x);
                nadd(bs, bc, red[t].y);
            }
            A.part[(size_t)blockIdx.x * A.V + v] = make_double2(bs, bc);
        }
        __syncthreads();
    }
}

__global__ void conserved_final(const double2* part, int blocks, int V, double* out) {
    const int v = threadIdx.x;
    if (v >= V) return;
    double s = 0, c = 0;
    for (int b = 0; b < blocks; b++) {
        nadd(s, c, part[(size_t)b * V + v].x);
        nadd(s, c, part[(size_t)b * V + v].y);
    }
    out[v] = s + c;
}

}  // namespace

extern "C" int spdk_hydro_conserved(spdk_hydro* h, double* sums, int count) {
    if (!h || !sums) return spdk::fail(SPDK_E_ARG, "null argument");
    if (count != h->V) return spdk::fail(SPDK_E_ARG, "count must be " + std::to_string(h->V));
    if (h->D < 2 || h->n > 8) return spdk::fail(SPDK_E_ARG, "2D or 3D, p <= 7");
    if (h->cfg.slab_n != 0)
        return spdk::fail(SPDK_E_ARG, "a slab solver holds halo rows: sum the whole domain's solver instead");
    ConservedArgs A{};
    A.u = h->u;
    A.fp32 = h->prec == SPDK_PRECISION_FP32;
    A.D = h->D;
    A.n = h->n;
    A.V = h->V;
    A.NPT = h->NPT;
    A.E = h->E;
    for (int d = 0; d < 3; d++) A.N[d] = h->G.N[d];
    for (int i = 0; i < h->n * h->n; i++) A.C[i] = h->mats.sp_to_cv[i];
    const int blocks = (int)std::min<long long>(h->E, 148LL * 8);
    // sub-cell widths of the active cells (frame index a + 2 .. a + 3) and
    // the block partials, in one allocation
    size_t nw[3] = {0, 0, 0}, total = 0;
    for (int d = 0; d < h->D; d++) {
        nw[d] = (size_t)h->G.N[d] * h->n;
        total += nw[d];
    }
    std::vector<double> host(total);
    size_t off = 0;
    for (int d = 0; d < h->D; d++) {
        const std::vector<double>& f = h->ax[d].fv_faces;
        for (size_t a = 0; a < nw[d]; a++) host[off + a] = f[a + 3] - f[a + 2];
        off += nw[d];
    }
    void* buf = nullptr;
    const size_t bytes = total * sizeof(double) + (size_t)blocks * h->V * sizeof(double2) + h->V * sizeof(double);
    if (cudaMalloc(&buf, bytes) != cudaSuccess) return spdk::fail(SPDK_E_NOMEM, "conserved sums: device allocation");
    double* wdev = (double*)buf;
    A.part = (double2*)(wdev + total);
    double* out = (double*)(A.part + (size_t)blocks * h->V);
    int rc = 0;
    if (cudaMemcpyAsync(wdev, host.data(), total * sizeof(double), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
        rc = spdk::fail(SPDK_E_CUDA, "conserved sums: widths");
    off = 0;
    for (int d = 0; d < 3; d++) {
        A.w[d] = d < h->D ? wdev + off : nullptr;
        if (d < h->D) off += nw[d];
    }
    if (!rc) {
        const size_t smem = 2 * (size_t)h->V * h->NPT * sizeof(double);
        conserved_partials<<<blocks, kThreadsC, smem, h->stream>>>(A);
        conserved_final<<<1, 32, 0, h->stream>>>(A.part, blocks, h->V, out);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(sums, out, h->V * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) rc = spdk::fail(SPDK_E_CUDA, std::string("conserved sums: ") + cudaGetErrorString(e));
    }
    cudaFree(buf);
    return rc;
}
