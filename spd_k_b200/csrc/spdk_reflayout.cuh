// Device arrays in the reference's own layout (LayoutRight views with ghost
// elements / ghost frames, src/define.hpp:99-130, src/fv_structs.hpp:41-100)
// and the generic kernels the reference-layout entry points share: the 1-D
// tensor transform, the SSP-RK combination and the SD interface ghost fill.
// One thread per output point, reference operation order.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "spdk.h"
#include "spdk_physics.cuh"

namespace spdk {
int fail(int code, const std::string& msg);
}

namespace {

using namespace spdk;

constexpr int kBlock = 256;

struct SDa {
    double* p;
    int e[8];  // t, var, k, j, i, kk, jj, ii
    __host__ __device__ long long pts() const { return (long long)e[2] * e[3] * e[4] * e[5] * e[6] * e[7]; }
    __device__ double& at(int t, int v, int k, int j, int i, int kk, int jj, int ii) const {
        long long o = (((((long long)t * e[1] + v) * e[2] + k) * e[3] + j) * e[4] + i);
        o = ((o * e[5] + kk) * e[6] + jj) * e[7] + ii;
        return p[o];
    }
};
struct FVa {
    double* p;
    int e[4];  // var, K, J, I
    __host__ __device__ long long cells() const { return (long long)e[1] * e[2] * e[3]; }
    __device__ double& at(int v, int k, int j, int i) const {
        return p[(((long long)v * e[1] + k) * e[2] + j) * e[3] + i];
    }
};
unsigned blocks_for(long long n) {
    long long b = (n + kBlock - 1) / kBlock;
    if (b > 148LL * 32) b = 148LL * 32;
    return (unsigned)(b < 1 ? 1 : b);
}
int launched(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return 0;
}
__host__ __device__ __forceinline__ int choose(int dim, int i, int j, int k) {
    return dim == 0 ? i : (dim == 1 ? j : k);
}

// decompose a linear index over the (k, j, i, kk, jj, ii) extents of a
__device__ __forceinline__ void point_of(const SDa& a, long long q, int c[6]) {
    for (int x = 5; x >= 0; x--) {
        c[x] = (int)(q % a.e[2 + x]);
        q /= a.e[2 + x];
    }
}

// ---- transforms: src/transforms.cpp:120-177 -------------------------------
__global__ void k_transform_1d(SDa A, SDa B, const double* __restrict__ M, int mcols, int dim, int tsrc) {
    const int q = choose(dim, A.e[7], A.e[6], A.e[5]);
    const int nt = tsrc < 0 ? A.e[0] : 1;
    const long long n = B.pts() * nt * A.e[1];
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
        const int var = (int)(o % A.e[1]);
        long long r = o / A.e[1];
        const int t = (int)(r % nt);
        r /= nt;
        int c[6];
        point_of(B, r, c);
        const int k = c[0], j = c[1], i = c[2], kk = c[3], jj = c[4], ii = c[5];
        const int id = choose(dim, ii, jj, kk);
        const int ts = tsrc < 0 ? t : tsrc;
        double u = 0;
        for (int ll = 0; ll < q; ll++) {
            const int n0 = dim == 0 ? ll : ii, n1 = dim == 1 ? ll : jj, n2 = dim == 2 ? ll : kk;
            u += A.at(ts, var, k, j, i, n2, n1, n0) * M[id * mcols + ll];
        }
        B.at(tsrc < 0 ? t : 0, var, k, j, i, kk, jj, ii) = u;
    }
}

// src/transforms.cpp:252-261 (slice 0 of U)
__global__ void k_combine(SDa U, SDa U0, double a) {
    const long long n = (long long)U.e[1] * U.pts();
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x)
        U.p[o] = a * U0.p[o] + (1.0 - a) * U.p[o];
}

// src/boundary.cpp:48-113: the interface point of the ghost elements of
// direction dim <- periodic partner / copy / mirror (normal slot 1+dim
// negated); reads only interior elements, so one pass equals the
// reference's pack-then-unpack
__global__ void k_boundaries_sd(SDa U, int dim, int type) {
    const int N = choose(dim, U.e[4], U.e[3], U.e[2]), n = choose(dim, U.e[7], U.e[6], U.e[5]);
    const int Ez = dim == 2 ? 1 : U.e[2], Ey = dim == 1 ? 1 : U.e[3], Ex = dim == 0 ? 1 : U.e[4];
    const int ez = dim == 2 ? 1 : U.e[5], ey = dim == 1 ? 1 : U.e[6], ex = dim == 0 ? 1 : U.e[7];
    const long long cnt = (long long)Ez * Ey * Ex * ez * ey * ex * U.e[0] * U.e[1];
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < cnt; o += (long long)gridDim.x * blockDim.x) {
        long long r = o;
        const int var = (int)(r % U.e[1]); r /= U.e[1];
        const int t = (int)(r % U.e[0]); r /= U.e[0];
        const int ii = (int)(r % ex); r /= ex;
        const int jj = (int)(r % ey); r /= ey;
        const int kk = (int)(r % ez); r /= ez;
        const int i = (int)(r % Ex); r /= Ex;
        const int j = (int)(r % Ey); r /= Ey;
        const int k = (int)r;
        auto at = [&](int E, int P) -> double& {
            return U.at(t, var, dim == 2 ? E : k, dim == 1 ? E : j, dim == 0 ? E : i, dim == 2 ? P : kk,
                        dim == 1 ? P : jj, dim == 0 ? P : ii);
        };
        double L, R;
        if (type == kPeriodic) { L = at(N - 2, n - 1); R = at(1, 0); }
        else if (type == kGradfree) { L = at(1, 0); R = at(N - 2, n - 1); }
        else {
            const double sgn = (var == 1 + dim) ? -1.0 : 1.0;
            L = sgn * at(1, 0);
            R = sgn * at(N - 2, n - 1);
        }
        at(0, n - 1) = L;
        at(N - 1, 0) = R;
    }
}

}  // namespace
