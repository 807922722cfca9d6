// The FP32 Picard pass's divergence contraction on CUDA cores and on tensor
// cores, for measurement. No counterpart in the reference.
//
// For every element-variable ev (count of them) of a 2D order-p run:
//   dudt[ev][jj][ii] = sum_ll Fx[ev][jj][ll] D[ii][ll] + Fy[ev][ii][ll] D[jj][ll]
// with D = dfp_to_sp (n x nf). This is the flux divergence of the Picard
// passes (src/transforms.cpp:296-303) in the FP32 form. Two kernels compute
// it from the same global arrays:
//   mode 0 (CUDA cores): the same staging, then one thread per 2 x 2 point
//     block of one ev, the form the Picard pass uses (FP32 FMAs);
//   mode 1 (tensor cores): one warp per 16 ev's as batched small GEMMs on
//     mma.sync m16n8k8 TF32 with FP32 accumulation and the 3xTF32 split
//     (x = hi + lo; lo*hi + hi*lo + hi*hi): the x term with rows (ev, jj),
//     K = ll, N = ii; the y term with rows jj, K = ll, N = (ev, ii); K padded
//     from nf = 5 to 8, the short sides to the MMA's 16 x 8.
// p = 3 only (n = 4, nf = 5), the headline order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "spdk.h"
#include "spdk_setup.h"

namespace spdk {
int fail(int code, const std::string& msg);
}

namespace {

using namespace spdk;

constexpr int kN = 4, kNF = 5;

struct StudyMats {
    float D[kN * kNF];  // dfp_to_sp [ii][ll]
};

// mode 0: one warp per 16 ev's, staged in shared memory exactly as mode 1
// stages them (so both modes read their operands the same way, as the
// Picard pass reads its flux points from shared memory); each lane then
// takes two (ev, 2 x 2 block) items -- the Picard pass's thread mapping --
// and computes them with FP32 FMAs
constexpr int kEvPerWarp = 16;
constexpr int kWarps = 8;

__global__ void __launch_bounds__(256) div_cuda_cores(StudyMats M, long long count, const float* __restrict__ fx,
                                                     const float* __restrict__ fy, float* __restrict__ dudt) {
    __shared__ float sx[kWarps][kEvPerWarp * kN * kNF];
    __shared__ float sy[kWarps][kEvPerWarp * kN * kNF];
    __shared__ float so[kWarps][kEvPerWarp * kN * kN];
    // the coefficients are read at lane-dependent offsets: shared memory, not
    // the parameter space
    __shared__ float D[kN * kNF];
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < kN * kNF; q++) D[q] = M.D[q];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long groups = (count + kEvPerWarp - 1) / kEvPerWarp;
    for (long long grp = (long long)blockIdx.x * kWarps + warp; grp < groups; grp += (long long)gridDim.x * kWarps) {
        const long long ev0 = grp * kEvPerWarp;
        const int nev = (int)min((long long)kEvPerWarp, count - ev0);
        for (int q = lane; q < kEvPerWarp * kN * kNF; q += 32) {
            const bool ok = q < nev * kN * kNF;
            sx[warp][q] = ok ? fx[ev0 * kN * kNF + q] : 0.f;
            sy[warp][q] = ok ? fy[ev0 * kN * kNF + q] : 0.f;
        }
        __syncwarp();
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int item = lane + 32 * k;  // (block, ev): block-major, 16 ev's per block
            const int ev = item % kEvPerWarp, b = item / kEvPerWarp;
            const int bx0 = (b & 1) * 2, by0 = (b >> 1) * 2;
            const float* X = sx[warp] + ev * kN * kNF;  // [jj][ll]
            const float* Y = sy[warp] + ev * kN * kNF;  // [ii][ll]
            float dd[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
            for (int ll = 0; ll < kNF; ll++) {
                const float x0 = X[(by0 + 0) * kNF + ll], x1 = X[(by0 + 1) * kNF + ll];
                const float y0 = Y[(bx0 + 0) * kNF + ll], y1 = Y[(bx0 + 1) * kNF + ll];
                const float c0 = D[(bx0 + 0) * kNF + ll], c1 = D[(bx0 + 1) * kNF + ll];
                const float r0 = D[(by0 + 0) * kNF + ll], r1 = D[(by0 + 1) * kNF + ll];
                dd[0][0] += x0 * c0 + y0 * r0;
                dd[0][1] += x0 * c1 + y1 * r0;
                dd[1][0] += x1 * c0 + y0 * r1;
                dd[1][1] += x1 * c1 + y1 * r1;
            }
            float* out = so[warp] + ev * kN * kN;
#pragma unroll
            for (int j = 0; j < 2; j++)
#pragma unroll
                for (int i = 0; i < 2; i++) out[(by0 + j) * kN + bx0 + i] = dd[j][i];
        }
        __syncwarp();
        for (int q = lane; q < nev * kN * kN; q += 32) dudt[ev0 * kN * kN + q] = so[warp][q];
        __syncwarp();
    }
}

__device__ __forceinline__ uint32_t tf32_bits(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
// x = hi + lo, both TF32 values
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
    hi = tf32_bits(x);
    lo = tf32_bits(x - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
// c += a b with the 3xTF32 split of both operands (small terms first)
__device__ __forceinline__ void mma_3xtf32(float (&c)[4], const uint32_t (&ah)[4], const uint32_t (&al)[4],
                                           const uint32_t (&bh)[2], const uint32_t (&bl)[2]) {
    mma_tf32(c, al, bh);
    mma_tf32(c, ah, bl);
    mma_tf32(c, ah, bh);
}

// mode 1: one warp per 16 ev's; the warp's Fx, Fy rows are staged in shared
// memory, the two GEMMs' results summed there and written back coalesced

__global__ void __launch_bounds__(256) div_tensor_cores(StudyMats M, long long count, const float* __restrict__ fx,
                                                       const float* __restrict__ fy, float* __restrict__ dudt) {
    __shared__ float sx[kWarps][kEvPerWarp * kN * kNF];
    __shared__ float sy[kWarps][kEvPerWarp * kN * kNF];
    __shared__ float so[kWarps][kEvPerWarp * kN * kN];
    __shared__ float D[kN * kNF];
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < kN * kNF; q++) D[q] = M.D[q];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;  // MMA fragment row group, thread in group
    // constant fragments: the x term's B = D^T (K = ll, N = ii), the y term's
    // A = D (rows jj, K = ll); entries outside n x nf are zero
    auto Dv = [&](int r, int c) { return (r < kN && c < kNF) ? D[r * kNF + c] : 0.f; };
    uint32_t bxh[2], bxl[2], ayh[4], ayl[4];
    split_tf32(Dv(g, t), bxh[0], bxl[0]);          // B(k = t, n = g) = D[g][t]
    split_tf32(Dv(g, t + 4), bxh[1], bxl[1]);      // B(k = t + 4, n = g)
    split_tf32(Dv(g, t), ayh[0], ayl[0]);          // A(row g, k = t)
    split_tf32(Dv(g + 8, t), ayh[1], ayl[1]);      // A(row g + 8, k = t)
    split_tf32(Dv(g, t + 4), ayh[2], ayl[2]);      // A(row g, k = t + 4)
    split_tf32(Dv(g + 8, t + 4), ayh[3], ayl[3]);  // A(row g + 8, k = t + 4)
    const long long groups = (count + kEvPerWarp - 1) / kEvPerWarp;
    for (long long grp = (long long)blockIdx.x * kWarps + warp; grp < groups; grp += (long long)gridDim.x * kWarps) {
        const long long ev0 = grp * kEvPerWarp;
        const int nev = (int)min((long long)kEvPerWarp, count - ev0);
        for (int q = lane; q < kEvPerWarp * kN * kNF; q += 32) {
            const bool ok = q < nev * kN * kNF;
            sx[warp][q] = ok ? fx[ev0 * kN * kNF + q] : 0.f;
            sy[warp][q] = ok ? fy[ev0 * kN * kNF + q] : 0.f;
        }
        __syncwarp();
        // x term: 64 rows (ev, jj) in 4 m-tiles, K = ll, N = ii
        const float* X = sx[warp];
        auto xa = [&](int row, int k) { return k < kNF ? X[row * kNF + k] : 0.f; };
#pragma unroll
        for (int mt = 0; mt < 4; mt++) {
            uint32_t ah[4], al[4];
            split_tf32(xa(mt * 16 + g, t), ah[0], al[0]);
            split_tf32(xa(mt * 16 + g + 8, t), ah[1], al[1]);
            split_tf32(xa(mt * 16 + g, t + 4), ah[2], al[2]);
            split_tf32(xa(mt * 16 + g + 8, t + 4), ah[3], al[3]);
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            mma_3xtf32(c, ah, al, bxh, bxl);
            // c0, c1: row g, cols 2t, 2t+1; c2, c3: row g + 8
            if (2 * t < kN) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int row = mt * 16 + g + 8 * h;  // = ev * n + jj
                    so[warp][row * kN + 2 * t] = c[2 * h];
                    so[warp][row * kN + 2 * t + 1] = c[2 * h + 1];
                }
            }
        }
        __syncwarp();
        // y term: rows jj (4 of 16), K = ll, N = (ev, ii) in 8 n-tiles
        const float* Y = sy[warp];
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            // B(k, n): n = column (ev, ii) = nt * 8 + g, k = ll
            const int col = nt * 8 + g;
            uint32_t bh[2], bl[2];
            split_tf32(t < kNF ? Y[col * kNF + t] : 0.f, bh[0], bl[0]);
            split_tf32(t + 4 < kNF ? Y[col * kNF + t + 4] : 0.f, bh[1], bl[1]);
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            mma_3xtf32(c, ayh, ayl, bh, bl);
            // c0, c1: row jj = g, cols nt * 8 + 2t, + 1 (rows >= n are zero)
            if (g < kN) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int cc = nt * 8 + 2 * t + h;  // = ev * n + ii
                    const int ev = cc / kN, ii = cc % kN;
                    so[warp][(ev * kN + g) * kN + ii] += c[h];
                }
            }
        }
        __syncwarp();
        for (int q = lane; q < nev * kN * kN; q += 32) dudt[ev0 * kN * kN + q] = so[warp][q];
        __syncwarp();
    }
}

}  // namespace

extern "C" int spdk_study_divergence(int mode, int p, long long count, const float* fx, const float* fy, float* dudt,
                                     void* stream) {
    if (p != 3) return fail(SPDK_E_ARG, "the divergence study covers p = 3");
    if (mode != 0 && mode != 1) return fail(SPDK_E_ARG, "mode must be 0 (CUDA cores) or 1 (tensor cores)");
    if (count < 0 || (count > 0 && (!fx || !fy || !dudt))) return fail(SPDK_E_ARG, "null argument");
    if (count == 0) return 0;
    Matrices m;
    build_matrices(p, true, &m);
    StudyMats M;
    for (int q = 0; q < kN * kNF; q++) M.D[q] = (float)m.dfp_to_sp[q];
    cudaStream_t s = (cudaStream_t)stream;
    const long long groups = (count + kEvPerWarp - 1) / kEvPerWarp;
    const unsigned blocks = (unsigned)std::min<long long>((groups + kWarps - 1) / kWarps, 148LL * 32);
    if (mode == 0) div_cuda_cores<<<blocks, 256, 0, s>>>(M, count, fx, fy, dudt);
    else div_tensor_cores<<<blocks, 256, 0, s>>>(M, count, fx, fy, dudt);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(SPDK_E_CUDA, std::string("divergence study: ") + cudaGetErrorString(e));
    return 0;
}
