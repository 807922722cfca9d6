// Learned a-priori troubled-cell indicator: feature rows of a solver state,
// and the MLP's forward, loss/gradient and Adam kernels (declarations and
// the model in include/spdk_learned.h).
//
// The network is tiny (about 7k parameters), so every kernel keeps the
// whole model in shared memory as BF16 and gives each block a tile of 32
// samples; products of BF16 values accumulate in FP32. The gradient is
// reduced deterministically: each block writes its partial sums, a second
// kernel adds the partials in block order.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "spdk.h"
#include "spdk_learned.h"
#include "spdk_learned_impl.h"

namespace spdk {
int fail(int code, const std::string& msg);
}

namespace {

using namespace spdk;

constexpr int kH = 64;        // hidden width
constexpr int kSB = 32;       // samples per block
constexpr int kThreadsM = 256;
constexpr int kMaxIn = 448;

__device__ __forceinline__ float bf(uint16_t v) { return __uint_as_float((uint32_t)v << 16); }
__device__ __forceinline__ uint16_t to_bf(float f) {
    __nv_bfloat16 b = __float2bfloat16_rn(f);
    return *reinterpret_cast<uint16_t*>(&b);
}
// GELU, erf form, and its derivative
__device__ __forceinline__ float gelu(float a) { return 0.5f * a * (1.0f + erff(a * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float a) {
    return 0.5f * (1.0f + erff(a * 0.70710678118654752f)) + a * 0.39894228040143268f * expf(-0.5f * a * a);
}

struct Layout {
    int n_in;
    int oW1, ob1, oW2, ob2, ow3, ob3, n;
};
__host__ __device__ inline Layout layout(int n_in) {
    Layout L;
    L.n_in = n_in;
    L.oW1 = 0;
    L.ob1 = n_in * kH;
    L.oW2 = L.ob1 + kH;
    L.ob2 = L.oW2 + kH * kH;
    L.ow3 = L.ob2 + kH;
    L.ob3 = L.ow3 + kH;
    L.n = L.ob3 + 1;
    return L;
}

// shared memory of one block: BF16 parameters, FP32 activations of kSB samples
struct Smem {
    int wbytes, xoff, a1, h1, a2, h2, d2, d1, z, total;
};
__host__ __device__ inline Smem smem_layout(int n_in) {
    const Layout L = layout(n_in);
    Smem s;
    s.wbytes = ((L.n * 2 + 15) / 16) * 16;
    s.xoff = s.wbytes;                               // float X [kSB][n_in]
    s.a1 = s.xoff + kSB * n_in * 4;                  // float [kSB][kH] each
    s.h1 = s.a1 + kSB * kH * 4;
    s.a2 = s.h1 + kSB * kH * 4;
    s.h2 = s.a2 + kSB * kH * 4;
    s.d2 = s.h2 + kSB * kH * 4;
    s.d1 = s.d2 + kSB * kH * 4;
    s.z = s.d1 + kSB * kH * 4;                       // float [kSB]
    s.total = s.z + kSB * 4;
    return s;
}

// forward pass of the block's samples into shared memory (A1, H1, A2, H2, z)
__device__ void forward_tile(const Layout& L, const Smem& S, unsigned char* sm, const uint16_t* __restrict__ x,
                             long long s0, int batch) {
    const uint16_t* W = reinterpret_cast<const uint16_t*>(sm);
    float* X = reinterpret_cast<float*>(sm + S.xoff);
    float* A1 = reinterpret_cast<float*>(sm + S.a1);
    float* H1 = reinterpret_cast<float*>(sm + S.h1);
    float* A2 = reinterpret_cast<float*>(sm + S.a2);
    float* H2 = reinterpret_cast<float*>(sm + S.h2);
    float* Z = reinterpret_cast<float*>(sm + S.z);
    const int n_in = L.n_in;
    for (int q = threadIdx.x; q < kSB * n_in; q += blockDim.x) {
        const int s = q / n_in, k = q % n_in;
        X[q] = (s0 + s < batch) ? bf(x[(s0 + s) * n_in + k]) : 0.0f;
    }
    __syncthreads();
    const int j = threadIdx.x % kH, g = threadIdx.x / kH;  // 4 sample groups
    constexpr int G = kThreadsM / kH, PS = kSB / G;
    {
        float acc[PS];
#pragma unroll
        for (int r = 0; r < PS; r++) acc[r] = 0.0f;
        for (int k = 0; k < n_in; k++) {
            const float w = bf(W[L.oW1 + k * kH + j]);
#pragma unroll
            for (int r = 0; r < PS; r++) acc[r] += X[(g + r * G) * n_in + k] * w;
        }
        const float b = bf(W[L.ob1 + j]);
#pragma unroll
        for (int r = 0; r < PS; r++) {
            const int s = g + r * G;
            const float a = acc[r] + b;
            A1[s * kH + j] = a;
            H1[s * kH + j] = gelu(a);
        }
    }
    __syncthreads();
    {
        float acc[PS];
#pragma unroll
        for (int r = 0; r < PS; r++) acc[r] = 0.0f;
        for (int k = 0; k < kH; k++) {
            const float w = bf(W[L.oW2 + k * kH + j]);
#pragma unroll
            for (int r = 0; r < PS; r++) acc[r] += H1[(g + r * G) * kH + k] * w;
        }
        const float b = bf(W[L.ob2 + j]);
#pragma unroll
        for (int r = 0; r < PS; r++) {
            const int s = g + r * G;
            const float a = acc[r] + b;
            A2[s * kH + j] = a;
            H2[s * kH + j] = gelu(a);
        }
    }
    __syncthreads();
    if (threadIdx.x < kSB) {
        const int s = threadIdx.x;
        float z = bf(W[L.ob3]);
        for (int k = 0; k < kH; k++) z += H2[s * kH + k] * bf(W[L.ow3 + k]);
        Z[s] = z;
    }
    __syncthreads();
}

__device__ void load_params(const Layout& L, unsigned char* sm, const uint16_t* __restrict__ wbf) {
    uint16_t* W = reinterpret_cast<uint16_t*>(sm);
    for (int q = threadIdx.x; q < L.n; q += blockDim.x) W[q] = wbf[q];
    __syncthreads();
}

__global__ void __launch_bounds__(kThreadsM) k_mlp_forward(int n_in, const uint16_t* __restrict__ wbf,
                                                             const uint16_t* __restrict__ x, int batch,
                                                             float* __restrict__ p, uint8_t* __restrict__ flags,
                                                             float thr) {
    extern __shared__ __align__(16) unsigned char sm[];
    const Layout L = layout(n_in);
    const Smem S = smem_layout(n_in);
    load_params(L, sm, wbf);
    const long long s0 = (long long)blockIdx.x * kSB;
    forward_tile(L, S, sm, x, s0, batch);
    const float* Z = reinterpret_cast<const float*>(sm + S.z);
    if (threadIdx.x < kSB && s0 + threadIdx.x < batch) {
        const float pr = 1.0f / (1.0f + expf(-Z[threadIdx.x]));
        if (p) p[s0 + threadIdx.x] = pr;
        if (flags) flags[s0 + threadIdx.x] = pr > thr ? 1 : 0;
    }
}

// Inference: a persistent grid; each block keeps the parameters in shared
// memory and walks tiles of 128 samples, each thread accumulating 4 hidden
// units x 8 samples in registers (12 shared loads per 32 FMAs). The sums
// run over k in the same order as forward_tile, so the probabilities are
// the same as the training kernels'.
constexpr int kSI = 128;  // samples per inference tile
constexpr size_t kInferSmemMax = 200 * 1024;
struct InferSmem {
    int wbytes, xoff, h1, total;
};
__host__ __device__ inline InferSmem infer_smem(int n_in) {
    const Layout L = layout(n_in);
    InferSmem s;
    s.wbytes = ((L.n * 2 + 15) / 16) * 16;
    s.xoff = s.wbytes;
    s.h1 = s.xoff + kSI * n_in * 4;
    s.total = s.h1 + kSI * kH * 4;
    return s;
}

__global__ void __launch_bounds__(kThreadsM) k_mlp_infer(int n_in, const uint16_t* __restrict__ wbf,
                                                           const uint16_t* __restrict__ x, long long batch,
                                                           float* __restrict__ p, uint8_t* __restrict__ flags,
                                                           float thr) {
    extern __shared__ __align__(16) unsigned char sm[];
    const Layout L = layout(n_in);
    const InferSmem S = infer_smem(n_in);
    load_params(L, sm, wbf);
    const uint16_t* W = reinterpret_cast<const uint16_t*>(sm);
    float* X = reinterpret_cast<float*>(sm + S.xoff);
    float* H1 = reinterpret_cast<float*>(sm + S.h1);
    const int j0 = threadIdx.x % 16, g = threadIdx.x / 16;  // units j0 + 16u, samples g + 16r
    const long long tiles = (batch + kSI - 1) / kSI;
    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const long long s0 = tile * kSI;
        for (int q = threadIdx.x; q < kSI * n_in; q += blockDim.x) {
            const int s = q / n_in, k = q % n_in;
            X[q] = (s0 + s < batch) ? bf(x[(s0 + s) * n_in + k]) : 0.0f;
        }
        __syncthreads();
        // two hidden layers: in [kSI][nk] -> gelu(in W + b); the first goes
        // to H1, the second straight into the output dot product
        float zp[8];
        for (int layer = 0; layer < 2; layer++) {
            const float* in = layer == 0 ? X : H1;
            const int nk = layer == 0 ? n_in : kH;
            const int oW = layer == 0 ? L.oW1 : L.oW2, ob = layer == 0 ? L.ob1 : L.ob2;
            float acc[8][4];
#pragma unroll
            for (int r = 0; r < 8; r++)
#pragma unroll
                for (int u = 0; u < 4; u++) acc[r][u] = 0.0f;
            for (int k = 0; k < nk; k++) {
                float w[4], xv[8];
#pragma unroll
                for (int u = 0; u < 4; u++) w[u] = bf(W[oW + k * kH + j0 + 16 * u]);
#pragma unroll
                for (int r = 0; r < 8; r++) xv[r] = in[(g + 16 * r) * nk + k];
#pragma unroll
                for (int r = 0; r < 8; r++)
#pragma unroll
                    for (int u = 0; u < 4; u++) acc[r][u] += xv[r] * w[u];
            }
            if (layer == 0) {
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const float b = bf(W[ob + j0 + 16 * u]);
#pragma unroll
                    for (int r = 0; r < 8; r++) H1[(g + 16 * r) * kH + j0 + 16 * u] = gelu(acc[r][u] + b);
                }
                __syncthreads();
            } else {
                // this thread's 4 units of w3 . H2 for its 8 samples, then the
                // 16 threads of a sample group (consecutive lanes) add up
#pragma unroll
                for (int r = 0; r < 8; r++) zp[r] = 0.0f;
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const float b = bf(W[ob + j0 + 16 * u]), w3 = bf(W[L.ow3 + j0 + 16 * u]);
#pragma unroll
                    for (int r = 0; r < 8; r++) zp[r] += gelu(acc[r][u] + b) * w3;
                }
#pragma unroll
                for (int r = 0; r < 8; r++)
#pragma unroll
                    for (int off = 8; off > 0; off >>= 1) zp[r] += __shfl_xor_sync(0xffffffffu, zp[r], off);
            }
        }
        if (j0 == 0) {
            const float b3 = bf(W[L.ob3]);
#pragma unroll
            for (int r = 0; r < 8; r++) {
                const long long s = s0 + g + 16 * r;
                if (s < batch) {
                    const float pr = 1.0f / (1.0f + expf(-(zp[r] + b3)));
                    if (p) p[s] = pr;
                    if (flags) flags[s] = pr > thr ? 1 : 0;
                }
            }
        }
        __syncthreads();
    }
}

// per block: sum_s w_s BCE_s, sum_s w_s and the unnormalised gradient
// sum_s w_s dBCE_s/dtheta into part[block][0 .. n+1]
__global__ void __launch_bounds__(kThreadsM) k_mlp_grad(int n_in, const uint16_t* __restrict__ wbf,
                                                          const uint16_t* __restrict__ x, const float* __restrict__ y,
                                                          const float* __restrict__ wt, int batch,
                                                          float* __restrict__ part) {
    extern __shared__ __align__(16) unsigned char sm[];
    const Layout L = layout(n_in);
    const Smem S = smem_layout(n_in);
    load_params(L, sm, wbf);
    const long long s0 = (long long)blockIdx.x * kSB;
    forward_tile(L, S, sm, x, s0, batch);
    const uint16_t* W = reinterpret_cast<const uint16_t*>(sm);
    float* X = reinterpret_cast<float*>(sm + S.xoff);
    float* A1 = reinterpret_cast<float*>(sm + S.a1);
    float* H1 = reinterpret_cast<float*>(sm + S.h1);
    float* A2 = reinterpret_cast<float*>(sm + S.a2);
    float* H2 = reinterpret_cast<float*>(sm + S.h2);
    float* D2 = reinterpret_cast<float*>(sm + S.d2);
    float* D1 = reinterpret_cast<float*>(sm + S.d1);
    float* Z = reinterpret_cast<float*>(sm + S.z);
    float* out = part + (size_t)blockIdx.x * (L.n + 2);
    __shared__ float dz[kSB], lw[kSB], ww[kSB];
    if (threadIdx.x < kSB) {
        const int s = threadIdx.x;
        float d = 0, l = 0, w = 0;
        if (s0 + s < batch) {
            const float z = Z[s], t = y[s0 + s];
            w = wt ? wt[s0 + s] : 1.0f;
            const float pr = 1.0f / (1.0f + expf(-z));
            d = w * (pr - t);
            // numerically stable BCE of the logit
            l = w * (fmaxf(z, 0.0f) - z * t + log1pf(expf(-fabsf(z))));
        }
        dz[s] = d;
        lw[s] = l;
        ww[s] = w;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float a = 0, b = 0;
        for (int s = 0; s < kSB; s++) {
            a += lw[s];
            b += ww[s];
        }
        out[0] = a;
        out[1] = b;
    }
    float* g = out + 2;
    // output layer and dA2
    for (int q = threadIdx.x; q < kSB * kH; q += blockDim.x) {
        const int s = q / kH, j = q % kH;
        D2[q] = dz[s] * bf(W[L.ow3 + j]) * gelu_d(A2[q]);
    }
    for (int j = threadIdx.x; j < kH; j += blockDim.x) {
        float a = 0;
        for (int s = 0; s < kSB; s++) a += dz[s] * H2[s * kH + j];
        g[L.ow3 + j] = a;
    }
    if (threadIdx.x == 0) {
        float a = 0;
        for (int s = 0; s < kSB; s++) a += dz[s];
        g[L.ob3] = a;
    }
    __syncthreads();
    // layer 2 weights, bias and dA1
    for (int q = threadIdx.x; q < kH * kH; q += blockDim.x) {
        const int i = q / kH, j = q % kH;
        float a = 0;
        for (int s = 0; s < kSB; s++) a += H1[s * kH + i] * D2[s * kH + j];
        g[L.oW2 + q] = a;
    }
    for (int j = threadIdx.x; j < kH; j += blockDim.x) {
        float a = 0;
        for (int s = 0; s < kSB; s++) a += D2[s * kH + j];
        g[L.ob2 + j] = a;
    }
    for (int q = threadIdx.x; q < kSB * kH; q += blockDim.x) {
        const int s = q / kH, i = q % kH;
        float a = 0;
        for (int j = 0; j < kH; j++) a += D2[s * kH + j] * bf(W[L.oW2 + i * kH + j]);
        D1[q] = a * gelu_d(A1[q]);
    }
    __syncthreads();
    // layer 1 weights and bias
    for (int q = threadIdx.x; q < n_in * kH; q += blockDim.x) {
        const int k = q / kH, i = q % kH;
        float a = 0;
        for (int s = 0; s < kSB; s++) a += X[s * n_in + k] * D1[s * kH + i];
        g[L.oW1 + q] = a;
    }
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        float a = 0;
        for (int s = 0; s < kSB; s++) a += D1[s * kH + i];
        g[L.ob1 + i] = a;
    }
}

// fixed-order sum of the block partials; loss and gradient normalised by sum w
__global__ void k_mlp_reduce(const float* __restrict__ part, int blocks, int n, float* __restrict__ loss,
                             float* __restrict__ grad) {
    const int stride = n + 2;
    float wsum = 0;
    for (int b = 0; b < blocks; b++) wsum += part[(size_t)b * stride + 1];
    const float inv = wsum > 0 ? 1.0f / wsum : 0.0f;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n + 1; q += gridDim.x * blockDim.x) {
        float a = 0;
        const int col = q == n ? 0 : q + 2;
        for (int b = 0; b < blocks; b++) a += part[(size_t)b * stride + col];
        if (q == n) {
            if (loss) *loss = a * inv;
        } else if (grad) {
            grad[q] = a * inv;
        }
    }
}

// Adam (Kingma & Ba 2015) on the FP32 master weights, BF16 copy refreshed
__global__ void k_mlp_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ g, uint16_t* __restrict__ wbf, int n, float lr, float c1,
                           float c2) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const float gq = g[q];
        const float mq = 0.9f * m[q] + 0.1f * gq;
        const float vq = 0.999f * v[q] + 0.001f * gq * gq;
        m[q] = mq;
        v[q] = vq;
        const float upd = lr * (mq * c1) / (sqrtf(vq * c2) + 1e-8f);
        const float nw = w[q] - upd;
        w[q] = nw;
        wbf[q] = to_bf(nw);
    }
}

__global__ void k_to_bf16(const float* __restrict__ w, uint16_t* __restrict__ wbf, int n) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) wbf[q] = to_bf(w[q]);
}

// ---- feature rows of a solver state -----------------------------------------
template <typename R>
__device__ __forceinline__ void rho_p_point(const R* u, int V, int NPT, int pt, double gm, double* rho, double* p) {
    const double r = (double)u[pt];
    double m2 = 0;
    for (int d = 1; d < V - 1; d++) {
        const double m = (double)u[d * NPT + pt];
        m2 += m * m;
    }
    *rho = r;
    *p = ((double)u[(V - 1) * NPT + pt] - 0.5 * m2 / r) * (gm - 1.0);
}

// per element: mean density and mean pressure over the solution points,
// summed in point order; one thread per (element, point), 256 threads =
// 256 / NPT elements (or one element and several rounds)
template <typename R>
__global__ void k_elem_means(const R* __restrict__ u, int V, int NPT, long long E, double gm,
                             float2* __restrict__ mean) {
    extern __shared__ double2 rp[];  // [elements of the block][NPT]
    const int per = NPT >= (int)blockDim.x ? 1 : (int)blockDim.x / NPT;
    const long long e0 = (long long)blockIdx.x * per;
    for (int q = threadIdx.x; q < per * NPT; q += blockDim.x) {
        const int el = q / NPT, pt = q % NPT;
        double r = 1.0, p = 1.0;
        if (e0 + el < E) rho_p_point(u + (e0 + el) * V * NPT, V, NPT, pt, gm, &r, &p);
        rp[q] = make_double2(r, p);
    }
    __syncthreads();
    if (threadIdx.x < per && e0 + threadIdx.x < E) {
        double sr = 0, sp = 0;
        for (int pt = 0; pt < NPT; pt++) {
            sr += rp[threadIdx.x * NPT + pt].x;
            sp += rp[threadIdx.x * NPT + pt].y;
        }
        mean[e0 + threadIdx.x] = make_float2((float)(sr / NPT), (float)(sp / NPT));
    }
}

__device__ __forceinline__ float safe_ratio(double a, double b) {
    const double r = (b > 0 && isfinite(b)) ? a / b - 1.0 : 0.0;
    return isfinite(r) ? (float)r : 0.0f;
}

// feature rows: the nodal part one thread per (element, point), the
// neighbour part one thread per (element, direction)
template <typename R>
__global__ void k_features(const R* __restrict__ u, const float2* __restrict__ mean, int D, int V, int NPT, int N0,
                           int N1, int N2, int bc0, int bc1, int bc2, long long E, double gm, int n_in,
                           uint16_t* __restrict__ x) {
    const int per = NPT >= (int)blockDim.x ? 1 : (int)blockDim.x / NPT;
    const long long e0 = (long long)blockIdx.x * per;
    for (int q = threadIdx.x; q < per * NPT; q += blockDim.x) {
        const int el = q / NPT, pt = q % NPT;
        const long long e = e0 + el;
        if (e >= E) continue;
        double r, p;
        rho_p_point(u + e * V * NPT, V, NPT, pt, gm, &r, &p);
        const float2 me = mean[e];
        x[e * n_in + pt] = to_bf(safe_ratio(r, me.x));
        x[e * n_in + NPT + pt] = to_bf(safe_ratio(p, me.y));
    }
    for (int q = threadIdx.x; q < per * D; q += blockDim.x) {
        const long long e = e0 + q / D;
        const int d = q % D;
        if (e >= E) continue;
        const float2 me = mean[e];
        const int N[3] = {N0, N1, N2}, bc[3] = {bc0, bc1, bc2};
        const int c[3] = {(int)(e % N0), (int)((e / N0) % N1), (int)(e / ((long long)N0 * N1))};
        float2 nb[2];
        for (int sd = 0; sd < 2; sd++) {
            int cc[3] = {c[0], c[1], c[2]};
            cc[d] += sd ? 1 : -1;
            if (cc[d] < 0 || cc[d] >= N[d]) {
                if (bc[d] == SPDK_BC_PERIODIC) cc[d] = cc[d] < 0 ? cc[d] + N[d] : cc[d] - N[d];
                else cc[d] = c[d];  // outside the domain: the element itself
            }
            nb[sd] = mean[((long long)cc[2] * N1 + cc[1]) * N0 + cc[0]];
        }
        const float r0 = safe_ratio(nb[0].x, me.x), r1 = safe_ratio(nb[1].x, me.x);
        const float p0 = safe_ratio(nb[0].y, me.y), p1 = safe_ratio(nb[1].y, me.y);
        uint16_t* row = x + e * n_in + 2 * NPT + 4 * d;
        row[0] = to_bf(fminf(r0, r1));
        row[1] = to_bf(fmaxf(r0, r1));
        row[2] = to_bf(fminf(p0, p1));
        row[3] = to_bf(fmaxf(p0, p1));
    }
}

unsigned grid_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    if (b > 148LL * 16) b = 148LL * 16;
    return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace

struct spdk_mlp {
    int n_in = 0, n = 0;
    float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr, *part = nullptr;
    uint16_t* wbf = nullptr;
    int part_blocks = 0;
    long long step = 0;
    size_t smem = 0, infer_smem = 0;
};

namespace spdk {

int mlp_infer_flags(spdk_mlp* m, const uint16_t* x, long long batch, float* p, uint8_t* flags, float thr,
                    cudaStream_t s) {
    if (m->infer_smem <= kInferSmemMax) {
        const long long tiles = (batch + kSI - 1) / kSI;
        const unsigned blocks = (unsigned)(tiles < 148LL * 2 ? tiles : 148LL * 2);
        k_mlp_infer<<<blocks, kThreadsM, m->infer_smem, s>>>(m->n_in, m->wbf, x, batch, p, flags, thr);
    } else {
        // wide inputs (3D, high order): the 32-sample tiles of the training kernels
        const unsigned blocks = (unsigned)((batch + kSB - 1) / kSB);
        k_mlp_forward<<<blocks, kThreadsM, m->smem, s>>>(m->n_in, m->wbf, x, (int)batch, p, flags, thr);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail(SPDK_E_CUDA, std::string("indicator: ") + cudaGetErrorString(e));
}

int feature_rows(const void* u, bool fp32, int D, int p, const int N[3], const int bc[3], double gm, long long E,
                 float2* means, uint16_t* x, cudaStream_t s) {
    const int n = p + 1, NPT = D == 2 ? n * n : n * n * n, V = D + 2, n_in = 2 * NPT + 4 * D;
    const int threads = 256;
    const int per = NPT >= threads ? 1 : threads / NPT;
    const unsigned g = (unsigned)((E + per - 1) / per);
    const size_t sm = (size_t)per * NPT * sizeof(double2);
    if (fp32) {
        k_elem_means<float><<<g, threads, sm, s>>>((const float*)u, V, NPT, E, gm, means);
        k_features<float><<<g, threads, 0, s>>>((const float*)u, means, D, V, NPT, N[0], N[1], N[2], bc[0], bc[1],
                                                 bc[2], E, gm, n_in, x);
    } else {
        k_elem_means<double><<<g, threads, sm, s>>>((const double*)u, V, NPT, E, gm, means);
        k_features<double><<<g, threads, 0, s>>>((const double*)u, means, D, V, NPT, N[0], N[1], N[2], bc[0], bc[1],
                                                  bc[2], E, gm, n_in, x);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail(SPDK_E_CUDA, std::string("features: ") + cudaGetErrorString(e));
}

int mlp_n_in(const spdk_mlp* m) { return m->n_in; }

}  // namespace spdk

extern "C" {

int spdk_mlp_create(int n_in, int hidden, unsigned long long seed, spdk_mlp** out) {
    if (!out) return fail(SPDK_E_ARG, "null argument");
    *out = nullptr;
    if (hidden != kH) return fail(SPDK_E_ARG, "hidden width must be 64");
    if (n_in < 1 || n_in > kMaxIn) return fail(SPDK_E_ARG, "n_in must be in 1..448");
    spdk_mlp* m = new spdk_mlp;
    m->n_in = n_in;
    const Layout L = layout(n_in);
    m->n = L.n;
    m->smem = (size_t)smem_layout(n_in).total;
    m->infer_smem = (size_t)infer_smem(n_in).total;
    // seeded Glorot-uniform weights (SplitMix64 stream), zero biases
    std::vector<float> w(L.n, 0.0f);
    uint64_t st = seed;
    auto uni = [&]() {
        uint64_t z = (st += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int fan_in, int fan_out, int count) {
        const double a = std::sqrt(6.0 / (fan_in + fan_out));
        for (int q = 0; q < count; q++) w[off + q] = (float)((2.0 * uni() - 1.0) * a);
    };
    fill(L.oW1, n_in, kH, n_in * kH);
    fill(L.oW2, kH, kH, kH * kH);
    fill(L.ow3, kH, 1, kH);
    int rc = 0;
    if (cudaMalloc((void**)&m->w, L.n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&m->m, L.n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&m->v, L.n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&m->g, L.n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void**)&m->wbf, L.n * sizeof(uint16_t)) != cudaSuccess)
        rc = fail(SPDK_E_NOMEM, "mlp parameters");
    if (!rc) {
        cudaMemset(m->m, 0, L.n * sizeof(float));
        cudaMemset(m->v, 0, L.n * sizeof(float));
        cudaMemcpy(m->w, w.data(), L.n * sizeof(float), cudaMemcpyHostToDevice);
        k_to_bf16<<<grid_for(L.n, 256), 256>>>(m->w, m->wbf, L.n);
        if (cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m->smem) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m->smem) != cudaSuccess ||
            (m->infer_smem <= kInferSmemMax &&
             cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m->infer_smem) !=
                 cudaSuccess))
            rc = fail(SPDK_E_CUDA, "mlp shared memory request");
        if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = fail(SPDK_E_CUDA, "mlp init");
    }
    if (rc) {
        spdk_mlp_destroy(m);
        return rc;
    }
    *out = m;
    return 0;
}

int spdk_mlp_destroy(spdk_mlp* m) {
    if (!m) return 0;
    cudaFree(m->w);
    cudaFree(m->m);
    cudaFree(m->v);
    cudaFree(m->g);
    cudaFree(m->wbf);
    cudaFree(m->part);
    delete m;
    return 0;
}

int spdk_mlp_num_params(spdk_mlp* m, int* count) {
    if (!m || !count) return fail(SPDK_E_ARG, "null argument");
    *count = m->n;
    return 0;
}

int spdk_mlp_get_params(spdk_mlp* m, float* host, int count) {
    if (!m || !host || count != m->n) return fail(SPDK_E_ARG, "count must be num_params");
    if (cudaMemcpy(host, m->w, count * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(SPDK_E_CUDA, "mlp get_params");
    return 0;
}

int spdk_mlp_set_params(spdk_mlp* m, const float* host, int count) {
    if (!m || !host || count != m->n) return fail(SPDK_E_ARG, "count must be num_params");
    if (cudaMemcpy(m->w, host, count * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(SPDK_E_CUDA, "mlp set_params");
    cudaMemset(m->m, 0, count * sizeof(float));
    cudaMemset(m->v, 0, count * sizeof(float));
    m->step = 0;
    k_to_bf16<<<grid_for(count, 256), 256>>>(m->w, m->wbf, count);
    if (cudaDeviceSynchronize() != cudaSuccess) return fail(SPDK_E_CUDA, "mlp set_params");
    return 0;
}

int spdk_mlp_forward(spdk_mlp* m, const uint16_t* x, int batch, float* p, void* stream) {
    if (!m || !x || !p || batch < 1) return fail(SPDK_E_ARG, "bad argument");
    return mlp_infer_flags(m, x, batch, p, nullptr, 0.5f, (cudaStream_t)stream);
}

int spdk_mlp_loss_grad(spdk_mlp* m, const uint16_t* x, const float* y, const float* w, int batch, float* loss,
                       float* grad, void* stream) {
    if (!m || !x || !y || batch < 1) return fail(SPDK_E_ARG, "bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    const int blocks = (batch + kSB - 1) / kSB;
    if (blocks > m->part_blocks) {
        // scratch for the block partials, grown outside any capture
        cudaStreamSynchronize(s);
        cudaFree(m->part);
        m->part = nullptr;
        if (cudaMalloc((void**)&m->part, (size_t)blocks * (m->n + 2) * sizeof(float)) != cudaSuccess) {
            m->part_blocks = 0;
            return fail(SPDK_E_NOMEM, "mlp gradient scratch");
        }
        m->part_blocks = blocks;
    }
    k_mlp_grad<<<blocks, kThreadsM, m->smem, s>>>(m->n_in, m->wbf, x, y, w, batch, m->part);
    k_mlp_reduce<<<grid_for(m->n + 1, 256), 256, 0, s>>>(m->part, blocks, m->n, loss, grad);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail(SPDK_E_CUDA, std::string("mlp gradient: ") + cudaGetErrorString(e));
}

int spdk_mlp_train_step(spdk_mlp* m, const uint16_t* x, const float* y, const float* w, int batch, float lr,
                        float* loss, void* stream) {
    if (!m) return fail(SPDK_E_ARG, "null argument");
    int rc = spdk_mlp_loss_grad(m, x, y, w, batch, loss, m->g, stream);
    if (rc) return rc;
    m->step++;
    const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, (double)m->step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow(0.999, (double)m->step)));
    k_mlp_adam<<<grid_for(m->n, 256), 256, 0, (cudaStream_t)stream>>>(m->w, m->m, m->v, m->g, m->wbf, m->n, lr, c1,
                                                                     c2);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail(SPDK_E_CUDA, std::string("mlp adam: ") + cudaGetErrorString(e));
}

}  // extern "C"
