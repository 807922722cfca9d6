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
#include "spdk_physics.cuh"

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
    feature_rho_p(u + pt, NPT, V, gm, rho, p);
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

__device__ __forceinline__ float safe_ratio(double a, double b) { return feature_ratio(a, b); }

// element grid of a feature row
struct FeatureGeom {
    int D, V, NPT;
    int N[3], bc[3];
    long long E;
};

// the nodal part of element e's row at point pt: rho / mean - 1 (column
// pt) and p / mean - 1 (column NPT + pt)
template <typename R>
__device__ __forceinline__ void own_features(const R* __restrict__ u, const float2* __restrict__ mean,
                                             const FeatureGeom& F, double gm, long long e, int pt, uint16_t* xr,
                                             uint16_t* xp) {
    double r, p;
    rho_p_point(u + e * F.V * F.NPT, F.V, F.NPT, pt, gm, &r, &p);
    const float2 me = mean[e];
    *xr = to_bf(safe_ratio(r, me.x));
    *xp = to_bf(safe_ratio(p, me.y));
}

// min and max over the two neighbours of a direction of the ratio of their
// mean to the element's, for rho then p
__device__ __forceinline__ void neighbour_values(float2 me, float2 lo, float2 hi, uint16_t f[4]) {
    const float r0 = safe_ratio(lo.x, me.x), r1 = safe_ratio(hi.x, me.x);
    const float p0 = safe_ratio(lo.y, me.y), p1 = safe_ratio(hi.y, me.y);
    f[0] = to_bf(fminf(r0, r1));
    f[1] = to_bf(fmaxf(r0, r1));
    f[2] = to_bf(fminf(p0, p1));
    f[3] = to_bf(fmaxf(p0, p1));
}

// the neighbour part of direction d (columns 2 NPT + 4d ..): min and max
// over the two neighbours of the ratio of their mean to the element's, for
// rho then p; outside a non-periodic boundary the neighbour is the element
__device__ __forceinline__ void neighbour_features(const float2* __restrict__ mean, const FeatureGeom& F,
                                                   long long e, int d, uint16_t f[4]) {
    const float2 me = mean[e];
    const int c[3] = {(int)(e % F.N[0]), (int)((e / F.N[0]) % F.N[1]), (int)(e / ((long long)F.N[0] * F.N[1]))};
    float2 nb[2];
    for (int sd = 0; sd < 2; sd++) {
        int cc[3] = {c[0], c[1], c[2]};
        cc[d] += sd ? 1 : -1;
        if (cc[d] < 0 || cc[d] >= F.N[d]) {
            if (F.bc[d] == SPDK_BC_PERIODIC) cc[d] = cc[d] < 0 ? cc[d] + F.N[d] : cc[d] - F.N[d];
            else cc[d] = c[d];
        }
        nb[sd] = mean[((long long)cc[2] * F.N[1] + cc[1]) * F.N[0] + cc[0]];
    }
    neighbour_values(me, nb[0], nb[1], f);
}

// feature rows: the nodal part one thread per (element, point), the
// neighbour part one thread per (element, direction)
template <typename R>
__global__ void k_features(const R* __restrict__ u, const float2* __restrict__ mean, FeatureGeom F, double gm,
                           int n_in, uint16_t* __restrict__ x) {
    const int NPT = F.NPT, D = F.D;
    const int per = NPT >= (int)blockDim.x ? 1 : (int)blockDim.x / NPT;
    const long long e0 = (long long)blockIdx.x * per;
    for (int q = threadIdx.x; q < per * NPT; q += blockDim.x) {
        const int el = q / NPT, pt = q % NPT;
        const long long e = e0 + el;
        if (e >= F.E) continue;
        own_features(u, mean, F, gm, e, pt, &x[e * n_in + pt], &x[e * n_in + NPT + pt]);
    }
    for (int q = threadIdx.x; q < per * D; q += blockDim.x) {
        const long long e = e0 + q / D;
        const int d = q % D;
        if (e >= F.E) continue;
        neighbour_features(mean, F, e, d, x + e * n_in + 2 * NPT + 4 * d);
    }
}

// ---------------------------------------------------------------------------
// Inference on the tensor cores: mma.sync m16n8k16 with BF16 operands and
// FP32 accumulators, one warp per 16 samples.
//
// Layer 1 takes the BF16 input rows (staged in shared memory) as the A
// operand and W1 as B. Its FP32 accumulators, after bias and GELU, are held
// in the layout of an m16n8k16 A operand (n-tiles 2c and 2c+1 of layer 1 are
// k-chunk c of layer 2), and each activation is split exactly into three
// BF16 terms (hi + mid + lo == the FP32 value; each residual has at most 16
// and then 8 significant bits), so layer 2 multiplies the same FP32
// activations as the training kernels, with products exact in FP32. The
// output layer is a dot product over the accumulators reduced across the 4
// lanes of a quad. Only the accumulation order differs from forward_tile.
//
// B fragments are pre-arranged in shared memory in lane order (one 8-byte
// load per lane per fragment, no bank conflicts); input rows have a stride
// of 16 kc + 8 BF16 (an odd multiple of 4 words), which makes the A-fragment
// loads conflict-free too.
// ---------------------------------------------------------------------------
constexpr int kTcWarps = 8;

struct TcSmem {
    int kc1, ldx, w1f, w2f, vec, xs, total;
};
__host__ __device__ inline TcSmem tc_smem(int n_in, int warps) {
    TcSmem s;
    s.kc1 = (n_in + 15) / 16;
    s.ldx = s.kc1 * 16 + 8;
    s.w1f = 0;                              // uint2 [kc1][8 n-tiles][32 lanes]
    s.w2f = s.w1f + s.kc1 * 8 * 32 * 8;     // uint2 [4][8][32]
    s.vec = s.w2f + 4 * 8 * 32 * 8;         // float b1[kH], b2[kH], w3[kH], b3 (+3 pad)
    s.xs = s.vec + (3 * kH + 4) * 4;        // uint16 [warps][16][ldx]
    s.total = s.xs + warps * 16 * s.ldx * 2;
    return s;
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf(uint16_t lo, uint16_t hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }

// (x0, x1) == hi + mid + lo exactly, each term a packed BF16 pair (x0 in
// the low half), round-to-nearest residuals
__device__ __forceinline__ void split3x2(float x0, float x1, uint32_t* hi, uint32_t* mid, uint32_t* lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
    const float2 hf = __bfloat1622float2(h);
    const float r0 = x0 - hf.x, r1 = x1 - hf.y;
    const __nv_bfloat162 m = __floats2bfloat162_rn(r0, r1);
    const float2 mf = __bfloat1622float2(m);
    const __nv_bfloat162 l = __floats2bfloat162_rn(r0 - mf.x, r1 - mf.y);
    *hi = *reinterpret_cast<const uint32_t*>(&h);
    *mid = *reinterpret_cast<const uint32_t*>(&m);
    *lo = *reinterpret_cast<const uint32_t*>(&l);
}

// B fragments of W1 (k < n_in, zero beyond) and W2, and the FP32 vectors
__device__ void load_tc_params(const Layout& L, const TcSmem& S, unsigned char* sm, const uint16_t* __restrict__ wbf) {
    uint2* W1f = reinterpret_cast<uint2*>(sm + S.w1f);
    uint2* W2f = reinterpret_cast<uint2*>(sm + S.w2f);
    float* vec = reinterpret_cast<float*>(sm + S.vec);
    const int n1 = S.kc1 * 8 * 32, n2 = 4 * 8 * 32;
    for (int q = threadIdx.x; q < n1 + n2; q += blockDim.x) {
        const bool first = q < n1;
        const int r = first ? q : q - n1;
        const int lane = r % 32, nt = (r / 32) % 8, kc = r / 256;
        const int g = lane >> 2, t = lane & 3;
        const int nk = first ? L.n_in : kH, oW = first ? L.oW1 : L.oW2;
        const int col = nt * 8 + g;
        const int k0 = kc * 16 + 2 * t;
        uint16_t v[4];
        const int ks[4] = {k0, k0 + 1, k0 + 8, k0 + 9};
#pragma unroll
        for (int i = 0; i < 4; i++) v[i] = ks[i] < nk ? wbf[oW + ks[i] * kH + col] : (uint16_t)0;
        (first ? W1f : W2f)[r] = make_uint2(pack_bf(v[0], v[1]), pack_bf(v[2], v[3]));
    }
    for (int q = threadIdx.x; q < kH; q += blockDim.x) {
        vec[q] = bf(wbf[L.ob1 + q]);
        vec[kH + q] = bf(wbf[L.ob2 + q]);
        vec[2 * kH + q] = bf(wbf[L.ow3 + q]);
    }
    if (threadIdx.x == 0) vec[3 * kH] = bf(wbf[L.ob3]);
    __syncthreads();
}

// the network on the warp's 16 rows in Xs ([16][ldx] BF16); z[0], z[1] are
// the logits of rows g and g + 8 (g = lane / 4), in every lane of the quad
__device__ __forceinline__ void mlp16_tc(const TcSmem& S, const unsigned char* sm, const uint16_t* Xs, float z[2]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const uint2* W1f = reinterpret_cast<const uint2*>(sm + S.w1f);
    const uint2* W2f = reinterpret_cast<const uint2*>(sm + S.w2f);
    const float* vec = reinterpret_cast<const float*>(sm + S.vec);
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
        for (int i = 0; i < 4; i++) acc[nt][i] = 0.0f;
    for (int kc = 0; kc < S.kc1; kc++) {
        const uint16_t* x0 = Xs + g * S.ldx + kc * 16 + 2 * t;
        const uint32_t a[4] = {*reinterpret_cast<const uint32_t*>(x0),
                               *reinterpret_cast<const uint32_t*>(x0 + 8 * S.ldx),
                               *reinterpret_cast<const uint32_t*>(x0 + 8),
                               *reinterpret_cast<const uint32_t*>(x0 + 8 * S.ldx + 8)};
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const uint2 b = W1f[(kc * 8 + nt) * 32 + lane];
            mma_bf16(acc[nt], a, b.x, b.y);
        }
    }
    // H1 = gelu(A1 + b1), in place: acc[nt][0..1] row g, [2..3] row g + 8,
    // columns nt * 8 + 2t + {0, 1}
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const int c0 = nt * 8 + 2 * t;
        acc[nt][0] = gelu(acc[nt][0] + vec[c0]);
        acc[nt][1] = gelu(acc[nt][1] + vec[c0 + 1]);
        acc[nt][2] = gelu(acc[nt][2] + vec[c0]);
        acc[nt][3] = gelu(acc[nt][3] + vec[c0 + 1]);
    }
    float acc2[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
        for (int i = 0; i < 4; i++) acc2[nt][i] = 0.0f;
#pragma unroll
    for (int kc = 0; kc < 4; kc++) {
        // A registers of k-chunk kc: {row g, cols 2t..}, {row g+8}, {row g, cols 8+2t..}, {row g+8, 8+}
        uint32_t ah[4], am[4], al[4];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const float* hp = acc[2 * kc + (r >> 1)] + 2 * (r & 1);
            split3x2(hp[0], hp[1], &ah[r], &am[r], &al[r]);
        }
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const uint2 b = W2f[(kc * 8 + nt) * 32 + lane];
            mma_bf16(acc2[nt], al, b.x, b.y);
            mma_bf16(acc2[nt], am, b.x, b.y);
            mma_bf16(acc2[nt], ah, b.x, b.y);
        }
    }
    float z0 = 0.0f, z1 = 0.0f;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const int c0 = nt * 8 + 2 * t;
        z0 += gelu(acc2[nt][0] + vec[kH + c0]) * vec[2 * kH + c0];
        z0 += gelu(acc2[nt][1] + vec[kH + c0 + 1]) * vec[2 * kH + c0 + 1];
        z1 += gelu(acc2[nt][2] + vec[kH + c0]) * vec[2 * kH + c0];
        z1 += gelu(acc2[nt][3] + vec[kH + c0 + 1]) * vec[2 * kH + c0 + 1];
    }
    z0 += __shfl_xor_sync(0xffffffffu, z0, 1);
    z0 += __shfl_xor_sync(0xffffffffu, z0, 2);
    z1 += __shfl_xor_sync(0xffffffffu, z1, 1);
    z1 += __shfl_xor_sync(0xffffffffu, z1, 2);
    z[0] = z0 + vec[3 * kH];
    z[1] = z1 + vec[3 * kH];
}

__device__ __forceinline__ void write_outputs(const float z[2], long long s0, long long batch, float* __restrict__ p,
                                              uint8_t* __restrict__ flags, float thr) {
    const int lane = threadIdx.x & 31;
    if ((lane & 3) != 0) return;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const long long s = s0 + (lane >> 2) + 8 * h;
        if (s < batch) {
            const float pr = 1.0f / (1.0f + expf(-z[h]));
            if (p) p[s] = pr;
            if (flags) flags[s] = pr > thr ? 1 : 0;
        }
    }
}

// probabilities / flags of BF16 feature rows x [batch][n_in]
__global__ void __launch_bounds__(kTcWarps * 32) k_mlp_infer_tc(int n_in, const uint16_t* __restrict__ wbf,
                                                                const float* __restrict__ z0,
                                                                const uint16_t* __restrict__ x, long long batch,
                                                                float* __restrict__ p, uint8_t* __restrict__ flags,
                                                                float thr) {
    extern __shared__ __align__(16) unsigned char sm[];
    const Layout L = layout(n_in);
    const TcSmem S = tc_smem(n_in, kTcWarps);
    load_tc_params(L, S, sm, wbf);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint16_t* Xs = reinterpret_cast<uint16_t*>(sm + S.xs) + warp * 16 * S.ldx;
    for (int q = lane; q < 16 * S.ldx; q += 32) Xs[q] = 0;  // padding columns stay zero
    __syncwarp();
    const float zz = *z0;
    const long long tiles = (batch + 15) / 16;
    for (long long tile = (long long)blockIdx.x * kTcWarps + warp; tile < tiles; tile += (long long)gridDim.x * kTcWarps) {
        const long long s0 = tile * 16;
        // the tile's 16 x n_in inputs in memory order, four loads in
        // flight per lane (row and column advanced without division); a
        // tile of all-zero rows takes the zero-input logit
        unsigned nz = 0;
        const int total = 16 * n_in;
        int row = lane / n_in, k = lane - row * n_in;
        const int drow = 32 / n_in, dk = 32 - drow * n_in;
        for (int q0 = 0; q0 < total; q0 += 128) {
            uint16_t v[4];
            int rr[4], kk[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                rr[i] = row;
                kk[i] = k;
                const bool ok = q0 + 32 * i + lane < total && s0 + row < batch;
                v[i] = ok ? x[(s0 + row) * n_in + k] : (uint16_t)0;
                row += drow;
                k += dk;
                if (k >= n_in) {
                    k -= n_in;
                    row++;
                }
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
                if (q0 + 32 * i + lane < total) {
                    Xs[rr[i] * S.ldx + kk[i]] = v[i];
                    nz |= v[i];
                }
        }
        __syncwarp();
        float z[2] = {zz, zz};
        if (__any_sync(0xffffffffu, nz != 0)) mlp16_tc(S, sm, Xs, z);
        write_outputs(z, s0, batch, p, flags, thr);
        __syncwarp();  // the next tile overwrites Xs
    }
}

// the logit of the all-zero input row, *z0 (one warp): a tile whose rows
// are all zero gives it for every row, so the inference kernels reuse it;
// recomputed whenever the BF16 weights change
__global__ void __launch_bounds__(32) k_mlp_zero_logit(int n_in, const uint16_t* __restrict__ wbf, float* z0) {
    extern __shared__ __align__(16) unsigned char sm[];
    const Layout L = layout(n_in);
    const TcSmem S = tc_smem(n_in, 1);
    load_tc_params(L, S, sm, wbf);
    uint16_t* Xs = reinterpret_cast<uint16_t*>(sm + S.xs);
    for (int q = threadIdx.x; q < 16 * S.ldx; q += 32) Xs[q] = 0;
    __syncwarp();
    float z[2];
    mlp16_tc(S, sm, Xs, z);
    if (threadIdx.x == 0) *z0 = z[0];
}

// the solver's a-priori flags from its stored feature rows: the nodal part
// of each row (columns < 2 NPT, written by the step's last update) and the
// neighbour part formed here from the element means; one warp per 16
// elements. Compiled for 3 resident blocks (80 registers, 72 bytes of
// spills; 127 registers and 2 blocks otherwise): the timed blast step with
// the indicator 0.8372 -> 0.8359 ms.
__global__ void __launch_bounds__(kTcWarps * 32, 3) k_indicator_rows_tc(const uint16_t* __restrict__ feat,
                                                                     const float2* __restrict__ mean, FeatureGeom F,
                                                                     int n_in, const uint16_t* __restrict__ wbf,
                                                                     const float* __restrict__ z0,
                                                                     uint8_t* __restrict__ flags, float thr,
                                                                     const int* gate) {
    if (gate && *gate) return;  // the solver's device time loop has ended
    extern __shared__ __align__(16) unsigned char sm[];
    const Layout L = layout(n_in);
    const TcSmem S = tc_smem(n_in, kTcWarps);
    load_tc_params(L, S, sm, wbf);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint16_t* Xs = reinterpret_cast<uint16_t*>(sm + S.xs) + warp * 16 * S.ldx;
    for (int q = lane; q < 16 * S.ldx; q += 32) Xs[q] = 0;
    __syncwarp();
    const float zz = *z0;
    const int nod = 2 * F.NPT;
    const long long tiles = (F.E + 15) / 16;
    for (long long tile = (long long)blockIdx.x * kTcWarps + warp; tile < tiles; tile += (long long)gridDim.x * kTcWarps) {
        const long long e0 = tile * 16;
        // the nodal columns of the 16 rows: all loads issued, then stored
        unsigned nz = 0;
        for (int k0 = 0; k0 < nod; k0 += 32) {
            const int k = k0 + lane;
            uint16_t v[16];
#pragma unroll
            for (int row = 0; row < 16; row++)
                v[row] = (k < nod && e0 + row < F.E) ? feat[(e0 + row) * n_in + k] : (uint16_t)0;
            if (k < nod) {
#pragma unroll
                for (int row = 0; row < 16; row++) {
                    Xs[row * S.ldx + k] = v[row];
                    nz |= v[row];
                }
            }
        }
        for (int q = lane; q < 16 * F.D; q += 32) {
            const int row = q / F.D, d = q - row * F.D;
            const long long e = e0 + row;
            uint16_t f[4] = {0, 0, 0, 0};
            if (e < F.E) neighbour_features(mean, F, e, d, f);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                Xs[row * S.ldx + nod + 4 * d + i] = f[i];
                nz |= f[i];
            }
        }
        __syncwarp();
        float z[2] = {zz, zz};
        if (__any_sync(0xffffffffu, nz != 0)) mlp16_tc(S, sm, Xs, z);
        write_outputs(z, e0, F.E, nullptr, flags, thr);
        __syncwarp();
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
    size_t smem = 0, tc_smem = 0, z0_smem = 0;
    float* z0 = nullptr;  // logit of the all-zero input row (device)
};

namespace spdk {

static FeatureGeom geom(int D, int p, const int N[3], const int bc[3], long long E) {
    FeatureGeom F;
    const int n = p + 1;
    F.D = D;
    F.V = D + 2;
    F.NPT = D == 2 ? n * n : n * n * n;
    for (int d = 0; d < 3; d++) {
        F.N[d] = N[d];
        F.bc[d] = bc[d];
    }
    F.E = E;
    return F;
}

static int launch_means(const void* u, bool fp32, const FeatureGeom& F, double gm, float2* means, cudaStream_t s) {
    const int threads = 256;
    const int per = F.NPT >= threads ? 1 : threads / F.NPT;
    const unsigned g = (unsigned)((F.E + per - 1) / per);
    const size_t sm = (size_t)per * F.NPT * sizeof(double2);
    if (fp32) k_elem_means<float><<<g, threads, sm, s>>>((const float*)u, F.V, F.NPT, F.E, gm, means);
    else k_elem_means<double><<<g, threads, sm, s>>>((const double*)u, F.V, F.NPT, F.E, gm, means);
    return 0;
}

static unsigned tc_blocks(long long rows) {
    const long long tiles = (rows + 15) / 16;
    const long long b = (tiles + kTcWarps - 1) / kTcWarps;
    return (unsigned)(b < 148LL * 4 ? (b < 1 ? 1 : b) : 148LL * 4);
}

int mlp_infer_flags(spdk_mlp* m, const uint16_t* x, long long batch, float* p, uint8_t* flags, float thr,
                    cudaStream_t s) {
    k_mlp_infer_tc<<<tc_blocks(batch), kTcWarps * 32, m->tc_smem, s>>>(m->n_in, m->wbf, m->z0, x, batch, p, flags,
                                                                       thr);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail(SPDK_E_CUDA, std::string("indicator: ") + cudaGetErrorString(e));
}

int feature_rows(const void* u, bool fp32, int D, int p, const int N[3], const int bc[3], double gm, long long E,
                 float2* means, uint16_t* x, cudaStream_t s) {
    const FeatureGeom F = geom(D, p, N, bc, E);
    const int n_in = 2 * F.NPT + 4 * D;
    launch_means(u, fp32, F, gm, means, s);
    const int threads = 256;
    const int per = F.NPT >= threads ? 1 : threads / F.NPT;
    const unsigned g = (unsigned)((E + per - 1) / per);
    if (fp32) k_features<float><<<g, threads, 0, s>>>((const float*)u, means, F, gm, n_in, x);
    else k_features<double><<<g, threads, 0, s>>>((const double*)u, means, F, gm, n_in, x);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail(SPDK_E_CUDA, std::string("features: ") + cudaGetErrorString(e));
}

int indicator_flags(spdk_mlp* m, const uint16_t* feat, const float2* means, int D, int p, const int N[3],
                    const int bc[3], long long E, uint8_t* flags, float thr, cudaStream_t s, const int* gate) {
    const FeatureGeom F = geom(D, p, N, bc, E);
    if (2 * F.NPT + 4 * D != m->n_in) return fail(SPDK_E_ARG, "indicator input width does not match the solver");
    k_indicator_rows_tc<<<tc_blocks(E), kTcWarps * 32, m->tc_smem, s>>>(feat, means, F, m->n_in, m->wbf, m->z0, flags,
                                                                        thr, gate);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail(SPDK_E_CUDA, std::string("indicator: ") + cudaGetErrorString(e));
}

// the zero-input logit after a change of the BF16 weights
static int update_zero_logit(spdk_mlp* m, cudaStream_t s) {
    k_mlp_zero_logit<<<1, 32, m->z0_smem, s>>>(m->n_in, m->wbf, m->z0);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail(SPDK_E_CUDA, std::string("mlp zero logit: ") + cudaGetErrorString(e));
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
    m->tc_smem = (size_t)tc_smem(n_in, kTcWarps).total;
    m->z0_smem = (size_t)tc_smem(n_in, 1).total;
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
        cudaMalloc((void**)&m->wbf, L.n * sizeof(uint16_t)) != cudaSuccess ||
        cudaMalloc((void**)&m->z0, sizeof(float)) != cudaSuccess)
        rc = fail(SPDK_E_NOMEM, "mlp parameters");
    if (!rc) {
        cudaMemset(m->m, 0, L.n * sizeof(float));
        cudaMemset(m->v, 0, L.n * sizeof(float));
        cudaMemcpy(m->w, w.data(), L.n * sizeof(float), cudaMemcpyHostToDevice);
        k_to_bf16<<<grid_for(L.n, 256), 256>>>(m->w, m->wbf, L.n);
        if (cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m->smem) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m->smem) != cudaSuccess ||
            cudaFuncSetAttribute(k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m->tc_smem) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k_indicator_rows_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)m->tc_smem) != cudaSuccess ||
            cudaFuncSetAttribute(k_mlp_zero_logit, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m->z0_smem) !=
                cudaSuccess)
            rc = fail(SPDK_E_CUDA, "mlp shared memory request");
        if (!rc) rc = update_zero_logit(m, 0);
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
    cudaFree(m->z0);
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
    if (int rc = update_zero_logit(m, 0)) return rc;
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
    if (int rc2 = update_zero_logit(m, (cudaStream_t)stream)) return rc2;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail(SPDK_E_CUDA, std::string("mlp adam: ") + cudaGetErrorString(e));
}

}  // extern "C"
