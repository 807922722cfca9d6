// Batched form: one launch of a pass covers the tiles of every problem of a
// group (same order p, same tile shape). Each problem contributes a table
// item -- its grid description, its pass arguments and the index of its
// first block in the launch -- and a block finds its item by binary search,
// copies it to shared memory and runs the same kernel body as the
// single-problem launch, on its problem-local tile index.
#pragma once
#include "spdk_kernelset.cuh"

namespace spdk {

struct DetectArgs {
    const double2* rpo;
    const double2* rpn;
    uint8_t* T;
};
struct DtArgs {
    double* dt;
    unsigned long long* dtmin;
};

template <typename Args>
struct BatchItem {
    DevGrid G;
    Args A;
    long long first;  // first block of this problem in the launch
};

// the item of this block, copied to shared memory (all threads return it)
template <typename Item>
__device__ __forceinline__ const Item& batch_item(const Item* __restrict__ items, int n, long long* local) {
    __shared__ __align__(16) unsigned char raw[sizeof(Item)];
    __shared__ int q;
    if (threadIdx.x == 0) {
        int lo = 0, hi = n - 1;
        const long long b = blockIdx.x;
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (items[mid].first <= b) lo = mid;
            else hi = mid - 1;
        }
        q = lo;
    }
    __syncthreads();
    const int* src = reinterpret_cast<const int*>(items + q);
    int* dst = reinterpret_cast<int*>(raw);
    static_assert(sizeof(Item) % 4 == 0, "item size");
    for (int w = threadIdx.x; w < (int)(sizeof(Item) / 4); w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    const Item& it = *reinterpret_cast<const Item*>(raw);
    *local = (long long)blockIdx.x - it.first;
    return it;
}

template <typename R, int D, int P, int TX, int TY, int TZ, int MODE>
__global__ void __launch_bounds__(kThreads, kPicardBlocksPerSM<R, D, P, MODE>)
    picard_batched(const BatchItem<PicardArgsT<R>>* __restrict__ items, int n, DevMatsT<R> M) {
    long long b;
    const BatchItem<PicardArgsT<R>>& it = batch_item(items, n, &b);
    if constexpr (D == 2) picard2d_body<R, P, TX, TY, MODE, false>(it.G, M, it.A, b);
    else picard_kernel_body<R, D, P, TX, TY, TZ, MODE>(it.G, M, it.A, b);
}

// the batched detect and update take one block per SM more than the
// single-problem kernels (the FP64 update excepted: it would spill 350
// bytes a thread): the groups' many small members leave the single-problem
// sizing's occupancy unused (measured on the first 16 problems of the
// ensemble, FP32: 44.7 -> 43.6 ms per step; the single 256^2 blast is
// 0.3 % slower with the same sizing, so it keeps its own)
template <int D>
constexpr int kDetectBlocksPerSMBatched = D == 2 ? 5 : kDetectBlocksPerSM<D>;
template <typename R, int D, int P>
constexpr int kUpdateBlocksPerSMBatched = (D == 2 && sizeof(R) == 4) ? 6 : kUpdateBlocksPerSM<D, P>;

template <typename R, int D, int P, int TX, int TY, int TZ>
__global__ void __launch_bounds__(kThreads, kDetectBlocksPerSMBatched<D>) detect_batched(const BatchItem<DetectArgs>* __restrict__ items, int n) {
    long long b;
    const BatchItem<DetectArgs>& it = batch_item(items, n, &b);
    fv_detect_kernel_body<R, D, P, TX, TY, TZ>(it.G, it.A.rpo, it.A.rpn, it.A.T, nullptr, b);
}

template <typename R, int D, int P, int TX, int TY, int TZ>
__global__ void __launch_bounds__(kThreads, kUpdateBlocksPerSMBatched<R, D, P>)
    update_batched(const BatchItem<FallbackArgsT<R>>* __restrict__ items, int n, DevMatsT<R> M) {
    long long b;
    const BatchItem<FallbackArgsT<R>>& it = batch_item(items, n, &b);
    fv_update_kernel_body<R, D, P, TX, TY, TZ>(it.G, M, it.A, b);
}

// dt hand-over of every problem of the batch: one thread per problem
__global__ void dt_batched(const DtArgs* __restrict__ a, int n);

template <typename R>
struct BatchSetT {
    void (*predict)(const BatchItem<PicardArgsT<R>>*, int, DevMatsT<R>) = nullptr;
    void (*correct)(const BatchItem<PicardArgsT<R>>*, int, DevMatsT<R>) = nullptr;
    void (*flux)(const BatchItem<PicardArgsT<R>>*, int, DevMatsT<R>) = nullptr;
    void (*detect)(const BatchItem<DetectArgs>*, int) = nullptr;
    void (*update)(const BatchItem<FallbackArgsT<R>>*, int, DevMatsT<R>) = nullptr;
    size_t picard_smem = 0, update_smem = 0;
    int tile[3] = {1, 1, 1};
};

template <typename R, int P, int TX, int TY>
BatchSetT<R> make_batch_set() {
    BatchSetT<R> k;
    k.predict = picard_batched<R, 2, P, TX, TY, 1, kPredict>;
    k.correct = picard_batched<R, 2, P, TX, TY, 1, kCorrect>;
    k.flux = picard_batched<R, 2, P, TX, TY, 1, kFlux>;
    k.detect = detect_batched<R, 2, P, TX, TY, 1>;
    k.update = update_batched<R, 2, P, TX, TY, 1>;
    k.picard_smem = picard_smem_bytes<R, 2, P, TX, TY, 1>();
    k.update_smem = UpdateSmem<R, 2, P, TX, TY, 1>::bytes;
    k.tile[0] = TX;
    k.tile[1] = TY;
    return k;
}

// the batched kernels of one (form, order, tile) -- false when not instantiated
// (2D; orders 2, 3, 5; tiles 1x1, 2x2 and, for p <= 3, 4x4)
bool batch_set(int p, int tile, BatchSetT<double>* k);
bool batch_set(int p, int tile, BatchSetT<float>* k);

}  // namespace spdk
