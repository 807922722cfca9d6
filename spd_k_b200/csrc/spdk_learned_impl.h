// Internal entry points of the learned indicator used by the hydro solver
// (spdk_hydro.cu); the public API is include/spdk_learned.h.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

struct spdk_mlp;

namespace spdk {

// probabilities (p may be NULL) and flags p > thr (flags may be NULL) of
// `batch` feature rows
int mlp_infer_flags(spdk_mlp* m, const uint16_t* x, long long batch, float* p, uint8_t* flags, float thr,
                    cudaStream_t s);
// feature rows x [E][2 NPT + 4 D] of a state u [E][D+2][NPT] (double or
// float); means is scratch [E]
int feature_rows(const void* u, bool fp32, int D, int p, const int N[3], const int bc[3], double gm, long long E,
                 float2* means, uint16_t* x, cudaStream_t s);
// flags p > thr of every element from stored feature rows: their nodal
// part (columns < 2 NPT, as feature_rows or the step's last update writes
// it) and the element means (the neighbour part is formed from them)
int indicator_flags(spdk_mlp* m, const uint16_t* feat, const float2* means, int D, int p, const int N[3],
                    const int bc[3], long long E, uint8_t* flags, float thr, cudaStream_t s,
                    const int* gate = nullptr);
int mlp_n_in(const spdk_mlp* m);

}  // namespace spdk
