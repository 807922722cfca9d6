// Batched kernels of the plain FP64 form (built without FMA contraction): 2D, orders 2, 3, 5.
#include "spdk_batch.cuh"

namespace spdk {

bool batch_set(int p, int tile, BatchSetT<double>* k) {
    switch (p) {
    case 2:
        if (tile == 1) { *k = make_batch_set<double, 2, 1, 1>(); return true; }
        if (tile == 2) { *k = make_batch_set<double, 2, 2, 2>(); return true; }
        if (tile == 4) { *k = make_batch_set<double, 2, 4, 4>(); return true; }
        return false;
    case 3:
        if (tile == 1) { *k = make_batch_set<double, 3, 1, 1>(); return true; }
        if (tile == 2) { *k = make_batch_set<double, 3, 2, 2>(); return true; }
        if (tile == 4) { *k = make_batch_set<double, 3, 4, 4>(); return true; }
        return false;
    case 5:
        if (tile == 1) { *k = make_batch_set<double, 5, 1, 1>(); return true; }
        if (tile == 2) { *k = make_batch_set<double, 5, 2, 2>(); return true; }
        return false;
    }
    return false;
}

}  // namespace spdk
