// Kernel instantiations of one group of (ndim, p) variants.
#include "spdk_kernelset.cuh"

namespace spdk {

bool select_2d_low(int p, const int N[3], KernelSetT<double>* k) {
    switch (p) {
    case 1: return pick2<double, 1>(N[0], N[1], k);
    case 2: return pick2<double, 2>(N[0], N[1], k);
    case 3: return pick2<double, 3>(N[0], N[1], k);
    }
    return false;
}

}  // namespace spdk
