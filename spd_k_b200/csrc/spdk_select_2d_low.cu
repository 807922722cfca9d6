// Kernel instantiations of one group of (ndim, p) variants.
#include "spdk_kernelset.cuh"

namespace spdk {

bool select_2d_low(int p, const int N[3], KernelSetT<double>* k, bool visc) {
    switch (p) {
    case 1: return pick2<double, 1>(N[0], N[1], k, visc);
    case 2: return pick2<double, 2>(N[0], N[1], k, visc);
    case 3: return pick2<double, 3>(N[0], N[1], k, visc);
    }
    return false;
}

}  // namespace spdk
