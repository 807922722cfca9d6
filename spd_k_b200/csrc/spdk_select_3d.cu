// Kernel instantiations of one group of (ndim, p) variants.
#include "spdk_kernelset.cuh"

namespace spdk {

bool select_3d(int p, const int N[3], KernelSetT<double>* k, bool visc) {
    switch (p) {
    case 1: return pick3<double, 1>(N[0], N[1], N[2], k, visc);
    case 2: return pick3<double, 2>(N[0], N[1], N[2], k, visc);
    case 3: return pick3<double, 3>(N[0], N[1], N[2], k, visc);
    case 4: return pick3<double, 4>(N[0], N[1], N[2], k, visc);
    case 5: return pick3<double, 5>(N[0], N[1], N[2], k, visc);
    }
    return false;
}

}  // namespace spdk
