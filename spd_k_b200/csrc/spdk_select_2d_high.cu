// Kernel instantiations of one group of (ndim, p) variants.
#include "spdk_kernelset.cuh"

namespace spdk {

bool select_2d_high(int p, const int N[3], KernelSetT<double>* k, bool visc) {
    switch (p) {
    case 4: return pick2<double, 4>(N[0], N[1], k, visc);
    case 5: return pick2<double, 5>(N[0], N[1], k, visc);
    case 6: return pick2<double, 6>(N[0], N[1], k, visc);
    case 7: return pick2<double, 7>(N[0], N[1], k, visc);
    }
    return false;
}

}  // namespace spdk
