// Kernel instantiations of one group of (ndim, p) variants.
#include "spdk_kernelset.cuh"

namespace spdk {

bool select_2d_low(int p, const int N[3], KernelSet* k) {
    switch (p) {
    case 1: return pick2<1>(N[0], N[1], k);
    case 2: return pick2<2>(N[0], N[1], k);
    case 3: return pick2<3>(N[0], N[1], k);
    }
    return false;
}

}  // namespace spdk
