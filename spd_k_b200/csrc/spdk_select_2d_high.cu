// Kernel instantiations of one group of (ndim, p) variants.
#include "spdk_kernelset.cuh"

namespace spdk {

bool select_2d_high(int p, const int N[3], KernelSet* k) {
    switch (p) {
    case 4: return pick2<4>(N[0], N[1], k);
    case 5: return pick2<5>(N[0], N[1], k);
    case 6: return pick2<6>(N[0], N[1], k);
    case 7: return pick2<7>(N[0], N[1], k);
    }
    return false;
}

}  // namespace spdk
