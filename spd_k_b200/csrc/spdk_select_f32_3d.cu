// FP32 (precision form) kernel instantiations, 3D. Compiled with FMA
// contraction.
#include "spdk_kernelset.cuh"

namespace spdk {

bool select_f32_3d(int p, const int N[3], KernelSetT<float>* k, bool visc) {
    switch (p) {
    case 1: return pick3<float, 1>(N[0], N[1], N[2], k, visc);
    case 2: return pick3<float, 2>(N[0], N[1], N[2], k, visc);
    case 3: return pick3<float, 3>(N[0], N[1], N[2], k, visc);
    case 4: return pick3<float, 4>(N[0], N[1], N[2], k, visc);
    case 5: return pick3<float, 5>(N[0], N[1], N[2], k, visc);
    }
    return false;
}

}  // namespace spdk
