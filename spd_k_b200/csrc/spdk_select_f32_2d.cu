// FP32 (precision form) kernel instantiations, 2D. Compiled with FMA
// contraction: this form is judged by its error against the FP64 form, not
// by bit equality.
#include "spdk_kernelset.cuh"

namespace spdk {

bool select_f32_2d(int p, const int N[3], KernelSetT<float>* k, bool visc) {
    switch (p) {
    case 1: return pick2<float, 1>(N[0], N[1], k, visc);
    case 2: return pick2<float, 2>(N[0], N[1], k, visc);
    case 3: return pick2<float, 3>(N[0], N[1], k, visc);
    case 4: return pick2<float, 4>(N[0], N[1], k, visc);
    case 5: return pick2<float, 5>(N[0], N[1], k, visc);
    case 6: return pick2<float, 6>(N[0], N[1], k, visc);
    case 7: return pick2<float, 7>(N[0], N[1], k, visc);
    }
    return false;
}

}  // namespace spdk
