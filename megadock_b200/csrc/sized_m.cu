// Kernels of FFT sizes 294, 300, 308, 320 (staged row/column forms; one translation unit
// per size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_m(int N) {
    switch (N) {
    case 294: return sized_ops_of<294>();
    case 300: return sized_ops_of<300>();
    case 308: return sized_ops_of<308>();
    case 320: return sized_ops_of<320>();
    default: return nullptr;
    }
}

}  // namespace mdb
