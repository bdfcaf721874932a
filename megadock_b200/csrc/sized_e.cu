// Kernels of FFT sizes 36, 40, 44, 56, 60, 84, 88 (one translation unit per size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_e(int N) {
    switch (N) {
    case 36: return sized_ops_of<36>();
    case 40: return sized_ops_of<40>();
    case 44: return sized_ops_of<44>();
    case 56: return sized_ops_of<56>();
    case 60: return sized_ops_of<60>();
    case 84: return sized_ops_of<84>();
    case 88: return sized_ops_of<88>();
    default: return nullptr;
    }
}

}  // namespace mdb
