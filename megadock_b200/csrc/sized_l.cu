// Kernels of FFT sizes 264, 270, 280, 288 (staged row/column forms; one translation unit
// per size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_l(int N) {
    switch (N) {
    case 264: return sized_ops_of<264>();
    case 270: return sized_ops_of<270>();
    case 280: return sized_ops_of<280>();
    case 288: return sized_ops_of<288>();
    default: return nullptr;
    }
}

}  // namespace mdb
