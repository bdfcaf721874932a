// Kernels of FFT sizes 108, 112, 120 (one translation unit per size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_c(int N) {
    switch (N) {
    case 108: return sized_ops_of<108>();
    case 112: return sized_ops_of<112>();
    case 120: return sized_ops_of<120>();
    default: return nullptr;
    }
}

}  // namespace mdb
