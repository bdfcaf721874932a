// Kernels of FFT sizes 128, 144, 160 (one translation unit per size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_d(int N) {
    switch (N) {
    case 128: return sized_ops_of<128>();
    case 144: return sized_ops_of<144>();
    case 160: return sized_ops_of<160>();
    default: return nullptr;
    }
}

}  // namespace mdb
