// Kernels of FFT sizes 132, 140 (one translation unit per size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_f(int N) {
    switch (N) {
    case 132: return sized_ops_of<132>();
    case 140: return sized_ops_of<140>();
    default: return nullptr;
    }
}

}  // namespace mdb
