// Kernels of FFT sizes 80, 96, 100 (one translation unit per size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_b(int N) {
    switch (N) {
    case 80: return sized_ops_of<80>();
    case 96: return sized_ops_of<96>();
    case 100: return sized_ops_of<100>();
    default: return nullptr;
    }
}

}  // namespace mdb
