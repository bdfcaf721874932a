// Kernels of FFT sizes 196 ... 224 (one translation unit per size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_j(int N) {
    switch (N) {
    case 196: return sized_ops_of<196>();
    case 198: return sized_ops_of<198>();
    case 200: return sized_ops_of<200>();
    case 210: return sized_ops_of<210>();
    case 216: return sized_ops_of<216>();
    case 220: return sized_ops_of<220>();
    case 224: return sized_ops_of<224>();
    default: return nullptr;
    }
}

}  // namespace mdb
