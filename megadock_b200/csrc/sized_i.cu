// Kernels of FFT sizes 162 ... 192 (one translation unit per size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_i(int N) {
    switch (N) {
    case 162: return sized_ops_of<162>();
    case 168: return sized_ops_of<168>();
    case 176: return sized_ops_of<176>();
    case 180: return sized_ops_of<180>();
    case 192: return sized_ops_of<192>();
    default: return nullptr;
    }
}

}  // namespace mdb
