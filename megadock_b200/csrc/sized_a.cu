// Kernels of FFT sizes 32, 48, 64, 72 (one translation unit per size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_a(int N) {
    switch (N) {
    case 32: return sized_ops_of<32>();
    case 48: return sized_ops_of<48>();
    case 64: return sized_ops_of<64>();
    case 72: return sized_ops_of<72>();
    default: return nullptr;
    }
}

}  // namespace mdb
