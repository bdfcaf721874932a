// Kernels of FFT sizes 42, 50, 54, 66, 70, 90, 98 (N/2 odd; one translation
// unit per size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_g(int N) {
    switch (N) {
    case 42: return sized_ops_of<42>();
    case 50: return sized_ops_of<50>();
    case 54: return sized_ops_of<54>();
    case 66: return sized_ops_of<66>();
    case 70: return sized_ops_of<70>();
    case 90: return sized_ops_of<90>();
    case 98: return sized_ops_of<98>();
    default: return nullptr;
    }
}

}  // namespace mdb
