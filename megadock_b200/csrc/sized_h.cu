// Kernels of FFT sizes 110, 126, 150, 154 (N/2 odd; one translation unit per
// size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_h(int N) {
    switch (N) {
    case 110: return sized_ops_of<110>();
    case 126: return sized_ops_of<126>();
    case 150: return sized_ops_of<150>();
    case 154: return sized_ops_of<154>();
    default: return nullptr;
    }
}

}  // namespace mdb
