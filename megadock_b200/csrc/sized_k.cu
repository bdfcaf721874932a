// Kernels of FFT sizes 240, 242, 250, 252, 256 (staged row/column forms; one translation unit
// per size group).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_k(int N) {
    switch (N) {
    case 240: return sized_ops_of<240>();
    case 242: return sized_ops_of<242>();
    case 250: return sized_ops_of<250>();
    case 252: return sized_ops_of<252>();
    case 256: return sized_ops_of<256>();
    default: return nullptr;
    }
}

}  // namespace mdb
