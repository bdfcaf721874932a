// Kernels of FFT sizes 486, 490, 500, 504, 512 (ng1 of the default grid table
// in (242, 256], the device receptor build's limit; staged row/column forms).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_r(int N) {
    switch (N) {
    case 486: return sized_ops_of<486>();
    case 490: return sized_ops_of<490>();
    case 500: return sized_ops_of<500>();
    case 504: return sized_ops_of<504>();
    case 512: return sized_ops_of<512>();
    default: return nullptr;
    }
}

}  // namespace mdb
