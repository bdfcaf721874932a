// Kernels of FFT sizes 324, 330, 336, 350, 352, 360, 378 (ng1 of the default
// grid table in (160, 189]; staged row/column forms).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_o(int N) {
    switch (N) {
    case 324: return sized_ops_of<324>();
    case 330: return sized_ops_of<330>();
    case 336: return sized_ops_of<336>();
    case 350: return sized_ops_of<350>();
    case 352: return sized_ops_of<352>();
    case 360: return sized_ops_of<360>();
    case 378: return sized_ops_of<378>();
    default: return nullptr;
    }
}

}  // namespace mdb
