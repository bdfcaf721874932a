// Kernels of FFT sizes 448, 450, 462, 480, 484 (ng1 of the default grid table in
// (220, 242]; staged row/column forms; from N = 462 the x-line kernel's
// 32-line tile passes a CTA's shared memory and 16-line tiles run instead).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_q(int N) {
    switch (N) {
    case 448: return sized_ops_of<448>();
    case 450: return sized_ops_of<450>();
    case 462: return sized_ops_of<462>();
    case 480: return sized_ops_of<480>();
    case 484: return sized_ops_of<484>();
    default: return nullptr;
    }
}

}  // namespace mdb
