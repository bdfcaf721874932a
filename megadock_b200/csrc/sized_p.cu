// Kernels of FFT sizes 384, 392, 396, 420, 432, 440 (ng1 of the default grid
// table in (189, 220] other than 200, whose N = 400 is in sized_n.cu; staged
// row/column forms; at N = 440 the x-line kernel's 32-line tile holds 220 KB
// of the 227 KB a CTA may use).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_p(int N) {
    switch (N) {
    case 384: return sized_ops_of<384>();
    case 392: return sized_ops_of<392>();
    case 396: return sized_ops_of<396>();
    case 420: return sized_ops_of<420>();
    case 432: return sized_ops_of<432>();
    case 440: return sized_ops_of<440>();
    default: return nullptr;
    }
}

}  // namespace mdb
