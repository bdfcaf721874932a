// Kernels of FFT size 400 (ng1 = 200; staged row/column forms, the voxel
// class kernel's bit planes in dynamic shared memory).
#include "context.cuh"

namespace mdb {

const SizedOps *sized_ops_n(int N) { return N == 400 ? sized_ops_of<400>() : nullptr; }

}  // namespace mdb
