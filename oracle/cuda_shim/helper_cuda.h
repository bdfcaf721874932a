/*
 * Test infrastructure (oracle side only).  The reference's GPU sources include
 * helper_cuda.h from the CUDA samples, which this image does not ship; the
 * only thing they use from it is checkCudaErrors(call) on CUDA runtime and
 * cuFFT status codes.  This project-written stand-in defines that one macro:
 * a non-zero status prints its code and location and exits, as the samples'
 * helper does.
 */
#ifndef MD_ORACLE_HELPER_CUDA_H
#define MD_ORACLE_HELPER_CUDA_H
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

template <typename T>
static inline void md_oracle_check(T status, const char *what, const char *file, int line) {
    if (status) {
        std::fprintf(stderr, "CUDA status %d at %s:%d (%s)\n", (int)status, file, line, what);
        std::exit(EXIT_FAILURE);
    }
}
#define checkCudaErrors(call) md_oracle_check((call), #call, __FILE__, __LINE__)
#endif
