// Minimal stand-in for the CUDA samples' helper_cuda.h, which the reference's
// SRC/cuda_pointer.h includes for checkCudaErrors (print and abort).
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>
#define checkCudaErrors(call)                                                          \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            std::fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_),   \
                         __FILE__, __LINE__);                                          \
            std::abort();                                                              \
        }                                                                              \
    } while (0)
