// Stand-in for the CUDA-samples helper header the reference includes, for the
// reference's own GPU build (plfbs_ref_gpu): the error-check macro reports a
// failed runtime call and ends the program, as the samples' version does.
#pragma once
#include <cstdio>
#include <cstdlib>

#include <cuda_runtime.h>

#define checkCudaErrors(val) plfbs_ref_check_cuda((val), #val, __FILE__, __LINE__)

template <typename T>
inline void plfbs_ref_check_cuda(T result, const char* call, const char* file, int line) {
  if (result) {
    std::fprintf(stderr, "CUDA error %d at %s:%d \"%s\"\n", (int)result, file, line, call);
    std::exit(EXIT_FAILURE);
  }
}
