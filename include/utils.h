/*
 * utils.h -- CUDA error check that prints the failing call and exits, as the
 * reference's CUDA_ERROR_CHECK does (include/utils.h:3-12).
 */
#ifndef BZ2GPU_B200_UTILS_H
#define BZ2GPU_B200_UTILS_H

#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>

#define CUDA_ERROR_CHECK(expr)                                                        \
  do {                                                                                \
    cudaError_t bz_status_ = (expr);                                                  \
    if (bz_status_ != cudaSuccess) {                                                  \
      fprintf(stderr, "%s failed! At line %d, in %s\nError: %s\n\t %s\n", #expr,      \
              __LINE__, __FILE__, cudaGetErrorName(bz_status_),                        \
              cudaGetErrorString(bz_status_));                                        \
      exit(EXIT_FAILURE);                                                             \
    }                                                                                 \
  } while (0)

#endif
