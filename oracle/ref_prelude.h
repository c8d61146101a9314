/*
 * Host-compilation shim for the reference treecode sources.
 *
 * TEST INFRASTRUCTURE ONLY.  This header lets g++ compile the reference's
 * own CUDA kernel file (CUDA-based/ext/wn_treecode/wn_treecode_cuda/
 * wn_treecode_cuda_kernels.cu) as plain host C++, so that every __global__
 * kernel becomes an ordinary function that a host loop can call once per
 * emulated thread.  Nothing here is shipped or linked into the product.
 *
 * What it does:
 *  - pulls in every system header the reference files include, before the
 *    reference text is wrapped in a namespace by the including .cpp file;
 *  - defines the include guards of <cuda.h> and <cuda_runtime.h> so those
 *    headers are skipped (no device toolchain is involved);
 *  - maps __global__/__device__/__forceinline__ to host equivalents;
 *  - provides thread-local blockIdx/blockDim/threadIdx so an OpenMP loop can
 *    emulate a 1-D launch (one host iteration per CUDA thread).
 */
#pragma once

#include <assert.h>
#include <math.h>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>
#include <omp.h>

#define __cuda_cuda_h__
#define __CUDA_RUNTIME_H__

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline

struct wnref_dim3 {
    unsigned int x, y, z;
};

extern thread_local wnref_dim3 blockIdx;
extern thread_local wnref_dim3 blockDim;
extern thread_local wnref_dim3 threadIdx;

/* Set the emulated thread coordinates so that
 * blockDim.x * blockIdx.x + threadIdx.x == linear_index. */
static inline void wnref_set_thread(long linear_index) {
    blockDim.x = 1;
    blockDim.y = 1;
    blockDim.z = 1;
    blockIdx.x = (unsigned int)linear_index;
    blockIdx.y = 0;
    blockIdx.z = 0;
    threadIdx.x = 0;
    threadIdx.y = 0;
    threadIdx.z = 0;
}
