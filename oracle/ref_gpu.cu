/*
 * GPU build of the reference's CUDA treecode kernels.
 *
 * TEST AND BASELINE INFRASTRUCTURE ONLY.  The reference file
 * CUDA-based/ext/wn_treecode/wn_treecode_cuda/wn_treecode_cuda_kernels.cu is
 * #included unchanged from where it lies (path from -DWN_REF_CUDA_KERNELS in
 * oracle/Makefile) and compiled by nvcc for sm_100a.  The extern "C"
 * launchers below replay the launch sequences of the reference's torch
 * interface (wn_treecode_cuda_torch_interface.cu:41-134 for the scatter,
 * :137-777 for the multiply_by_* kernels: <<<ceil(n/1024), 1024>>>), on the
 * given stream, and -- unlike the reference -- check every launch, so a
 * launch that fails (e.g. too many registers for 1024-thread blocks) is an
 * error instead of silent zeros.  The Makefile builds with -maxrregcount=64
 * for that reason (a build flag, not a source change).
 */
#include <assert.h>
#include <cuda.h>
#include <cuda_runtime.h>

#include <iostream>
#include <vector>

namespace wnref_gpu {
#include WN_REF_CUDA_KERNELS
}

namespace {

typedef long idx_t;

template <typename T>
int scatter(idx_t M, const idx_t* parent, const idx_t* children, const T* points,
            const T* weights, const T* attrs, idx_t attr_dim, const idx_t* n2p,
            const idx_t* n2p_start, const idx_t* npts, const bool* is_leaf, idx_t tree_depth,
            T* out_attrs, T* out_rep, T* out_w, bool* scattered, bool* next, cudaStream_t s) {
    using namespace wnref_gpu;
    // torch::zeros of the outputs and masks (wn_treecode_cuda_torch_interface.cu:65-72)
    cudaMemsetAsync(scattered, 0, M, s);
    cudaMemsetAsync(next, 0, M, s);
    cudaMemsetAsync(out_attrs, 0, sizeof(T) * M * attr_dim, s);
    cudaMemsetAsync(out_rep, 0, sizeof(T) * M * 3, s);
    cudaMemsetAsync(out_w, 0, sizeof(T) * M, s);
    const idx_t blocks = (M + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK;
    scatter_point_attrs_to_nodes_leaf_cuda_kernel<T><<<blocks, THREADS_PER_BLOCK, 0, s>>>(
        parent, points, weights, attrs, n2p, n2p_start, npts, is_leaf, scattered, out_attrs,
        out_rep, out_w, attr_dim, M);
    if (cudaGetLastError() != cudaSuccess) return 2;
    for (idx_t depth = tree_depth - 1; depth >= 0; depth--) {
        find_next_to_scatter_cuda_kernel<T><<<blocks, THREADS_PER_BLOCK, 0, s>>>(
            children, is_leaf, scattered, next, n2p, M);
        scatter_point_attrs_to_nodes_nonleaf_cuda_kernel<T><<<blocks, THREADS_PER_BLOCK, 0, s>>>(
            parent, children, points, weights, attrs, n2p, n2p_start, npts, is_leaf, scattered,
            next, out_attrs, out_rep, out_w, attr_dim, M);
        if (cudaGetLastError() != cudaSuccess) return 2;
    }
    return 0;
}

template <typename T>
int multiply(int op, const T* q, const T* qw, idx_t nq, const T* points, const T* attrs,
             const idx_t* n2p, const idx_t* n2p_start, const idx_t* children,
             const T* node_attrs, const bool* is_leaf, const T* half_w, const T* rep,
             const idx_t* npts, T* out, int continuous, cudaStream_t s) {
    using namespace wnref_gpu;
    const idx_t blocks = (nq + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK;
    const bool cont = continuous != 0;
#define WNREF_LAUNCH(K, ...) K<T><<<blocks, THREADS_PER_BLOCK, 0, s>>>(__VA_ARGS__)
#define WNREF_ARGS q, qw, points, attrs, n2p, n2p_start, children, node_attrs, is_leaf, half_w, rep, npts, out, nq
    switch (op) {
        case 0: WNREF_LAUNCH(multiply_by_A_cuda_kernel, WNREF_ARGS, cont); break;
        case 1: WNREF_LAUNCH(multiply_by_AT_cuda_kernel, WNREF_ARGS); break;
        case 2: WNREF_LAUNCH(multiply_by_A3_cuda_kernel, WNREF_ARGS, cont); break;
        case 3: WNREF_LAUNCH(multiply_by_A21_cuda_kernel, WNREF_ARGS, cont); break;
        case 4: WNREF_LAUNCH(multiply_by_A22_cuda_kernel, WNREF_ARGS, cont); break;
        case 5: WNREF_LAUNCH(multiply_by_A23_cuda_kernel, WNREF_ARGS, cont); break;
        case 6: WNREF_LAUNCH(multiply_by_A2T1_cuda_kernel, WNREF_ARGS); break;
        case 7: WNREF_LAUNCH(multiply_by_A2T2_cuda_kernel, WNREF_ARGS); break;
        case 8: WNREF_LAUNCH(multiply_by_A2T3_cuda_kernel, WNREF_ARGS); break;
        case 9: WNREF_LAUNCH(multiply_by_G_cuda_kernel, WNREF_ARGS); break;
        default: return 1;
    }
#undef WNREF_ARGS
#undef WNREF_LAUNCH
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace

extern "C" {

const char* wnref_gpu_last_error(void) { return cudaGetErrorString(cudaPeekAtLastError()); }

int wnref_gpu_scatter(int f64, long M, const long* parent, const long* children,
                      const void* points, const void* weights, const void* attrs, long attr_dim,
                      const long* n2p, const long* n2p_start, const long* npts,
                      const bool* is_leaf, long tree_depth, void* out_attrs, void* out_rep,
                      void* out_w, bool* scattered, bool* next, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (f64)
        return scatter<double>(M, parent, children, (const double*)points, (const double*)weights,
                               (const double*)attrs, attr_dim, n2p, n2p_start, npts, is_leaf,
                               tree_depth, (double*)out_attrs, (double*)out_rep, (double*)out_w,
                               scattered, next, s);
    return scatter<float>(M, parent, children, (const float*)points, (const float*)weights,
                          (const float*)attrs, attr_dim, n2p, n2p_start, npts, is_leaf,
                          tree_depth, (float*)out_attrs, (float*)out_rep, (float*)out_w,
                          scattered, next, s);
}

int wnref_gpu_multiply(int f64, int op, const void* q, const void* qw, long nq,
                       const void* points, const void* attrs, const long* n2p,
                       const long* n2p_start, const long* children, const void* node_attrs,
                       const bool* is_leaf, const void* half_w, const void* rep, const long* npts,
                       void* out, int continuous, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (f64)
        return multiply<double>(op, (const double*)q, (const double*)qw, nq,
                                (const double*)points, (const double*)attrs, n2p, n2p_start,
                                children, (const double*)node_attrs, is_leaf,
                                (const double*)half_w, (const double*)rep, npts, (double*)out,
                                continuous, s);
    return multiply<float>(op, (const float*)q, (const float*)qw, nq, (const float*)points,
                           (const float*)attrs, n2p, n2p_start, children,
                           (const float*)node_attrs, is_leaf, (const float*)half_w,
                           (const float*)rep, npts, (float*)out, continuous, s);
}

}  // extern "C"
