/*
 * Host build of the reference's CUDA treecode kernels.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  The reference
 * file CUDA-based/ext/wn_treecode/wn_treecode_cuda/wn_treecode_cuda_kernels.cu
 * is #included unchanged from where it lies (path given by -DWN_REF_CUDA_KERNELS
 * in oracle/Makefile) inside a private namespace, with ref_prelude.h turning
 * its __global__ kernels into host functions.  The extern "C" functions below
 * replay the launch sequences of the reference's torch interface
 * (wn_treecode_cuda_torch_interface.cu:41-134 for the node scatter and
 * :137-777 for the multiply_by_* launches), one host iteration per CUDA
 * thread, so the results are the reference algorithm evaluated with host
 * libm instead of CUDA's math library.
 */
#include "ref_prelude.h"

thread_local wnref_dim3 blockIdx;
thread_local wnref_dim3 blockDim;
thread_local wnref_dim3 threadIdx;

namespace wnref_cuda {
#include WN_REF_CUDA_KERNELS
}

namespace {

typedef long idx_t;

/* Operator codes shared with oracle/oracle.py (REF_OPS). */
enum RefOp {
    REF_A = 0,
    REF_AT = 1,
    REF_A3 = 2,
    REF_A21 = 3,
    REF_A22 = 4,
    REF_A23 = 5,
    REF_A2T1 = 6,
    REF_A2T2 = 7,
    REF_A2T3 = 8,
    REF_G = 9,
};

/* Replays wn_treecode_cuda_torch_interface.cu:41-134: one leaf-kernel launch
 * over all nodes, then `tree_depth` rounds of find_next + nonleaf launches.
 * Each emulated launch runs to completion before the next one starts, which
 * is what the default-stream ordering of the reference guarantees. */
template <typename T>
void scatter(idx_t num_nodes, const idx_t* parent, const idx_t* children, const T* points,
             const T* weights, const T* attrs, idx_t attr_dim, const idx_t* n2p,
             const idx_t* n2p_start, const idx_t* npts, const bool* is_leaf, idx_t tree_depth,
             T* out_attrs, T* out_rep, T* out_w) {
    std::vector<char> scattered(num_nodes, 0), next(num_nodes, 0);
    bool* sc = reinterpret_cast<bool*>(scattered.data());
    bool* nx = reinterpret_cast<bool*>(next.data());
    std::memset(out_attrs, 0, sizeof(T) * num_nodes * attr_dim);
    std::memset(out_rep, 0, sizeof(T) * num_nodes * 3);
    std::memset(out_w, 0, sizeof(T) * num_nodes);
#pragma omp parallel for schedule(static)
    for (idx_t i = 0; i < num_nodes; i++) {
        wnref_set_thread(i);
        wnref_cuda::scatter_point_attrs_to_nodes_leaf_cuda_kernel<T>(
            parent, points, weights, attrs, n2p, n2p_start, npts, is_leaf, sc, out_attrs, out_rep,
            out_w, attr_dim, num_nodes);
    }
    for (idx_t depth = tree_depth - 1; depth >= 0; depth--) {
#pragma omp parallel for schedule(static)
        for (idx_t i = 0; i < num_nodes; i++) {
            wnref_set_thread(i);
            wnref_cuda::find_next_to_scatter_cuda_kernel<T>(children, is_leaf, sc, nx, n2p,
                                                            num_nodes);
        }
#pragma omp parallel for schedule(static)
        for (idx_t i = 0; i < num_nodes; i++) {
            wnref_set_thread(i);
            wnref_cuda::scatter_point_attrs_to_nodes_nonleaf_cuda_kernel<T>(
                parent, children, points, weights, attrs, n2p, n2p_start, npts, is_leaf, sc, nx,
                out_attrs, out_rep, out_w, attr_dim, num_nodes);
        }
    }
}

template <typename T>
int multiply(int op, const T* qpts, const T* qw, idx_t nq, const T* points, const T* attrs,
             const idx_t* n2p, const idx_t* n2p_start, const idx_t* children, const T* node_attrs,
             const bool* is_leaf, const T* half_w, const T* rep, const idx_t* npts, T* out,
             int continuous) {
    using namespace wnref_cuda;
    const bool cont = continuous != 0;
#pragma omp parallel for schedule(dynamic, 64)
    for (idx_t i = 0; i < nq; i++) {
        wnref_set_thread(i);
        switch (op) {
            case REF_A:
                multiply_by_A_cuda_kernel<T>(qpts, qw, points, attrs, n2p, n2p_start, children,
                                             node_attrs, is_leaf, half_w, rep, npts, out, nq, cont);
                break;
            case REF_AT:
                multiply_by_AT_cuda_kernel<T>(qpts, qw, points, attrs, n2p, n2p_start, children,
                                              node_attrs, is_leaf, half_w, rep, npts, out, nq);
                break;
            case REF_A3:
                multiply_by_A3_cuda_kernel<T>(qpts, qw, points, attrs, n2p, n2p_start, children,
                                              node_attrs, is_leaf, half_w, rep, npts, out, nq, cont);
                break;
            case REF_A21:
                multiply_by_A21_cuda_kernel<T>(qpts, qw, points, attrs, n2p, n2p_start, children,
                                               node_attrs, is_leaf, half_w, rep, npts, out, nq,
                                               cont);
                break;
            case REF_A22:
                multiply_by_A22_cuda_kernel<T>(qpts, qw, points, attrs, n2p, n2p_start, children,
                                               node_attrs, is_leaf, half_w, rep, npts, out, nq,
                                               cont);
                break;
            case REF_A23:
                multiply_by_A23_cuda_kernel<T>(qpts, qw, points, attrs, n2p, n2p_start, children,
                                               node_attrs, is_leaf, half_w, rep, npts, out, nq,
                                               cont);
                break;
            case REF_A2T1:
                multiply_by_A2T1_cuda_kernel<T>(qpts, qw, points, attrs, n2p, n2p_start, children,
                                                node_attrs, is_leaf, half_w, rep, npts, out, nq);
                break;
            case REF_A2T2:
                multiply_by_A2T2_cuda_kernel<T>(qpts, qw, points, attrs, n2p, n2p_start, children,
                                                node_attrs, is_leaf, half_w, rep, npts, out, nq);
                break;
            case REF_A2T3:
                multiply_by_A2T3_cuda_kernel<T>(qpts, qw, points, attrs, n2p, n2p_start, children,
                                                node_attrs, is_leaf, half_w, rep, npts, out, nq);
                break;
            case REF_G:
                multiply_by_G_cuda_kernel<T>(qpts, qw, points, attrs, n2p, n2p_start, children,
                                             node_attrs, is_leaf, half_w, rep, npts, out, nq);
                break;
            default:
                break;
        }
    }
    return (op >= REF_A && op <= REF_G) ? 0 : -1;
}

}  // namespace

extern "C" {

void wnref_scatter_f32(long num_nodes, const long* parent, const long* children,
                       const float* points, const float* weights, const float* attrs,
                       long attr_dim, const long* n2p, const long* n2p_start, const long* npts,
                       const bool* is_leaf, long tree_depth, float* out_attrs, float* out_rep,
                       float* out_w) {
    scatter<float>(num_nodes, parent, children, points, weights, attrs, attr_dim, n2p, n2p_start,
                   npts, is_leaf, tree_depth, out_attrs, out_rep, out_w);
}

void wnref_scatter_f64(long num_nodes, const long* parent, const long* children,
                       const double* points, const double* weights, const double* attrs,
                       long attr_dim, const long* n2p, const long* n2p_start, const long* npts,
                       const bool* is_leaf, long tree_depth, double* out_attrs, double* out_rep,
                       double* out_w) {
    scatter<double>(num_nodes, parent, children, points, weights, attrs, attr_dim, n2p, n2p_start,
                    npts, is_leaf, tree_depth, out_attrs, out_rep, out_w);
}

int wnref_multiply_f32(int op, const float* qpts, const float* qw, long nq, const float* points,
                       const float* attrs, const long* n2p, const long* n2p_start,
                       const long* children, const float* node_attrs, const bool* is_leaf,
                       const float* half_w, const float* rep, const long* npts, float* out,
                       int continuous) {
    return multiply<float>(op, qpts, qw, nq, points, attrs, n2p, n2p_start, children, node_attrs,
                           is_leaf, half_w, rep, npts, out, continuous);
}

int wnref_multiply_f64(int op, const double* qpts, const double* qw, long nq,
                       const double* points, const double* attrs, const long* n2p,
                       const long* n2p_start, const long* children, const double* node_attrs,
                       const bool* is_leaf, const double* half_w, const double* rep,
                       const long* npts, double* out, int continuous) {
    return multiply<double>(op, qpts, qw, nq, points, attrs, n2p, n2p_start, children, node_attrs,
                            is_leaf, half_w, rep, npts, out, continuous);
}

}  // extern "C"
