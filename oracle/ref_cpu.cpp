/*
 * Host build of the reference's OpenMP CPU treecode (plain Gauss A / AT / G).
 *
 * TEST INFRASTRUCTURE ONLY.  The reference file
 * CUDA-based/ext/wn_treecode/wn_treecode_cpu/wn_treecode_cpu_kernels.cpp is
 * #included unchanged (path from -DWN_REF_CPU_KERNELS) inside a private
 * namespace.  These are the reference's own CPU launchers; note their A has
 * the opposite sign of the CUDA A (wn_treecode_cpu_kernels.cpp:94) and they
 * call omp_set_num_threads(20) themselves.
 */
#include "ref_prelude.h"

namespace wnref_cpu {
#include WN_REF_CPU_KERNELS
}

namespace {
typedef long idx_t;

template <typename T>
void scatter(idx_t num_nodes, const idx_t* parent, const idx_t* children, const T* points,
             const T* weights, const T* attrs, idx_t attr_dim, const idx_t* n2p,
             const idx_t* n2p_start, const idx_t* npts, const bool* is_leaf, idx_t tree_depth,
             T* out_attrs, T* out_rep, T* out_w) {
    using namespace wnref_cpu;
    std::vector<char> scattered(num_nodes, 0), next(num_nodes, 0);
    bool* sc = reinterpret_cast<bool*>(scattered.data());
    bool* nx = reinterpret_cast<bool*>(next.data());
    std::memset(out_attrs, 0, sizeof(T) * num_nodes * attr_dim);
    std::memset(out_rep, 0, sizeof(T) * num_nodes * 3);
    std::memset(out_w, 0, sizeof(T) * num_nodes);
    scatter_point_attrs_to_nodes_leaf_cpu_kernel_launcher<T>(parent, points, weights, attrs, n2p,
                                                             n2p_start, npts, is_leaf, sc,
                                                             out_attrs, out_rep, out_w, attr_dim,
                                                             num_nodes);
    for (idx_t depth = tree_depth - 1; depth >= 0; depth--) {
        find_next_to_scatter_cpu_kernel_launcher<T>(children, is_leaf, sc, nx, n2p, num_nodes);
        scatter_point_attrs_to_nodes_nonleaf_cpu_kernel_launcher<T>(
            parent, children, points, weights, attrs, n2p, n2p_start, npts, is_leaf, sc, nx,
            out_attrs, out_rep, out_w, attr_dim, num_nodes);
    }
}
}  // namespace

extern "C" {

void wnref_cpu_scatter_f32(long num_nodes, const long* parent, const long* children,
                           const float* points, const float* weights, const float* attrs,
                           long attr_dim, const long* n2p, const long* n2p_start, const long* npts,
                           const bool* is_leaf, long tree_depth, float* out_attrs, float* out_rep,
                           float* out_w) {
    scatter<float>(num_nodes, parent, children, points, weights, attrs, attr_dim, n2p, n2p_start,
                   npts, is_leaf, tree_depth, out_attrs, out_rep, out_w);
}

/* op: 0 = A (CPU sign), 1 = AT, 9 = G; same codes as the CUDA host build. */
int wnref_cpu_multiply_f32(int op, const float* qpts, const float* qw, long nq,
                           const float* points, const float* attrs, const long* n2p,
                           const long* n2p_start, const long* children, const float* node_attrs,
                           const bool* is_leaf, const float* half_w, const float* rep,
                           const long* npts, float* out, int continuous) {
    using namespace wnref_cpu;
    switch (op) {
        case 0:
            multiply_by_A_cpu_kernel_launcher<float>(qpts, qw, points, attrs, n2p, n2p_start,
                                                     children, node_attrs, is_leaf, half_w, rep,
                                                     npts, out, nq, continuous != 0);
            return 0;
        case 1:
            multiply_by_AT_cpu_kernel_launcher<float>(qpts, qw, points, attrs, n2p, n2p_start,
                                                      children, node_attrs, is_leaf, half_w, rep,
                                                      npts, out, nq);
            return 0;
        case 9:
            multiply_by_G_cpu_kernel_launcher<float>(qpts, qw, points, attrs, n2p, n2p_start,
                                                     children, node_attrs, is_leaf, half_w, rep,
                                                     npts, out, nq);
            return 0;
        default:
            return -1;
    }
}

}  // extern "C"
