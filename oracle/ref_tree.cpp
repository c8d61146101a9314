/*
 * Host build of the reference's octree builder.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference file
 * CUDA-based/ext/wn_treecode/wn_treecode_cpu/wn_treecode_cpu_treeutils.cpp is
 * #included unchanged (path from -DWN_REF_TREEUTILS) inside a private
 * namespace.  wnref_build_tree_* replays build_tree_cpu
 * (wn_treecode_cpu_torch_interface.cpp:42-102): recursive build with root
 * centre 0 and half-width 1, then preorder serialisation.  The only change
 * is that max_points_per_node is a parameter (the reference hard-codes 1 at
 * wn_treecode_cpu_torch_interface.cpp:60) and the console prints are dropped.
 */
#include "ref_prelude.h"

namespace wnref_tree {
#include WN_REF_TREEUTILS
}

namespace {

template <typename T>
struct RefTree {
    long num_nodes = 0, num_leaves = 0, depth = 0;
    std::vector<long> parent, children, npts, n2p_start, n2p;
    std::vector<char> is_leaf;
    std::vector<T> half_w;
};

template <typename T>
void* build(const T* pts, long n, long max_depth, long max_points_per_node) {
    using namespace wnref_tree;
    std::vector<long> idx(n);
    for (long i = 0; i < n; i++) idx[i] = i;
    long cur = 0;
    auto* t = new RefTree<T>();
    if (n == 0) return t;
    OctNode<T>* root = build_tree_cpu_recursive<T>(pts, idx, nullptr, T(0), T(0), T(0), T(1), 0,
                                                   cur, max_depth, max_points_per_node);
    compute_tree_attributes<T>(root, t->num_nodes, t->num_leaves, t->depth);
    long m = t->num_nodes;
    t->parent.assign(m, 0);
    t->children.assign(m * 8, 0);
    t->npts.assign(m, 0);
    t->n2p_start.assign(m, 0);
    t->is_leaf.assign(m, 0);
    t->half_w.assign(m, T(0));
    serialize_tree_recursive<T>(root, t->parent.data(), t->children.data(),
                                reinterpret_cast<bool*>(t->is_leaf.data()), t->half_w.data(),
                                t->npts.data(), t->n2p_start.data(), t->n2p);
    free_tree_recursive<T>(root);
    return t;
}

template <typename T>
void fill(void* h, long* parent, long* children, bool* is_leaf, T* half_w, long* npts, long* n2p,
          long* n2p_start) {
    auto* t = static_cast<RefTree<T>*>(h);
    long m = t->num_nodes;
    std::memcpy(parent, t->parent.data(), sizeof(long) * m);
    std::memcpy(children, t->children.data(), sizeof(long) * m * 8);
    std::memcpy(is_leaf, t->is_leaf.data(), m);
    std::memcpy(half_w, t->half_w.data(), sizeof(T) * m);
    std::memcpy(npts, t->npts.data(), sizeof(long) * m);
    std::memcpy(n2p, t->n2p.data(), sizeof(long) * t->n2p.size());
    std::memcpy(n2p_start, t->n2p_start.data(), sizeof(long) * m);
}

template <typename T>
void sizes(void* h, long* num_nodes, long* num_leaves, long* depth, long* n2p_len) {
    auto* t = static_cast<RefTree<T>*>(h);
    *num_nodes = t->num_nodes;
    *num_leaves = t->num_leaves;
    *depth = t->depth;
    *n2p_len = (long)t->n2p.size();
}

}  // namespace

extern "C" {

void* wnref_build_tree_f32(const float* pts, long n, long max_depth, long max_points_per_node) {
    return build<float>(pts, n, max_depth, max_points_per_node);
}
void* wnref_build_tree_f64(const double* pts, long n, long max_depth, long max_points_per_node) {
    return build<double>(pts, n, max_depth, max_points_per_node);
}
void wnref_tree_sizes_f32(void* h, long* nn, long* nl, long* d, long* l) {
    sizes<float>(h, nn, nl, d, l);
}
void wnref_tree_sizes_f64(void* h, long* nn, long* nl, long* d, long* l) {
    sizes<double>(h, nn, nl, d, l);
}
void wnref_tree_fill_f32(void* h, long* parent, long* children, bool* is_leaf, float* half_w,
                         long* npts, long* n2p, long* n2p_start) {
    fill<float>(h, parent, children, is_leaf, half_w, npts, n2p, n2p_start);
}
void wnref_tree_fill_f64(void* h, long* parent, long* children, bool* is_leaf, double* half_w,
                         long* npts, long* n2p, long* n2p_start) {
    fill<double>(h, parent, children, is_leaf, half_w, npts, n2p, n2p_start);
}
void wnref_tree_free_f32(void* h) { delete static_cast<RefTree<float>*>(h); }
void wnref_tree_free_f64(void* h) { delete static_cast<RefTree<double>*>(h); }

}  // extern "C"
