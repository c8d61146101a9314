// extern "C" entry points declared in include/cagr.h.
#include <string>

#include "../../include/cagr.h"
#include "internal.h"

struct cagr_tree {
    cagr::Tree* t;
};

namespace cagr {

namespace {
thread_local std::string g_last_error;
}

int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

}  // namespace cagr

using cagr::set_error;

namespace {

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int check_tree(const cagr_tree* h) {
    if (!h || !h->t) return set_error(CAGR_ERR_INVALID, "tree handle is null");
    return CAGR_OK;
}

// Entry points that exist in the reference far-field mode only.
int reference_mode_only(const cagr_tree* h, const char* what) {
    if (h->t->interp)
        return set_error(CAGR_ERR_STATE, std::string(what) +
                                             " needs the reference far-field mode "
                                             "(cagr_tree_set_far_field(tree, CAGR_FAR_REFERENCE, ...))");
    return CAGR_OK;
}

int op_attr_dim(int op) {
    switch (op) {
        case CAGR_OP_AT:
        case CAGR_OP_A2T1:
        case CAGR_OP_A2T2:
        case CAGR_OP_A2T3: return 1;
        case CAGR_OP_A:
        case CAGR_OP_A3:
        case CAGR_OP_A21:
        case CAGR_OP_A22:
        case CAGR_OP_A23:
        case CAGR_OP_G:
        case CAGR_OP_A2_FUSED: return 3;
        case CAGR_OP_A2T_SUM: return 3;         // three scalar columns, one per slot
        case CAGR_OP_A2T_SUM_SHARED: return 1;  // one scalar column shared by the three
        case CAGR_OP_COUNT: return -1;  // any: counts with whatever slot 0 holds
        case CAGR_OP_A2_INSIDE: return 3;
        case CAGR_OP_A2T_RHS: return 3;
        default: return 0;
    }
}

}  // namespace

extern "C" {

int cagr_version(void) { return 100; }

const char* cagr_status_string(int status) {
    switch (status) {
        case CAGR_OK: return "ok";
        case CAGR_ERR_INVALID: return "invalid argument";
        case CAGR_ERR_CUDA: return "CUDA error";
        case CAGR_ERR_ALLOC: return "device allocation failed";
        case CAGR_ERR_OVERFLOW: return "size exceeds index range";
        case CAGR_ERR_STATE: return "invalid call order";
        default: return "unknown status";
    }
}

const char* cagr_last_error(void) { return cagr::g_last_error.c_str(); }

int cagr_tree_build(const void* points_dev, int64_t n, int dtype, int max_depth, int leaf_size,
                    void* stream, cagr_tree** out_tree) {
    if (!out_tree) return set_error(CAGR_ERR_INVALID, "out_tree is null");
    *out_tree = nullptr;
    cagr::Tree* t = nullptr;
    int rc = cagr::tree_build(points_dev, n, dtype, max_depth, leaf_size, as_stream(stream), &t);
    if (rc != CAGR_OK) return rc;
    *out_tree = new cagr_tree{t};
    return CAGR_OK;
}

int cagr_tree_destroy(cagr_tree* tree) {
    if (!tree) return CAGR_OK;
    cagr::tree_free(tree->t);
    delete tree;
    return CAGR_OK;
}

int cagr_tree_info(const cagr_tree* tree, int64_t* num_points, int64_t* num_nodes,
                   int64_t* num_leaves, int64_t* depth, int64_t* n2p_len) {
    if (int rc = check_tree(tree)) return rc;
    const cagr::Tree* t = tree->t;
    if (num_points) *num_points = t->n;
    if (num_nodes) *num_nodes = t->m;
    if (num_leaves) *num_leaves = t->num_leaves;
    if (depth) *depth = t->depth;
    if (n2p_len) *n2p_len = t->n2p_len;
    return CAGR_OK;
}

int cagr_tree_export(const cagr_tree* tree, int64_t* parent_dev, int64_t* children_dev,
                     uint8_t* is_leaf_dev, void* half_w_dev, int64_t* npts_dev, int64_t* n2p_dev,
                     int64_t* n2p_start_dev, void* stream) {
    if (int rc = check_tree(tree)) return rc;
    return cagr::tree_export(tree->t, parent_dev, children_dev, is_leaf_dev, half_w_dev, npts_dev,
                             n2p_dev, n2p_start_dev, as_stream(stream));
}

int cagr_tree_morton_order(const cagr_tree* tree, int32_t* perm_dev, void* stream) {
    if (int rc = check_tree(tree)) return rc;
    if (!perm_dev) return set_error(CAGR_ERR_INVALID, "perm_dev is null");
    cudaError_t e = cudaMemcpyAsync(perm_dev, tree->t->perm, sizeof(int32_t) * tree->t->n,
                                    cudaMemcpyDeviceToDevice, as_stream(stream));
    if (e != cudaSuccess) return set_error(CAGR_ERR_CUDA, cudaGetErrorString(e));
    return CAGR_OK;
}

int cagr_scatter(cagr_tree* tree, int slot, const void* attrs_dev, int attr_dim,
                 const void* weights_dev, void* stream) {
    if (int rc = check_tree(tree)) return rc;
    if (tree->t->interp) {
        if (slot < 0 || slot > 2) return set_error(CAGR_ERR_INVALID, "slot must be 0..2");
        return cagr::interp_scatter(tree->t, slot, attrs_dev, attr_dim, as_stream(stream));
    }
    return cagr::moments(tree->t, slot, attrs_dev, attr_dim, weights_dev, as_stream(stream));
}

int cagr_scatter_import(cagr_tree* tree, int slot, const void* node_attrs_dev,
                        const void* reppoints_dev, const void* attrs_dev, int attr_dim,
                        void* stream) {
    if (int rc = check_tree(tree)) return rc;
    if (int rc = reference_mode_only(tree, "cagr_scatter_import")) return rc;
    return cagr::moments_import(tree->t, slot, node_attrs_dev, reppoints_dev, attrs_dev, attr_dim,
                                as_stream(stream));
}

int cagr_scatter3(cagr_tree* tree, const void* values3_dev, void* stream) {
    if (int rc = check_tree(tree)) return rc;
    if (tree->t->interp) return cagr::interp_scatter(tree->t, 3, values3_dev, 3, as_stream(stream));
    return cagr::moments3(tree->t, values3_dev, as_stream(stream));
}

int cagr_scatter_export(const cagr_tree* tree, int slot, void* node_attrs_dev,
                        void* reppoints_dev, void* node_weights_dev, void* stream) {
    if (int rc = check_tree(tree)) return rc;
    if (int rc = reference_mode_only(tree, "cagr_scatter_export")) return rc;
    return cagr::moments_export(tree->t, slot, node_attrs_dev, reppoints_dev, node_weights_dev,
                                as_stream(stream));
}

int cagr_multiply(const cagr_tree* tree, int op, const void* queries_dev,
                  const int32_t* query_order_dev, int64_t nq, const void* widths_dev,
                  double width, int flags, void* out_dev, int64_t out_stride, void* stream) {
    if (int rc = check_tree(tree)) return rc;
    if (op_attr_dim(op) == 0) return set_error(CAGR_ERR_INVALID, "unknown operator");
    if (flags & ~(CAGR_FLAG_CONTINUOUS | CAGR_FLAG_ACCUMULATE | CAGR_FLAG_NEGATE))
        return set_error(CAGR_ERR_INVALID, "unknown flag bits");
    if (out_stride < 0 || out_stride > (1 << 20))
        return set_error(CAGR_ERR_INVALID, "out_stride out of range");
    cagr::TraverseArgs a;
    a.op = op;
    if (op == CAGR_OP_A2T_SUM || op == CAGR_OP_A2T_SUM_SHARED || op == CAGR_OP_A2T_RHS) {
        a.op = cagr::kOpA2TFused;
        a.slots = op == CAGR_OP_A2T_SUM ? 3 : (op == CAGR_OP_A2T_RHS ? 4 : 1);
    }
    a.continuous = (flags & CAGR_FLAG_CONTINUOUS) ? 1 : 0;
    a.accumulate = (flags & CAGR_FLAG_ACCUMULATE) ? 1 : 0;
    a.negate = (flags & CAGR_FLAG_NEGATE) ? 1 : 0;
    a.queries = queries_dev;
    a.qorder = query_order_dev;
    a.nq = nq;
    a.widths = widths_dev;
    a.width = width;
    a.out = out_dev;
    a.out_stride = (int)out_stride;
    if (tree->t->interp) return cagr::interp_traverse(tree->t, a, as_stream(stream));
    return cagr::traverse(tree->t, a, as_stream(stream));
}

int cagr_multiply_rhs_window(const cagr_tree* tree, const void* widths_dev, double width,
                             const void* widths_hi_dev, int flags, void* out_dev, void* stream) {
    if (int rc = check_tree(tree)) return rc;
    if (int rc = reference_mode_only(tree, "cagr_multiply_rhs_window")) return rc;
    if (flags & ~CAGR_FLAG_ACCUMULATE) return set_error(CAGR_ERR_INVALID, "unknown flag bits");
    if (!widths_hi_dev) return set_error(CAGR_ERR_INVALID, "widths_hi must be a device buffer");
    cagr::TraverseArgs a;
    a.op = cagr::kOpA2TFused;
    a.slots = 4;
    a.accumulate = (flags & CAGR_FLAG_ACCUMULATE) ? 1 : 0;
    a.widths = widths_dev;
    a.width = width;
    a.widths_hi = widths_hi_dev;
    a.out = out_dev;
    return cagr::traverse(tree->t, a, as_stream(stream));
}

int cagr_b_window_table(const cagr_tree* tree, const void* base_dev, const void* scales_dev,
                        int num_scales, void* out_dev, void* stream) {
    if (int rc = check_tree(tree)) return rc;
    if (int rc = reference_mode_only(tree, "cagr_b_window_table")) return rc;
    return cagr::b_window_table(tree->t, base_dev, scales_dev, num_scales, out_dev,
                                as_stream(stream));
}

int cagr_adjoint(cagr_tree* tree, int op, const void* widths_dev, double width, int flags,
                 const void* grad_out_dev, void* grad_attrs_dev, void* stream) {
    if (int rc = check_tree(tree)) return rc;
    if (int rc = reference_mode_only(tree, "cagr_adjoint")) return rc;
    if (op != CAGR_OP_A2_FUSED)
        return set_error(CAGR_ERR_INVALID, "the adjoint is implemented for CAGR_OP_A2_FUSED");
    if (flags & ~CAGR_FLAG_CONTINUOUS) return set_error(CAGR_ERR_INVALID, "unknown flag bits");
    if (!grad_out_dev || !grad_attrs_dev)
        return set_error(CAGR_ERR_INVALID, "grad_out and grad_attrs must be device buffers");
    cagr::TraverseArgs a;
    a.op = cagr::kOpA2Fused;
    a.continuous = (flags & CAGR_FLAG_CONTINUOUS) ? 1 : 0;
    a.widths = widths_dev;
    a.width = width;
    return cagr::adjoint(tree->t, a, grad_out_dev, grad_attrs_dev, as_stream(stream));
}

int cagr_field_grid(const cagr_tree* tree, int op, int nx, int ny, int nz,
                    const double* origin, double spacing, const void* widths_dev, double width,
                    int flags, void* out_dev, void* stream) {
    if (int rc = check_tree(tree)) return rc;
    if (op_attr_dim(op) <= 0 || op == CAGR_OP_A2T_SUM || op == CAGR_OP_A2T_SUM_SHARED ||
        op == CAGR_OP_A2T_RHS)
        return set_error(CAGR_ERR_INVALID, "unsupported operator for grid queries");
    if (!origin) return set_error(CAGR_ERR_INVALID, "origin is null");
    if (flags & ~(CAGR_FLAG_CONTINUOUS | CAGR_FLAG_ACCUMULATE | CAGR_FLAG_NEGATE))
        return set_error(CAGR_ERR_INVALID, "unknown flag bits");
    cagr::TraverseArgs a;
    a.op = op;
    a.continuous = (flags & CAGR_FLAG_CONTINUOUS) ? 1 : 0;
    a.accumulate = (flags & CAGR_FLAG_ACCUMULATE) ? 1 : 0;
    a.negate = (flags & CAGR_FLAG_NEGATE) ? 1 : 0;
    a.grid = 1;
    a.gx = nx;
    a.gy = ny;
    a.gz = nz;
    for (int d = 0; d < 3; d++) a.gorigin[d] = origin[d];
    a.gspacing = spacing;
    a.widths = widths_dev;
    a.width = width;
    a.out = out_dev;
    if (tree->t->interp) return cagr::interp_traverse(tree->t, a, as_stream(stream));
    return cagr::traverse(tree->t, a, as_stream(stream));
}

int cagr_mc_table(int8_t* tri, uint8_t* ntri) { return cagr::mc_table(tri, ntri); }

int cagr_marching_cubes(const float* values_dev, int nx, int ny, int nz, const double* origin,
                        double spacing, double iso, float* vertices_dev, int64_t max_vertices,
                        int32_t* faces_dev, int64_t max_faces, int64_t* num_vertices,
                        int64_t* num_faces, void* stream) {
    if (!origin) return set_error(CAGR_ERR_INVALID, "origin is null");
    return cagr::marching_cubes(values_dev, nx, ny, nz, origin, spacing, iso, nullptr,
                                vertices_dev, max_vertices, faces_dev, max_faces, num_vertices,
                                num_faces, as_stream(stream));
}

int cagr_marching_cubes_table(const float* values_dev, int nx, int ny, int nz,
                              const double* origin, double spacing, double iso,
                              const int8_t* triangles, float* vertices_dev, int64_t max_vertices,
                              int32_t* faces_dev, int64_t max_faces, int64_t* num_vertices,
                              int64_t* num_faces, void* stream) {
    if (!origin) return set_error(CAGR_ERR_INVALID, "origin is null");
    if (!triangles) return set_error(CAGR_ERR_INVALID, "triangles is null");
    return cagr::marching_cubes(values_dev, nx, ny, nz, origin, spacing, iso, triangles,
                                vertices_dev, max_vertices, faces_dev, max_faces, num_vertices,
                                num_faces, as_stream(stream));
}

int cagr_forward(cagr_tree* tree, int op, const void* values_dev, const void* widths_dev,
                 double width, int flags, void* out_dev, void* stream) {
    if (int rc = check_tree(tree)) return rc;
    const int dim = op_attr_dim(op);
    if (dim <= 0) return set_error(CAGR_ERR_INVALID, "unknown operator for cagr_forward");
    if (op == CAGR_OP_A2T_SUM) {
        if (int rc = cagr_scatter3(tree, values_dev, stream)) return rc;
    } else if (int rc = cagr_scatter(tree, 0, values_dev, dim, nullptr, stream)) {
        return rc;
    }
    return cagr_multiply(tree, op, nullptr, nullptr, 0, widths_dev, width, flags, out_dev, 0,
                         stream);
}

int cagr_tree_set_far_field(cagr_tree* tree, int mode, int degree, double theta, int direct_max,
                            void* stream) {
    if (int rc = check_tree(tree)) return rc;
    if (mode == CAGR_FAR_REFERENCE) {
        if (tree->t->interp) {
            if (cudaStreamSynchronize(as_stream(stream)) != cudaSuccess)
                return set_error(CAGR_ERR_CUDA, "stream synchronisation failed");
            cagr::interp_free(tree->t);
        }
        return CAGR_OK;
    }
    if (mode != CAGR_FAR_INTERP) return set_error(CAGR_ERR_INVALID, "unknown far-field mode");
    return cagr::interp_setup(tree->t, degree, theta, direct_max, as_stream(stream));
}

int cagr_tree_far_field(const cagr_tree* tree, int* mode, int* degree, double* theta,
                        int* direct_max, int64_t* num_interp_nodes) {
    if (int rc = check_tree(tree)) return rc;
    if (mode) *mode = tree->t->interp ? CAGR_FAR_INTERP : CAGR_FAR_REFERENCE;
    cagr::interp_info(tree->t, degree, theta, direct_max, num_interp_nodes);
    return cagr::interp_status(tree->t);
}

int cagr_debug_interp_wait_limit(cagr_tree* tree, int64_t spin) {
    if (int rc = check_tree(tree)) return rc;
    return cagr::interp_set_wait_limit(tree->t, spin);
}

int cagr_tree_query_groups(const cagr_tree* tree, int32_t* order_dev, void* stream) {
    if (int rc = check_tree(tree)) return rc;
    if (!order_dev) return set_error(CAGR_ERR_INVALID, "order_dev is null");
    return cagr::query_groups(tree->t, order_dev, as_stream(stream));
}

}  // extern "C"
