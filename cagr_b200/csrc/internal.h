// Host-side structures shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "common.cuh"

namespace cagr {

// Records the message for cagr_last_error() and returns `code`.
int set_error(int code, const std::string& msg);

// CUDA call check inside functions returning a status code.
#define CAGR_CUDA(call)                                                                  \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            return ::cagr::set_error(::cagr::kErrCuda, std::string(#call) + ": " +       \
                                                           cudaGetErrorString(e_));      \
        }                                                                                \
    } while (0)

// Stream-ordered device memory from the library's per-device pool (memory.cu):
// freed blocks stay reserved for later calls.
int pool_alloc(void** p, size_t bytes, cudaStream_t s);
void pool_free(void* p, cudaStream_t s);

struct Interp;  // interpolated far field (interp.cu), null in the reference mode

// Device arrays owned by one tree.  All pointers are device pointers.
struct Tree {
    int dtype = 0;  // 0 = float32, 1 = float64
    int max_depth = 15;
    int leaf_size = 1;
    int device = 0;
    int64_t n = 0;           // points
    int64_t m = 0;           // nodes
    int64_t num_leaves = 0;
    int64_t depth = 0;       // deepest node
    int64_t n2p_len = 0;     // total length of the per-node point lists

    int32_t* perm = nullptr;       // [N] sorted position -> original index
    int32_t* invperm = nullptr;    // [N] original index -> sorted position
    int4* meta = nullptr;          // [M]
    uint8_t* nchild = nullptr;     // [M]
    int32_t* parent = nullptr;     // [M]
    int32_t* children = nullptr;   // [M*8], -1 = none
    int32_t* leaf_ids = nullptr;   // [num_leaves]
    int64_t* n2p_start = nullptr;  // [M]
    int32_t* n2p = nullptr;        // [n2p_len] original indices (built by the first export)
    int32_t* lorder = nullptr;     // [N] leaves' points in original-index order, by sorted
                                   // position (null: perm is that order, leaf size 1)
    void* spos = nullptr;          // [N*3] T, positions in sorted order
    int32_t* qgroup = nullptr;     // [N] self-query qi is the point at sorted position qgroup[qi]
                                   // (3-D Hilbert order: the traversals' warp grouping)
    uint32_t* counters = nullptr;  // [M], zero between moment passes
    void* rec[3] = {nullptr, nullptr, nullptr};  // [(M+N)*CAGR_REC_STRIDE] T per slot
    int rec_dim[3] = {0, 0, 0};    // attribute dim the slot was filled with (0 = empty)
    // Packed records of the three-slot adjoint (written with slots 0..2 by moments3):
    //   node  [M*12]: for k = 0..2  (c_k.x, c_k.y, c_k.z, exp(-c_k[k]/2) * s_k)
    //   point [N*8] : (y.x, y.y, y.z, e_0 s_0), (e_1 s_1, e_2 s_2, 0, 0),  e_k = exp(-y_k/2)
    void* adj_nodes = nullptr;
    void* adj_points = nullptr;
    //   sums  [M*8] : (W_0, W_1, W_2, 0), (A_0, A_1, A_2, 0)  (the climb's running sums)
    void* adj_sums = nullptr;
    bool adj_valid = false;
    bool slot_adj[3] = {false, false, false};  // slot k's latest moments are the adjoint's
    // Far-field mode: null = the reference's monopole at the weighted centroid
    // with per-query acceptance (bit-exact decisions); else the interpolated
    // far field (Chebyshev proxy grids per node, one acceptance test per warp).
    Interp* interp = nullptr;
};

int tree_build(const void* points, int64_t n, int dtype, int max_depth, int leaf_size,
               cudaStream_t stream, Tree** out);
void tree_free(Tree* t);
int tree_export(Tree* t, int64_t* parent, int64_t* children, uint8_t* is_leaf, void* half_w,
                int64_t* npts, int64_t* n2p, int64_t* n2p_start, cudaStream_t stream);

// Bottom-up node moments into record slot `slot`.  attrs: [N, dim] in the
// tree dtype (original point order); weights: [N] or null (then |attr|).
int moments(Tree* t, int slot, const void* attrs, int dim, const void* weights,
            cudaStream_t stream);
// Three scalar attributes at once (values3: [N, 3], column k -> slot k, weights |v_k|):
// the node moments of the reference's three A2Tk calls, in one launch.
int moments3(Tree* t, const void* values3, cudaStream_t stream);
// The records of slot `slot` from moments given in the reference layout
// (node_attrs [M, dim], reppoints [M, 3]) and point attributes [N, dim].
int moments_import(Tree* t, int slot, const void* node_attrs, const void* reppoints,
                   const void* attrs, int dim, cudaStream_t stream);
// Copy node moments of a slot out in the reference layout:
// node_attrs [M, dim], reppoints [M, 3], weights [M].
int moments_export(const Tree* t, int slot, void* node_attrs, void* reppoints, void* weights,
                   cudaStream_t stream);

// Operator codes (mirrored in include/cagr.h).
enum Op : int {
    kOpA = 0,
    kOpAT = 1,
    kOpA3 = 2,
    kOpA21 = 3,
    kOpA22 = 4,
    kOpA23 = 5,
    kOpA2T1 = 6,
    kOpA2T2 = 7,
    kOpA2T3 = 8,
    kOpG = 9,
    kOpA2Fused = 10,    // (A21, A22, A23) in one traversal -> [N', 3]
    kOpA2TFused = 11,   // sum_k A2Tk(s_k) with slot k holding s_k -> [N', 3]
    kOpCount = 12,      // pair terms per query with the slot-0 moments -> [N', 1]
    kOpA2Inside = 14,   // sums over inside-width pair terms (d.m, m_0, m_1, m_2) -> [N', 4]
};

struct TraverseArgs {
    int op = 0;
    int continuous = 0;
    int accumulate = 0;
    int negate = 0;                    // write (or add) -op
    int slots = 1;                     // kOpA2TFused: 3 = slot k holds s_k, 1 = shared slot 0
    const void* queries = nullptr;     // [nq, 3] T or null (= the tree's points)
    const int32_t* qorder = nullptr;   // [nq] processing order or null
    int64_t nq = 0;
    const void* widths = nullptr;      // [nq] T or null (then `width`)
    double width = 0.0;
    const void* widths_hi = nullptr;   // [nq] T or null: A2T right-hand side, b's terms
                                       // only for t(widths) <= r^2 < t(widths_hi)
    void* out = nullptr;               // [nq, out_dim] T
    int out_stride = 0;                // scalars between consecutive queries (0 = out_dim)
    // regular-grid queries (instead of `queries`): node (i, j, k) at
    // gorigin + (i, j, k) * gspacing, output row (k * gy + j) * gx + i
    int grid = 0;
    int gx = 0, gy = 0, gz = 0;
    double gorigin[3] = {0, 0, 0};
    double gspacing = 0;
};

int traverse(const Tree* t, const TraverseArgs& a, cudaStream_t stream);

// For the widths w_i = base * scales[i] (scales ascending, device [S], S <= 64;
// base device [n], original order) with b's moments in record slot 1:
// out[i] [n, 3] = b's A2T terms (summed over the three directions) kept at w_i
// and below w_hi = base * scales[S-1].
int b_window_table(const Tree* t, const void* base, const void* scales, int S, void* out,
                   cudaStream_t stream);

// J^T grad for the fused A2 on the tree's points (a.op = kOpA2Fused; a.widths,
// a.width, a.continuous as in the forward); grad and grad_attrs [n,3] in
// original point order.
int adjoint(const Tree* t, const TraverseArgs& a, const void* grad, void* grad_attrs,
            cudaStream_t stream);

// Interpolated far field (interp.cu).  interp_setup switches the tree to it
// (degree 1..8 of the Chebyshev grid per axis, acceptance parameter theta,
// nodes of at most direct_max points summed directly when near); interp_free
// returns it to the reference mode.  interp_scatter fills slot 0..2 (cagr_scatter)
// or 3 (cagr_scatter3's three scalar columns) with point and proxy records;
// interp_traverse evaluates an operator with them.
int interp_setup(Tree* t, int degree, double theta, int direct_max, cudaStream_t stream);
void interp_free(Tree* t);
int interp_scatter(Tree* t, int slot, const void* attrs, int dim, cudaStream_t stream);
int interp_traverse(const Tree* t, const TraverseArgs& a, cudaStream_t stream);
int interp_info(const Tree* t, int* degree, double* theta, int* direct_max, int64_t* num_interp);
// Reads the walks' error flag (synchronises the device): kErrCuda if a walk
// abandoned a staging wait since the mode was set up.
int interp_status(const Tree* t);
// Test hook: try_wait rounds before a staging wait is abandoned.
int interp_set_wait_limit(Tree* t, int64_t spin);
// The original index of the i-th self-query in processing order (consecutive
// groups of 32 walk together): perm[qgroup[i]].
int query_groups(const Tree* t, int32_t* order, cudaStream_t stream);

// Marching cubes (mcubes.cu).  The case table: tri[256][36] edge ids (12
// triangles at most) and ntri[256].
int mc_table(int8_t* tri, uint8_t* ntri);
// ref_table: null (the generated table, inside = value > iso) or triangles[256][16]
// in the reference's layout (inside = value < iso).
int marching_cubes(const float* values, int nx, int ny, int nz, const double* origin,
                   double spacing, double iso, const int8_t* ref_table, float* verts,
                   int64_t max_verts, int32_t* faces, int64_t max_faces, int64_t* nverts,
                   int64_t* nfaces, cudaStream_t s);

}  // namespace cagr
