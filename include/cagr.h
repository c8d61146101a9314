/*
 * cagr.h -- C ABI of the B200 treecode library (libcagr_b200.so).
 *
 * Drop-in boundary for the hot path of mayueji/CAGR: the Barnes-Hut treecode
 * evaluation of the convection-augmented Gauss operator A.mu and its
 * transpose-form A^T.w.  Every pointer argument named *_dev is a device
 * pointer on the current CUDA device; `stream` is a cudaStream_t (NULL = the
 * legacy default stream).  No entry point synchronises the stream unless it
 * says so.  Outputs are caller-owned; the tree handle owns its own device
 * memory.  Every function returns a cagr_status; on failure
 * cagr_last_error() gives a message (thread-local).
 *
 * Reference interfaces replaced (paths inside mayueji/CAGR):
 *   build_tree ............ CUDA-based/ext/wn_treecode/wn_treecode_cpu/
 *                           wn_treecode_cpu_torch_interface.cpp:104-118 (-> :42-102)
 *   scatter_point_attrs_to_nodes
 *                           CUDA-based/ext/wn_treecode/wn_treecode_cuda/
 *                           wn_treecode_cuda_torch_interface.cu:41-134
 *   multiply_by_{A,AT,A3,A21,A22,A23,A2T1,A2T2,A2T3,G}
 *                           wn_treecode_cuda_torch_interface.cu:137-777
 *                           (pybind names at :779-793)
 *   WindingNumberTreecode.forward_*
 *                           CUDA-based/ext/wn_treecode/wn_treecode_func.py:45-392
 */
#ifndef CAGR_H
#define CAGR_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cagr_tree cagr_tree;

/* Status codes. */
enum {
    CAGR_OK = 0,
    CAGR_ERR_INVALID = 1,  /* bad argument (null pointer, size, dtype, op) */
    CAGR_ERR_CUDA = 2,     /* a CUDA call or kernel launch failed */
    CAGR_ERR_ALLOC = 3,    /* device allocation failed */
    CAGR_ERR_OVERFLOW = 4, /* a size exceeds the 32-bit index range of the tree */
    CAGR_ERR_STATE = 5     /* call order: e.g. multiply before scatter */
};

/* Element types (the reference dispatches float and double,
 * AT_DISPATCH_FLOATING_TYPES in wn_treecode_cuda_torch_interface.cu). */
enum { CAGR_F32 = 0, CAGR_F64 = 1 };

/* Operators.  Reference kernels in wn_treecode_cuda_kernels.cu:
 *   A    :556-621   [N',1]   sum d.mu / r^3 (CUDA sign)
 *   AT   :623-692   [N',3]   sum d s / r^3
 *   A3   :694-763   [N',1]   (A21 + A22 + A23) / 3
 *   A21..A23 :843-1042 [N',1] sum exp(d_k/2) (d.mu / r^3 + mu_k / (2r))
 *   A2T1..A2T3 :1046-1257 [N',3] sum exp(d_k/2) (d s / r^3 + e_k s / (2r))
 *   G    :1259-1322 [N',3]   sum mu / r^3 - 3 d (d.mu) / r^5
 * A2_FUSED has no reference counterpart: A21, A22, A23 from one traversal,
 * written as the three columns of an [N',3] output.
 * A2T_SUM replaces the reference composition A2T1(s1) + A2T2(s2) + A2T3(s3)
 * (main_CAGR.py:110,137-139) with one traversal over the moments of s_k in
 * slot k (cagr_scatter3): every direction keeps its own |s_k|-weighted
 * centroids and acceptance decisions, as the three reference calls do.
 * A2T_SUM_SHARED is the same sum when s1 = s2 = s3 = s (the right-hand side
 * A2T1(b) + A2T2(b) + A2T3(b), main_CAGR.py:108): one slot, [N',3] output.
 * COUNT has no reference counterpart (the reference has no instrumentation):
 * the number of pair terms (accepted nodes + near leaf points) each query
 * sums with the moments in slot 0 -- the algorithmic work of a traversal. */
enum {
    CAGR_OP_A = 0,
    CAGR_OP_AT = 1,
    CAGR_OP_A3 = 2,
    CAGR_OP_A21 = 3,
    CAGR_OP_A22 = 4,
    CAGR_OP_A23 = 5,
    CAGR_OP_A2T1 = 6,
    CAGR_OP_A2T2 = 7,
    CAGR_OP_A2T3 = 8,
    CAGR_OP_G = 9,
    CAGR_OP_A2_FUSED = 10,
    CAGR_OP_A2T_SUM = 11,
    CAGR_OP_COUNT = 12,
    CAGR_OP_A2T_SUM_SHARED = 13,
    CAGR_OP_A2_INSIDE = 14,
    CAGR_OP_A2T_RHS = 15
};

/* cagr_multiply / cagr_forward flags. */
enum {
    CAGR_FLAG_CONTINUOUS = 1, /* the reference's continuous_kernel argument (A, A3, A2x) */
    CAGR_FLAG_ACCUMULATE = 2, /* add into out_dev instead of overwriting it */
    CAGR_FLAG_NEGATE = 4      /* write (or add) -op: the GaussRecon driver's grid value -A3
                                 (main_GaussRecon_cuda.cu:478); cagr_multiply, cagr_field_grid */
};

/* Library identification. */
int cagr_version(void);
const char* cagr_status_string(int status);
const char* cagr_last_error(void);

/* Builds the octree of `n` points (points_dev: [n,3], dtype) on the device.
 * Same tree as the reference build_tree (root centre 0, half-width 1, octant
 * code x>=cx | y>=cy<<1 | z>=cz<<2, leaf at max_depth or <= leaf_size points,
 * preorder node ids); the reference hard-codes leaf_size 1
 * (wn_treecode_cpu_torch_interface.cpp:60) and callers pass max_depth 15.
 * Replaces build_tree, wn_treecode_cpu_torch_interface.cpp:104-118.
 * Synchronises `stream` (node counts are needed on the host). */
int cagr_tree_build(const void* points_dev, int64_t n, int dtype, int max_depth, int leaf_size,
                    void* stream, cagr_tree** out_tree);

/* Frees the tree and all its device memory (after the device is idle for it). */
int cagr_tree_destroy(cagr_tree* tree);

/* Sizes of a built tree.  Any output pointer may be NULL. */
int cagr_tree_info(const cagr_tree* tree, int64_t* num_points, int64_t* num_nodes,
                   int64_t* num_leaves, int64_t* depth, int64_t* n2p_len);

/* Writes the tree in the reference layout (build_tree's seven tensors,
 * wn_treecode_cpu_torch_interface.cpp:73-101): parent[M] i64 (-1 root),
 * children[M,8] i64 (-1 none), is_leaf[M] u8, half_w[M] (tree dtype),
 * npts[M] i64, n2p[L] i64, n2p_start[M] i64.  Any output may be NULL.  The
 * per-node point lists (n2p) are built, and kept with the tree, by the first
 * call that asks for them (a walk over every point's leaf-to-root path and a
 * radix sort); the build itself does not make them. */
int cagr_tree_export(const cagr_tree* tree, int64_t* parent_dev, int64_t* children_dev,
                     uint8_t* is_leaf_dev, void* half_w_dev, int64_t* npts_dev, int64_t* n2p_dev,
                     int64_t* n2p_start_dev, void* stream);

/* Copies the Morton order (sorted position -> original index, int32[n]). */
int cagr_tree_morton_order(const cagr_tree* tree, int32_t* perm_dev, void* stream);

/* Node moments of per-point attributes (attrs_dev: [n, attr_dim], attr_dim 1
 * or 3, original point order) into moment slot `slot` (0..2) of the tree:
 * node attribute sums, weights (sum of weights_dev, or of |attr| when
 * weights_dev is NULL, as wn_treecode_func.py:131 computes them) and weighted
 * centroids.  Replaces scatter_point_attrs_to_nodes,
 * wn_treecode_cuda_torch_interface.cu:41-134; results are bit-identical to
 * the reference kernels :419-553 evaluated in IEEE arithmetic. */
int cagr_scatter(cagr_tree* tree, int slot, const void* attrs_dev, int attr_dim,
                 const void* weights_dev, void* stream);

/* Loads node moments given in the reference layout into record slot `slot`
 * (0..2): node_attrs_dev [M, attr_dim] and reppoints_dev [M, 3] as
 * scatter_point_attrs_to_nodes returns them (node ids = the reference's
 * preorder ids, which are this tree's), and the point attributes attrs_dev
 * [n, attr_dim] (original order).  The reference's multiply_by_* take these
 * arrays as arguments (wn_treecode_cuda_torch_interface.cu:137-777): this is
 * how a caller holding them evaluates with them.  With the moments of
 * cagr_scatter_export the records are those of cagr_scatter (same bits). */
int cagr_scatter_import(cagr_tree* tree, int slot, const void* node_attrs_dev,
                        const void* reppoints_dev, const void* attrs_dev, int attr_dim,
                        void* stream);

/* Node moments of three scalar attributes at once: column k of values3_dev
 * ([n,3], original point order) is scattered with weights |v_k| -- the three
 * scatter_point_attrs_to_nodes calls the reference makes before its A2T1,
 * A2T2 and A2T3 kernels (wn_treecode_func.py:271-351), in one launch.  The
 * result is held in the packed records CAGR_OP_A2T_SUM reads, not in the
 * record slots, which keep what the last cagr_scatter put there (single-slot
 * operators, and CAGR_OP_A2T_RHS's b in slot 1, read those);
 * cagr_scatter_export(tree, k, ...) returns column k's moments (attr dim 1)
 * until the next cagr_scatter into slot k. */
int cagr_scatter3(cagr_tree* tree, const void* values3_dev, void* stream);

/* Copies slot `slot` out in the reference layout: node_attrs [M, attr_dim],
 * reppoints [M,3], node_weights [M] (any may be NULL). */
int cagr_scatter_export(const cagr_tree* tree, int slot, void* node_attrs_dev,
                        void* reppoints_dev, void* node_weights_dev, void* stream);

/* Evaluates operator `op` with the moments in slot 0 (attr_dim 3 for
 * A/A3/A2x/G/A2_FUSED, 1 for AT/A2Tx/A2T_SUM_SHARED; slots 0..2 for
 * A2T_SUM).  Queries: queries_dev [nq,3], or NULL
 * for the tree's own points (then nq is ignored and outputs follow the
 * original point order).  query_order_dev (int32[nq], optional) gives the
 * order in which queries are processed (Morton order is fastest); outputs
 * always land at the query's own row.  Width per query: widths_dev [nq] or,
 * when NULL, the scalar `width`.  flags: CAGR_FLAG_CONTINUOUS (the
 * reference's continuous kernel, for A, A3, A2x) and CAGR_FLAG_ACCUMULATE
 * (sum into out_dev).  out_dev: [nq, out_stride] with out_stride 0 =
 * the operator's output width.  Replaces multiply_by_*,
 * wn_treecode_cuda_torch_interface.cu:137-777. */
int cagr_multiply(const cagr_tree* tree, int op, const void* queries_dev,
                  const int32_t* query_order_dev, int64_t nq, const void* widths_dev,
                  double width, int flags, void* out_dev, int64_t out_stride, void* stream);

/* One WindingNumberTreecode.forward_* call (wn_treecode_func.py:45-392):
 * node moments of values_dev ([n,3] for A/A3/A2x/G/A2_FUSED, [n,1] for
 * AT/A2Tx/A2T_SUM_SHARED; [n,3] scalar columns for A2T_SUM, via
 * cagr_scatter3), then `op` at the tree's own points. */
int cagr_forward(cagr_tree* tree, int op, const void* values_dev, const void* widths_dev,
                 double width, int flags, void* out_dev, void* stream);

/* Evaluates `op` (A, A3, A2x, G, A2_FUSED, AT, A2Tx; moments in slot 0) at the
 * nodes of a regular nx x ny x nz grid, node (i, j, k) at origin + (i, j, k) *
 * spacing (origin: 3 doubles in host memory), written to out_dev row
 * (k * ny + j) * nx + i; no query array is materialised.  Widths: widths_dev
 * (grid-shaped) or the scalar `width`.  The field evaluation of the GaussRecon
 * driver (multiply_by_A3 with the continuous kernel at grid corners,
 * main_GaussRecon_cuda.cu:427-445) on a regular grid. */
int cagr_field_grid(const cagr_tree* tree, int op, int nx, int ny, int nz, const double* origin,
                    double spacing, const void* widths_dev, double width, int flags, void* out_dev,
                    void* stream);

/* Marching cubes on float32 field values of a regular grid (values_dev
 * [nz, ny, nx], x fastest; node (i, j, k) at origin + (i, j, k) * spacing):
 * the surface value = iso, corners with value > iso inside, triangles wound
 * outward (toward decreasing values).  Writes *num_vertices / *num_faces; when
 * vertices_dev and faces_dev are non-NULL also the mesh (vertices [V,3]
 * float32, faces [F,3] int32 indices, vertices shared between cells) in the
 * same pass over the grid; if V or F exceed the given maxima, nothing beyond
 * them is written, the sizes are still set and the call returns
 * CAGR_ERR_OVERFLOW (call again with buffers of those sizes).  With NULL
 * buffers only the sizes are computed.  Synchronises `stream`.
 * The reference extracts the surface with PoissonRecon's adaptive octree MC
 * (gaussrecon_src/Octree.cpp:852-1090, tables MarchingCubes.cpp:32-324); this
 * uniform-grid MC uses its own generated case table (cagr_mc_table), or the
 * reference's table through cagr_marching_cubes_table. */
int cagr_marching_cubes(const float* values_dev, int nx, int ny, int nz, const double* origin,
                        double spacing, double iso, float* vertices_dev, int64_t max_vertices,
                        int32_t* faces_dev, int64_t max_faces, int64_t* num_vertices,
                        int64_t* num_faces, void* stream);

/* cagr_marching_cubes with a caller-supplied case table in the reference's
 * layout (gaussrecon_src/MarchingCubes.cpp:32-324 triangles[256][16] with
 * GetIndex at :333-345), replacing PoissonRecon's per-cube table lookup
 * (MarchingCubes::AddTriangleIndices, :573-584) on a regular grid.
 * triangles (host memory, 256 * 16 int8): row = case index whose bit k is set
 * when corner {0, 1, 3, 2, 4, 5, 7, 6}[k] (corner c = x + 2y + 4z) has
 * value < iso; entries = edge ids 4a + u + 2v as in cagr_mc_table, three per
 * triangle, -1 after the last (at most 5 triangles).  Corners with value < iso
 * are inside; vertices (one per crossed grid edge, in the same order and at
 * the same positions as cagr_marching_cubes) are shared between cells, and the
 * triangles of each cell are the table's, in its order and winding, cells in
 * index order.  Returns CAGR_ERR_INVALID for a table with other entries or
 * with a triangle on an edge its case does not cross; otherwise as
 * cagr_marching_cubes. */
int cagr_marching_cubes_table(const float* values_dev, int nx, int ny, int nz,
                              const double* origin, double spacing, double iso,
                              const int8_t* triangles, float* vertices_dev, int64_t max_vertices,
                              int32_t* faces_dev, int64_t max_faces, int64_t* num_vertices,
                              int64_t* num_faces, void* stream);

/* The marching-cubes case table (host memory): tri[256 * 36] edge ids, three
 * per triangle, and ntri[256] triangle counts.  Corner c = x + 2y + 4z; edge
 * 4a + u + 2v runs along axis a with the other two coordinates (u, v) in
 * increasing axis order.  No counterpart in the reference (its tables use
 * PoissonRecon's numbering). */
int cagr_mc_table(int8_t* tri, uint8_t* ntri);

/* No counterpart in the reference.  Node moments (the outputs of
 * cagr_scatter_export) computed from tree arrays in the reference layout
 * (parent, children, is_leaf, npts, n2p, n2p_start as cagr_tree_export
 * writes them; num_nodes = M) WITHOUT ANY DEVICE ALLOCATION, for callers that
 * cannot allocate at this point (under a fixed memory budget owned by another
 * allocator, or holding only the reference arrays and no tree handle).  Inputs (points [n,3], weights [n] or NULL for
 * |attr|, attrs [n, attr_dim]) and outputs (node_attrs [M, attr_dim],
 * reppoints [M,3], node_weights [M]) are the caller's; dtype CAGR_F32 or
 * CAGR_F64.  The per-node scratch lives in one fixed device array of
 * 2,097,152 nodes (8 MiB, held by every GPU that loads the library until
 * exit); larger trees return CAGR_ERR_INVALID.  All calls share that array:
 * calls that overlap on the GPU race, so order them on one stream.  The first
 * call on a device looks the array up.
 * Every buffer and the stream must belong to the CURRENT device (the scratch
 * array is the current device's; a buffer of another device is not detected). */
int cagr_scatter_noalloc(const int64_t* parent_dev, const int64_t* children_dev,
                         const uint8_t* is_leaf_dev, const int64_t* npts_dev,
                         const int64_t* n2p_dev, const int64_t* n2p_start_dev, int64_t num_nodes,
                         int dtype, const void* points_dev, const void* weights_dev,
                         const void* attrs_dev, int attr_dim, void* node_attrs_dev,
                         void* reppoints_dev, void* node_weights_dev, void* stream);

/* CAGR_OP_A2T_RHS (cagr_multiply; no reference counterpart as one call):
 * sum_k A2Tk(b) - sum_k A2Tk(s_k) in one traversal, the residual the CAGR
 * steepest-descent step forms from the reference's calls at one width
 * (main_CAGR.py:108-115): b's moments in record slot 1 (cagr_scatter(tree, 1,
 * b, 1, ...)), the s_k's from cagr_scatter3.  Every input keeps its own
 * moments and acceptance decisions, as in the separate calls; out [N',3]. */

/* CAGR_OP_A2T_RHS on the tree's own points with b's terms restricted to
 * t(w) <= r^2 < t(w_hi) (widths_dev or `width` give w, widths_hi_dev [n] gives
 * w_hi >= w per point; t is the reference's `r >= w` test on r^2).  The
 * acceptance decisions do not depend on the width, so with out holding
 * sum_k A2Tk(b) at the widths w_hi (cagr_multiply, CAGR_OP_A2T_SUM_SHARED,
 * b's moments in slot 0) and CAGR_FLAG_ACCUMULATE, out becomes exactly the
 * CAGR_OP_A2T_RHS value at w, up to summation order: the b terms at r >= w_hi
 * are the same in both, and those below are added here.  For the CAGR solve,
 * whose widths shrink or grow along one schedule: b's far terms are evaluated
 * once per solve instead of once per step.  The tree's points only; out [n,3]
 * (original order); flags: CAGR_FLAG_ACCUMULATE. */
int cagr_multiply_rhs_window(const cagr_tree* tree, const void* widths_dev, double width,
                             const void* widths_hi_dev, int flags, void* out_dev, void* stream);

/* b's part of the right-hand side for a whole schedule of widths in one walk:
 * for w_i = base * scales[i] (scales_dev [num_scales] ascending, 1..64 of
 * them; base_dev [n]; both in the tree dtype on the device, the product
 * rounded once as the caller's own base * scale), with b's moments in record
 * slot 1, out_dev [num_scales, n, 3] receives for each i the sum of b's
 * sum_k A2Tk terms kept at w_i (r >= w_i, the reference's test) with
 * r < w_hi = base * scales[num_scales - 1].  Adding
 * cagr_multiply(CAGR_OP_A2T_SUM_SHARED) at w_hi (b's moments in slot 0) gives
 * sum_k A2Tk(b) at every w_i, up to summation order: the acceptance decisions
 * do not depend on the width.  Allocates n * num_scales * 3 scalars of
 * scratch from the pool. */
int cagr_b_window_table(const cagr_tree* tree, const void* base_dev, const void* scales_dev,
                        int num_scales, void* out_dev, void* stream);

/* Exact adjoint of CAGR_OP_A2_FUSED on the tree's own points (no counterpart
 * in the reference, whose A2T1..A2T3 are a different operator:
 * wn_treecode_cuda_kernels.cu:263-379 against :113-224).  With the slot-0
 * moments of the forward call (the same centroids, hence the same acceptance
 * decisions and pair terms), the forward is linear in the point attributes mu;
 * this returns grad_attrs = J^T grad_out for grad_out [n,3] (d loss / d out,
 * original point order): grad_attrs [n,3] (original order), the sum over the
 * pair terms of the forward of grad_out . d(term)/d(mu).  op must be
 * CAGR_OP_A2_FUSED; widths / width / flags (CAGR_FLAG_CONTINUOUS only) as in
 * the forward call.  The traversal is recomputed, not stored.  Allocates
 * 3 (M + n) scalars of scratch from the library's pool.
 *
 * CAGR_OP_A2_INSIDE (for cagr_multiply, no reference counterpart) returns per
 * query [N',4] the sums over the pair terms inside the width (r < w) of
 * (d . m, m_0, m_1, m_2): with them the derivative of the continuous
 * kernel's output with respect to the query's width is closed-form. */
int cagr_adjoint(cagr_tree* tree, int op, const void* widths_dev, double width, int flags,
                 const void* grad_out_dev, void* grad_attrs_dev, void* stream);

/* Diagnostic with no counterpart in the reference: measures this GPU's FP32
 * FMA throughput (a long chain of independent fused multiply-adds on every
 * SM) and writes it to *gflops.  The roofline denominator for the
 * FP32-bound traversal kernels.  Synchronises `stream`. */
int cagr_probe_fp32_peak(int64_t iters, double* gflops, void* stream);

/* Diagnostic: out[i] = 1/sqrt(in[i]) for n doubles, computed as the FP64
 * traversals compute it (a hardware approximation and one third-order
 * correction), for comparison with CUDA's rsqrt(double): within 2 ulp for
 * normal positive arguments; 0 and +inf give NaN (the traversals never pass
 * them). */
int cagr_probe_rsqrt64(const double* in_dev, double* out_dev, int64_t n, void* stream);

/* Device memory (no counterpart in the reference, whose allocations are
 * torch's): every array the library allocates -- trees, node records, build
 * and marching-cubes scratch -- comes from one stream-ordered pool per device
 * that keeps freed memory reserved for later calls.  cagr_pool_trim
 * synchronises the current device and releases reserved, unused memory beyond
 * keep_bytes; cagr_pool_reserved reports the bytes the current device's pool
 * holds from the CUDA driver and the bytes in use. */
int cagr_pool_trim(int64_t keep_bytes);
int cagr_pool_reserved(int64_t* reserved_bytes, int64_t* used_bytes);

/* Fault injection for tests (no counterpart in the reference, which checks no
 * allocation at all): after n more library allocations succeed, every further
 * one fails with CAGR_ERR_ALLOC, as a full device would make it; n < 0 turns
 * this off (the default).  Process-wide. */
int cagr_debug_fail_allocations_after(int64_t n);

/* Far-field modes of a tree (no counterpart in the reference, whose treecode
 * has the first one only).
 *
 * CAGR_FAR_REFERENCE (the default): the reference's algorithm,
 * wn_treecode_cuda_kernels.cu:556-1322 -- one term per accepted node at its
 * |attr|-weighted centroid, accepted per query when |x - c|^2 > (4 half_w)^2;
 * every query sums exactly the reference's pair set (the parity mode).
 *
 * CAGR_FAR_INTERP: the same operators with an interpolated far field -- the
 * pair kernel interpolated in the source position on a (degree+1)^3
 * Chebyshev grid of each node's bounding box (proxy charges from the node's
 * points), accepted once per group of queries (32 consecutive ones, split
 * when they straddle a jump of the curve) when r_node + theta * r_group <
 * theta * distance -- so r_node < theta * |x - c| for every query x -- and no
 * pair lies within a query's width; near nodes of at most direct_max points
 * are summed directly.  Its error against the exact
 * (direct) sums falls geometrically with the degree.  In this mode
 * cagr_scatter / cagr_scatter3 compute proxy charges (weights_dev is
 * ignored: there are no centroids); cagr_multiply, cagr_forward and
 * cagr_field_grid evaluate A, AT, A3, A21..A23, A2T1..A2T3, G, A2_FUSED,
 * A2T_SUM, A2T_SUM_SHARED and COUNT; cagr_scatter_export, cagr_adjoint,
 * cagr_multiply_rhs_window, cagr_b_window_table, CAGR_OP_A2T_RHS and
 * CAGR_OP_A2_INSIDE return CAGR_ERR_STATE / CAGR_ERR_INVALID.  Explicit
 * queries should come in a spatially coherent order (query_order_dev: e.g.
 * Morton order), since the acceptance test is per group of 32. */
enum { CAGR_FAR_REFERENCE = 0, CAGR_FAR_INTERP = 1 };

/* Sets the far-field mode (degree 1..8, theta in (0, 1), direct_max >= 1 are
 * used by CAGR_FAR_INTERP only).  Switching to CAGR_FAR_INTERP computes the
 * nodes' bounding boxes and proxy layout (synchronises `stream`); the
 * moments / charges must be recomputed after any switch. */
int cagr_tree_set_far_field(cagr_tree* tree, int mode, int degree, double theta, int direct_max,
                            void* stream);

/* The current mode and its parameters; num_interp_nodes = nodes with proxy
 * grids.  Any output may be NULL.  Synchronises the device and returns
 * CAGR_ERR_CUDA if a walk of the interpolated far field abandoned one of its
 * bounded waits for the records it stages into shared memory (its outputs are
 * then incomplete); such a wait is bounded so that no kernel can hang. */
int cagr_tree_far_field(const cagr_tree* tree, int* mode, int* degree, double* theta,
                        int* direct_max, int64_t* num_interp_nodes);

/* Test hook (no counterpart in the reference): the number of try_wait rounds
 * after which a walk of the interpolated far field abandons a staging wait
 * (default 4194304).  0 makes every walk abandon its first wait at once: it
 * sets the error flag that cagr_tree_far_field reports, waits for the copies
 * it has in flight and stops, so the error path can be tested without a
 * fault. */
int cagr_debug_interp_wait_limit(cagr_tree* tree, int64_t spin);

/* The order in which self-queries (queries_dev NULL) are processed: order_dev
 * [n] int32 receives the original index of the i-th one; each consecutive
 * group of 32 walks the tree together (a 3-D Hilbert order of the points).
 * No counterpart in the reference (one thread per query there). */
int cagr_tree_query_groups(const cagr_tree* tree, int32_t* order_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CAGR_H */
