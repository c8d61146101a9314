/*
 * cagr_oracle.c -- CPU restatement of the reference treecode.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product in
 * cagr_b200/; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  Nothing in the product calls it.
 *
 * Parity is pinned: tests/test_oracle.py compares every function here against
 * the reference's own sources compiled on the host (oracle/_ref, built by
 * `make -C oracle ref`), and against the committed golden vectors in
 * tests/golden/ that were generated from those sources.
 *
 * Contents (reference = mayueji/CAGR, paths inside that project):
 *  - octree build + serialisation, restating build_tree_cpu_recursive
 *    (CUDA-based/ext/wn_treecode/wn_treecode_cpu/wn_treecode_cpu_treeutils.cpp:90-177)
 *    and serialize_tree_recursive (same file :202-258), with the root placed
 *    as in build_tree_cpu (wn_treecode_cpu_torch_interface.cpp:42-102);
 *  - bottom-up node moments, restating scatter_point_attrs_to_nodes
 *    (wn_treecode_cuda_torch_interface.cu:41-134 and the leaf / nonleaf
 *    kernels wn_treecode_cuda_kernels.cu:419-523), in the same floating-point
 *    operation order so the node arrays come out bit-identical;
 *  - per-query depth-first traversal with the reference acceptance rule
 *    (wn_treecode_cuda_kernels.cu:586-618) for the operators A, AT, A3,
 *    A21/A22/A23, A2T1/A2T2/A2T3 and G (pair terms at :80-414);
 *  - an FP64 direct sum (no tree) of every operator: the accuracy oracle;
 *  - an instrumented traversal that counts pair interactions per query.
 *
 * Build: oracle/Makefile (gcc -O3 -ffp-contract=off -fopenmp).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t idx_t;

/* Operator codes (same numbering as oracle/ref_cuda_host.cpp and oracle.py). */
enum {
    OP_A = 0,
    OP_AT = 1,
    OP_A3 = 2,
    OP_A21 = 3,
    OP_A22 = 4,
    OP_A23 = 5,
    OP_A2T1 = 6,
    OP_A2T2 = 7,
    OP_A2T3 = 8,
    OP_G = 9,
};

/* ------------------------------------------------------------------------ */
/* Octree build                                                              */
/* ------------------------------------------------------------------------ */

typedef struct {
    idx_t m, cap;             /* nodes so far, capacity */
    idx_t l, lcap;            /* node2point entries so far, capacity */
    idx_t depth, num_leaves;  /* deepest node depth, leaf count */
    idx_t *parent, *children, *npts, *n2p_start, *n2p;
    unsigned char* is_leaf;
    double* half_w;
    /* build parameters */
    const double* xyz;
    idx_t max_depth, leaf_size;
} OTree;

static int ot_grow_nodes(OTree* t) {
    if (t->m < t->cap) return 0;
    idx_t nc = t->cap ? t->cap * 2 : 1024;
    idx_t* p = realloc(t->parent, sizeof(idx_t) * nc);
    if (!p) return -1;
    t->parent = p;
    p = realloc(t->children, sizeof(idx_t) * nc * 8);
    if (!p) return -1;
    t->children = p;
    p = realloc(t->npts, sizeof(idx_t) * nc);
    if (!p) return -1;
    t->npts = p;
    p = realloc(t->n2p_start, sizeof(idx_t) * nc);
    if (!p) return -1;
    t->n2p_start = p;
    unsigned char* b = realloc(t->is_leaf, nc);
    if (!b) return -1;
    t->is_leaf = b;
    double* h = realloc(t->half_w, sizeof(double) * nc);
    if (!h) return -1;
    t->half_w = h;
    t->cap = nc;
    return 0;
}

static int ot_append_points(OTree* t, const idx_t* ids, idx_t n) {
    if (t->l + n > t->lcap) {
        idx_t nc = t->lcap ? t->lcap : 4096;
        while (nc < t->l + n) nc *= 2;
        idx_t* p = realloc(t->n2p, sizeof(idx_t) * nc);
        if (!p) return -1;
        t->n2p = p;
        t->lcap = nc;
    }
    memcpy(t->n2p + t->l, ids, sizeof(idx_t) * n);
    t->l += n;
    return 0;
}

/*
 * Creates the node for `ids` (ascending original indices) and its subtree.
 * Node ids are handed out on creation, parents before children and octants
 * in order 0..7, so ids are preorder ids; each node's point list is appended
 * to n2p when the node is created, which is the same preorder concatenation
 * the reference serialiser produces.  A node is a leaf when it is at
 * max_depth or holds at most leaf_size points.  Octant code: +1 if x >= cx,
 * +2 if y >= cy, +4 if z >= cz.  All centres are dyadic rationals, exactly
 * representable in float and double, so comparing in double gives the same
 * answer as the reference's comparison in the input precision.
 */
static int ot_build(OTree* t, const idx_t* ids, idx_t n, double cx, double cy, double cz,
                    double hw, idx_t depth, idx_t parent, idx_t* scratch) {
    if (ot_grow_nodes(t)) return -1;
    idx_t id = t->m++;
    t->parent[id] = parent;
    for (int k = 0; k < 8; k++) t->children[id * 8 + k] = -1;
    t->npts[id] = n;
    t->n2p_start[id] = t->l;
    t->half_w[id] = hw;
    if (depth > t->depth) t->depth = depth;
    if (ot_append_points(t, ids, n)) return -1;
    int leaf = (t->max_depth >= 0 && depth >= t->max_depth) || n <= t->leaf_size;
    t->is_leaf[id] = (unsigned char)leaf;
    if (leaf) {
        t->num_leaves++;
        return 0;
    }
    /* stable counting partition of ids into octants */
    idx_t cnt[8] = {0}, off[8];
    for (idx_t i = 0; i < n; i++) {
        const double* p = t->xyz + 3 * ids[i];
        int o = (p[0] >= cx) | ((p[1] >= cy) << 1) | ((p[2] >= cz) << 2);
        cnt[o]++;
    }
    off[0] = 0;
    for (int k = 1; k < 8; k++) off[k] = off[k - 1] + cnt[k - 1];
    idx_t* part = scratch; /* n entries, reused below for the children */
    idx_t pos[8];
    memcpy(pos, off, sizeof(pos));
    for (idx_t i = 0; i < n; i++) {
        const double* p = t->xyz + 3 * ids[i];
        int o = (p[0] >= cx) | ((p[1] >= cy) << 1) | ((p[2] >= cz) << 2);
        part[pos[o]++] = ids[i];
    }
    /* the partition must outlive the recursion into children, which reuse
     * the scratch space after it */
    double q = hw / 2.0;
    for (int k = 0; k < 8; k++) {
        if (cnt[k] == 0) continue;
        double ncx = (k & 1) ? cx + q : cx - q;
        double ncy = (k & 2) ? cy + q : cy - q;
        double ncz = (k & 4) ? cz + q : cz - q;
        idx_t child = t->m;
        t->children[id * 8 + k] = child;
        if (ot_build(t, part + off[k], cnt[k], ncx, ncy, ncz, q, depth + 1, id, scratch + n))
            return -1;
    }
    return 0;
}

static OTree* ot_new(const double* xyz, idx_t n, idx_t max_depth, idx_t leaf_size) {
    OTree* t = calloc(1, sizeof(OTree));
    if (!t) return NULL;
    t->xyz = xyz;
    t->max_depth = max_depth;
    t->leaf_size = leaf_size;
    if (n == 0) return t;
    idx_t* ids = malloc(sizeof(idx_t) * n);
    /* scratch: one partition buffer of size n per level on the current path */
    idx_t levels = (max_depth >= 0 ? max_depth : 64) + 2;
    idx_t* scratch = malloc(sizeof(idx_t) * n * levels);
    if (!ids || !scratch) {
        free(ids);
        free(scratch);
        free(t);
        return NULL;
    }
    for (idx_t i = 0; i < n; i++) ids[i] = i;
    int rc = ot_build(t, ids, n, 0.0, 0.0, 0.0, 1.0, 0, -1, scratch);
    free(ids);
    free(scratch);
    if (rc) return NULL;
    return t;
}

void* oracle_build_tree_f32(const float* pts, idx_t n, idx_t max_depth, idx_t leaf_size) {
    double* xyz = malloc(sizeof(double) * 3 * (n > 0 ? n : 1));
    if (!xyz) return NULL;
    for (idx_t i = 0; i < 3 * n; i++) xyz[i] = (double)pts[i];
    OTree* t = ot_new(xyz, n, max_depth, leaf_size);
    free(xyz);
    return t;
}

void* oracle_build_tree_f64(const double* pts, idx_t n, idx_t max_depth, idx_t leaf_size) {
    return ot_new(pts, n, max_depth, leaf_size);
}

void oracle_tree_sizes(void* h, idx_t* num_nodes, idx_t* num_leaves, idx_t* depth,
                       idx_t* n2p_len) {
    OTree* t = h;
    *num_nodes = t->m;
    *num_leaves = t->num_leaves;
    *depth = t->depth;
    *n2p_len = t->l;
}

void oracle_tree_fill(void* h, idx_t* parent, idx_t* children, unsigned char* is_leaf,
                      double* half_w, idx_t* npts, idx_t* n2p, idx_t* n2p_start) {
    OTree* t = h;
    idx_t m = t->m;
    if (m == 0) return;
    memcpy(parent, t->parent, sizeof(idx_t) * m);
    memcpy(children, t->children, sizeof(idx_t) * m * 8);
    memcpy(is_leaf, t->is_leaf, m);
    memcpy(half_w, t->half_w, sizeof(double) * m);
    memcpy(npts, t->npts, sizeof(idx_t) * m);
    memcpy(n2p, t->n2p, sizeof(idx_t) * t->l);
    memcpy(n2p_start, t->n2p_start, sizeof(idx_t) * m);
}

void oracle_tree_free(void* h) {
    OTree* t = h;
    if (!t) return;
    free(t->parent);
    free(t->children);
    free(t->npts);
    free(t->n2p_start);
    free(t->n2p);
    free(t->is_leaf);
    free(t->half_w);
    free(t);
}

/* ------------------------------------------------------------------------ */
/* Node moments and traversals, instantiated for float and double            */
/* ------------------------------------------------------------------------ */

/*
 * Node moments (node attribute sums, weights, weighted centroids).
 * Children always carry larger preorder ids than their parent, so one sweep
 * over the nodes in decreasing id order sees every child before its parent.
 * Operation order follows the reference kernels exactly: for a leaf, the
 * points in node2point order accumulate weight, attribute sum, weight-scaled
 * position and plain position; for an internal node, the existing children
 * in octant order do the same with their own sums.  The centroid is the
 * weighted sum times (1/W); with W == 0 it is the plain sum times (1/npts),
 * which for an internal node divides a sum of child centroids by the point
 * count (wn_treecode_cuda_kernels.cu:510-517).
 */
#define DEFINE_MOMENTS(T, SUF)                                                                 \
    void oracle_moments_##SUF(idx_t m, const idx_t* children, const unsigned char* is_leaf,    \
                              const idx_t* npts, const idx_t* n2p, const idx_t* n2p_start,      \
                              const T* pts, const T* w, const T* attrs, idx_t c, T* out_attrs,  \
                              T* out_rep, T* out_w) {                                           \
        for (idx_t n = m - 1; n >= 0; n--) {                                                    \
            T W = 0, acc[3] = {0, 0, 0}, rep[3] = {0, 0, 0}, plain[3] = {0, 0, 0};             \
            for (idx_t a = 0; a < c; a++) acc[a] = 0;                                           \
            if (is_leaf[n]) {                                                                   \
                for (idx_t j = 0; j < npts[n]; j++) {                                           \
                    idx_t p = n2p[n2p_start[n] + j];                                            \
                    W = W + w[p];                                                               \
                    for (idx_t a = 0; a < c; a++) acc[a] = acc[a] + attrs[p * c + a];           \
                    for (int d = 0; d < 3; d++) {                                               \
                        T s = pts[p * 3 + d] * w[p];                                            \
                        rep[d] = rep[d] + s;                                                    \
                        plain[d] = plain[d] + pts[p * 3 + d];                                   \
                    }                                                                           \
                }                                                                               \
            } else {                                                                            \
                for (int k = 0; k < 8; k++) {                                                   \
                    idx_t ch = children[n * 8 + k];                                             \
                    if (ch < 0) continue;                                                       \
                    W = W + out_w[ch];                                                          \
                    for (idx_t a = 0; a < c; a++) acc[a] = acc[a] + out_attrs[ch * c + a];      \
                    for (int d = 0; d < 3; d++) {                                               \
                        T s = out_rep[ch * 3 + d] * out_w[ch];                                  \
                        rep[d] = rep[d] + s;                                                    \
                        plain[d] = plain[d] + out_rep[ch * 3 + d];                              \
                    }                                                                           \
                }                                                                               \
            }                                                                                   \
            if (W > 0) {                                                                        \
                T inv = (T)1 / W;                                                               \
                for (int d = 0; d < 3; d++) out_rep[n * 3 + d] = rep[d] * inv;                  \
            } else {                                                                            \
                T inv = (T)1 / (T)npts[n];                                                      \
                for (int d = 0; d < 3; d++) out_rep[n * 3 + d] = plain[d] * inv;                \
            }                                                                                   \
            out_w[n] = W;                                                                       \
            for (idx_t a = 0; a < c; a++) out_attrs[n * c + a] = acc[a];                        \
        }                                                                                       \
    }

DEFINE_MOMENTS(float, f32)
DEFINE_MOMENTS(double, f64)

/*
 * Pair terms.  d = x - y (query minus source), r2 = (d0*d0 + d1*d1) + d2*d2
 * in the working precision, r = sqrt(r2); a pair contributes only when
 * r >= w (w = the query's smoothing width), except for the continuous
 * variants of A / A2k which use w in place of r inside the width.
 *   A   : d.mu / r^3                                   (:80-110, CUDA sign)
 *   A2k : exp(d_k/2) (d.mu / r^3 + mu_k / (2r))        (:113-224)
 *         continuous, inside: exp(w) (d.mu / w^3 + mu_k / (2w))
 *   AT  : d s / r^3                      -> R^3        (:229-258)
 *   A2Tk: exp(d_k/2) (d s / r^3 + e_k s / (2r)) -> R^3 (:263-379)
 *   G   : mu / r^3 - 3 d (d.mu) / r^5    -> R^3        (:385-414)
 * A3 sums A21+A22+A23 per interaction and divides by 3 at the end (:694-763).
 */
#define DEFINE_TRAVERSE(T, SUF, SQRT, EXP)                                                     \
    static void pair_##SUF(int op, const T* d, const T* a, T w, int cont, T* out) {            \
        T r2 = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];                                     \
        T r = SQRT(r2);                                                                        \
        int outside = r >= w;                                                                  \
        if (op == OP_A) {                                                                      \
            T dm = (d[0] * a[0] + d[1] * a[1]) + d[2] * a[2];                                 \
            if (outside)                                                                       \
                out[0] += dm / (r * r2);                                                       \
            else if (cont)                                                                     \
                out[0] += dm / (w * w * w);                                                    \
        } else if (op == OP_A21 || op == OP_A22 || op == OP_A23 || op == OP_A3) {              \
            int k0 = (op == OP_A3) ? 0 : op - OP_A21, k1 = (op == OP_A3) ? 3 : k0 + 1;         \
            T dm = (d[0] * a[0] + d[1] * a[1]) + d[2] * a[2];                                 \
            for (int k = k0; k < k1; k++) {                                                    \
                if (outside) {                                                                 \
                    T e = EXP(d[k] * (T)0.5);                                                  \
                    out[0] += e * (dm / (r * r2) + a[k] * (T)0.5 / r);                         \
                } else if (cont) {                                                             \
                    T e = EXP(w);                                                              \
                    out[0] += e * (dm / (w * w * w) + a[k] * (T)0.5 / w);                      \
                }                                                                              \
            }                                                                                  \
        } else if (op == OP_AT) {                                                              \
            if (outside)                                                                       \
                for (int j = 0; j < 3; j++) out[j] += d[j] * a[0] / (r * r2);                  \
        } else if (op == OP_A2T1 || op == OP_A2T2 || op == OP_A2T3) {                          \
            int k = op - OP_A2T1;                                                              \
            if (outside) {                                                                     \
                T e = EXP(d[k] * (T)0.5);                                                      \
                for (int j = 0; j < 3; j++) {                                                  \
                    T t = d[j] * a[0] / (r * r2);                                              \
                    if (j == k) t += a[0] * (T)0.5 / r;                                        \
                    out[j] += e * t;                                                           \
                }                                                                              \
            }                                                                                  \
        } else if (op == OP_G) {                                                               \
            if (outside) {                                                                     \
                T dm = (d[0] * a[0] + d[1] * a[1]) + d[2] * a[2];                             \
                T r3 = r * r2, r5 = r2 * r3;                                                   \
                for (int j = 0; j < 3; j++) out[j] += a[j] / r3 - 3 * d[j] * dm / r5;          \
            }                                                                                  \
        }                                                                                      \
    }                                                                                          \
                                                                                               \
    static int attr_dim_##SUF(int op) {                                                        \
        return (op == OP_AT || op == OP_A2T1 || op == OP_A2T2 || op == OP_A2T3) ? 1 : 3;       \
    }                                                                                          \
    static int out_dim_##SUF(int op) {                                                         \
        return (op == OP_A || op == OP_A3 || op == OP_A21 || op == OP_A22 || op == OP_A23) ? 1 \
                                                                                           : 3; \
    }                                                                                          \
                                                                                               \
    /* Depth-first traversal with an explicit stack; children are pushed in octant order and \
     * popped last-first, as at wn_treecode_cuda_kernels.cu:588-618, so contributions are     \
     * accumulated in the reference order.  A node is far when                                 \
     * |x - c|^2 > (4 half_w)^2 with c the node centroid (:595).  Far nodes contribute one     \
     * pair term with the node's attribute sum at c; near leaves contribute each point.  The   \
     * instrumented variant counts terms (far + near) and node visits per query. */            \
    int oracle_multiply_##SUF(int op, const T* q, const T* qw, idx_t nq, const T* pts,         \
                              const T* attrs, const idx_t* n2p, const idx_t* n2p_start,         \
                              const idx_t* children, const T* node_attrs,                       \
                              const unsigned char* is_leaf, const T* half_w, const T* rep,      \
                              const idx_t* npts, T* out, int cont, idx_t* n_terms,              \
                              idx_t* n_visits) {                                                \
        if (op < OP_A || op > OP_G) return -1;                                                 \
        int ca = attr_dim_##SUF(op), co = out_dim_##SUF(op);                                   \
        int fail = 0;                                                                          \
        _Pragma("omp parallel for schedule(dynamic, 64) reduction(|:fail)")                    \
        for (idx_t i = 0; i < nq; i++) {                                                       \
            idx_t stack[22 * 7 + 2];                                                           \
            int top = 0;                                                                       \
            T acc[3] = {0, 0, 0};                                                              \
            idx_t terms = 0, visits = 0;                                                       \
            const T* x = q + 3 * i;                                                            \
            stack[top++] = 0;                                                                  \
            while (top > 0) {                                                                  \
                idx_t n = stack[--top];                                                        \
                visits++;                                                                      \
                const T* c = rep + 3 * n;                                                      \
                T dx = x[0] - c[0], dy = x[1] - c[1], dz = x[2] - c[2];                        \
                T dist2 = ((dx * dx) + (dy * dy)) + (dz * dz);                                 \
                T lim = (T)4 * half_w[n];                                                      \
                if (dist2 > lim * lim) {                                                       \
                    T d[3] = {dx, dy, dz};                                                     \
                    pair_##SUF(op, d, node_attrs + ca * n, qw[i], cont, acc);                  \
                    terms++;                                                                   \
                } else if (!is_leaf[n]) {                                                      \
                    for (int k = 0; k < 8; k++) {                                              \
                        idx_t ch = children[n * 8 + k];                                        \
                        if (ch < 0) continue;                                                  \
                        if (top >= 22 * 7 + 2) {                                               \
                            fail = 1;                                                          \
                            break;                                                             \
                        }                                                                      \
                        stack[top++] = ch;                                                     \
                    }                                                                          \
                } else {                                                                       \
                    for (idx_t j = 0; j < npts[n]; j++) {                                      \
                        idx_t p = n2p[n2p_start[n] + j];                                       \
                        T d[3] = {x[0] - pts[3 * p], x[1] - pts[3 * p + 1],                    \
                                  x[2] - pts[3 * p + 2]};                                      \
                        pair_##SUF(op, d, attrs + ca * p, qw[i], cont, acc);                   \
                        terms++;                                                               \
                    }                                                                          \
                }                                                                              \
            }                                                                                  \
            if (op == OP_A3) acc[0] = acc[0] / (T)3;                                           \
            if (out)                                                                           \
                for (int j = 0; j < co; j++) out[co * i + j] = acc[j];                         \
            if (n_terms) n_terms[i] = terms;                                                   \
            if (n_visits) n_visits[i] = visits;                                                \
        }                                                                                      \
        return fail ? -2 : 0;                                                                  \
    }

DEFINE_TRAVERSE(float, f32, sqrtf, expf)
DEFINE_TRAVERSE(double, f64, sqrt, exp)

/* ------------------------------------------------------------------------ */
/* FP64 direct sum (no tree): the accuracy oracle                             */
/* ------------------------------------------------------------------------ */

/* Sums every source for every query in double precision with the same pair
 * terms (and width rule) as the treecode.  Sources/queries are given in
 * double.  Cost O(nq * n): use for small cases and sampled queries. */
int oracle_direct_f64(int op, const double* q, const double* qw, idx_t nq, const double* pts,
                      const double* attrs, idx_t n, double* out, int cont) {
    if (op < OP_A || op > OP_G) return -1;
    int ca = attr_dim_f64(op), co = out_dim_f64(op);
#pragma omp parallel for schedule(dynamic, 16)
    for (idx_t i = 0; i < nq; i++) {
        double acc[3] = {0, 0, 0};
        for (idx_t j = 0; j < n; j++) {
            double d[3] = {q[3 * i] - pts[3 * j], q[3 * i + 1] - pts[3 * j + 1],
                           q[3 * i + 2] - pts[3 * j + 2]};
            pair_f64(op, d, attrs + ca * j, qw[i], cont, acc);
        }
        if (op == OP_A3) acc[0] /= 3.0;
        for (int j = 0; j < co; j++) out[co * i + j] = acc[j];
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Marching cubes on a regular grid (checker for cagr_marching_cubes)         */
/* ------------------------------------------------------------------------ */

/* Values v[(k*ny + j)*nx + i]; node (i,j,k) at origin + (i,j,k)*h in float as
 * fmaf(i, h, o).  A corner is inside when v > iso.  Vertices: one per crossed
 * grid edge, grid points in index order and axes x, y, z, at
 * o + i*h + ((iso - v0) / (v1 - v0)) * h along the edge.  Triangles: cells in
 * index order, each with the case table's triangles (tri[256][36] edge ids,
 * ntri[256]); edge 4a + u + 2w of cell (i,j,k) starts at the grid point offset
 * by (u, w) along the two other axes in increasing order.  With NULL outputs
 * only the counts are returned. */
int oracle_marching_cubes(const float* v, int nx, int ny, int nz, double ox, double oy, double oz,
                          double h, float iso, const signed char* tri, const unsigned char* ntri,
                          float* verts, idx_t maxv, int* faces, idx_t maxf, idx_t* nv_out,
                          idx_t* nf_out) {
    const idx_t P = (idx_t)nx * ny * nz;
    unsigned char* mask = calloc(P, 1);
    idx_t* vbase = malloc(sizeof(idx_t) * (P + 1));
    if (!mask || !vbase) {
        free(mask);
        free(vbase);
        return -1;
    }
    const float fh = (float)h, fox = (float)ox, foy = (float)oy, foz = (float)oz;
    idx_t nv = 0;
    for (idx_t p = 0; p < P; p++) {
        const int i = (int)(p % nx), j = (int)((p / nx) % ny), k = (int)(p / ((idx_t)nx * ny));
        const int a = v[p] > iso;
        unsigned char m = 0;
        if (i + 1 < nx && (v[p + 1] > iso) != a) m |= 1;
        if (j + 1 < ny && (v[p + nx] > iso) != a) m |= 2;
        if (k + 1 < nz && (v[p + (idx_t)nx * ny] > iso) != a) m |= 4;
        mask[p] = m;
        vbase[p] = nv;
        if (verts && m) {
            const float x = fmaf((float)i, fh, fox), y = fmaf((float)j, fh, foy),
                        z = fmaf((float)k, fh, foz);
            const idx_t step[3] = {1, nx, (idx_t)nx * ny};
            idx_t o = nv;
            for (int ax = 0; ax < 3; ax++) {
                if (!((m >> ax) & 1)) continue;
                if (o >= maxv) break;
                const float t = (iso - v[p]) / (v[p + step[ax]] - v[p]);
                const float d = t * fh;
                verts[3 * o + 0] = ax == 0 ? x + d : x;
                verts[3 * o + 1] = ax == 1 ? y + d : y;
                verts[3 * o + 2] = ax == 2 ? z + d : z;
                o++;
            }
        }
        nv += (m & 1) + ((m >> 1) & 1) + ((m >> 2) & 1);
    }
    vbase[P] = nv;
    idx_t nf = 0;
    const int cx = nx - 1, cy = ny - 1, cz = nz - 1;
    for (idx_t c = 0; c < (idx_t)cx * cy * cz; c++) {
        const int i = (int)(c % cx), j = (int)((c / cx) % cy), k = (int)(c / ((idx_t)cx * cy));
        const idx_t p = ((idx_t)k * ny + j) * nx + i;
        int cs = 0;
        for (int q = 0; q < 8; q++) {
            const idx_t o = (q & 1) + ((q >> 1) & 1) * (idx_t)nx + (q >> 2) * (idx_t)nx * ny;
            if (v[p + o] > iso) cs |= 1 << q;
        }
        for (int t = 0; t < ntri[cs]; t++, nf++) {
            if (!faces || nf >= maxf) continue;
            for (int s = 0; s < 3; s++) {
                const int e = tri[cs * 36 + 3 * t + s];
                const int ax = e >> 2, u = e & 1, w = (e >> 1) & 1;
                int oi = i, oj = j, ok = k;
                if (ax == 0) {
                    oj += u;
                    ok += w;
                } else if (ax == 1) {
                    oi += u;
                    ok += w;
                } else {
                    oi += u;
                    oj += w;
                }
                const idx_t q = ((idx_t)ok * ny + oj) * nx + oi;
                int rank = 0;
                for (int b = 0; b < ax; b++) rank += (mask[q] >> b) & 1;
                faces[3 * nf + s] = (int)(vbase[q] + rank);
            }
        }
    }
    *nv_out = nv;
    *nf_out = nf;
    free(mask);
    free(vbase);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* The interpolated far-field mode of the library (CAGR_FAR_INTERP), FP64    */
/* ------------------------------------------------------------------------ */

/* The checker of cagr_b200's second evaluation mode, which has no
 * counterpart in the reference: the same operators (the exact pair sums of
 * the pair terms above) with the far field of the barycentric Lagrange
 * treecode (L. Wang, R. Krasny, S. Tlupova, Commun. Comput. Phys. 28 (2020)):
 *  - box of a node = the tight bounding box of its points (centre (lo+hi)/2,
 *    half extents floored at 1e-3 of the largest), radius |half extents|;
 *  - nodes with >= (p+1)^3 points carry proxy charges
 *    q_m = sum_j L_a(u_x) L_b(u_y) L_c(u_z) a_j on the tensor grid of
 *    Chebyshev points of the second kind cos(pi k / p) scaled to the box
 *    (barycentric Lagrange basis L, weights (-1)^k halved at both ends);
 *  - queries are processed in groups of 32 (in `order`), split top-down
 *    into aligned subgroups: a group of 2^k is split when its radius
 *    exceeds 5 times that of its more compact half (ip_group); a final
 *    subgroup's batch is the bounding box of its
 *    queries (centre, radius r_B) and its largest width w_B, walked on its
 *    own; a node is far when r_C + theta r_B < theta R and
 *    R >= r_B + r_C + w_B (R = distance of the centres; radii and w_B scaled
 *    by 1 + 2^-16 as the library scales them); the walk is the preorder of
 *    the tree: far -> proxy grid (nodes with proxies) or the node's points;
 *    near leaves and near nodes of <= direct_max points -> their points;
 *    otherwise the children.
 * Operators: the ten above plus 10 = A2_FUSED (A21, A22, A23 as three
 * columns), 11 = A2T_SUM (sum_k A2Tk of the k-th of three scalar columns),
 * 12 = COUNT (pair terms per query), 13 = A2T_SUM_SHARED (sum_k A2Tk(s)).
 * kind: 0 = attrs [n,3] vectors, 1 = [n,1] scalars, 2 = [n,3] three scalar
 * columns.  terms (optional): pair terms per query. */
enum { OP_A2_FUSED = 10, OP_A2T_SUM = 11, OP_COUNT = 12, OP_A2T_SHARED = 13 };

static void ip_pair(int op, const double* d, const double* a, double w, int cont, double* acc) {
    switch (op) {
        case OP_A2_FUSED:
            pair_f64(OP_A21, d, a, w, cont, acc);
            pair_f64(OP_A22, d, a, w, cont, acc + 1);
            pair_f64(OP_A23, d, a, w, cont, acc + 2);
            break;
        case OP_A2T_SUM:
            for (int k = 0; k < 3; k++) pair_f64(OP_A2T1 + k, d, a + k, w, 0, acc);
            break;
        case OP_A2T_SHARED:
            for (int k = 0; k < 3; k++) pair_f64(OP_A2T1 + k, d, a, w, 0, acc);
            break;
        case OP_COUNT: break;
        default: pair_f64(op, d, a, w, cont, acc);
    }
}

static void ip_lagrange(double u, int P, const double* t, const double* om, double* L) {
    for (int k = 0; k < P; k++)
        if (u == t[k]) {
            for (int l = 0; l < P; l++) L[l] = l == k ? 1.0 : 0.0;
            return;
        }
    double sum = 0.0;
    for (int k = 0; k < P; k++) {
        L[k] = om[k] / (u - t[k]);
        sum += L[k];
    }
    for (int k = 0; k < P; k++) L[k] /= sum;
}

/* Box of the queries [a, min(b, end)) in `order`: centre c, radius r (half
 * extents from the farther end, |h| * (1 + 2^-16)), largest width w (NaN ->
 * inf, scaled alike); r = w = 0 for an empty range. */
static void ip_group(const double* q, const double* qw, const idx_t* order, idx_t a, idx_t b,
                     idx_t end, double* c, double* r, double* w) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    double wm = 0.0;
    if (b > end) b = end;
    for (idx_t k = a; k < b; k++) {
        const idx_t qi = order ? order[k] : k;
        for (int x = 0; x < 3; x++) {
            lo[x] = fmin(lo[x], q[3 * qi + x]);
            hi[x] = fmax(hi[x], q[3 * qi + x]);
        }
        wm = fmax(wm, qw[qi] == qw[qi] ? qw[qi] : INFINITY);
    }
    if (!(lo[0] <= hi[0])) {
        c[0] = c[1] = c[2] = 0.0;
        *r = *w = 0.0;
        return;
    }
    double h[3];
    for (int x = 0; x < 3; x++) {
        c[x] = 0.5 * (lo[x] + hi[x]);
        h[x] = fmax(hi[x] - c[x], c[x] - lo[x]);
    }
    *r = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]) * (1.0 + 1.0 / 65536);
    *w = wm * (1.0 + 1.0 / 65536);
}

int oracle_interp_f64(int op, int cont, const double* q, const double* qw, const idx_t* order,
                      idx_t nq, const double* pts, const double* attrs, idx_t n, int kind,
                      const idx_t* children, const unsigned char* is_leaf, const idx_t* npts,
                      const idx_t* n2p, const idx_t* n2p_start, idx_t M, int degree,
                      double theta, int direct_max, double* out, idx_t* terms) {
    (void)n;
    if (degree < 1 || degree > 8) return -1;
    const int P = degree + 1, P3 = P * P * P;
    const int ca = kind == 1 ? 1 : 3;
    const int co = (op == OP_A || op == OP_A3 || op == OP_A21 || op == OP_A22 || op == OP_A23 ||
                    op == OP_COUNT) ? 1 : 3;
    double tch[9], om[9];
    for (int k = 0; k <= degree; k++) {
        tch[k] = cos(acos(-1.0) * (double)k / (double)degree);
        om[k] = ((k & 1) ? -1.0 : 1.0) * ((k == 0 || k == degree) ? 0.5 : 1.0);
    }
    double* box = malloc(sizeof(double) * 7 * M);   /* c[3], h[3], r */
    idx_t* iidx = malloc(sizeof(idx_t) * M);
    if (!box || !iidx) {
        free(box);
        free(iidx);
        return -1;
    }
    idx_t ni = 0;
    for (idx_t i = 0; i < M; i++) {
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (idx_t j = 0; j < npts[i]; j++) {
            const double* y = pts + 3 * n2p[n2p_start[i] + j];
            for (int a = 0; a < 3; a++) {
                lo[a] = fmin(lo[a], y[a]);
                hi[a] = fmax(hi[a], y[a]);
            }
        }
        double* b = box + 7 * i;
        double hmax = 0.0;
        for (int a = 0; a < 3; a++) {
            if (!(lo[a] <= hi[a])) lo[a] = hi[a] = 0.0;
            b[a] = 0.5 * (lo[a] + hi[a]);
            b[3 + a] = fmax(hi[a] - b[a], b[a] - lo[a]);
            hmax = fmax(hmax, b[3 + a]);
        }
        const double fl = fmax(hmax * 1e-3, 1e-30);
        for (int a = 0; a < 3; a++) b[3 + a] = fmax(b[3 + a], fl);
        b[6] = sqrt(b[3] * b[3] + b[4] * b[4] + b[5] * b[5]) * (1.0 + 1.0 / 65536);
        iidx[i] = npts[i] >= P3 ? ni++ : -1;
    }
    /* proxy grids: positions [ni][P3][3], charges [ni][P3][3] */
    double* ppos = malloc(sizeof(double) * 3 * (size_t)(ni > 0 ? ni : 1) * P3);
    double* pchg = calloc(3 * (size_t)(ni > 0 ? ni : 1) * P3, sizeof(double));
    if (!ppos || !pchg) {
        free(box);
        free(iidx);
        free(ppos);
        free(pchg);
        return -1;
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (idx_t i = 0; i < M; i++) {
        if (iidx[i] < 0) continue;
        const double* b = box + 7 * i;
        double* pp = ppos + 3 * (size_t)iidx[i] * P3;
        double* pc = pchg + 3 * (size_t)iidx[i] * P3;
        for (int m = 0; m < P3; m++) {
            const int ia = m / (P * P), ib = (m / P) % P, ic = m % P;
            pp[3 * m] = b[0] + b[3] * tch[ia];
            pp[3 * m + 1] = b[1] + b[4] * tch[ib];
            pp[3 * m + 2] = b[2] + b[5] * tch[ic];
        }
        for (idx_t j = 0; j < npts[i]; j++) {
            const idx_t pj = n2p[n2p_start[i] + j];
            double L[3][9];
            for (int a = 0; a < 3; a++) {
                double u = (pts[3 * pj + a] - b[a]) / b[3 + a];
                u = fmin(fmax(u, -1.0), 1.0);
                ip_lagrange(u, P, tch, om, L[a]);
            }
            const double* aj = attrs + ca * pj;
            for (int m = 0; m < P3; m++) {
                const double wgt = L[0][m / (P * P)] * L[1][(m / P) % P] * L[2][m % P];
                for (int c = 0; c < ca; c++) pc[3 * m + c] += wgt * aj[c];
            }
        }
    }
    const double th2 = theta * theta;
    const idx_t ngroups = (nq + 31) / 32;
#pragma omp parallel for schedule(dynamic, 4)
    for (idx_t g = 0; g < ngroups; g++) {
        const idx_t q0 = g * 32, q1 = q0 + 32 < nq ? q0 + 32 : nq;
        /* each query's group, top-down: the aligned group of 2^k queries is
         * split when its radius exceeds 5 times that of its more compact half */
        int kq_of[32];
        for (idx_t i = q0; i < q1; i++) {
            int k = 5;
            while (k > 0) {
                const idx_t a = q0 + (((i - q0) >> k) << k), h = (idx_t)1 << (k - 1);
                double c[3], r, r0, r1, w;
                ip_group(q, qw, order, a, a + 2 * h, q1, c, &r, &w);
                ip_group(q, qw, order, a, a + h, q1, c, &r0, &w);
                ip_group(q, qw, order, a + h, a + 2 * h, q1, c, &r1, &w);
                if (!(r > 5.0 * fmin(r0, r1))) break;
                k--;
            }
            kq_of[i - q0] = k;
        }
        double acc[32][3];
        idx_t cnt[32];
        memset(acc, 0, sizeof(acc));
        memset(cnt, 0, sizeof(cnt));
        for (idx_t sa = q0; sa < q1; sa += (idx_t)1 << kq_of[sa - q0]) {
            const idx_t sb = sa + ((idx_t)1 << kq_of[sa - q0]) < q1 ? sa + ((idx_t)1 << kq_of[sa - q0]) : q1;
            double bc[3], br, wm;
            ip_group(q, qw, order, sa, sb, q1, bc, &br, &wm);
            idx_t stack[8 * 64];
            int sp = 0;
            stack[sp++] = 0;
            while (sp > 0) {
                const idx_t nd = stack[--sp];
                const double* b = box + 7 * nd;
                const double dx = bc[0] - b[0], dy = bc[1] - b[1], dz = bc[2] - b[2];
                const double R2 = dx * dx + dy * dy + dz * dz;
                const double sr = br + b[6], sw = sr + wm, a = b[6] + theta * br;
                const int far = a * a < th2 * R2 && R2 >= sw * sw;
                if (far && iidx[nd] >= 0) {
                    const double* pp = ppos + 3 * (size_t)iidx[nd] * P3;
                    const double* pc = pchg + 3 * (size_t)iidx[nd] * P3;
                    for (idx_t kq = sa; kq < sb; kq++) {
                        const idx_t qi = order ? order[kq] : kq;
                        for (int m = 0; m < P3; m++) {
                            const double d[3] = {q[3 * qi] - pp[3 * m], q[3 * qi + 1] - pp[3 * m + 1],
                                                 q[3 * qi + 2] - pp[3 * m + 2]};
                            ip_pair(op, d, pc + 3 * m, qw[qi], cont, acc[kq - q0]);
                        }
                        cnt[kq - q0] += P3;
                    }
                } else if (far || is_leaf[nd] || npts[nd] <= direct_max) {
                    for (idx_t kq = sa; kq < sb; kq++) {
                        const idx_t qi = order ? order[kq] : kq;
                        for (idx_t j = 0; j < npts[nd]; j++) {
                            const idx_t pj = n2p[n2p_start[nd] + j];
                            const double d[3] = {q[3 * qi] - pts[3 * pj], q[3 * qi + 1] - pts[3 * pj + 1],
                                                 q[3 * qi + 2] - pts[3 * pj + 2]};
                            ip_pair(op, d, attrs + ca * pj, qw[qi], cont, acc[kq - q0]);
                        }
                        cnt[kq - q0] += npts[nd];
                    }
                } else {
                    for (int c = 7; c >= 0; c--)
                        if (children[8 * nd + c] >= 0) stack[sp++] = children[8 * nd + c];
                }
            }
        }
        for (idx_t kq = q0; kq < q1; kq++) {
            const idx_t qi = order ? order[kq] : kq;
            if (op == OP_A3) acc[kq - q0][0] /= 3.0;
            if (op == OP_COUNT) acc[kq - q0][0] = (double)cnt[kq - q0];
            for (int j = 0; j < co; j++) out[co * qi + j] = acc[kq - q0][j];
            if (terms) terms[qi] = cnt[kq - q0];
        }
    }
    free(box);
    free(iidx);
    free(ppos);
    free(pchg);
    return 0;
}

/* Marching cubes with a case table in the reference's layout, restating its
 * per-cube lookup: MarchingCubes::GetIndex (gaussrecon_src/MarchingCubes.cpp:
 * 333-345; bit k set when the k-th corner of (0,0,0), (1,0,0), (1,1,0), (0,1,0),
 * (0,0,1), (1,0,1), (1,1,1), (0,1,1) has value < iso), AddTriangleIndices
 * (:573-584; the case's row of triangles[256][16] until -1) and
 * Cube::EdgeCorners / FactorEdgeIndex (Cube.cpp:86-108; edge e runs along axis
 * e >> 2 from corner (.., e & 1, (e >> 1) & 1) in the other two axes' order).
 * Inside = value < iso.  Vertices: one per crossed grid edge, numbered and
 * placed as in oracle_marching_cubes; faces: cells in index order, each case's
 * triangles in the table's order.  Returns -2 for an entry that is not an
 * edge the case crosses. */
int oracle_marching_cubes_reftable(const float* v, int nx, int ny, int nz, double ox, double oy,
                                   double oz, double h, float iso, const signed char* tri16,
                                   float* verts, idx_t maxv, int* faces, idx_t maxf,
                                   idx_t* nv_out, idx_t* nf_out) {
    static const int corner_xyz[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                         {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    const idx_t P = (idx_t)nx * ny * nz, sx = 1, sy = nx, sz = (idx_t)nx * ny;
    unsigned char* mask = calloc(P, 1);
    idx_t* vbase = malloc(sizeof(idx_t) * (P + 1));
    if (!mask || !vbase) {
        free(mask);
        free(vbase);
        return -1;
    }
    const float fh = (float)h, fo[3] = {(float)ox, (float)oy, (float)oz};
    idx_t nv = 0;
    for (idx_t p = 0; p < P; p++) {
        const int c[3] = {(int)(p % nx), (int)((p / nx) % ny), (int)(p / sz)};
        const int n[3] = {nx, ny, nz};
        const idx_t step[3] = {sx, sy, sz};
        const int below = v[p] < iso;
        unsigned char m = 0;
        for (int ax = 0; ax < 3; ax++)
            if (c[ax] + 1 < n[ax] && (v[p + step[ax]] < iso) != below) m |= (unsigned char)(1 << ax);
        mask[p] = m;
        vbase[p] = nv;
        for (int ax = 0; ax < 3; ax++) {
            if (!((m >> ax) & 1)) continue;
            if (verts && nv < maxv) {
                const float t = (iso - v[p]) / (v[p + step[ax]] - v[p]);
                for (int d = 0; d < 3; d++) {
                    const float x = fmaf((float)c[d], fh, fo[d]);
                    verts[3 * nv + d] = d == ax ? x + t * fh : x;
                }
            }
            nv++;
        }
    }
    vbase[P] = nv;
    idx_t nf = 0;
    int rc = 0;
    for (int k = 0; k + 1 < nz && !rc; k++) {
        for (int j = 0; j + 1 < ny && !rc; j++) {
            for (int i = 0; i + 1 < nx && !rc; i++) {
                const idx_t p = (idx_t)k * sz + (idx_t)j * sy + i;
                int idx = 0;
                for (int q = 0; q < 8; q++) {
                    const int* o = corner_xyz[q];
                    if (v[p + o[0] * sx + o[1] * sy + o[2] * sz] < iso) idx |= 1 << q;
                }
                const signed char* row = tri16 + 16 * idx;
                for (int q = 0; q < 15 && row[q] != -1; q += 3, nf++) {
                    for (int s = 0; s < 3; s++) {
                        const int e = row[q + s];
                        if (e < 0 || e > 11) {
                            rc = -2;
                            break;
                        }
                        const int ax = e >> 2, a = e & 1, b = (e >> 1) & 1;
                        int off[3];
                        off[ax] = 0;
                        off[ax == 0 ? 1 : 0] = a;
                        off[ax == 2 ? 1 : 2] = b;
                        const idx_t g = p + off[0] * sx + off[1] * sy + off[2] * sz;
                        if (!((mask[g] >> ax) & 1)) {
                            rc = -2;
                            break;
                        }
                        int rank = 0;
                        for (int t = 0; t < ax; t++) rank += (mask[g] >> t) & 1;
                        if (faces && nf < maxf) faces[3 * nf + s] = (int)(vbase[g] + rank);
                    }
                    if (rc) break;
                }
            }
        }
    }
    *nv_out = nv;
    *nf_out = nf;
    free(mask);
    free(vbase);
    return rc;
}
