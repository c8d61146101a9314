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
