// Bottom-up node moments ("scatter point attributes to nodes").
//
// Reference: mayueji/CAGR CUDA-based/ext/wn_treecode/wn_treecode_cuda/
// wn_treecode_cuda_torch_interface.cu:41-134 launches one leaf kernel and then
// 2*tree_depth kernels over ALL M nodes (find-next + nonleaf,
// wn_treecode_cuda_kernels.cu:419-553).  Here one launch does the whole
// reduction: one thread per leaf computes the leaf moments, then climbs; at
// every parent the last-arriving child (arrival counter incremented by an
// acquire-release atomic, so the last arrival sees its siblings' records; reset
// by the thread that completes the node) computes the parent from its children
// in octant order.  No thread ever waits for another.  (A level-synchronous
// variant -- one launch per depth -- measured slower at 1M points: its ~15
// dependent launches cost more than the arrival counters.)  The
// floating-point operation order is the reference's, so node sums, weights and
// centroids are bit-identical to the reference kernels evaluated in IEEE
// arithmetic:
//   leaf:     for points in node2point order  W += w;  A += a;  R += y*w;  P += y
//   internal: for children in octant order    W += Wc; A += Ac; R += Rc*Wc; P += Rc
//   centroid: W > 0 ? R * (1/W) : P * (1/npts)            (:456-461, :510-517)
// The same launch writes the Morton-ordered point records the traversal reads.  Every record carries exp(-c/2) per axis so the traversal forms the
// convection factor exp((x-c)_k/2) as exp(x_k/2) * exp(-c_k/2), and node
// records carry the acceptance radius (4 half_w)^2.
//
// NS = 3 computes three independent scalar attributes (the three inputs of
// the reference's A2T1/A2T2/A2T3 calls, each with its own |s_k| weights and
// centroids) in the same launch, and also writes the packed adjoint records.
#include <string>

#include "internal.h"

namespace cagr {
namespace {

constexpr int kBlock = 256;
// The climb's blocks are small: a block stays resident until its last thread
// has climbed, so a 256-thread block held 8 warps for one climbing lane
// (measured at 1M points: 64 threads 0.208 -> 0.190 ms, with the parent
// prefetch below 0.162 ms; 32 threads 0.166 ms).
constexpr int kClimbBlock = 64;

template <typename T>
__device__ __forceinline__ T weight_of(const T* a, int dim) {
    if (dim == 1) return sqrt_rn(mul_rn(a[0], a[0]));
    return sqrt_rn(add_rn(add_rn(mul_rn(a[0], a[0]), mul_rn(a[1], a[1])), mul_rn(a[2], a[2])));
}

// r0 = (x, y, z, r0w), r1 = (e1, e2, e3, a0), r2 = (a1, a2, W, 0)
template <typename T, int DIM>
__device__ __forceinline__ void write_record(T* r, const T* pos, const T* e, const T* a, T W,
                                             T r0w) {
    st4<T>(r, make4(pos[0], pos[1], pos[2], r0w));
    st4<T>(r + 4, make4(e[0], e[1], e[2], a[0]));
    st4<T>(r + 8, make4(DIM == 3 ? a[1] : T(0), DIM == 3 ? a[2] : T(0), W, T(0)));
}

template <typename T>
__device__ __forceinline__ void exps(const T* c, T* e) {
    e[0] = exp_t(c[0] * T(-0.5));
    e[1] = exp_t(c[1] * T(-0.5));
    e[2] = exp_t(c[2] * T(-0.5));
}

template <typename T, int DIM, int NS>
struct MomParams {
    int64_t num_leaves = 0, M = 0;
    const int32_t* leaf_ids = nullptr;
    const int4* meta = nullptr;
    const uint8_t* nchild = nullptr;
    const int32_t* parent = nullptr;
    const int32_t* children = nullptr;
    const int32_t* perm = nullptr;
    const int32_t* invperm = nullptr;
    const int32_t* lorder = nullptr;  // leaves' points in original-index order (null: perm)
    const T* spos = nullptr;
    const T* attrs = nullptr;    // row stride astride; slot k reads columns [k*DIM, k*DIM+DIM)
    int astride = DIM;
    const T* weights = nullptr;  // NS == 1 only; null = |attr|
    uint32_t* counters = nullptr;
    T* rec[NS];
    T* adjn = nullptr;  // NS == 3: packed adjoint node records [M*12]
    T* adjp = nullptr;  // NS == 3: packed adjoint point records [N*8]
    T* adjs = nullptr;  // NS == 3: node sums (W_k), (A_k) [M*8]
};

// Running sums of one node, per slot.
template <typename T, int NS>
struct Sums {
    T W[NS], A[NS][3], R[NS][3], P[NS][3];
    __device__ __forceinline__ void clear() {
#pragma unroll
        for (int k = 0; k < NS; k++) {
            W[k] = T(0);
            for (int d = 0; d < 3; d++) A[k][d] = R[k][d] = P[k][d] = T(0);
        }
    }
};

// Point records of a leaf's Morton range, and the leaf sums over its points in
// node2point (ascending original index) order.
template <typename T, int DIM, int NS>
__device__ __forceinline__ void leaf_pass(const MomParams<T, DIM, NS>& p, int node, const int4& lm,
                                         Sums<T, NS>& S) {
    const int64_t M = p.M;
    const int pstart = lm.y, np = node_npts(lm);
    for (int j = 0; j < np; j++) {
        const int s = pstart + j;
        const int pt = p.perm[s];
        const T pos[3] = {p.spos[3 * s], p.spos[3 * s + 1], p.spos[3 * s + 2]};
        T e[3];
        exps(pos, e);
        T es[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int k = 0; k < NS; k++) {
            T a[3] = {T(0), T(0), T(0)};
#pragma unroll
            for (int c = 0; c < DIM; c++) a[c] = p.attrs[(int64_t)pt * p.astride + k * DIM + c];
            const T w = (NS == 1 && p.weights) ? p.weights[pt] : weight_of(a, DIM);
            if constexpr (NS == 1)
                write_record<T, DIM>(p.rec[k] + (M + s) * CAGR_REC_STRIDE, pos, e, a, w, T(0));
            es[k] = e[k] * a[0];
        }
        if constexpr (NS == 3) {
            st4<T>(p.adjp + (int64_t)s * 8, make4(pos[0], pos[1], pos[2], es[0]));
            st4<T>(p.adjp + (int64_t)s * 8 + 4, make4(es[1], es[2], T(0), T(0)));
        }
    }
    S.clear();
    for (int j = 0; j < np; j++) {
        // the leaf's points in ascending original index (node2point order)
        const int pt = p.lorder ? p.lorder[pstart + j] : p.perm[pstart + j];
        const int s = p.lorder ? p.invperm[pt] : pstart + j;
        const T y[3] = {p.spos[3 * s], p.spos[3 * s + 1], p.spos[3 * s + 2]};
#pragma unroll
        for (int k = 0; k < NS; k++) {
            T a[3] = {T(0), T(0), T(0)};
#pragma unroll
            for (int c = 0; c < DIM; c++) a[c] = p.attrs[(int64_t)pt * p.astride + k * DIM + c];
            const T w = (NS == 1 && p.weights) ? p.weights[pt] : weight_of(a, DIM);
            S.W[k] = add_rn(S.W[k], w);
            for (int c = 0; c < DIM; c++) S.A[k][c] = add_rn(S.A[k][c], a[c]);
            for (int d = 0; d < 3; d++) {
                S.R[k][d] = add_rn(S.R[k][d], mul_rn(y[d], w));
                S.P[k][d] = add_rn(S.P[k][d], y[d]);
            }
        }
    }
}

// Sums over the children of `node` in octant order.  CG: read through L2
// (children written by other threads of the same launch).
template <bool CG, typename T, int DIM, int NS>
__device__ __forceinline__ void children_pass(const MomParams<T, DIM, NS>& p, const int4 c0,
                                              const int4 c1, Sums<T, NS>& S) {
    S.clear();
    const int ch[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
#pragma unroll
    for (int q = 0; q < 8; q++) {
        if (ch[q] < 0) continue;
        if constexpr (NS == 3) {
            // the packed records: centroids (adjn) and sums (adjs) of the three slots
            const T* a = p.adjn + (int64_t)ch[q] * 12;
            const T* sm = p.adjs + (int64_t)ch[q] * 8;
            const Vec4<T> cq[3] = {CG ? ld4_cg(a) : ld4(a), CG ? ld4_cg(a + 4) : ld4(a + 4),
                                   CG ? ld4_cg(a + 8) : ld4(a + 8)};
            const Vec4<T> sw = CG ? ld4_cg(sm) : ld4(sm);
            const Vec4<T> sa = CG ? ld4_cg(sm + 4) : ld4(sm + 4);
            const T wcs[3] = {sw.x, sw.y, sw.z};
            const T acs[3] = {sa.x, sa.y, sa.z};
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const T wc = wcs[k];
                const T rc[3] = {cq[k].x, cq[k].y, cq[k].z};
                S.W[k] = add_rn(S.W[k], wc);
                S.A[k][0] = add_rn(S.A[k][0], acs[k]);
                for (int d = 0; d < 3; d++) {
                    S.R[k][d] = add_rn(S.R[k][d], mul_rn(rc[d], wc));
                    S.P[k][d] = add_rn(S.P[k][d], rc[d]);
                }
            }
            continue;
        }
#pragma unroll
        for (int k = 0; k < NS; k++) {
            const T* r = p.rec[k] + (int64_t)ch[q] * CAGR_REC_STRIDE;
            const Vec4<T> r0 = CG ? ld4_cg(r) : ld4(r);
            const Vec4<T> r1 = CG ? ld4_cg(r + 4) : ld4(r + 4);
            const Vec4<T> r2 = CG ? ld4_cg(r + 8) : ld4(r + 8);
            const T wc = r2.z;
            const T ac[3] = {r1.w, r2.x, r2.y};
            const T rc[3] = {r0.x, r0.y, r0.z};
            S.W[k] = add_rn(S.W[k], wc);
            for (int c = 0; c < DIM; c++) S.A[k][c] = add_rn(S.A[k][c], ac[c]);
            for (int d = 0; d < 3; d++) {
                S.R[k][d] = add_rn(S.R[k][d], mul_rn(rc[d], wc));
                S.P[k][d] = add_rn(S.P[k][d], rc[d]);
            }
        }
    }
}

// Centroid (with the reference's zero-weight fallback) and node record(s).
template <typename T, int DIM, int NS>
__device__ __forceinline__ void finish_node(const MomParams<T, DIM, NS>& p, int node, int depth,
                                            int count, const Sums<T, NS>& S) {
#pragma unroll
    for (int k = 0; k < NS; k++) {
        T c[3], e[3];
        if (S.W[k] > T(0)) {
            const T inv = div_rn(T(1), S.W[k]);
            for (int d = 0; d < 3; d++) c[d] = mul_rn(S.R[k][d], inv);
        } else {
            // (wn_treecode_cuda_kernels.cu:459-460 for leaves, :515-517 for internal
            // nodes, where it divides a sum of child centroids by the point count)
            const T inv = div_rn(T(1), T(count));
            for (int d = 0; d < 3; d++) c[d] = mul_rn(S.P[k][d], inv);
        }
        if constexpr (NS == 1) {
            exps(c, e);
            T r0w = mac_radius2<T>(depth);
            // a one-point leaf whose centroid is its point exactly: the node
            // record equals the point record for every pair term (marked by the
            // sign of the acceptance radius)
            if (count == 1 && c[0] == S.P[k][0] && c[1] == S.P[k][1] && c[2] == S.P[k][2])
                r0w = -r0w;
            write_record<T, DIM>(p.rec[k] + (int64_t)node * CAGR_REC_STRIDE, c, e, S.A[k], S.W[k],
                                 r0w);
        } else {
            // slot k of the adjoint needs exp(-c_k[k]/2) only
            const T ek = exp_t(c[k] * T(-0.5));
            st4<T>(p.adjn + (int64_t)node * 12 + 4 * k, make4(c[0], c[1], c[2], ek * S.A[k][0]));
        }
    }
    if constexpr (NS == 3) {
        st4<T>(p.adjs + (int64_t)node * 8, make4(S.W[0], S.W[1], S.W[2], T(0)));
        st4<T>(p.adjs + (int64_t)node * 8 + 4, make4(S.A[0][0], S.A[1][0], S.A[2][0], T(0)));
    }
}

// Arrival at a parent: add 1 with release (this thread's records are visible to
// whoever arrives later).  Only the last arrival reads its siblings' records,
// so only it orders its later loads after the atomic, with an acquire fence
// (the release sequence of the counter's adds synchronises with it); the
// others skip the acquire (and the L1 invalidation it implies).
__device__ __forceinline__ bool arrive_last(uint32_t* counter, uint32_t need) {
    uint32_t old;
    asm volatile("atom.release.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(counter) : "memory");
    if (old + 1u != need) return false;
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    return true;
}

// Each leaf thread climbs while it is the last child to arrive at the parent.
template <typename T, int DIM, int NS>
__global__ void __launch_bounds__(kClimbBlock) k_moments_climb(const MomParams<T, DIM, NS> p) {
    const int64_t li = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= p.num_leaves) return;
    int node = p.leaf_ids[li];
    const int4 lm = p.meta[node];
    Sums<T, NS> S;
    leaf_pass(p, node, lm, S);
    int count = node_npts(lm), depth = node_depth(lm);
    // the parent's structure (read-only) is loaded while the arrival is in
    // flight; only the children's records wait for it (measured at 1M points:
    // 0.190 -> 0.162 ms for [n,3] moments)
    int par = node == 0 ? 0 : p.parent[node];
    while (true) {
        finish_node(p, node, depth, count, S);
        if (node == 0) return;
        const int4 pm = p.meta[par];
        const uint32_t need = p.nchild[par];
        const int4 c0 = reinterpret_cast<const int4*>(p.children)[2 * (int64_t)par];
        const int4 c1 = reinterpret_cast<const int4*>(p.children)[2 * (int64_t)par + 1];
        if (!arrive_last(&p.counters[par], need)) return;
        p.counters[par] = 0u;
        node = par;
        par = par == 0 ? 0 : p.parent[par];  // the next level's, in flight meanwhile
        count = node_npts(pm);
        depth = node_depth(pm);
        children_pass<true>(p, c0, c1, S);
    }
}

// Slot k of the packed adjoint records in the reference layout.
template <typename T>
__global__ void k_export_adj(const T* __restrict__ adjn, const T* __restrict__ adjs, int64_t M,
                             int k, T* __restrict__ node_attrs, T* __restrict__ reppoints,
                             T* __restrict__ weights) {
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M) return;
    if (node_attrs) node_attrs[n] = adjs[n * 8 + 4 + k];
    if (reppoints)
        for (int d = 0; d < 3; d++) reppoints[n * 3 + d] = adjn[n * 12 + 4 * k + d];
    if (weights) weights[n] = adjs[n * 8 + k];
}

template <typename T, int DIM>
__global__ void k_export_moments(const T* __restrict__ rec, int64_t M, T* __restrict__ node_attrs,
                                 T* __restrict__ reppoints, T* __restrict__ weights) {
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M) return;
    const T* r = rec + n * CAGR_REC_STRIDE;
    const T a[3] = {r[7], r[8], r[9]};
    if (node_attrs)
        for (int c = 0; c < DIM; c++) node_attrs[n * DIM + c] = a[c];
    if (reppoints)
        for (int d = 0; d < 3; d++) reppoints[n * 3 + d] = r[d];
    if (weights) weights[n] = r[10];
}

int ensure_slot(Tree* t, int slot, size_t elem, cudaStream_t s) {
    if (t->rec[slot]) return kOk;
    return pool_alloc(&t->rec[slot], elem * (size_t)(t->m + t->n) * CAGR_REC_STRIDE, s);
}

template <typename T, int DIM, int NS>
int run(Tree* t, MomParams<T, DIM, NS> p, cudaStream_t s) {
    p.num_leaves = t->num_leaves;
    p.M = t->m;
    p.leaf_ids = t->leaf_ids;
    p.meta = t->meta;
    p.nchild = t->nchild;
    p.parent = t->parent;
    p.children = t->children;
    p.perm = t->perm;
    p.invperm = t->invperm;
    p.lorder = t->lorder;
    p.spos = (const T*)t->spos;
    p.counters = t->counters;
    const unsigned grid = (unsigned)((t->num_leaves + kClimbBlock - 1) / kClimbBlock);
    k_moments_climb<T, DIM, NS><<<grid, kClimbBlock, 0, s>>>(p);
    CAGR_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int launch_moments(Tree* t, int slot, const void* attrs, int dim, const void* weights,
                   cudaStream_t s) {
    if (int rc = ensure_slot(t, slot, sizeof(T), s)) return rc;
    int rc;
    if (dim == 3) {
        MomParams<T, 3, 1> p;
        p.attrs = (const T*)attrs;
        p.astride = 3;
        p.weights = (const T*)weights;
        p.rec[0] = (T*)t->rec[slot];
        rc = run(t, p, s);
    } else {
        MomParams<T, 1, 1> p;
        p.attrs = (const T*)attrs;
        p.astride = 1;
        p.weights = (const T*)weights;
        p.rec[0] = (T*)t->rec[slot];
        rc = run(t, p, s);
    }
    if (rc) return rc;
    t->rec_dim[slot] = dim;
    return kOk;
}

// Three scalar attributes into the packed adjoint records only (the record
// slots are not written: the three-slot traversal reads the packed layout,
// and export reads centroids and sums from it).  The record slots keep what
// the last cagr_scatter into each put there.
template <typename T>
int launch_moments3(Tree* t, const void* values3, cudaStream_t s) {
    if (!t->adj_nodes)
        if (int rc = pool_alloc(&t->adj_nodes, sizeof(T) * 12 * (size_t)t->m, s)) return rc;
    if (!t->adj_points)
        if (int rc = pool_alloc(&t->adj_points, sizeof(T) * 8 * (size_t)t->n, s)) return rc;
    if (!t->adj_sums)
        if (int rc = pool_alloc(&t->adj_sums, sizeof(T) * 8 * (size_t)t->m, s)) return rc;
    MomParams<T, 1, 3> p;
    p.attrs = (const T*)values3;
    p.astride = 3;
    for (int k = 0; k < 3; k++) p.rec[k] = nullptr;
    p.adjn = (T*)t->adj_nodes;
    p.adjp = (T*)t->adj_points;
    p.adjs = (T*)t->adj_sums;
    if (int rc = run(t, p, s)) return rc;
    for (int k = 0; k < 3; k++) {
        t->slot_adj[k] = true;
    }
    t->adj_valid = true;
    return kOk;
}


// Records of slot from moments given in the reference layout -- node_attrs
// [M, DIM] and reppoints [M, 3] as scatter_point_attrs_to_nodes returns them,
// and the point attributes [N, DIM] -- exactly as the moment pass writes them
// from the same values (node weights are not carried: no traversal reads them).
template <typename T, int DIM>
__global__ void k_import(const int4* __restrict__ meta, const T* __restrict__ spos,
                         const int32_t* __restrict__ perm, int64_t M, int64_t N,
                         const T* __restrict__ node_attrs, const T* __restrict__ rep,
                         const T* __restrict__ attrs, T* __restrict__ rec) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M) {
        const int4 mt = meta[i];
        const T c[3] = {rep[3 * i], rep[3 * i + 1], rep[3 * i + 2]};
        T e[3], a[3] = {T(0), T(0), T(0)};
        exps(c, e);
        for (int d = 0; d < DIM; d++) a[d] = node_attrs[i * DIM + d];
        T r0w = mac_radius2<T>(node_depth(mt));
        if (node_npts(mt) == 1) {
            const int64_t s = mt.y;
            if (c[0] == spos[3 * s] && c[1] == spos[3 * s + 1] && c[2] == spos[3 * s + 2])
                r0w = -r0w;
        }
        write_record<T, DIM>(rec + i * CAGR_REC_STRIDE, c, e, a, T(0), r0w);
    } else if (i < M + N) {
        const int64_t s = i - M;
        const int64_t pt = perm[s];
        const T pos[3] = {spos[3 * s], spos[3 * s + 1], spos[3 * s + 2]};
        T e[3], a[3] = {T(0), T(0), T(0)};
        exps(pos, e);
        for (int d = 0; d < DIM; d++) a[d] = attrs[pt * DIM + d];
        write_record<T, DIM>(rec + i * CAGR_REC_STRIDE, pos, e, a, weight_of(a, DIM), T(0));
    }
}

template <typename T>
int launch_import(Tree* t, int slot, const void* node_attrs, const void* rep, const void* attrs,
                  int dim, cudaStream_t s) {
    if (int rc = ensure_slot(t, slot, sizeof(T), s)) return rc;
    const int64_t total = t->m + t->n;
    const unsigned grid = (unsigned)((total + kBlock - 1) / kBlock);
    if (dim == 3)
        k_import<T, 3><<<grid, kBlock, 0, s>>>(t->meta, (const T*)t->spos, t->perm, t->m, t->n,
                                               (const T*)node_attrs, (const T*)rep,
                                               (const T*)attrs, (T*)t->rec[slot]);
    else
        k_import<T, 1><<<grid, kBlock, 0, s>>>(t->meta, (const T*)t->spos, t->perm, t->m, t->n,
                                               (const T*)node_attrs, (const T*)rep,
                                               (const T*)attrs, (T*)t->rec[slot]);
    CAGR_CUDA(cudaGetLastError());
    t->rec_dim[slot] = dim;
    t->slot_adj[slot] = false;
    return kOk;
}
}  // namespace

int moments_import(Tree* t, int slot, const void* node_attrs, const void* reppoints,
                   const void* attrs, int dim, cudaStream_t stream) {
    if (slot < 0 || slot > 2) return set_error(kErrInvalid, "moment slot must be 0, 1 or 2");
    if (dim != 1 && dim != 3) return set_error(kErrInvalid, "attribute dim must be 1 or 3");
    if (!node_attrs || !reppoints || !attrs) return set_error(kErrInvalid, "null buffer");
    return t->dtype == 0 ? launch_import<float>(t, slot, node_attrs, reppoints, attrs, dim, stream)
                         : launch_import<double>(t, slot, node_attrs, reppoints, attrs, dim, stream);
}

int moments(Tree* t, int slot, const void* attrs, int dim, const void* weights,
            cudaStream_t stream) {
    if (slot < 0 || slot > 2) return set_error(kErrInvalid, "moment slot must be 0, 1 or 2");
    if (dim != 1 && dim != 3) return set_error(kErrInvalid, "attribute dim must be 1 or 3");
    if (!attrs) return set_error(kErrInvalid, "attrs is null");
    t->slot_adj[slot] = false;  // export of this slot reads the record slot again
    return t->dtype == 0 ? launch_moments<float>(t, slot, attrs, dim, weights, stream)
                         : launch_moments<double>(t, slot, attrs, dim, weights, stream);
}

int moments3(Tree* t, const void* values3, cudaStream_t stream) {
    if (!values3) return set_error(kErrInvalid, "values is null");
    return t->dtype == 0 ? launch_moments3<float>(t, values3, stream)
                         : launch_moments3<double>(t, values3, stream);
}

int moments_export(const Tree* t, int slot, void* node_attrs, void* reppoints, void* weights,
                   cudaStream_t stream) {
    if (slot < 0 || slot > 2) return set_error(kErrInvalid, "moment slot must be 0, 1 or 2");
    const unsigned grid = (unsigned)((t->m + kBlock - 1) / kBlock);
    if (t->slot_adj[slot] && t->adj_valid) {
        if (t->dtype == 0)
            k_export_adj<float><<<grid, kBlock, 0, stream>>>(
                (const float*)t->adj_nodes, (const float*)t->adj_sums, t->m, slot,
                (float*)node_attrs, (float*)reppoints, (float*)weights);
        else
            k_export_adj<double><<<grid, kBlock, 0, stream>>>(
                (const double*)t->adj_nodes, (const double*)t->adj_sums, t->m, slot,
                (double*)node_attrs, (double*)reppoints, (double*)weights);
        CAGR_CUDA(cudaGetLastError());
        return kOk;
    }
    if (!t->rec[slot] || t->rec_dim[slot] == 0)
        return set_error(kErrState, "no moments computed in this slot");
    const int dim = t->rec_dim[slot];
    if (t->dtype == 0) {
        if (dim == 3)
            k_export_moments<float, 3><<<grid, kBlock, 0, stream>>>(
                (const float*)t->rec[slot], t->m, (float*)node_attrs, (float*)reppoints,
                (float*)weights);
        else
            k_export_moments<float, 1><<<grid, kBlock, 0, stream>>>(
                (const float*)t->rec[slot], t->m, (float*)node_attrs, (float*)reppoints,
                (float*)weights);
    } else {
        if (dim == 3)
            k_export_moments<double, 3><<<grid, kBlock, 0, stream>>>(
                (const double*)t->rec[slot], t->m, (double*)node_attrs, (double*)reppoints,
                (double*)weights);
        else
            k_export_moments<double, 1><<<grid, kBlock, 0, stream>>>(
                (const double*)t->rec[slot], t->m, (double*)node_attrs, (double*)reppoints,
                (double*)weights);
    }
    CAGR_CUDA(cudaGetLastError());
    return kOk;
}

}  // namespace cagr
