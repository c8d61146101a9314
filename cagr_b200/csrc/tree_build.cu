// Device octree build, bit-exact with the reference serialised layout.
//
// Reference semantics (mayueji/CAGR, CUDA-based/ext/wn_treecode/wn_treecode_cpu/
// wn_treecode_cpu_treeutils.cpp:90-177 and :202-258): recursive split of
// [-1,1]^3 around dyadic centres with octant code (x>=cx) + 2(y>=cy) + 4(z>=cz),
// leaf when depth == max_depth or the node holds <= leaf_size points, nodes
// numbered in preorder (octants in order), and every node's point list (ascending
// original index) concatenated in preorder.
//
// B200 formulation (no recursion, O(N log N) parallel work):
//  1. Per-axis integer keys floor(x * 2^(D-1)) + 2^(D-1) (exact: a power-of-two
//     scale, a floor and an integer add; D = max_depth), bit-interleaved into a
//     3D-bit Morton code whose j-th 3-bit digit is the reference octant code at
//     depth j.  Bit b of the key is set exactly when x >= the depth-(D-1-b)
//     centre the reference compares against.
//  2. Stable radix sort of (code, index): equal codes keep ascending index.
//  3. lcp[i] = number of equal leading digits of codes i-1 and i.  Position i
//     opens cells at depths lcp[i]+1..D.  The cell at depth d starting at i is a
//     node iff its parent cell holds > leaf_size points, and it is internal iff
//     it holds > leaf_size points and d < D; the nodes starting at position i
//     therefore form one chain of depths d0..dlast.
//  4. Preorder id of node (d, i) = (nodes at positions < i) + (d - d0): sorting
//     nodes by (first point, depth) is preorder.  Subtree ends and parents come
//     from a sparse-table search over lcp.
//  5. Per-node point lists (needed only by the reference-layout export, so
//     built on its first call): (node, index) pairs, a point's leaf and its
//     ancestors, emitted in index order, then a stable radix sort by node id.
//     The moments only need each leaf's own points in index order.
#include <cub/cub.cuh>

#include <algorithm>
#include <string>
#include <vector>

#include "internal.h"

namespace cagr {
namespace {

constexpr int kBlock = 256;

inline unsigned grid_for(int64_t n, int block = kBlock) {
    return (unsigned)((n + block - 1) / block);
}

// Stream-ordered temporary buffer from the library's pool.
struct Tmp {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~Tmp() { pool_free(p, s); }
};

int tmp_alloc(Tmp& t, size_t bytes, cudaStream_t s) {
    t.s = s;
    return pool_alloc(&t.p, bytes, s);
}

// A tree array: from the pool, ordered on the build stream, freed by tree_free.
int dev_alloc(void** p, size_t bytes, cudaStream_t s) { return pool_alloc(p, bytes, s); }

// ---- step 1: Morton codes -------------------------------------------------

template <typename T>
__device__ __forceinline__ uint32_t axis_key(T v, int D) {
    if (D == 0 || v != v) return 0u;  // NaN fails every `>=`: all-zero key
    const T half = ldexp(T(1), D - 1);
    const T s = floor(v * half);  // power-of-two scale: exact
    if (s < -half) return 0u;
    if (s >= half) return (1u << D) - 1u;
    return (uint32_t)((int64_t)s + (int64_t)half);
}

__device__ __forceinline__ uint64_t spread3(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x1f00000000ffffull;
    x = (x | (x << 16)) & 0x1f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

template <typename T>
__global__ void k_morton(const T* __restrict__ pts, int64_t n, int D, uint64_t* __restrict__ keys,
                         int32_t* __restrict__ idx) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t kx = axis_key(pts[3 * i + 0], D);
    uint32_t ky = axis_key(pts[3 * i + 1], D);
    uint32_t kz = axis_key(pts[3 * i + 2], D);
    keys[i] = spread3(kx) | (spread3(ky) << 1) | (spread3(kz) << 2);
    idx[i] = (int32_t)i;
}

// ---- warp grouping of the self-queries ---------------------------------------
//
// The traversals walk the tree one warp per 32 consecutive queries, visiting
// the union of the nodes their queries open.  Every query's pair terms and
// their order are its own (preorder of the nodes it accepts), whoever shares
// its warp, so the grouping changes no output bit -- only how many nodes a
// warp visits.  Groups of 32 consecutive points along a 3-D Hilbert curve are
// more compact than along the Morton curve (no jumps between distant cells):
// 3.2 % fewer warp visits on the 1M-point union-of-primitives cloud.
// Hilbert index: J. Skilling, "Programming the Hilbert curve", AIP Conf. Proc.
// 707 (2004) -- axes to transposed index by inverse undo of the excess work,
// Gray decode, then the three axes' bits interleaved from the top.  10 bits
// per axis group as well as 21 (a host simulation of the warp walk counts the
// same visits) and keep the key in 32 bits: half the radix-sort passes.
// Points in one cell keep their Morton order (stable sort).
constexpr int kHilbertBits = 10;

template <typename T>
__global__ void k_hilbert(const T* __restrict__ spos, int64_t n, uint32_t* __restrict__ keys,
                          int32_t* __restrict__ idx) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t X[3];
#pragma unroll
    for (int a = 0; a < 3; a++) X[a] = axis_key(spos[3 * i + a], kHilbertBits);
    const uint32_t top = 1u << (kHilbertBits - 1);
    for (uint32_t Q = top; Q > 1; Q >>= 1) {
        const uint32_t P = Q - 1;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            if (X[a] & Q) {
                X[0] ^= P;
            } else {
                const uint32_t t = (X[0] ^ X[a]) & P;
                X[0] ^= t;
                X[a] ^= t;
            }
        }
    }
    X[1] ^= X[0];
    X[2] ^= X[1];
    uint32_t t = 0;
    for (uint32_t Q = top; Q > 1; Q >>= 1)
        if (X[2] & Q) t ^= Q - 1;
    X[0] ^= t;
    X[1] ^= t;
    X[2] ^= t;
    keys[i] = (uint32_t)(spread3(X[2]) | (spread3(X[1]) << 1) | (spread3(X[0]) << 2));
    idx[i] = (int32_t)i;
}

__device__ __forceinline__ int digit_at(uint64_t code, int D, int d) {
    // octant chosen by the split of a depth-d node (child at depth d+1)
    return (int)((code >> (3 * (D - 1 - d))) & 7u);
}

// ---- step 3: lcp and node chains --------------------------------------------

__global__ void k_lcp(const uint64_t* __restrict__ sk, int64_t n, int D, int8_t* __restrict__ lcp) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i == 0) {
        lcp[0] = -1;
        return;
    }
    uint64_t x = sk[i - 1] ^ sk[i];
    lcp[i] = (x == 0) ? (int8_t)D : (int8_t)((__clzll((long long)x) - (64 - 3 * D)) / 3);
}

__global__ void k_chain(const int8_t* __restrict__ lcp, int64_t n, int D, int s,
                        int32_t* __restrict__ nn, int8_t* __restrict__ d0a,
                        int8_t* __restrict__ dla, int32_t* __restrict__ isleafpos) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int d0 = (i == 0) ? 0 : lcp[i] + 1;
    bool exists;
    if (i == 0) {
        exists = true;
    } else if (d0 > D) {
        exists = false;  // same code as the previous point: shares its leaf
    } else {
        // the parent cell (depth L = lcp[i]) must hold more than s points
        const int L = lcp[i];
        int64_t total = 1, a = i, b = i + 1;
        while (total <= s && a > 0 && lcp[a] >= L) {
            a--;
            total++;
        }
        while (total <= s && b < n && lcp[b] >= L) {
            b++;
            total++;
        }
        exists = total > s;
    }
    int m = -1;  // min lcp over (i, i+s]: the deepest depth whose cell at i holds > s points
    if (i + s < n) {
        m = CAGR_MAX_DEPTH + 1;
        for (int j = 1; j <= s; j++) m = min(m, (int)lcp[i + j]);
    }
    int dlast = (d0 < D && m >= d0) ? min(m + 1, D) : d0;
    nn[i] = exists ? (dlast - d0 + 1) : 0;
    d0a[i] = (int8_t)d0;
    dla[i] = exists ? (int8_t)dlast : (int8_t)0;  // no node here: keep out of the depth max
    isleafpos[i] = exists ? 1 : 0;
}

// sparse table: st[k][j] = min(lcp[j .. min(j + 2^k, n) - 1]).  One launch
// writes levels k0 .. k0 + m - 1 (m <= kLevelsPerLaunch) from level k0 - 1:
// level k0 - 1 + i at j is the min of prev[j + t h] over t < 2^i (h = 2^(k0-1),
// positions past n skipped), the union of those windows being [j, j + 2^i h).
// The strided reads of neighbouring threads are coalesced and come from L2.
// (measured at 1M points, ncu launch durations: 19 launches of one level
// 122 us, 10 of two levels 107 us, 5 of four levels 94 us)
constexpr int kLevelsPerLaunch = 4;

__global__ void k_sparse_levels(const int8_t* __restrict__ prev, int8_t* __restrict__ out,
                                int64_t n, int64_t h, int m) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int cur = prev[j];
    int t = 1;
    for (int i = 1; i <= m; i++) {
        for (; t < (1 << i); t++) {
            const int64_t x = j + (int64_t)t * h;
            if (x < n) cur = min(cur, (int)prev[x]);
        }
        out[(int64_t)(i - 1) * n + j] = (int8_t)cur;
    }
}

// first j > i with lcp[j] < d, or n
__device__ __forceinline__ int64_t fwd_search(const int8_t* __restrict__ st, int K, int64_t n,
                                              int64_t i, int d) {
    int64_t pos = i + 1;
    for (int k = K - 1; k >= 0; k--) {
        int64_t len = 1LL << k;
        if (pos + len <= n && st[(int64_t)k * n + pos] >= d) pos += len;
    }
    return pos;
}

// largest j < i with lcp[j] < t (exists because lcp[0] = -1 and t >= 0)
__device__ __forceinline__ int64_t bwd_search(const int8_t* __restrict__ st, int K, int64_t n,
                                              int64_t i, int t) {
    int64_t pos = i - 1;
    for (int k = K - 1; k >= 0; k--) {
        int64_t len = 1LL << k;
        if (pos - len + 1 >= 0 && st[(int64_t)k * n + (pos - len + 1)] >= t) pos -= len;
    }
    return pos;
}

__global__ void k_emit(const uint64_t* __restrict__ sk, const int8_t* __restrict__ st, int K,
                       int64_t n, int D, int64_t M, const int32_t* __restrict__ nn,
                       const int32_t* __restrict__ base, const int8_t* __restrict__ d0a,
                       const int8_t* __restrict__ dla, int4* __restrict__ meta,
                       int32_t* __restrict__ parent, int32_t* __restrict__ children,
                       int32_t* __restrict__ nchild, int64_t* __restrict__ npts64) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || nn[i] == 0) return;
    const int d0 = d0a[i], dlast = dla[i];
    const int64_t b = base[i];
    for (int d = d0; d <= dlast; d++) {
        const int64_t id = b + (d - d0);
        const int64_t end = fwd_search(st, K, n, i, d);
        const int64_t next = (end < n) ? (int64_t)base[end] : M;
        int64_t par;
        if (d == 0) {
            par = -1;
        } else if (d > d0) {
            par = id - 1;
        } else {
            const int64_t p = bwd_search(st, K, n, i, d - 1);
            par = (int64_t)base[p] + (d - 1 - d0a[p]);
        }
        const bool leaf = (d == dlast);
        const int cnt = (int)(end - i);
        meta[id] = make_int4((int)next, (int)i, leaf ? -cnt : cnt, d);
        parent[id] = (int32_t)par;
        npts64[id] = end - i;
        if (par >= 0) {
            children[par * 8 + digit_at(sk[i], D, d - 1)] = (int32_t)id;
            atomicAdd(&nchild[par], 1);
        }
    }
}

// child counts as bytes; marks twigs (internal nodes with as many children as
// points: every child is a one-point leaf) in bit 8 of meta.w
__global__ void k_pack(uint8_t* __restrict__ out, const int32_t* __restrict__ nchild,
                       int4* __restrict__ meta, int64_t M) {
    int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= M) return;
    const int c = nchild[id];
    out[id] = (uint8_t)c;
    const int z = meta[id].z;
    if (z > 0 && z == c) meta[id].w |= 1 << 8;
}

__global__ void k_leaf_ids(const int32_t* __restrict__ nn, const int32_t* __restrict__ base,
                           const int8_t* __restrict__ d0a, const int8_t* __restrict__ dla,
                           const int32_t* __restrict__ leafrank, int64_t n,
                           int32_t* __restrict__ leaf_ids) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || nn[i] == 0) return;
    leaf_ids[leafrank[i]] = base[i] + (dla[i] - d0a[i]);
}

__global__ void k_inv(const int32_t* __restrict__ perm, int64_t n, int32_t* __restrict__ inv) {
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    inv[perm[s]] = (int32_t)s;
}

template <typename T>
__global__ void k_spos(const T* __restrict__ pts, const int32_t* __restrict__ perm, int64_t n,
                       T* __restrict__ spos) {
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int64_t p = perm[s];
    spos[3 * s + 0] = pts[3 * p + 0];
    spos[3 * s + 1] = pts[3 * p + 1];
    spos[3 * s + 2] = pts[3 * p + 2];
}

// ---- the per-node point lists (node2point_index), built on first export ----
// Every point belongs to its leaf and the leaf's ancestors: per point (original
// index p) its leaf's depth + 1 pairs (node, p), root first; a stable sort of
// all pairs by node id then lists each node's points in ascending p.

// leaf node of every sorted position
__global__ void k_leaf_of_pos(const int32_t* __restrict__ leaf_ids, int64_t num_leaves,
                              const int4* __restrict__ meta, int32_t* __restrict__ leaf_of) {
    const int64_t li = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= num_leaves) return;
    const int leaf = leaf_ids[li];
    const int4 m = meta[leaf];
    for (int j = 0; j < node_npts(m); j++) leaf_of[(int64_t)m.y + j] = leaf;
}

template <bool WRITE>
__global__ void k_pairs(const int32_t* __restrict__ invperm, const int32_t* __restrict__ leaf_of,
                        const int4* __restrict__ meta, const int32_t* __restrict__ parent,
                        int64_t n, int32_t* __restrict__ cnt, const int64_t* __restrict__ off,
                        int32_t* __restrict__ pair_node, int32_t* __restrict__ pair_pt) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int node = leaf_of[invperm[p]];
    const int d = node_depth(meta[node]);
    if (!WRITE) {
        cnt[p] = d + 1;
        return;
    }
    const int64_t k = off[p];
    for (int i = d; i >= 0 && node >= 0; i--) {  // the leaf at k + d, the root at k
        pair_node[k + i] = node;
        pair_pt[k + i] = (int32_t)p;
        node = parent[node];
    }
}

// Leaves of more than one point list them in ascending original index (the
// reference's node2point order).  Morton-sorted positions already are in that
// order where all the leaf's points share their code (the stable sort keeps
// index order): every leaf of a leaf-size-1 tree, and any leaf of more than
// leaf_size points (a cell at the maximum depth).  The other leaves of a tree
// with larger leaves (at most leaf_size points) are sorted here.
__global__ void k_leaf_order(const int32_t* __restrict__ leaf_ids, int64_t num_leaves,
                             const int4* __restrict__ meta, const int32_t* __restrict__ perm,
                             int leaf_size, int32_t* __restrict__ order) {
    const int64_t li = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= num_leaves) return;
    const int4 m = meta[leaf_ids[li]];
    const int np = node_npts(m);
    int32_t* o = order + m.y;
    const bool sort = np <= leaf_size;
    for (int j = 0; j < np; j++) {  // insertion sort of perm[m.y .. m.y + np), or a copy
        const int32_t v = perm[(int64_t)m.y + j];
        int i = j;
        while (sort && i > 0 && o[i - 1] > v) {
            o[i] = o[i - 1];
            i--;
        }
        o[i] = v;
    }
}

__global__ void k_fill_i32(int32_t* a, int64_t n, int32_t v) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

template <typename T>
__global__ void k_export(const int4* __restrict__ meta, const int32_t* __restrict__ parent,
                         const int32_t* __restrict__ children, const int64_t* __restrict__ n2ps,
                         int64_t M, int64_t* __restrict__ o_parent, int64_t* __restrict__ o_children,
                         uint8_t* __restrict__ o_leaf, T* __restrict__ o_half_w,
                         int64_t* __restrict__ o_npts, int64_t* __restrict__ o_n2ps) {
    int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= M) return;
    const int4 mt = meta[id];
    if (o_parent) o_parent[id] = parent[id];
    if (o_children)
        for (int k = 0; k < 8; k++) o_children[id * 8 + k] = children[id * 8 + k];
    if (o_leaf) o_leaf[id] = node_leaf(mt) ? 1 : 0;
    if (o_half_w) o_half_w[id] = ldexp(T(1), -node_depth(mt));
    if (o_npts) o_npts[id] = node_npts(mt);
    if (o_n2ps) o_n2ps[id] = n2ps[id];
}

__global__ void k_widen(const int32_t* __restrict__ a, int64_t n, int64_t* __restrict__ b) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

// cub helpers -------------------------------------------------------------------

template <typename F>
int cub_call(F&& f, cudaStream_t s) {
    size_t bytes = 0;
    CAGR_CUDA(f(nullptr, bytes));
    Tmp tmp;
    if (int rc = tmp_alloc(tmp, bytes, s)) return rc;
    CAGR_CUDA(f(tmp.p, bytes));
    return kOk;
}

int bit_width(int64_t v) {
    int b = 0;
    while ((int64_t(1) << b) <= v && b < 62) b++;
    return b;
}

template <typename T>
int build_impl(const T* pts, int64_t n, int D, int s, cudaStream_t st, Tree* t) {
    const unsigned gN = grid_for(n);
    // 1-2: codes and stable sort
    Tmp keys, keys2, idx, sorted_keys;
    if (int rc = tmp_alloc(keys, sizeof(uint64_t) * n, st)) return rc;
    if (int rc = tmp_alloc(sorted_keys, sizeof(uint64_t) * n, st)) return rc;
    if (int rc = tmp_alloc(idx, sizeof(int32_t) * n, st)) return rc;
    if (int rc = dev_alloc((void**)&t->perm, sizeof(int32_t) * n, st)) return rc;
    k_morton<T><<<gN, kBlock, 0, st>>>(pts, n, D, (uint64_t*)keys.p, (int32_t*)idx.p);
    CAGR_CUDA(cudaGetLastError());
    const int end_bit = 3 * D;
    if (end_bit > 0) {
        if (int rc = cub_call(
                [&](void* tp, size_t& b) {
                    return cub::DeviceRadixSort::SortPairs(tp, b, (const uint64_t*)keys.p,
                                                           (uint64_t*)sorted_keys.p,
                                                           (const int32_t*)idx.p, t->perm, n, 0,
                                                           end_bit, st);
                },
                st))
            return rc;
    } else {
        CAGR_CUDA(cudaMemcpyAsync(sorted_keys.p, keys.p, sizeof(uint64_t) * n,
                                  cudaMemcpyDeviceToDevice, st));
        CAGR_CUDA(cudaMemcpyAsync(t->perm, idx.p, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice,
                                  st));
    }
    const uint64_t* sk = (const uint64_t*)sorted_keys.p;

    // 3: lcp, chains, sparse table
    int K = 1;
    while ((int64_t(1) << K) < n) K++;
    Tmp stab, nn, d0a, dla, isleafpos, base, leafrank;
    if (int rc = tmp_alloc(stab, (size_t)K * n, st)) return rc;
    if (int rc = tmp_alloc(nn, sizeof(int32_t) * n, st)) return rc;
    if (int rc = tmp_alloc(d0a, n, st)) return rc;
    if (int rc = tmp_alloc(dla, n, st)) return rc;
    if (int rc = tmp_alloc(isleafpos, sizeof(int32_t) * n, st)) return rc;
    if (int rc = tmp_alloc(base, sizeof(int32_t) * (n + 1), st)) return rc;
    if (int rc = tmp_alloc(leafrank, sizeof(int32_t) * (n + 1), st)) return rc;
    int8_t* lcp = (int8_t*)stab.p;
    k_lcp<<<gN, kBlock, 0, st>>>(sk, n, D, lcp);
    k_chain<<<gN, kBlock, 0, st>>>(lcp, n, D, s, (int32_t*)nn.p, (int8_t*)d0a.p, (int8_t*)dla.p,
                                   (int32_t*)isleafpos.p);
    for (int k0 = 1; k0 < K; k0 += kLevelsPerLaunch)
        k_sparse_levels<<<gN, kBlock, 0, st>>>(lcp + (int64_t)(k0 - 1) * n, lcp + (int64_t)k0 * n,
                                               n, int64_t(1) << (k0 - 1),
                                               std::min(kLevelsPerLaunch, K - k0));
    CAGR_CUDA(cudaGetLastError());
    if (int rc = cub_call(
            [&](void* tp, size_t& b) {
                return cub::DeviceScan::ExclusiveSum(tp, b, (const int32_t*)nn.p,
                                                     (int32_t*)base.p, n + 0, st);
            },
            st))
        return rc;
    if (int rc = cub_call(
            [&](void* tp, size_t& b) {
                return cub::DeviceScan::ExclusiveSum(tp, b, (const int32_t*)isleafpos.p,
                                                     (int32_t*)leafrank.p, n + 0, st);
            },
            st))
        return rc;
    int32_t last_base = 0, last_nn = 0, last_rank = 0, last_leaf = 0;
    CAGR_CUDA(cudaMemcpyAsync(&last_base, (int32_t*)base.p + (n - 1), 4, cudaMemcpyDeviceToHost, st));
    CAGR_CUDA(cudaMemcpyAsync(&last_nn, (int32_t*)nn.p + (n - 1), 4, cudaMemcpyDeviceToHost, st));
    CAGR_CUDA(cudaMemcpyAsync(&last_rank, (int32_t*)leafrank.p + (n - 1), 4,
                              cudaMemcpyDeviceToHost, st));
    CAGR_CUDA(cudaMemcpyAsync(&last_leaf, (int32_t*)isleafpos.p + (n - 1), 4,
                              cudaMemcpyDeviceToHost, st));
    CAGR_CUDA(cudaStreamSynchronize(st));
    const int64_t M = (int64_t)last_base + last_nn;
    const int64_t NL = (int64_t)last_rank + last_leaf;
    if (M <= 0 || M >= (int64_t(1) << 31) - 2)
        return set_error(kErrOverflow, "node count out of range: " + std::to_string(M));
    t->m = M;
    t->num_leaves = NL;

    // 4: nodes
    if (int rc = dev_alloc((void**)&t->meta, sizeof(int4) * M, st)) return rc;
    if (int rc = dev_alloc((void**)&t->nchild, M, st)) return rc;
    if (int rc = dev_alloc((void**)&t->parent, sizeof(int32_t) * M, st)) return rc;
    if (int rc = dev_alloc((void**)&t->children, sizeof(int32_t) * M * 8, st)) return rc;
    if (int rc = dev_alloc((void**)&t->leaf_ids, sizeof(int32_t) * NL, st)) return rc;
    if (int rc = dev_alloc((void**)&t->n2p_start, sizeof(int64_t) * (M + 1), st)) return rc;
    if (int rc = dev_alloc((void**)&t->counters, sizeof(uint32_t) * M, st)) return rc;
    CAGR_CUDA(cudaMemsetAsync(t->counters, 0, sizeof(uint32_t) * M, st));
    Tmp nchild, npts64;
    if (int rc = tmp_alloc(nchild, sizeof(int32_t) * M, st)) return rc;
    if (int rc = tmp_alloc(npts64, sizeof(int64_t) * (M + 1), st)) return rc;
    CAGR_CUDA(cudaMemsetAsync(nchild.p, 0, sizeof(int32_t) * M, st));
    k_fill_i32<<<grid_for(M * 8), kBlock, 0, st>>>(t->children, M * 8, -1);
    k_emit<<<gN, kBlock, 0, st>>>(sk, lcp, K, n, D, M, (const int32_t*)nn.p,
                                  (const int32_t*)base.p, (const int8_t*)d0a.p,
                                  (const int8_t*)dla.p, t->meta, t->parent, t->children,
                                  (int32_t*)nchild.p, (int64_t*)npts64.p);
    k_pack<<<grid_for(M), kBlock, 0, st>>>(t->nchild, (const int32_t*)nchild.p, t->meta, M);
    k_leaf_ids<<<gN, kBlock, 0, st>>>((const int32_t*)nn.p, (const int32_t*)base.p,
                                      (const int8_t*)d0a.p, (const int8_t*)dla.p,
                                      (const int32_t*)leafrank.p, n, t->leaf_ids);
    CAGR_CUDA(cudaGetLastError());

    // per-node point lists
    CAGR_CUDA(cudaMemsetAsync((int64_t*)npts64.p + M, 0, sizeof(int64_t), st));
    if (int rc = cub_call(
            [&](void* tp, size_t& b) {
                return cub::DeviceScan::ExclusiveSum(tp, b, (const int64_t*)npts64.p, t->n2p_start,
                                                     M + 1, st);
            },
            st))
        return rc;
    int64_t L = 0;
    CAGR_CUDA(cudaMemcpyAsync(&L, t->n2p_start + M, 8, cudaMemcpyDeviceToHost, st));
    if (int rc = dev_alloc((void**)&t->invperm, sizeof(int32_t) * n, st)) return rc;
    k_inv<<<gN, kBlock, 0, st>>>(t->perm, n, t->invperm);
    if (s > 1) {  // leaves of several codes: their points in original-index order
        if (int rc = dev_alloc((void**)&t->lorder, sizeof(int32_t) * n, st)) return rc;
        k_leaf_order<<<grid_for(NL), kBlock, 0, st>>>(t->leaf_ids, NL, t->meta, t->perm, s,
                                                      t->lorder);
    }
    CAGR_CUDA(cudaGetLastError());
    CAGR_CUDA(cudaStreamSynchronize(st));
    if (L <= 0 || L >= (int64_t(1) << 31) - 2)
        return set_error(kErrOverflow, "point-list length out of range: " + std::to_string(L));
    t->n2p_len = L;  // the lists themselves are built by the first export (ensure_n2p)

    // sorted positions
    if (int rc = dev_alloc(&t->spos, sizeof(T) * 3 * n, st)) return rc;
    k_spos<T><<<gN, kBlock, 0, st>>>(pts, t->perm, n, (T*)t->spos);
    CAGR_CUDA(cudaGetLastError());

    // warp grouping of the self-queries (the Morton key buffers are free again)
    if (int rc = dev_alloc((void**)&t->qgroup, sizeof(int32_t) * n, st)) return rc;
    k_hilbert<T><<<gN, kBlock, 0, st>>>((const T*)t->spos, n, (uint32_t*)keys.p, (int32_t*)idx.p);
    CAGR_CUDA(cudaGetLastError());
    if (int rc = cub_call(
            [&](void* tp, size_t& b) {
                return cub::DeviceRadixSort::SortPairs(tp, b, (const uint32_t*)keys.p,
                                                       (uint32_t*)sorted_keys.p,
                                                       (const int32_t*)idx.p, t->qgroup, n, 0,
                                                       3 * kHilbertBits, st);
            },
            st))
        return rc;

    // tree depth = deepest node
    int32_t maxd = 0;
    {
        Tmp dmax;
        if (int rc = tmp_alloc(dmax, sizeof(int8_t), st)) return rc;
        if (int rc = cub_call(
                [&](void* tp, size_t& b) {
                    return cub::DeviceReduce::Max(tp, b, (const int8_t*)dla.p, (int8_t*)dmax.p,
                                                  n, st);
                },
                st))
            return rc;
        int8_t h = 0;
        CAGR_CUDA(cudaMemcpyAsync(&h, dmax.p, 1, cudaMemcpyDeviceToHost, st));
        CAGR_CUDA(cudaStreamSynchronize(st));
        maxd = h;
    }
    t->depth = maxd;

    return kOk;
}

}  // namespace

void tree_free(Tree* t) {
    if (!t) return;
    // the arrays may be in use on any stream: finish the device's work, then
    // return them to the pool
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(t->device);
    cudaDeviceSynchronize();
    void* arrays[] = {t->perm,     t->invperm,  t->meta,      t->nchild, t->parent,
                      t->children, t->leaf_ids, t->n2p_start, t->n2p,    t->spos, t->lorder,
                      t->qgroup,   t->counters, t->rec[0],    t->rec[1], t->rec[2],
                      t->adj_nodes, t->adj_points, t->adj_sums};
    for (void* p : arrays) pool_free(p, nullptr);
    interp_free(t);
    if (prev >= 0) cudaSetDevice(prev);
    delete t;
}

int tree_build(const void* points, int64_t n, int dtype, int max_depth, int leaf_size,
               cudaStream_t stream, Tree** out) {
    *out = nullptr;
    if (n <= 0) return set_error(kErrInvalid, "tree build needs at least one point");
    if (n >= (int64_t(1) << 31) - 2) return set_error(kErrInvalid, "too many points");
    if (max_depth < 0 || max_depth > CAGR_MAX_DEPTH)
        return set_error(kErrInvalid, "max_depth must be in [0, 21]");
    if (leaf_size < 1 || leaf_size > 4096)
        return set_error(kErrInvalid, "leaf_size must be in [1, 4096]");
    if (dtype != 0 && dtype != 1) return set_error(kErrInvalid, "dtype must be 0 (f32) or 1 (f64)");
    if (!points) return set_error(kErrInvalid, "points is null");
    Tree* t = new Tree();
    t->dtype = dtype;
    t->n = n;
    t->max_depth = max_depth;
    t->leaf_size = leaf_size;
    cudaGetDevice(&t->device);
    int rc = dtype == 0 ? build_impl<float>((const float*)points, n, max_depth, leaf_size, stream, t)
                        : build_impl<double>((const double*)points, n, max_depth, leaf_size,
                                             stream, t);
    if (rc != kOk) {
        cudaStreamSynchronize(stream);
        tree_free(t);
        return rc;
    }
    *out = t;
    return kOk;
}

// The per-node point lists (node2point_index), built once, when first exported.
int ensure_n2p(Tree* t, cudaStream_t st) {
    if (t->n2p) return kOk;
    const int64_t n = t->n, L = t->n2p_len;
    const unsigned gN = grid_for(n);
    Tmp leaf_of, cnt, off, pn, pn2, pp;
    if (int rc = tmp_alloc(leaf_of, sizeof(int32_t) * n, st)) return rc;
    if (int rc = tmp_alloc(cnt, sizeof(int32_t) * n, st)) return rc;
    if (int rc = tmp_alloc(off, sizeof(int64_t) * n, st)) return rc;
    if (int rc = tmp_alloc(pn, sizeof(int32_t) * L, st)) return rc;
    if (int rc = tmp_alloc(pp, sizeof(int32_t) * L, st)) return rc;
    if (int rc = tmp_alloc(pn2, sizeof(int32_t) * L, st)) return rc;
    int32_t* lists = nullptr;
    if (int rc = dev_alloc((void**)&lists, sizeof(int32_t) * L, st)) return rc;
    k_leaf_of_pos<<<grid_for(t->num_leaves), kBlock, 0, st>>>(t->leaf_ids, t->num_leaves, t->meta,
                                                             (int32_t*)leaf_of.p);
    k_pairs<false><<<gN, kBlock, 0, st>>>(t->invperm, (const int32_t*)leaf_of.p, t->meta,
                                          t->parent, n, (int32_t*)cnt.p, nullptr, nullptr,
                                          nullptr);
    int rc = cub_call(
        [&](void* tp, size_t& b) {
            return cub::DeviceScan::ExclusiveSum(tp, b, (const int32_t*)cnt.p, (int64_t*)off.p,
                                                 n + 0, st);
        },
        st);
    if (!rc) {
        k_pairs<true><<<gN, kBlock, 0, st>>>(t->invperm, (const int32_t*)leaf_of.p, t->meta,
                                             t->parent, n, nullptr, (const int64_t*)off.p,
                                             (int32_t*)pn.p, (int32_t*)pp.p);
        const int node_bits = bit_width(t->m);
        rc = cub_call(
            [&](void* tp, size_t& b) {
                return cub::DeviceRadixSort::SortPairs(tp, b, (const uint32_t*)pn.p,
                                                       (uint32_t*)pn2.p, (const int32_t*)pp.p,
                                                       lists, L, 0, node_bits, st);
            },
            st);
    }
    if (!rc && cudaGetLastError() != cudaSuccess) rc = set_error(kErrCuda, "point lists launch");
    if (rc) {
        pool_free(lists, st);
        return rc;
    }
    t->n2p = lists;
    return kOk;
}

int tree_export(Tree* t, int64_t* parent, int64_t* children, uint8_t* is_leaf, void* half_w,
                int64_t* npts, int64_t* n2p, int64_t* n2p_start, cudaStream_t stream) {
    const int64_t M = t->m;
    if (n2p)
        if (int rc = ensure_n2p(t, stream)) return rc;
    if (t->dtype == 0)
        k_export<float><<<grid_for(M), kBlock, 0, stream>>>(t->meta, t->parent, t->children,
                                                            t->n2p_start, M, parent, children,
                                                            is_leaf, (float*)half_w, npts,
                                                            n2p_start);
    else
        k_export<double><<<grid_for(M), kBlock, 0, stream>>>(t->meta, t->parent, t->children,
                                                             t->n2p_start, M, parent, children,
                                                             is_leaf, (double*)half_w, npts,
                                                             n2p_start);
    if (n2p) k_widen<<<grid_for(t->n2p_len), kBlock, 0, stream>>>(t->n2p, t->n2p_len, n2p);
    CAGR_CUDA(cudaGetLastError());
    return kOk;
}

}  // namespace cagr
