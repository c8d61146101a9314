// Treecode traversal kernels (the hot path).
//
// Reference: mayueji/CAGR CUDA-based/ext/wn_treecode/wn_treecode_cuda/
// wn_treecode_cuda_kernels.cu:556-1322 -- one thread per query, a 106-entry
// depth-first stack in local memory, and per visited node: far if
// |x - c|^2 > (4 half_w)^2 (c = weighted centroid), then one pair term with the
// node's attribute sum at c; otherwise push the children, or at a leaf add one
// pair term per point.
//
// B200 formulation: one WARP walks the tree for 32 Morton-consecutive queries.
//  * The walk is stackless: nodes are in preorder, so "descend" is n+1 and
//    "skip the subtree" is meta.next.  Every node load is warp-uniform (one
//    L1 wavefront) and the loop control is uniform across the warp.
//  * Each query keeps exactly its own reference decisions with one integer:
//    kd = the deepest depth at which the query is still "active" (has opened
//    every ancestor).  At a node of depth d an active lane (d <= kd) sets
//    kd = d + 1 if it opens an internal node and kd = d otherwise.  Because
//    the walk only ever moves to the first child (depth d + 1) or to the next
//    node after a subtree (depth <= d), "active at the next node" is exactly
//    "depth <= kd".  The warp descends when any lane opened the node.  So the
//    set of pair terms of every query is the reference's set; only the
//    summation order differs.
//  * Acceptance and width tests use the reference's rounding (common.cuh) and
//    are decided bit-identically; the inner loop compares squared distances
//    and needs one rsqrt per pair.  The width rule is a select, not a branch.
//  * exp((x-y)_k/2) = exp(x_k/2) * exp(-y_k/2): the second factor is stored in
//    every source record, the first is per query, so a pair term costs no
//    transcendental beyond the rsqrt.
//  * A2Fused evaluates A21, A22, A23 in one walk (one set of node moments and
//    acceptance decisions, as in the reference, which walks three times).
//  * k_traverse_a2t walks once for sum_k A2Tk(s_k): with three moment slots
//    (the reference's three calls, each with its own |s_k|-weighted centroids
//    and therefore its own acceptance decisions, tracked by three kd's), or
//    with one shared slot when s_1 = s_2 = s_3 (the constant right-hand side).
//  * In the three-slot walk a twig (an internal node whose children are all
//    one-point leaves, flagged in meta.w) evaluates its children in an inner
//    loop for the lanes that opened it, without a metadata load, vote or
//    active-depth update per child; per-lane terms and their order are those of
//    visiting the children one by one.  (Measured: 4.31 -> 3.98 ms at 1M points;
//    the same loop slowed the single-slot walks, which keep the plain visit.)
#include <string>

#include "internal.h"

namespace cagr {
namespace {

#ifndef CAGR_TRAV_WARPS
#define CAGR_TRAV_WARPS 4
#endif
constexpr int kWarps = CAGR_TRAV_WARPS;  // warps (32 consecutive queries each) per block
constexpr unsigned kFull = 0xffffffffu;

template <typename T>
struct TravParams {
    int64_t M = 0, N = 0, nq = 0;
    const int4* meta = nullptr;
    const T* rec[3] = {nullptr, nullptr, nullptr};
    const T* adjn = nullptr;   // packed adjoint records (k_traverse_a2t3)
    const T* adjp = nullptr;
    const T* spos = nullptr;   // sorted tree points (queries == points)
    const int32_t* perm = nullptr;
    const int32_t* qgroup = nullptr;  // queries == points: sorted position of query qi
                                      // (null: qi itself, the Morton order)
    const T* queries = nullptr;
    const int32_t* qorder = nullptr;
    const T* widths = nullptr;
    T width = T(0);
    const T* widths_hi = nullptr;  // A2T right-hand side: b's terms only below these widths
    int grid = 0;              // queries are the nodes of a regular grid
    int gx = 0, gy = 0, gz = 0;
    T gox = T(0), goy = T(0), goz = T(0), gh = T(0);
    T* out = nullptr;
    int out_stride = 1;
    int accumulate = 0;  // bit 0: add into `out` instead of overwriting it; bit 1: write -op
    const T* g = nullptr;  // adjoint: d loss / d out per query [nq, 3], original order
    // adjoint: fixed-point accumulators (integers: their sums do not depend on
    // the order of the atomic adds), the per-node [M, 3] and per-point [N, 3]
    // (Morton order) sums of round(v * scale)
    unsigned long long* accn = nullptr;
    unsigned long long* accp = nullptr;
    unsigned long long* vmax = nullptr;  // pass 1: the largest |v| (as double bits)
    const double* scale = nullptr;       // pass 2: 2^e from vmax
};

template <typename T>
__device__ __forceinline__ void put(T* o, int j, T v, int mode) {
    const T u = (mode & 2) ? -v : v;
    o[j] = (mode & 1) ? o[j] + u : u;
}

template <int OP>
struct OpInfo {
    static constexpr bool a2 = OP == kOpA21 || OP == kOpA22 || OP == kOpA23 || OP == kOpA3 ||
                               OP == kOpA2Fused;
    static constexpr bool a2t = OP == kOpA2T1 || OP == kOpA2T2 || OP == kOpA2T3;
    static constexpr bool uses_exp = a2 || a2t;
    static constexpr bool dim3 = a2 || OP == kOpA || OP == kOpG || OP == kOpA2Inside;
    // which convection direction a single-direction operator uses
    static constexpr int k [[maybe_unused]] = (OP == kOpA21 || OP == kOpA2T1)   ? 0
                                              : (OP == kOpA22 || OP == kOpA2T2) ? 1
                                              : (OP == kOpA23 || OP == kOpA2T3) ? 2
                                                                                : -1;
    static constexpr bool sums0 = k == 0 || OP == kOpA3 || OP == kOpA2Fused;
    static constexpr bool sums1 = k == 1 || OP == kOpA3 || OP == kOpA2Fused;
    static constexpr bool sums2 = k == 2 || OP == kOpA3 || OP == kOpA2Fused;
};

// Per-lane state of one query.
template <typename T>
struct Lane {
    T q0, q1, q2;
    T tw;                 // width threshold on r^2 (r >= w  <=>  r^2 >= tw)
    T twh;                // A2T right-hand side: b's terms need r^2 < twh as well
    T iw, iw3;            // 1/w, 1/w^3 (continuous kernel inside the width)
    T acc0, acc1, acc2;   // outside-width sums (without the per-query exp factor)
    T in0, in1, in2;      // inside-width sums (continuous kernel)
};

// One pair term.  d = x - y, d2 = |d|^2 (reference rounding), src = record.
template <typename T, int OP, bool CONT>
__device__ __forceinline__ void pair_term(Lane<T>& L, const T* __restrict__ src, T dx, T dy, T dz,
                                          T d2) {
    if constexpr (OP == kOpCount) {
        L.acc0 += T(1);  // one pair term, whichever branch the reference takes
        return;
    } else {
        const bool outside = d2 >= L.tw;
        const T rinv = outside ? rsqrt_t(d2) : T(0);  // zero: the pair contributes nothing
        const T rinv3 = rinv * rinv * rinv;
        const Vec4<T> r1 = ld4(src + 4);  // (e1, e2, e3, a0)
        if constexpr (OpInfo<OP>::dim3) {
            const Vec4<T> r2 = ld4(src + 8);  // (a1, a2, W, 0)
            const T m0 = r1.w, m1 = r2.x, m2 = r2.y;
            const T dm = dx * m0 + dy * m1 + dz * m2;
            if constexpr (OP == kOpA) {
                L.acc0 += dm * rinv3;
                if (CONT && !outside) L.in0 += dm * L.iw3;
            } else if constexpr (OP == kOpA2Inside) {
                // the continuous kernel's inside-width sums (the width derivative)
                if (!outside) {
                    L.acc0 += dm;
                    L.in0 += m0;
                    L.in1 += m1;
                    L.in2 += m2;
                }
            } else if constexpr (OP == kOpG) {
                const T rinv5 = rinv3 * rinv * rinv;
                const T c = T(3) * dm * rinv5;
                L.acc0 += m0 * rinv3 - dx * c;
                L.acc1 += m1 * rinv3 - dy * c;
                L.acc2 += m2 * rinv3 - dz * c;
            } else {
                // A2k: exp(d_k/2) (dm / r^3 + m_k / (2r))
                const T t = dm * rinv3;
                const T h = T(0.5) * rinv;
                if constexpr (OpInfo<OP>::sums0) L.acc0 += r1.x * (t + h * m0);
                if constexpr (OpInfo<OP>::sums1) L.acc1 += r1.y * (t + h * m1);
                if constexpr (OpInfo<OP>::sums2) L.acc2 += r1.z * (t + h * m2);
                if constexpr (CONT) {
                    // continuous, inside the width: exp(w) (dm / w^3 + m_k / (2w))
                    if (!outside) {
                        const T ti = dm * L.iw3;
                        const T hi = T(0.5) * L.iw;
                        if constexpr (OpInfo<OP>::sums0) L.in0 += ti + hi * m0;
                        if constexpr (OpInfo<OP>::sums1) L.in1 += ti + hi * m1;
                        if constexpr (OpInfo<OP>::sums2) L.in2 += ti + hi * m2;
                    }
                }
            }
        } else if constexpr (OP == kOpAT) {
            const T c = r1.w * rinv3;
            L.acc0 += dx * c;
            L.acc1 += dy * c;
            L.acc2 += dz * c;
        } else if constexpr (OpInfo<OP>::a2t) {
            // exp(d_k/2) (d s / r^3 + e_k s / (2r)); no continuous branch (:293-299)
            constexpr int k = OpInfo<OP>::k;
            const T e = k == 0 ? r1.x : (k == 1 ? r1.y : r1.z);
            const T g = e * r1.w;
            const T c = g * rinv3;
            L.acc0 += dx * c;
            L.acc1 += dy * c;
            L.acc2 += dz * c;
            const T h = g * T(0.5) * rinv;
            if constexpr (k == 0) L.acc0 += h;
            if constexpr (k == 1) L.acc1 += h;
            if constexpr (k == 2) L.acc2 += h;
        }
    }
}

// Inverse of the 3-way bit interleave: every third bit of x, packed.
__device__ __forceinline__ uint32_t compact3(uint64_t x) {
    x &= 0x1249249249249249ull;
    x = (x ^ (x >> 2)) & 0x10c30c30c30c30c3ull;
    x = (x ^ (x >> 4)) & 0x100f00f00f00f00full;
    x = (x ^ (x >> 8)) & 0x1f0000ff0000ffull;
    x = (x ^ (x >> 16)) & 0x1f00000000ffffull;
    x = (x ^ (x >> 32)) & 0x1fffffull;
    return (uint32_t)x;
}

// Loads this lane's query; returns false past the end.  Three query sources:
// the tree's own points (in the tree's Hilbert grouping), an explicit array
// (optional order), or
// the nodes of a regular grid, visited in Morton order of (i, j, k) and
// written at (k * gy + j) * gx + i.
template <typename T>
__device__ __forceinline__ bool load_query(const TravParams<T>& p, int64_t qi, Lane<T>& L,
                                           int64_t& oidx, T& w) {
    w = p.width;
    oidx = 0;
    L.q0 = L.q1 = L.q2 = T(0);
    bool valid = qi < p.nq;
    if (valid && p.grid) {
        const uint32_t i = compact3((uint64_t)qi), j = compact3((uint64_t)qi >> 1),
                       k = compact3((uint64_t)qi >> 2);
        valid = i < (uint32_t)p.gx && j < (uint32_t)p.gy && k < (uint32_t)p.gz;
        if (valid) {
            oidx = ((int64_t)k * p.gy + j) * p.gx + i;
            L.q0 = fma(T(i), p.gh, p.gox);  // one rounding: node = origin + index * spacing
            L.q1 = fma(T(j), p.gh, p.goy);
            L.q2 = fma(T(k), p.gh, p.goz);
            if (p.widths) w = p.widths[oidx];
        }
    } else if (valid) {
        if (p.queries == nullptr) {
            const int64_t s = p.qgroup ? (int64_t)p.qgroup[qi] : qi;
            oidx = p.perm[s];
            L.q0 = p.spos[3 * s];
            L.q1 = p.spos[3 * s + 1];
            L.q2 = p.spos[3 * s + 2];
        } else {
            oidx = p.qorder ? (int64_t)p.qorder[qi] : qi;
            L.q0 = p.queries[3 * oidx];
            L.q1 = p.queries[3 * oidx + 1];
            L.q2 = p.queries[3 * oidx + 2];
        }
        if (p.widths) w = p.widths[oidx];
    }
    L.tw = width_threshold(w);
    L.iw = T(1) / w;
    L.iw3 = T(1) / (w * w * w);
    L.acc0 = L.acc1 = L.acc2 = T(0);
    L.in0 = L.in1 = L.in2 = T(0);
    return valid;
}

// This lane's query index: warp w of block b walks queries 32 (b * kWarps + w)
// onwards.  (A persistent launch whose warps take groups from a counter
// measured slower: neighbouring groups then run on different SMs and no longer
// share node records in L1.)
__device__ __forceinline__ int64_t lane_query() {
    return ((int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5)) * 32 + (threadIdx.x & 31);
}

// walk(qi) for this lane's query of every group of 32 queries that falls to
// this warp in a grid-stride loop (one group per warp at the launch's grid).
// Measured at 1M points against the single call walk(lane_query()): faster for
// the A2T walks (three-slot 3.71 -> 3.53 ms, right-hand side 5.41 -> 5.29,
// shared slot 2.55 -> 2.52), slower for some single-slot ones (G 2.02 -> 2.18),
// which keep the single call.
template <typename F>
__device__ __forceinline__ void stride_groups(int64_t nq, F&& walk) {
    const int lane = threadIdx.x & 31;
    const int64_t ngroups = (nq + 31) / 32;
    for (int64_t g = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5); g < ngroups;
         g += (int64_t)gridDim.x * kWarps)
        walk(g * 32 + lane);
}

template <typename T, int OP, bool CONT>
__device__ __forceinline__ void walk_query(const TravParams<T>& p, const int64_t qi) {
    if (__all_sync(kFull, qi >= p.nq)) return;  // whole warp past the end
    Lane<T> L;
    int64_t oidx;
    T w;
    const bool valid = load_query(p, qi, L, oidx, w);

    const int M = (int)p.M;
    const T* __restrict__ rec = p.rec[0];
    int kd = valid ? 0 : -1;  // active at depth d  <=>  d <= kd
    int n = 0;
    while (n < M) {
        const int4 mt = __ldg(p.meta + n);
        const int d = node_depth(mt);
        const bool leaf = node_leaf(mt);
        const T* r = rec + (int64_t)n * CAGR_REC_STRIDE;
        const Vec4<T> r0 = ld4(r);  // (cx, cy, cz, (4 half_w)^2)
        T dx = sub_rn(L.q0, r0.x);
        T dy = sub_rn(L.q1, r0.y);
        T dz = sub_rn(L.q2, r0.z);
        T d2 = dist2_exact(dx, dy, dz);
        const bool active = d <= kd;
        const bool far = d2 > rec_radius2(r0.w);
        const bool open = active && !far;
        if (active) kd = (open && !leaf) ? d + 1 : d;
        if (mt.z == -1) {
            // single-point leaf: far lanes take the node term, near lanes the point
            const T* src = r;
            if (open && !rec_same_leaf(r0.w)) {
                src = rec + ((int64_t)M + mt.y) * CAGR_REC_STRIDE;
                const Vec4<T> s0 = ld4(src);
                dx = sub_rn(L.q0, s0.x);
                dy = sub_rn(L.q1, s0.y);
                dz = sub_rn(L.q2, s0.z);
                d2 = dist2_exact(dx, dy, dz);
            }
            if (active) pair_term<T, OP, CONT>(L, src, dx, dy, dz, d2);
            n = mt.x;
            continue;
        }
        // (the vote after the one-point-leaf path, which does not need it: mt
        // is warp-uniform, so every lane of the warp gets here or none)
        const bool any_open = __any_sync(kFull, open);
        if (active && far) pair_term<T, OP, CONT>(L, r, dx, dy, dz, d2);
        if (leaf) {
            const int np = -mt.z;
            if (any_open) {
                const T* pr = rec + ((int64_t)M + mt.y) * CAGR_REC_STRIDE;
                for (int j = 0; j < np; j++, pr += CAGR_REC_STRIDE) {
                    if (open) {
                        const Vec4<T> s0 = ld4(pr);
                        const T ex = sub_rn(L.q0, s0.x);
                        const T ey = sub_rn(L.q1, s0.y);
                        const T ez = sub_rn(L.q2, s0.z);
                        pair_term<T, OP, CONT>(L, pr, ex, ey, ez, dist2_exact(ex, ey, ez));
                    }
                }
            }
            n = mt.x;
        } else {
            n = any_open ? n + 1 : mt.x;
        }
    }

    if (!valid) return;
    T* o = p.out + oidx * (int64_t)p.out_stride;
    const int acc = p.accumulate;
    if constexpr (OpInfo<OP>::uses_exp) {
        const T ex0 = exp_t(L.q0 * T(0.5)), ex1 = exp_t(L.q1 * T(0.5)), ex2 = exp_t(L.q2 * T(0.5));
        const T ew = CONT ? exp_t(w) : T(0);
        const T v0 = ex0 * L.acc0 + ew * L.in0;
        const T v1 = ex1 * L.acc1 + ew * L.in1;
        const T v2 = ex2 * L.acc2 + ew * L.in2;
        if constexpr (OP == kOpA21) put(o, 0, v0, acc);
        if constexpr (OP == kOpA22) put(o, 0, v1, acc);
        if constexpr (OP == kOpA23) put(o, 0, v2, acc);
        if constexpr (OP == kOpA3) put(o, 0, (v0 + v1 + v2) / T(3), acc);
        if constexpr (OP == kOpA2Fused) {
            put(o, 0, v0, acc);
            put(o, 1, v1, acc);
            put(o, 2, v2, acc);
        }
        if constexpr (OpInfo<OP>::a2t) {
            constexpr int k = OpInfo<OP>::k;
            const T ek = k == 0 ? ex0 : (k == 1 ? ex1 : ex2);
            put(o, 0, ek * L.acc0, acc);
            put(o, 1, ek * L.acc1, acc);
            put(o, 2, ek * L.acc2, acc);
        }
    } else if constexpr (OP == kOpA) {
        put(o, 0, L.acc0 + L.in0, acc);
    } else if constexpr (OP == kOpCount) {
        put(o, 0, L.acc0, acc);
    } else if constexpr (OP == kOpA2Inside) {
        put(o, 0, L.acc0, acc);
        put(o, 1, L.in0, acc);
        put(o, 2, L.in1, acc);
        put(o, 3, L.in2, acc);
    } else {
        put(o, 0, L.acc0, acc);
        put(o, 1, L.acc1, acc);
        put(o, 2, L.acc2, acc);
    }
}

template <typename T, int OP, bool CONT>
__global__ void __launch_bounds__(kWarps * 32) k_traverse(const TravParams<T> p) {
    walk_query<T, OP, CONT>(p, lane_query());
}

// One A2T term of the directions [klo, khi) with weight s:
//   acc += sum_k g_k (d / r^3 + e_k / (2r)),  g_k = exp(x_k/2) e_k(y) s,
// where e(y) = exp(-y/2) comes from the record (folded per term so that the
// three directions, which may use different sources, share one accumulator).
template <typename T, bool WINDOW = false>
__device__ __forceinline__ void a2t_term(Lane<T>& L, const T* ex, const T* e, T s, T dx, T dy,
                                         T dz, T d2, int klo, int khi) {
    // WINDOW: b's term in the right-hand side, kept only for tw <= r^2 < twh
    const bool outside = d2 >= L.tw && (!WINDOW || d2 < L.twh);
    const T rinv = outside ? rsqrt_t(d2) : T(0);
    const T rinv3 = rinv * rinv * rinv;
    const T hr = T(0.5) * rinv;
    T gsum = T(0);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (k < klo || k >= khi) continue;
        const T g = ex[k] * e[k] * s;
        gsum += g;
        if (k == 0) L.acc0 += g * hr;
        if (k == 1) L.acc1 += g * hr;
        if (k == 2) L.acc2 += g * hr;
    }
    const T c = gsum * rinv3;
    L.acc0 += dx * c;
    L.acc1 += dy * c;
    L.acc2 += dz * c;
}

// A2T1(s) + A2T2(s) + A2T3(s) in one walk for ONE input s (one slot, the three
// directions share its centroids and acceptance decisions): the solve's
// right-hand side A2T(b) (main_CAGR.py:98,108).
template <typename T>
__device__ __forceinline__ void walk_a2t_shared(const TravParams<T>& p, const int64_t qi) {
    if (__all_sync(kFull, qi >= p.nq)) return;
    Lane<T> L;
    int64_t oidx;
    T w;
    const bool valid = load_query(p, qi, L, oidx, w);
    const T ex[3] = {exp_t(L.q0 * T(0.5)), exp_t(L.q1 * T(0.5)), exp_t(L.q2 * T(0.5))};
    const int M = (int)p.M;
    const T* __restrict__ rec = p.rec[0];
    int kd = valid ? 0 : -1;
    int n = 0;
    while (n < M) {
        const int4 mt = __ldg(p.meta + n);
        const int d = node_depth(mt);
        const bool leaf = node_leaf(mt);
        const T* r = rec + (int64_t)n * CAGR_REC_STRIDE;
        const Vec4<T> r0 = ld4(r);
        T dx = sub_rn(L.q0, r0.x);
        T dy = sub_rn(L.q1, r0.y);
        T dz = sub_rn(L.q2, r0.z);
        T d2 = dist2_exact(dx, dy, dz);
        const bool active = d <= kd;
        const bool far = d2 > rec_radius2(r0.w);
        const bool open = active && !far;
        if (active) kd = (open && !leaf) ? d + 1 : d;
        const bool any_open = __any_sync(kFull, open);
        const T* src = r;
        if (leaf && open) {  // (the same-point flag measured slower here)
            src = rec + ((int64_t)M + mt.y) * CAGR_REC_STRIDE;
            const Vec4<T> s0 = ld4(src);
            dx = sub_rn(L.q0, s0.x);
            dy = sub_rn(L.q1, s0.y);
            dz = sub_rn(L.q2, s0.z);
            d2 = dist2_exact(dx, dy, dz);
        }
        if (active && (far || leaf)) {
            const Vec4<T> r1 = ld4(src + 4);  // (e1, e2, e3, s)
            const T e[3] = {r1.x, r1.y, r1.z};
            a2t_term(L, ex, e, r1.w, dx, dy, dz, d2, 0, 3);
        }
        if (leaf) {
            const int np = -mt.z;
            if (np > 1 && any_open) {
                const T* pr = rec + ((int64_t)M + mt.y + 1) * CAGR_REC_STRIDE;
                for (int j = 1; j < np; j++, pr += CAGR_REC_STRIDE) {
                    if (open) {
                        const Vec4<T> s0 = ld4(pr);
                        const Vec4<T> r1 = ld4(pr + 4);
                        const T e[3] = {r1.x, r1.y, r1.z};
                        const T px = sub_rn(L.q0, s0.x);
                        const T py = sub_rn(L.q1, s0.y);
                        const T pz = sub_rn(L.q2, s0.z);
                        a2t_term(L, ex, e, r1.w, px, py, pz, dist2_exact(px, py, pz), 0, 3);
                    }
                }
            }
            n = mt.x;
        } else {
            n = any_open ? n + 1 : mt.x;
        }
    }
    if (!valid) return;
    T* o = p.out + oidx * (int64_t)p.out_stride;
    put(o, 0, L.acc0, p.accumulate);
    put(o, 1, L.acc1, p.accumulate);
    put(o, 2, L.acc2, p.accumulate);
}

template <typename T>
__global__ void __launch_bounds__(kWarps * 32) k_traverse_a2t_shared(const TravParams<T> p) {
    stride_groups(p.nq, [&](int64_t qi) { walk_a2t_shared<T>(p, qi); });
}

// One direction-K A2T term with g = exp(x_K/2) exp(-y_K/2) s (premultiplied):
//   acc += g (d / r^3 + e_K / (2r)).
template <typename T, int K>
__device__ __forceinline__ void a2t_term1(Lane<T>& L, bool take, T g, T dx, T dy, T dz, T d2) {
    const bool outside = take && d2 >= L.tw;  // not taken: contributes exactly zero
    const T rinv = outside ? rsqrt_t(d2) : T(0);
    // g/r once, then g/r^3 from it, and the g/(2r) term as one FMA into the
    // accumulator (two operations fewer than forming r^-3 and g/2 apart:
    // A2T_SUM 3.53 -> 3.48 ms at 1M points, FP64 6.05 -> 5.92 ms)
    const T gr = g * rinv;
    const T c = gr * (rinv * rinv);
    L.acc0 += dx * c;
    L.acc1 += dy * c;
    L.acc2 += dz * c;
    if constexpr (K == 0) L.acc0 += T(0.5) * gr;
    if constexpr (K == 1) L.acc1 += T(0.5) * gr;
    if constexpr (K == 2) L.acc2 += T(0.5) * gr;
}

// The shared-slot (b) term of a near point: record (y, 0), (e(y), s).
template <typename T>
__device__ __forceinline__ void rhs_b_point(Lane<T>& L, const T* pr, const T* ex) {
    const Vec4<T> s0 = ld4(pr);
    const Vec4<T> r1 = ld4(pr + 4);
    const T px = sub_rn(L.q0, s0.x);
    const T py = sub_rn(L.q1, s0.y);
    const T pz = sub_rn(L.q2, s0.z);
    const T e[3] = {r1.x, r1.y, r1.z};
    a2t_term<T, true>(L, ex, e, r1.w, px, py, pz, dist2_exact(px, py, pz), 0, 3);
}

// Slot K of the three-slot adjoint walk: acceptance test against the slot's
// own centroid and the lane's own active depth kd.
template <typename T>
struct SlotTest {
    T dx, dy, dz, d2;
    bool active, far, open;
};
template <typename T>
__device__ __forceinline__ SlotTest<T> slot_test(const Lane<T>& L, const Vec4<T>& c, T R2, int d,
                                                 bool leaf, int& kd) {
    SlotTest<T> s;
    s.dx = sub_rn(L.q0, c.x);
    s.dy = sub_rn(L.q1, c.y);
    s.dz = sub_rn(L.q2, c.z);
    s.d2 = dist2_exact(s.dx, s.dy, s.dz);
    s.active = d <= kd;
    s.far = s.d2 > R2;
    s.open = s.active && !s.far;
    if (s.active) kd = (s.open && !leaf) ? d + 1 : d;
    return s;
}

// Near-point term of the three-slot adjoint: the point's geometry is shared by
// the slots that take it (open_k), each weighted by its own g_k.
template <typename T>
__device__ __forceinline__ void a2t3_point(Lane<T>& L, const T* pp, bool o0, bool o1, bool o2,
                                           T ex0, T ex1, T ex2) {
    const Vec4<T> P0 = ld4(pp);      // (y, e_0 s_0)
    const Vec4<T> P1 = ld4(pp + 4);  // (e_1 s_1, e_2 s_2, 0, 0)
    const T px = sub_rn(L.q0, P0.x);
    const T py = sub_rn(L.q1, P0.y);
    const T pz = sub_rn(L.q2, P0.z);
    const T dd = dist2_exact(px, py, pz);
    const bool outside = dd >= L.tw;
    const T rinv = outside ? rsqrt_t(dd) : T(0);
    const T hr = T(0.5) * rinv;
    const T g0 = o0 ? ex0 * P0.w : T(0);
    const T g1 = o1 ? ex1 * P1.x : T(0);
    const T g2 = o2 ? ex2 * P1.y : T(0);
    const T c = (g0 + g1 + g2) * (rinv * rinv * rinv);
    // two FMAs into each accumulator
    L.acc0 += px * c;
    L.acc0 += g0 * hr;
    L.acc1 += py * c;
    L.acc1 += g1 * hr;
    L.acc2 += pz * c;
    L.acc2 += g2 * hr;
}

// A one-point-leaf child of a twig for one slot: active = the lane opened the
// twig in that slot; far = node term at the child's centroid, near = point term.
template <typename T>
struct ChildTest {
    T dx, dy, dz, d2;
    bool far, near;
};
template <typename T>
__device__ __forceinline__ ChildTest<T> child_test(const Lane<T>& L, const Vec4<T>& c, T R2,
                                                   bool active) {
    ChildTest<T> t;
    t.dx = sub_rn(L.q0, c.x);
    t.dy = sub_rn(L.q1, c.y);
    t.dz = sub_rn(L.q2, c.z);
    t.d2 = dist2_exact(t.dx, t.dy, t.dz);
    const bool f = t.d2 > R2;
    t.far = active && f;
    t.near = active && !f;
    return t;
}

// sum_k A2Tk(s_k) in one walk over the packed adjoint records (Tree::adj_*):
// slot k holds the moments of s_k with its own |s_k|-weighted centroids, hence
// its own acceptance decisions, tracked by its own kd -- the three reference
// calls A2T1(s1), A2T2(s2), A2T3(s3) with their own scatters.  A near point's
// geometry is shared by the three directions.
//
// RHS: sum_k A2Tk(b) - sum_k A2Tk(s_k) in the same walk -- the right-hand side
// minus the normal-equation product of one CAGR iteration (main_CAGR.py:108,
// 114-115), at the same width.  b is a fourth slot with its own moments
// (record slot 1, the shared three-direction form of k_traverse_a2t_shared),
// its own centroids and its own kd; its terms are added, the s_k slots' terms
// subtracted.
template <typename T, bool RHS>
__device__ __forceinline__ void walk_a2t3(const TravParams<T>& p, const int64_t qi) {
    if (__all_sync(kFull, qi >= p.nq)) return;
    Lane<T> L;
    int64_t oidx;
    T w;
    const bool valid = load_query(p, qi, L, oidx, w);
    L.twh = T(INFINITY);
    if (RHS && valid && p.widths_hi) L.twh = width_threshold(p.widths_hi[oidx]);
    const T ex0 = exp_t(L.q0 * T(0.5)), ex1 = exp_t(L.q1 * T(0.5)), ex2 = exp_t(L.q2 * T(0.5));
    // the s_k slots' sign: subtracted in the RHS form
    const T sg = RHS ? T(-1) : T(1);
    const T gx0 = sg * ex0, gx1 = sg * ex1, gx2 = sg * ex2;
    const T exb[3] = {ex0, ex1, ex2};
    const int M = (int)p.M;
    const T* __restrict__ an = p.adjn;
    const T* __restrict__ ap = p.adjp;
    const T* __restrict__ rb = p.rec[1];  // RHS: b's records
    int kd0 = valid ? 0 : -1, kd1 = kd0, kd2 = kd0, kdb = kd0;
    int n = 0;
    while (n < M) {
        const int4 mt = __ldg(p.meta + n);
        const int d = node_depth(mt);
        const bool leaf = node_leaf(mt);
        const T R2 = mac_radius2_bits(d, T(0));
        const T* q = an + (int64_t)n * 12;
        const Vec4<T> c0 = ld4(q), c1 = ld4(q + 4), c2 = ld4(q + 8);
        const SlotTest<T> s0 = slot_test(L, c0, R2, d, leaf, kd0);
        const SlotTest<T> s1 = slot_test(L, c1, R2, d, leaf, kd1);
        const SlotTest<T> s2 = slot_test(L, c2, R2, d, leaf, kd2);
        bool open_any = s0.open || s1.open || s2.open;
        SlotTest<T> sb;
        Vec4<T> b1;
        if constexpr (RHS) {
            const T* r = rb + (int64_t)n * CAGR_REC_STRIDE;
            const Vec4<T> b0 = ld4(r);  // (c_b, (4h)^2)
            b1 = ld4(r + 4);            // (e(c_b), s_b)
            sb = slot_test(L, b0, rec_radius2(b0.w), d, leaf, kdb);
            open_any = open_any || sb.open;
        }
        const bool any_open = __any_sync(kFull, open_any);
        // node terms, each slot against its own centroid
        if (s0.active && s0.far) a2t_term1<T, 0>(L, true, gx0 * c0.w, s0.dx, s0.dy, s0.dz, s0.d2);
        if (s1.active && s1.far) a2t_term1<T, 1>(L, true, gx1 * c1.w, s1.dx, s1.dy, s1.dz, s1.d2);
        if (s2.active && s2.far) a2t_term1<T, 2>(L, true, gx2 * c2.w, s2.dx, s2.dy, s2.dz, s2.d2);
        if constexpr (RHS) {
            if (sb.active && sb.far && sb.d2 < L.twh) {
                const T e[3] = {b1.x, b1.y, b1.z};
                a2t_term<T, true>(L, exb, e, b1.w, sb.dx, sb.dy, sb.dz, sb.d2, 0, 3);
            }
        }
        if (leaf) {
            if (any_open) {
                const int np = -mt.z;
                const T* pp = ap + (int64_t)mt.y * 8;
                for (int j = 0; j < np; j++, pp += 8) {
                    if (s0.open || s1.open || s2.open)
                        a2t3_point(L, pp, s0.open, s1.open, s2.open, gx0, gx1, gx2);
                    if constexpr (RHS) {
                        if (sb.open) rhs_b_point(L, rb + ((int64_t)M + mt.y + j) * CAGR_REC_STRIDE, exb);
                    }
                }
            }
            n = mt.x;
        } else if (node_twig(mt)) {
            // one-point-leaf children n+1 .. n+npts: for each slot, the lanes that
            // opened this node are the lanes active at each child (same order of
            // terms as visiting the children one by one)
            if (any_open) {
                const int nc = mt.z;
                const T R2c = mac_radius2_bits(d + 1, T(0));
                const T* cq = q + 12;
                const T* pp = ap + (int64_t)mt.y * 8;
                for (int c = 0; c < nc; c++, cq += 12, pp += 8) {
                    if (s0.open || s1.open || s2.open) {
                        const Vec4<T> C0 = ld4(cq), C1 = ld4(cq + 4), C2 = ld4(cq + 8);
                        const ChildTest<T> t0 = child_test(L, C0, R2c, s0.open);
                        const ChildTest<T> t1 = child_test(L, C1, R2c, s1.open);
                        const ChildTest<T> t2 = child_test(L, C2, R2c, s2.open);
                        if (t0.far) a2t_term1<T, 0>(L, true, gx0 * C0.w, t0.dx, t0.dy, t0.dz, t0.d2);
                        if (t1.far) a2t_term1<T, 1>(L, true, gx1 * C1.w, t1.dx, t1.dy, t1.dz, t1.d2);
                        if (t2.far) a2t_term1<T, 2>(L, true, gx2 * C2.w, t2.dx, t2.dy, t2.dz, t2.d2);
                        if (t0.near || t1.near || t2.near)
                            a2t3_point(L, pp, t0.near, t1.near, t2.near, gx0, gx1, gx2);
                    }
                    if constexpr (RHS) {
                        if (sb.open) {
                            // b's one-point-leaf child: its node record if far, else its point
                            const T* cr = rb + ((int64_t)n + 1 + c) * CAGR_REC_STRIDE;
                            const Vec4<T> B0 = ld4(cr);
                            const ChildTest<T> tb = child_test(L, B0, rec_radius2(B0.w), true);
                            if (tb.far) {
                                if (tb.d2 < L.twh) {
                                    const Vec4<T> B1 = ld4(cr + 4);
                                    const T e[3] = {B1.x, B1.y, B1.z};
                                    a2t_term<T, true>(L, exb, e, B1.w, tb.dx, tb.dy, tb.dz,
                                                      tb.d2, 0, 3);
                                }
                            } else {
                                rhs_b_point(L, rb + ((int64_t)M + mt.y + c) * CAGR_REC_STRIDE, exb);
                            }
                        }
                    }
                }
            }
            n = mt.x;
        } else {
            n = any_open ? n + 1 : mt.x;
        }
    }
    if (!valid) return;
    T* o = p.out + oidx * (int64_t)p.out_stride;
    put(o, 0, L.acc0, p.accumulate);
    put(o, 1, L.acc1, p.accumulate);
    put(o, 2, L.acc2, p.accumulate);
}

template <typename T, bool RHS>
__global__ void __launch_bounds__(kWarps * 32) k_traverse_a2t3(const TravParams<T> p) {
    stride_groups(p.nq, [&](int64_t qi) { walk_a2t3<T, RHS>(p, qi); });
}

// Launches a traversal over p.nq queries, one warp per group of 32.
template <typename T>
int launch_groups(void (*kernel)(TravParams<T>), const TravParams<T>& p, cudaStream_t s) {
    const int64_t groups = (p.nq + 31) / 32;
    const int64_t blocks = (groups + kWarps - 1) / kWarps;
    if (blocks > 0x7fffffffLL) return set_error(kErrInvalid, "too many queries");
    kernel<<<(unsigned)blocks, kWarps * 32, 0, s>>>(p);
    CAGR_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T, int OP>
int launch_op(const TravParams<T>& p, int cont, int slots, cudaStream_t s) {
    if constexpr (OP == kOpA2TFused) {
        if (slots == 3) return launch_groups<T>(k_traverse_a2t3<T, false>, p, s);
        if (slots == 4) return launch_groups<T>(k_traverse_a2t3<T, true>, p, s);
        return launch_groups<T>(k_traverse_a2t_shared<T>, p, s);
    } else if (cont) {
        return launch_groups<T>(k_traverse<T, OP, true>, p, s);
    } else {
        return launch_groups<T>(k_traverse<T, OP, false>, p, s);
    }
}

template <typename T>
int dispatch(const Tree* t, const TraverseArgs& a, cudaStream_t s) {
    TravParams<T> p;
    p.M = t->m;
    p.N = t->n;
    p.nq = a.queries ? a.nq : t->n;
    if (a.grid) {
        // Morton indices over the smallest power-of-two cube holding the grid
        int bits = 0;
        while ((1 << bits) < a.gx || (1 << bits) < a.gy || (1 << bits) < a.gz) bits++;
        p.grid = 1;
        p.gx = a.gx;
        p.gy = a.gy;
        p.gz = a.gz;
        p.gox = (T)a.gorigin[0];
        p.goy = (T)a.gorigin[1];
        p.goz = (T)a.gorigin[2];
        p.gh = (T)a.gspacing;
        p.nq = int64_t(1) << (3 * bits);
    }
    p.meta = t->meta;
    p.spos = (const T*)t->spos;
    p.perm = t->perm;
    // warp grouping of self-queries, chosen per walk by measurement at 1M
    // points (outputs are the same bits either way): the Hilbert grouping
    // speeds up the A2T walks (three-slot 3.89 -> 3.70 ms, right-hand side
    // 5.68 -> 5.40, shared slot 2.62 -> 2.56) and slows the single-slot walks
    // (A2_FUSED 1.94 -> 2.01, AT 2.06 -> 2.24), which keep the Morton order
    p.qgroup = a.op == kOpA2TFused ? t->qgroup : nullptr;
    p.queries = (const T*)a.queries;
    p.qorder = a.qorder;
    p.widths = (const T*)a.widths;
    p.width = (T)a.width;
    p.widths_hi = (const T*)a.widths_hi;
    p.out = (T*)a.out;
    p.accumulate = (a.accumulate ? 1 : 0) | (a.negate ? 2 : 0);
    const bool scalar_in = a.op == kOpAT || a.op == kOpA2T1 || a.op == kOpA2T2 ||
                           a.op == kOpA2T3 || a.op == kOpA2TFused;
    const int slots = a.op == kOpA2TFused ? a.slots : 1;
    if (slots >= 3) {
        if (!t->adj_valid || !t->adj_nodes)
            return set_error(kErrState, "A2T sum needs the three-slot moments (cagr_scatter3)");
        p.adjn = (const T*)t->adj_nodes;
        p.adjp = (const T*)t->adj_points;
        if (slots == 4) {
            if (!t->rec[1] || t->rec_dim[1] != 1)
                return set_error(kErrState, "the A2T right-hand side needs b's moments in slot 1");
            p.rec[1] = (const T*)t->rec[1];
        }
    } else {
        const int need_dim = a.op == kOpCount ? t->rec_dim[0] : (scalar_in ? 1 : 3);
        if (!t->rec[0] || t->rec_dim[0] == 0 || t->rec_dim[0] != need_dim)
            return set_error(kErrState, "node moments of the right attribute dim are not computed");
        for (int k = 0; k < 3; k++) p.rec[k] = (const T*)t->rec[0];
    }
    const int out_dim = (a.op == kOpA || a.op == kOpA3 || a.op == kOpA21 || a.op == kOpA22 ||
                         a.op == kOpA23 || a.op == kOpCount)
                            ? 1
                            : (a.op == kOpA2Inside ? 4 : 3);
    p.out_stride = a.out_stride > 0 ? a.out_stride : out_dim;
    if (p.nq == 0) return kOk;
    switch (a.op) {
        case kOpA: return launch_op<T, kOpA>(p, a.continuous, 1, s);
        case kOpAT: return launch_op<T, kOpAT>(p, 0, 1, s);
        case kOpA3: return launch_op<T, kOpA3>(p, a.continuous, 1, s);
        case kOpA21: return launch_op<T, kOpA21>(p, a.continuous, 1, s);
        case kOpA22: return launch_op<T, kOpA22>(p, a.continuous, 1, s);
        case kOpA23: return launch_op<T, kOpA23>(p, a.continuous, 1, s);
        case kOpA2T1: return launch_op<T, kOpA2T1>(p, 0, 1, s);
        case kOpA2T2: return launch_op<T, kOpA2T2>(p, 0, 1, s);
        case kOpA2T3: return launch_op<T, kOpA2T3>(p, 0, 1, s);
        case kOpG: return launch_op<T, kOpG>(p, 0, 1, s);
        case kOpA2Fused: return launch_op<T, kOpA2Fused>(p, a.continuous, 1, s);
        case kOpA2TFused: return launch_op<T, kOpA2TFused>(p, 0, slots, s);
        case kOpCount: return launch_op<T, kOpCount>(p, 0, 1, s);
        case kOpA2Inside: return launch_op<T, kOpA2Inside>(p, 0, 1, s);
        default: return set_error(kErrInvalid, "unknown operator " + std::to_string(a.op));
    }
}

// ---- adjoint of the fused A2 ------------------------------------------------
//
// With the forward's moments (same centroids, decisions and pair terms) the
// fused A2 is linear in the attributes: out_k(x) = sum over terms of
// ex_k(x) e_k(src) (d . m / r^3 + m_k / (2r)) outside the width, plus
// e^w (d . m / w^3 + m_k / (2w)) inside it (continuous kernel), where m is the
// source's attribute sum (a node: the sum over its points).  So
//   d loss / d m_src = sum over the terms using src of
//       sum_k g_k ex_k e_k (d / r^3 + u_k / (2r))     (outside)
//       sum_k g_k e^w (d / w^3 + u_k / (2w))          (inside, continuous)
// and d loss / d mu_j = the sum of that over j's point terms and over every
// node containing j.  k_adjoint_a2 walks exactly as k_traverse<A2Fused> and
// adds each term's vector into the node or point it used (all lanes taking a
// term at a visit use the same node or point: one warp sum, one atomic add per
// component); k_adj_push adds the leaf-to-root node sums to each point's own.

// The warp sum of (a, b, c) over the lanes with `take` (all of them use the
// same node or point).  PASS 1 keeps its largest magnitude in the leader
// lane's running maximum vm (non-finite sums as infinity; each warp publishes
// its maximum once, at the end of its walk); pass 2 adds round(sum * sc) to
// the integer accumulators dst[0..2].  The
// warp sum has a fixed shuffle order and integer addition is associative, so
// the accumulated gradient is the same bits on every run (float atomics would
// add in the order the warps arrive).
template <bool PASS1, typename T>
__device__ __forceinline__ void warp_red3(bool take, T a, T b, T c, unsigned long long* dst,
                                          double& vm, double sc) {
    const unsigned m = __ballot_sync(kFull, take);
    if (m == 0u) return;
    if (!take) a = b = c = T(0);
    if (__popc(m) > 1) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(kFull, a, o);
            b += __shfl_xor_sync(kFull, b, o);
            c += __shfl_xor_sync(kFull, c, o);
        }
    }
    if ((int)(threadIdx.x & 31) == __ffs(m) - 1) {
        if constexpr (PASS1) {
            const double mx = fmax(fabs((double)a), fmax(fabs((double)b), fabs((double)c)));
            const bool bad = !(mx <= 1.0e300);  // NaN or infinite
            vm = fmax(vm, bad ? (double)INFINITY : mx);
        } else {
            atomicAdd(dst, (unsigned long long)llrint((double)a * sc));
            atomicAdd(dst + 1, (unsigned long long)llrint((double)b * sc));
            atomicAdd(dst + 2, (unsigned long long)llrint((double)c * sc));
        }
    }
}

// The fixed-point scale from the largest warp sum: a power of two with
// vmax * scale * bound < 2^62, bound = the most terms one accumulator can
// receive and the push can add (one per warp, times the levels of a path).
// 0 when a sum is not finite (the push then writes NaN).
__global__ void k_adj_scale(const unsigned long long* vmax, double bound, double* scale) {
    const double v = __longlong_as_double((long long)*vmax);
    if (!(v < (double)INFINITY)) {
        *scale = 0.0;
        return;
    }
    if (v == 0.0) {
        *scale = 1.0;
        return;
    }
    int e;
    frexp(v * bound, &e);  // v * bound < 2^e
    *scale = ldexp(1.0, 62 - e);
}

// d loss / d m of one term; G_k = g_k ex_k(x) (query side), gs_k = g_k, ew = e^w
template <typename T, bool CONT>
__device__ __forceinline__ void adj_term(const Lane<T>& L, const T* src, T dx, T dy, T dz, T d2,
                                         const T* G, const T* gs, T ew, T* v) {
    if (d2 >= L.tw) {
        const T rinv = rsqrt_t(d2);
        const Vec4<T> r1 = ld4(src + 4);  // (e1, e2, e3, a0)
        const T G0 = G[0] * r1.x, G1 = G[1] * r1.y, G2 = G[2] * r1.z;
        const T c = (G0 + G1 + G2) * (rinv * rinv * rinv);
        const T h = T(0.5) * rinv;
        v[0] = dx * c + h * G0;
        v[1] = dy * c + h * G1;
        v[2] = dz * c + h * G2;
    } else if (CONT) {
        const T c = (gs[0] + gs[1] + gs[2]) * ew * L.iw3;
        const T h = T(0.5) * ew * L.iw;
        v[0] = dx * c + h * gs[0];
        v[1] = dy * c + h * gs[1];
        v[2] = dz * c + h * gs[2];
    } else {
        v[0] = v[1] = v[2] = T(0);
    }
}

template <typename T, bool CONT, bool PASS1>
__global__ void __launch_bounds__(kWarps * 32) k_adjoint_a2(const TravParams<T> p) {
    const int lane = threadIdx.x & 31;
    const int64_t qi = ((int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5)) * 32 + lane;
    if (__all_sync(kFull, qi >= p.nq)) return;
    Lane<T> L;
    int64_t oidx;
    T w;
    const bool valid = load_query(p, qi, L, oidx, w);
    T gs[3] = {T(0), T(0), T(0)};
    if (valid)
        for (int k = 0; k < 3; k++) gs[k] = p.g[oidx * 3 + k];
    const T G[3] = {gs[0] * exp_t(L.q0 * T(0.5)), gs[1] * exp_t(L.q1 * T(0.5)),
                    gs[2] * exp_t(L.q2 * T(0.5))};
    const T ew = CONT ? exp_t(w) : T(0);
    double vm = 0.0;                          // pass 1: this lane's largest warp sum
    const double sc = PASS1 ? 0.0 : *p.scale;  // pass 2: the fixed-point scale

    const int M = (int)p.M;
    const T* __restrict__ rec = p.rec[0];
    int kd = valid ? 0 : -1;
    int n = 0;
    while (n < M) {
        const int4 mt = __ldg(p.meta + n);
        const int d = node_depth(mt);
        const bool leaf = node_leaf(mt);
        const T* r = rec + (int64_t)n * CAGR_REC_STRIDE;
        const Vec4<T> r0 = ld4(r);
        T dx = sub_rn(L.q0, r0.x);
        T dy = sub_rn(L.q1, r0.y);
        T dz = sub_rn(L.q2, r0.z);
        T d2 = dist2_exact(dx, dy, dz);
        const bool active = d <= kd;
        const bool far = d2 > rec_radius2(r0.w);
        const bool open = active && !far;
        if (active) kd = (open && !leaf) ? d + 1 : d;
        const bool any_open = __any_sync(kFull, open);
        if (mt.z == -1) {
            // one-point leaf: the node record for far lanes, the point for near ones
            const bool use_pt = open && !rec_same_leaf(r0.w);
            const T* src = r;
            if (use_pt) {
                src = rec + ((int64_t)M + mt.y) * CAGR_REC_STRIDE;
                const Vec4<T> s0 = ld4(src);
                dx = sub_rn(L.q0, s0.x);
                dy = sub_rn(L.q1, s0.y);
                dz = sub_rn(L.q2, s0.z);
                d2 = dist2_exact(dx, dy, dz);
            }
            T v[3];
            adj_term<T, CONT>(L, src, dx, dy, dz, d2, G, gs, ew, v);
            warp_red3<PASS1>(active && !use_pt, v[0], v[1], v[2], p.accn + (int64_t)n * 3, vm, sc);
            warp_red3<PASS1>(active && use_pt, v[0], v[1], v[2], p.accp + (int64_t)mt.y * 3, vm, sc);
            n = mt.x;
            continue;
        }
        {
            T v[3];
            adj_term<T, CONT>(L, r, dx, dy, dz, d2, G, gs, ew, v);
            warp_red3<PASS1>(active && far, v[0], v[1], v[2], p.accn + (int64_t)n * 3, vm, sc);
        }
        if (leaf) {
            const int np = -mt.z;
            if (any_open) {
                const T* pr = rec + ((int64_t)M + mt.y) * CAGR_REC_STRIDE;
                for (int j = 0; j < np; j++, pr += CAGR_REC_STRIDE) {
                    const Vec4<T> s0 = ld4(pr);
                    const T ex = sub_rn(L.q0, s0.x);
                    const T ey = sub_rn(L.q1, s0.y);
                    const T ez = sub_rn(L.q2, s0.z);
                    T v[3];
                    adj_term<T, CONT>(L, pr, ex, ey, ez, dist2_exact(ex, ey, ez), G, gs, ew, v);
                    warp_red3<PASS1>(open, v[0], v[1], v[2], p.accp + ((int64_t)mt.y + j) * 3, vm,
                                     sc);
                }
            }
            n = mt.x;
        } else {
            n = any_open ? n + 1 : mt.x;
        }
    }
    if constexpr (PASS1) {
        // one atomic per warp (the bits of a non-negative double order as its value)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vm = fmax(vm, __shfl_xor_sync(kFull, vm, o));
        if (lane == 0) atomicMax(p.vmax, (unsigned long long)__double_as_longlong(vm));
    }
}

// per leaf: the sum of its and its ancestors' node vectors, added to each of
// its points' own vector (all in the fixed point, exactly), converted once and
// written in original point order
template <typename T>
__global__ void k_adj_push(const int32_t* __restrict__ leaf_ids, int64_t num_leaves,
                           const int4* __restrict__ meta, const int32_t* __restrict__ parent,
                           const int32_t* __restrict__ perm,
                           const unsigned long long* __restrict__ accn,
                           const unsigned long long* __restrict__ accp,
                           const double* __restrict__ scale, T* __restrict__ grad) {
    const int64_t li = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= num_leaves) return;
    const double sc = *scale;
    const double inv = sc > 0.0 ? 1.0 / sc : (double)NAN;  // a power of two: exact
    const int leafn = leaf_ids[li];
    unsigned long long s0 = 0, s1 = 0, s2 = 0;
    for (int n = leafn; n >= 0; n = parent[n]) {
        s0 += accn[(int64_t)n * 3];
        s1 += accn[(int64_t)n * 3 + 1];
        s2 += accn[(int64_t)n * 3 + 2];
    }
    const int4 lm = meta[leafn];
    const int np = node_npts(lm);
    for (int j = 0; j < np; j++) {
        const int64_t s = (int64_t)lm.y + j;
        const int64_t pt = perm[s];
        grad[pt * 3] = (T)((double)(long long)(accp[s * 3] + s0) * inv);
        grad[pt * 3 + 1] = (T)((double)(long long)(accp[s * 3 + 1] + s1) * inv);
        grad[pt * 3 + 2] = (T)((double)(long long)(accp[s * 3 + 2] + s2) * inv);
    }
}

template <typename T>
int adjoint_impl(const Tree* t, const TraverseArgs& a, const void* grad, void* grad_attrs,
                 cudaStream_t s) {
    TravParams<T> p;
    p.M = t->m;
    p.N = t->n;
    p.nq = t->n;
    p.meta = t->meta;
    p.spos = (const T*)t->spos;
    p.perm = t->perm;
    p.qgroup = t->qgroup;  // Hilbert grouping: 3.42 -> 3.29 ms at 1M points
    p.widths = (const T*)a.widths;
    p.width = (T)a.width;
    for (int k = 0; k < 3; k++) p.rec[k] = (const T*)t->rec[0];
    p.g = (const T*)grad;
    if (p.nq == 0) return kOk;
    const size_t bn = sizeof(unsigned long long) * 3 * (size_t)t->m;
    const size_t bp = sizeof(unsigned long long) * 3 * (size_t)t->n;
    void *accn = nullptr, *accp = nullptr, *aux = nullptr;
    int rc = pool_alloc(&accn, bn, s);
    if (!rc) rc = pool_alloc(&accp, bp, s);
    if (!rc) rc = pool_alloc(&aux, 16, s);  // vmax bits, scale
    if (!rc) {
        p.accn = (unsigned long long*)accn;
        p.accp = (unsigned long long*)accp;
        p.vmax = (unsigned long long*)aux;
        p.scale = (const double*)((char*)aux + 8);
        cudaMemsetAsync(accn, 0, bn, s);
        cudaMemsetAsync(accp, 0, bp, s);
        cudaMemsetAsync(aux, 0, 16, s);
        const int64_t nwarps = (p.nq + 31) / 32;
        const int64_t blocks = (nwarps + kWarps - 1) / kWarps;
        // an accumulator gets at most one sum per warp; a point adds its own and
        // its ancestors' (at most CAGR_MAX_DEPTH + 2 accumulators)
        const double bound = (double)nwarps * (CAGR_MAX_DEPTH + 2);
        if (a.continuous) {
            k_adjoint_a2<T, true, true><<<(unsigned)blocks, kWarps * 32, 0, s>>>(p);
            k_adj_scale<<<1, 1, 0, s>>>(p.vmax, bound, (double*)p.scale);
            k_adjoint_a2<T, true, false><<<(unsigned)blocks, kWarps * 32, 0, s>>>(p);
        } else {
            k_adjoint_a2<T, false, true><<<(unsigned)blocks, kWarps * 32, 0, s>>>(p);
            k_adj_scale<<<1, 1, 0, s>>>(p.vmax, bound, (double*)p.scale);
            k_adjoint_a2<T, false, false><<<(unsigned)blocks, kWarps * 32, 0, s>>>(p);
        }
        k_adj_push<T><<<(unsigned)((t->num_leaves + 255) / 256), 256, 0, s>>>(
            t->leaf_ids, t->num_leaves, t->meta, t->parent, t->perm, p.accn, p.accp, p.scale,
            (T*)grad_attrs);
        if (cudaGetLastError() != cudaSuccess) rc = set_error(kErrCuda, "adjoint launch");
    }
    pool_free(accn, s);
    pool_free(accp, s);
    pool_free(aux, s);
    return rc;
}


// ---- b's window table for a schedule of widths -------------------------------
//
// The CAGR solve forms sum_k A2Tk(b) at the widths w_i = base * s_i of its
// steepest-descent steps (main_CAGR.py:98,108), b constant.  The acceptance
// decisions do not depend on the width, and a term is kept at width w iff
// sqrt_rn(r^2) >= w (the reference's test), so one walk over b's moments can
// serve every step: each of b's terms with r < w_hi (w_hi = base * s_max; the
// terms beyond are the same at every step and summed once, at w_hi) goes to
// the bucket of the number of step widths it passes; out[i] is then the sum of
// the buckets of the steps >= i (scales ascending), i.e. exactly b's terms at
// w_i below w_hi.  Each query's buckets are a row of `rows` [nq][S*3] owned by
// its lane (no atomics), zeroed by the caller.
template <typename T>
__device__ __forceinline__ void b_bucket(T* row, const T* sc, int S, T base, T twh, const T* ex,
                                         const Vec4<T>& r1, T dx, T dy, T dz, T d2) {
    if (!(d2 < twh)) return;  // r >= w_hi: kept at every step, summed at w_hi
    const T r = sqrt_rn(d2);
    int lo = 0, hi = S;       // number of i with base * s_i <= r (s ascending)
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (mul_rn(base, sc[mid]) <= r) lo = mid + 1;
        else hi = mid;
    }
    if (lo == 0) return;      // kept at no step
    const T rinv = rsqrt_t(d2);
    const T rinv3 = rinv * rinv * rinv;
    const T hr = T(0.5) * rinv;
    const T g0 = ex[0] * r1.x * r1.w, g1 = ex[1] * r1.y * r1.w, g2 = ex[2] * r1.z * r1.w;
    const T c = (g0 + g1 + g2) * rinv3;
    T* b = row + (lo - 1) * 3;
    b[0] += dx * c + g0 * hr;
    b[1] += dy * c + g1 * hr;
    b[2] += dz * c + g2 * hr;
}

template <typename T>
__global__ void __launch_bounds__(kWarps * 32) k_b_window(const TravParams<T> p, const T* base,
                                                          const T* scales, int S, T* rows,
                                                          T* out) {
    __shared__ T sc[64];
    for (int i = threadIdx.x; i < S; i += blockDim.x) sc[i] = scales[i];
    __syncthreads();
    const int64_t qi = lane_query();
    if (__all_sync(kFull, qi >= p.nq)) return;
    Lane<T> L;
    int64_t oidx;
    T w;
    const bool valid = load_query(p, qi, L, oidx, w);
    const T bq = valid ? base[oidx] : T(0);
    const T twh = valid ? width_threshold(mul_rn(bq, sc[S - 1])) : T(0);
    T* row = rows + (valid ? oidx : 0) * (int64_t)S * 3;
    const T ex[3] = {exp_t(L.q0 * T(0.5)), exp_t(L.q1 * T(0.5)), exp_t(L.q2 * T(0.5))};
    const int M = (int)p.M;
    const T* __restrict__ rec = p.rec[1];
    int kd = valid ? 0 : -1;
    int n = 0;
    while (n < M) {
        const int4 mt = __ldg(p.meta + n);
        const int d = node_depth(mt);
        const bool leaf = node_leaf(mt);
        const T* r = rec + (int64_t)n * CAGR_REC_STRIDE;
        const Vec4<T> r0 = ld4(r);
        T dx = sub_rn(L.q0, r0.x);
        T dy = sub_rn(L.q1, r0.y);
        T dz = sub_rn(L.q2, r0.z);
        T d2 = dist2_exact(dx, dy, dz);
        const bool active = d <= kd;
        const bool far = d2 > rec_radius2(r0.w);
        const bool open = active && !far;
        if (active) kd = (open && !leaf) ? d + 1 : d;
        const bool any_open = __any_sync(kFull, open);
        const T* src = r;
        if (leaf && open) {
            src = rec + ((int64_t)M + mt.y) * CAGR_REC_STRIDE;
            const Vec4<T> s0 = ld4(src);
            dx = sub_rn(L.q0, s0.x);
            dy = sub_rn(L.q1, s0.y);
            dz = sub_rn(L.q2, s0.z);
            d2 = dist2_exact(dx, dy, dz);
        }
        if (active && (far || leaf) && d2 < twh)
            b_bucket(row, sc, S, bq, twh, ex, ld4(src + 4), dx, dy, dz, d2);
        if (leaf) {
            const int np = -mt.z;
            if (np > 1 && any_open) {
                const T* pr = rec + ((int64_t)M + mt.y + 1) * CAGR_REC_STRIDE;
                for (int j = 1; j < np; j++, pr += CAGR_REC_STRIDE) {
                    if (open) {
                        const Vec4<T> s0 = ld4(pr);
                        const T px = sub_rn(L.q0, s0.x);
                        const T py = sub_rn(L.q1, s0.y);
                        const T pz = sub_rn(L.q2, s0.z);
                        const T pd2 = dist2_exact(px, py, pz);
                        if (pd2 < twh) b_bucket(row, sc, S, bq, twh, ex, ld4(pr + 4), px, py, pz, pd2);
                    }
                }
            }
            n = mt.x;
        } else {
            n = any_open ? n + 1 : mt.x;
        }
    }
    if (!valid) return;
    // out[i] = sum of the buckets of the steps >= i: the exp(x/2) factors are in g
    T a0 = T(0), a1 = T(0), a2 = T(0);
    const int64_t stride = p.nq * 3;
    for (int i = S - 1; i >= 0; i--) {
        a0 += row[i * 3];
        a1 += row[i * 3 + 1];
        a2 += row[i * 3 + 2];
        T* o = out + i * stride + oidx * 3;
        o[0] = a0;
        o[1] = a1;
        o[2] = a2;
    }
}

template <typename T>
int b_window_impl(const Tree* t, const void* base, const void* scales, int S, void* out,
                  cudaStream_t s) {
    if (!t->rec[1] || t->rec_dim[1] != 1)
        return set_error(kErrState, "b's window table needs b's moments in slot 1");
    TravParams<T> p;
    p.M = t->m;
    p.N = t->n;
    p.nq = t->n;
    p.meta = t->meta;
    p.spos = (const T*)t->spos;
    p.perm = t->perm;
    p.qgroup = t->qgroup;
    p.rec[1] = (const T*)t->rec[1];
    p.width = T(0);
    void* rows = nullptr;
    const size_t row_bytes = sizeof(T) * (size_t)t->n * S * 3;
    if (int rc = pool_alloc(&rows, row_bytes, s)) return rc;
    int rc = kOk;
    if (cudaMemsetAsync(rows, 0, row_bytes, s) != cudaSuccess) {
        rc = set_error(kErrCuda, "window table scratch");
    } else {
        const int64_t blocks = ((t->n + 31) / 32 + kWarps - 1) / kWarps;
        k_b_window<T><<<(unsigned)blocks, kWarps * 32, 0, s>>>(p, (const T*)base, (const T*)scales,
                                                               S, (T*)rows, (T*)out);
        if (cudaGetLastError() != cudaSuccess) rc = set_error(kErrCuda, "window table launch");
    }
    pool_free(rows, s);
    return rc;
}
}  // namespace

int traverse(const Tree* t, const TraverseArgs& a, cudaStream_t stream) {
    if (!a.out) return set_error(kErrInvalid, "output is null");
    if (a.queries && a.nq < 0) return set_error(kErrInvalid, "negative query count");
    if (!a.widths && !(a.width == a.width)) return set_error(kErrInvalid, "width is NaN");
    if (a.grid && (a.queries || a.qorder || a.gx <= 0 || a.gy <= 0 || a.gz <= 0 ||
                   a.gx > (1 << 20) || a.gy > (1 << 20) || a.gz > (1 << 20)))
        return set_error(kErrInvalid, "grid queries need positive dims <= 2^20 and no query array");
    if (a.qorder && !a.queries)
        return set_error(kErrInvalid, "a query order needs explicit queries");
    if (a.widths_hi && !(a.op == kOpA2TFused && a.slots == 4))
        return set_error(kErrInvalid, "upper widths apply to the A2T right-hand side only");
    return t->dtype == 0 ? dispatch<float>(t, a, stream) : dispatch<double>(t, a, stream);
}

int b_window_table(const Tree* t, const void* base, const void* scales, int S, void* out,
                   cudaStream_t stream) {
    if (S < 1 || S > 64) return set_error(kErrInvalid, "1 to 64 scales");
    if (!base || !scales || !out) return set_error(kErrInvalid, "null buffer");
    return t->dtype == 0 ? b_window_impl<float>(t, base, scales, S, out, stream)
                         : b_window_impl<double>(t, base, scales, S, out, stream);
}

int adjoint(const Tree* t, const TraverseArgs& a, const void* grad, void* grad_attrs,
            cudaStream_t stream) {
    if (a.op != kOpA2Fused) return set_error(kErrInvalid, "the adjoint covers the fused A2 only");
    if (!t->rec[0] || t->rec_dim[0] != 3)
        return set_error(kErrState, "the adjoint needs the forward's [n,3] moments in slot 0");
    if (!a.widths && !(a.width == a.width)) return set_error(kErrInvalid, "width is NaN");
    return t->dtype == 0 ? adjoint_impl<float>(t, a, grad, grad_attrs, stream)
                         : adjoint_impl<double>(t, a, grad, grad_attrs, stream);
}

}  // namespace cagr
