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
//    L1 wavefront), and control flow stays uniform across the warp.
//  * Each query keeps exactly its own reference acceptance decisions through a
//    per-depth lane mask in shared memory: mask[d+1] = the lanes that opened the
//    depth-d ancestor.  A lane contributes at a node only if it is in the mask
//    for that depth; far lanes add the node term, near lanes descend, and at a
//    leaf near lanes add the leaf's points.  The set of pair terms per query is
//    therefore the reference's set; only the summation order differs.
//  * Acceptance and width tests use the reference's rounding (see common.cuh),
//    so they are decided bit-identically; the inner loop compares squared
//    distances and needs one rsqrt per pair.
//  * exp((x-y)_k/2) = exp(x_k/2) * exp(-y_k/2): the second factor is stored in
//    every source record, the first is per query and applied once at the end,
//    so a pair term costs no transcendental beyond the rsqrt.
//  * A2Fused evaluates A21, A22, A23 in one walk (they share node moments and
//    acceptance decisions in the reference, which walks three times).
#include <string>

#include "internal.h"

namespace cagr {
namespace {

constexpr int kWarps = 4;  // warps per block
constexpr unsigned kFull = 0xffffffffu;

template <typename T>
struct TravParams {
    int64_t M = 0, N = 0, nq = 0;
    const int4* meta = nullptr;
    const T* rec = nullptr;
    const T* rec1 = nullptr;   // A2TFused: slot 1
    const T* rec2 = nullptr;   // A2TFused: slot 2
    const T* spos = nullptr;   // sorted tree points (queries == points)
    const int32_t* perm = nullptr;
    const T* queries = nullptr;
    const int32_t* qorder = nullptr;
    const T* widths = nullptr;
    T width = T(0);
    T* out = nullptr;
    int out_stride = 1;
};

template <int OP>
struct OpInfo {
    static constexpr bool a2 = OP == kOpA21 || OP == kOpA22 || OP == kOpA23 || OP == kOpA3 ||
                               OP == kOpA2Fused;
    static constexpr bool a2t = OP == kOpA2T1 || OP == kOpA2T2 || OP == kOpA2T3;
    static constexpr bool uses_exp = a2 || a2t;
    // which convection direction a single-direction operator uses
    static constexpr int k [[maybe_unused]] = (OP == kOpA21 || OP == kOpA2T1)   ? 0
                             : (OP == kOpA22 || OP == kOpA2T2) ? 1
                             : (OP == kOpA23 || OP == kOpA2T3) ? 2
                                                               : -1;
};

// Per-lane state of one query.
template <typename T>
struct Lane {
    T q0, q1, q2;
    T tw;                 // width threshold on r^2 (r >= w  <=>  r^2 >= tw)
    T iw, iw3;            // 1/w, 1/w^3 (continuous kernel inside the width)
    T acc0, acc1, acc2;   // outside-width sums (without the per-query exp factor)
    T in0, in1, in2;      // inside-width sums (continuous kernel)
};

// One pair term.  d = x - y, d2 = |d|^2 (reference rounding), src = record.
template <typename T, int OP, bool CONT>
__device__ __forceinline__ void pair_term(Lane<T>& L, const T* __restrict__ src, T dx, T dy, T dz,
                                          T d2) {
    const bool outside = d2 >= L.tw;
    const T rinv = rsqrt_t(d2);
    const T rinv3 = rinv * rinv * rinv;
    if constexpr (OP == kOpA || OpInfo<OP>::a2 || OP == kOpG) {
        const T m0 = src[REC_A0], m1 = src[REC_A1], m2 = src[REC_A2];
        const T dm = dx * m0 + dy * m1 + dz * m2;
        if constexpr (OP == kOpA) {
            if (outside) L.acc0 += dm * rinv3;
            else if (CONT) L.in0 += dm * L.iw3;
        } else if constexpr (OP == kOpG) {
            if (outside) {
                const T rinv5 = rinv3 * rinv * rinv;
                const T c = T(3) * dm * rinv5;
                L.acc0 += m0 * rinv3 - dx * c;
                L.acc1 += m1 * rinv3 - dy * c;
                L.acc2 += m2 * rinv3 - dz * c;
            }
        } else {
            // A2k: exp(d_k/2) (dm / r^3 + m_k / (2r)); continuous inside:
            // exp(w) (dm / w^3 + m_k / (2w))
            if (outside) {
                const T t = dm * rinv3;
                const T h = T(0.5) * rinv;
                constexpr int k = OpInfo<OP>::k;
                if constexpr (k == 0 || OP == kOpA3 || OP == kOpA2Fused)
                    L.acc0 += src[REC_E1] * (t + h * m0);
                if constexpr (k == 1 || OP == kOpA3 || OP == kOpA2Fused)
                    L.acc1 += src[REC_E2] * (t + h * m1);
                if constexpr (k == 2 || OP == kOpA3 || OP == kOpA2Fused)
                    L.acc2 += src[REC_E3] * (t + h * m2);
            } else if (CONT) {
                const T t = dm * L.iw3;
                const T h = T(0.5) * L.iw;
                constexpr int k = OpInfo<OP>::k;
                if constexpr (k == 0 || OP == kOpA3 || OP == kOpA2Fused) L.in0 += t + h * m0;
                if constexpr (k == 1 || OP == kOpA3 || OP == kOpA2Fused) L.in1 += t + h * m1;
                if constexpr (k == 2 || OP == kOpA3 || OP == kOpA2Fused) L.in2 += t + h * m2;
            }
        }
    } else if constexpr (OP == kOpAT) {
        if (outside) {
            const T c = src[REC_A0] * rinv3;
            L.acc0 += dx * c;
            L.acc1 += dy * c;
            L.acc2 += dz * c;
        }
    } else if constexpr (OpInfo<OP>::a2t) {
        // exp(d_k/2) (d s / r^3 + e_k s / (2r)); no continuous branch (:293-299)
        if (outside) {
            constexpr int k = OpInfo<OP>::k;
            const T s = src[REC_A0];
            const T e = src[REC_E1 + k];
            const T c = e * s * rinv3;
            L.acc0 += dx * c;
            L.acc1 += dy * c;
            L.acc2 += dz * c;
            const T h = e * s * T(0.5) * rinv;
            if constexpr (k == 0) L.acc0 += h;
            if constexpr (k == 1) L.acc1 += h;
            if constexpr (k == 2) L.acc2 += h;
        }
    }
}

template <typename T, int OP, bool CONT>
__global__ void __launch_bounds__(kWarps * 32) k_traverse(const TravParams<T> p) {
    __shared__ unsigned smask[kWarps][CAGR_MAX_DEPTH + 2];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int64_t qi = ((int64_t)blockIdx.x * kWarps + wid) * 32 + lane;
    const bool valid = qi < p.nq;
    const unsigned vmask = __ballot_sync(kFull, valid);
    if (vmask == 0) return;  // whole warp past the end

    // this lane's query
    int64_t oidx = 0;
    Lane<T> L;
    T w = p.width;
    L.q0 = L.q1 = L.q2 = T(0);
    if (valid) {
        if (p.queries == nullptr) {
            oidx = p.perm[qi];
            L.q0 = p.spos[3 * qi];
            L.q1 = p.spos[3 * qi + 1];
            L.q2 = p.spos[3 * qi + 2];
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

    unsigned* sm = smask[wid];
    if (lane == 0) sm[0] = vmask;
    __syncwarp();

    const int64_t M = p.M;
    const T* __restrict__ rec = p.rec;
    int n = 0;
    while (n < M) {
        const int4 mt = p.meta[n];
        const int depth = meta_depth(mt.w);
        const bool leaf = meta_leaf(mt.w);
        const bool active = (sm[depth] >> lane) & 1u;
        const T* r = rec + (int64_t)n * CAGR_REC_STRIDE;
        T dx = sub_rn(L.q0, r[REC_X]);
        T dy = sub_rn(L.q1, r[REC_Y]);
        T dz = sub_rn(L.q2, r[REC_Z]);
        T d2 = dist2_exact(dx, dy, dz);
        const bool far = d2 > mac_radius2<T>(depth);
        const bool open = active && !far;
        const unsigned omask = __ballot_sync(kFull, open);
        if (leaf && mt.z == 1) {
            // single-point leaf: far lanes use the node term, near lanes the point
            const T* src = r;
            if (open) {
                src = rec + (M + mt.y) * CAGR_REC_STRIDE;
                dx = sub_rn(L.q0, src[REC_X]);
                dy = sub_rn(L.q1, src[REC_Y]);
                dz = sub_rn(L.q2, src[REC_Z]);
                d2 = dist2_exact(dx, dy, dz);
            }
            if (active) pair_term<T, OP, CONT>(L, src, dx, dy, dz, d2);
            n = mt.x;
            continue;
        }
        if (active && far) pair_term<T, OP, CONT>(L, r, dx, dy, dz, d2);
        if (leaf) {
            if (omask) {
                const T* pr = rec + (M + mt.y) * CAGR_REC_STRIDE;
                for (int j = 0; j < mt.z; j++, pr += CAGR_REC_STRIDE) {
                    if (open) {
                        const T ex = sub_rn(L.q0, pr[REC_X]);
                        const T ey = sub_rn(L.q1, pr[REC_Y]);
                        const T ez = sub_rn(L.q2, pr[REC_Z]);
                        pair_term<T, OP, CONT>(L, pr, ex, ey, ez, dist2_exact(ex, ey, ez));
                    }
                }
            }
            n = mt.x;
        } else if (omask) {
            if (lane == 0) sm[depth + 1] = omask;
            __syncwarp();
            n = n + 1;
        } else {
            n = mt.x;
        }
    }

    if (!valid) return;
    T* o = p.out + oidx * (int64_t)p.out_stride;
    if constexpr (OpInfo<OP>::uses_exp) {
        const T ex0 = exp_t(L.q0 * T(0.5)), ex1 = exp_t(L.q1 * T(0.5)), ex2 = exp_t(L.q2 * T(0.5));
        const T ew = CONT ? exp_t(w) : T(0);
        const T v0 = ex0 * L.acc0 + ew * L.in0;
        const T v1 = ex1 * L.acc1 + ew * L.in1;
        const T v2 = ex2 * L.acc2 + ew * L.in2;
        if constexpr (OP == kOpA21) o[0] = v0;
        if constexpr (OP == kOpA22) o[0] = v1;
        if constexpr (OP == kOpA23) o[0] = v2;
        if constexpr (OP == kOpA3) o[0] = (v0 + v1 + v2) / T(3);
        if constexpr (OP == kOpA2Fused) {
            o[0] = v0;
            o[1] = v1;
            o[2] = v2;
        }
        if constexpr (OpInfo<OP>::a2t) {
            constexpr int k = OpInfo<OP>::k;
            const T ek = k == 0 ? ex0 : (k == 1 ? ex1 : ex2);
            o[0] = ek * L.acc0;
            o[1] = ek * L.acc1;
            o[2] = ek * L.acc2;
        }
    } else if constexpr (OP == kOpA) {
        o[0] = L.acc0 + L.in0;
    } else {
        o[0] = L.acc0;
        o[1] = L.acc1;
        o[2] = L.acc2;
    }
}

template <typename T, int OP>
int launch_op(const TravParams<T>& p, int cont, cudaStream_t s) {
    const int64_t warps = (p.nq + 31) / 32;
    const int64_t blocks = (warps + kWarps - 1) / kWarps;
    if (blocks > 0x7fffffffLL) return set_error(kErrInvalid, "too many queries");
    if (cont)
        k_traverse<T, OP, true><<<(unsigned)blocks, kWarps * 32, 0, s>>>(p);
    else
        k_traverse<T, OP, false><<<(unsigned)blocks, kWarps * 32, 0, s>>>(p);
    CAGR_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int dispatch(const Tree* t, const TraverseArgs& a, cudaStream_t s) {
    TravParams<T> p;
    p.M = t->m;
    p.N = t->n;
    p.nq = a.queries ? a.nq : t->n;
    p.meta = t->meta;
    p.spos = (const T*)t->spos;
    p.perm = t->perm;
    p.queries = (const T*)a.queries;
    p.qorder = a.qorder;
    p.widths = (const T*)a.widths;
    p.width = (T)a.width;
    p.out = (T*)a.out;
    const bool vec_in = a.op == kOpAT || a.op == kOpA2T1 || a.op == kOpA2T2 || a.op == kOpA2T3;
    const int need_dim = vec_in ? 1 : 3;
    const int slot = 0;
    if (!t->rec[slot] || t->rec_dim[slot] != need_dim)
        return set_error(kErrState, "node moments of the right attribute dim are not computed");
    p.rec = (const T*)t->rec[slot];
    int out_dim = (a.op == kOpA || a.op == kOpA3 || a.op == kOpA21 || a.op == kOpA22 ||
                   a.op == kOpA23)
                      ? 1
                      : 3;
    p.out_stride = a.out_stride > 0 ? a.out_stride : out_dim;
    if (p.nq == 0) return kOk;
    switch (a.op) {
        case kOpA: return launch_op<T, kOpA>(p, a.continuous, s);
        case kOpAT: return launch_op<T, kOpAT>(p, 0, s);
        case kOpA3: return launch_op<T, kOpA3>(p, a.continuous, s);
        case kOpA21: return launch_op<T, kOpA21>(p, a.continuous, s);
        case kOpA22: return launch_op<T, kOpA22>(p, a.continuous, s);
        case kOpA23: return launch_op<T, kOpA23>(p, a.continuous, s);
        case kOpA2T1: return launch_op<T, kOpA2T1>(p, 0, s);
        case kOpA2T2: return launch_op<T, kOpA2T2>(p, 0, s);
        case kOpA2T3: return launch_op<T, kOpA2T3>(p, 0, s);
        case kOpG: return launch_op<T, kOpG>(p, 0, s);
        case kOpA2Fused: return launch_op<T, kOpA2Fused>(p, a.continuous, s);
        default: return set_error(kErrInvalid, "unknown operator " + std::to_string(a.op));
    }
}

}  // namespace

int traverse(const Tree* t, const TraverseArgs& a, cudaStream_t stream) {
    if (!a.out) return set_error(kErrInvalid, "output is null");
    if (a.queries && a.nq < 0) return set_error(kErrInvalid, "negative query count");
    if (!a.widths && !(a.width == a.width)) return set_error(kErrInvalid, "width is NaN");
    return t->dtype == 0 ? dispatch<float>(t, a, stream) : dispatch<double>(t, a, stream);
}

}  // namespace cagr
