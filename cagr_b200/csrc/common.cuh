// Shared definitions for the CAGR treecode library (sm_100a).
//
// Layout in HBM (one tree, N points, M nodes, nodes numbered in preorder
// exactly as the reference serialiser numbers them):
//   perm[N]        int32  Morton-sorted position -> original point index
//   meta[M]        int4   {next (preorder skip pointer), pstart (first sorted
//                          position covered), npts (points under the node,
//                          negated for a leaf), depth}
//   nchild[M]      uint8  number of children
//   parent[M]      int32  parent id (-1 for the root)
//   children[M*8]  int32  child ids in octant order (-1 = none)
//   leaf_ids[NL]   int32  leaf node ids in preorder
//   rec[(M+N)*12]  T      source records, three 4-vectors each:
//                          node  i < M  : (cx, cy, cz, (4 half_w)^2)
//                                         (e1, e2, e3, a0) (a1, a2, W, 0)
//                          point M + s  : (x, y, z, 0) (e1, e2, e3, a0) (a1, a2, w, 0)
//                          with c the weighted centroid, e_k = exp(-c_k / 2)
//                          (resp. exp(-y_k / 2)), a the attribute (sum) and W / w
//                          the weight; points in Morton order.  Rewritten by every
//                          moment pass; one array per moment slot.
//   counters[M]    uint32 arrival counters for the bottom-up moment pass
//                          (self-resetting).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define CAGR_MAX_DEPTH 21
#define CAGR_REC_STRIDE 12  // scalars per source record

namespace cagr {

// Status codes returned by every extern "C" entry point (mirrored in include/cagr.h).
enum Status : int {
    kOk = 0,
    kErrInvalid = 1,
    kErrCuda = 2,
    kErrAlloc = 3,
    kErrOverflow = 4,
    kErrState = 5,
};

__host__ __device__ inline bool node_leaf(const int4& m) { return m.z < 0; }
__host__ __device__ inline int node_npts(const int4& m) { return m.z < 0 ? -m.z : m.z; }
__host__ __device__ inline int node_depth(const int4& m) { return m.w & 0xff; }
// A node record's r0.w is its acceptance radius (4 half_w)^2, negated for a
// one-point leaf whose centroid equals its point bit for bit (then the node
// record and the point record give identical pair terms).
template <typename T>
__device__ __forceinline__ T rec_radius2(T r0w) { return fabs(r0w); }
template <typename T>
__device__ __forceinline__ bool rec_same_leaf(T r0w) { return r0w < T(0); }
// internal node whose children are all one-point leaves: children n+1 .. n+npts,
// child c holding sorted point pstart + c
__host__ __device__ inline bool node_twig(const int4& m) { return (m.w >> 8) & 1; }

// 4-vector of T and aligned loads of one record component.
template <typename T>
struct Vec4Of;
template <>
struct Vec4Of<float> {
    using type = float4;
};
template <>
struct Vec4Of<double> {
    using type = double4;
};
template <typename T>
using Vec4 = typename Vec4Of<T>::type;

template <typename T>
__device__ __forceinline__ Vec4<T> ld4(const T* p) {
    return *reinterpret_cast<const Vec4<T>*>(p);
}
template <typename T>
__device__ __forceinline__ void st4(T* p, Vec4<T> v) {
    *reinterpret_cast<Vec4<T>*>(p) = v;
}
// L2-coherent load (data written by other threads of the same launch)
__device__ __forceinline__ float4 ld4_cg(const float* p) {
    return __ldcg(reinterpret_cast<const float4*>(p));
}
__device__ __forceinline__ double4 ld4_cg(const double* p) {
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 make4(float a, float b, float c, float d) {
    return make_float4(a, b, c, d);
}
__device__ __forceinline__ double4 make4(double a, double b, double c, double d) {
    return make_double4(a, b, c, d);
}

// Squared distance in the reference's operation order: d = x - c per axis,
// then ((dx*dx + dy*dy) + dz*dz), each step rounded (no FMA contraction), so
// acceptance and width decisions match the reference bit for bit.
__device__ __forceinline__ float dist2_exact(float dx, float dy, float dz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}
__device__ __forceinline__ double dist2_exact(double dx, double dy, double dz) {
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float sqrt_rn(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double sqrt_rn(double a) { return __dsqrt_rn(a); }
// The hardware reciprocal square root as one instruction.  Inside the traversal
// its argument is a squared distance at or above the width threshold: a normal
// number (or +0, giving +inf as rsqrtf does), where the flush-to-zero form
// returns what rsqrtf returns while skipping rsqrtf's scaling of denormal
// inputs (measured: identical outputs, 5-7 % less time per traversal).  A
// denormal argument -- points closer than ~1e-19 yet not coincident -- would
// give +inf here instead of a finite value.
__device__ __forceinline__ float rsqrt_t(float a) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}
// 1/sqrt(a) in double: the hardware approximation rsqrt.approx.f64 (relative
// error about 2^-22), refined by one third-order step from the series
// (1 - e)^(-1/2) = 1 + e/2 + 3e^2/8 + O(e^3) with e = 1 - a y^2, which takes
// the error to the rounding level (measured within 2 ulp of CUDA's
// rsqrt(double), and 1.3e-16 relative on the traversals' outputs, while the
// FP64 walks run 6.46 -> 6.05 ms (A2T_SUM) and 3.41 -> 3.09 ms (A2_FUSED) at
// 1M points).  a = 0 and a = +inf give NaN (CUDA's rsqrt gives inf and 0):
// the traversals call it only for r^2 >= t(w) > 0, finite; with a width
// w <= 0 a query on its own point divides by zero in the reference too.
// (Keeping the approximation's exact 0 and inf by a select cost the whole
// gain.)
__device__ __forceinline__ double rsqrt_t(double a) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
    const double e = fma(-a * y, y, 1.0);
    return fma(y * e, fma(0.375, e, 0.5), y);
}
__device__ __forceinline__ float exp_t(float a) { return expf(a); }
__device__ __forceinline__ double exp_t(double a) { return exp(a); }

// Smallest t >= 0 with sqrt_rn(t) >= w, so that for any r2 computed with
// dist2_exact:  sqrt_rn(r2) >= w  <=>  r2 >= t.  The reference tests
// `sqrt(r2) >= w` (wn_treecode_cuda_kernels.cu:90,127); this lets the inner
// loop compare squares without losing bit-exactness of the decision.
template <typename T>
__device__ __forceinline__ T width_threshold(T w) {
    if (w != w) return T(INFINITY);  // NaN width: `r >= w` is false for every pair
    if (!(w > T(0))) return T(0);    // w <= 0: every pair passes `r >= w`
    T t = mul_rn(w, w);
    if (!(t < T(INFINITY))) return t;
    // walk down while the predecessor still satisfies the test, then up
    for (int it = 0; it < 8; it++) {
        T prev = nextafter(t, T(0));
        if (sqrt_rn(prev) >= w) t = prev;
        else break;
    }
    for (int it = 0; it < 8; it++) {
        if (sqrt_rn(t) >= w) break;
        t = nextafter(t, T(INFINITY));
    }
    return t;
}

// (4 * half_w)^2 for a node at `depth` (half_w = 2^-depth): the reference
// acceptance threshold `pow(4 * half_w, 2)` (wn_treecode_cuda_kernels.cu:595),
// exact in both precisions.
template <typename T>
__host__ __device__ __forceinline__ T mac_radius2(int depth) {
    return T(16.0) * ldexp(T(1.0), -2 * depth);
}
// The same power of two, 2^(4 - 2 depth), built directly from its exponent
// field (valid for depth <= CAGR_MAX_DEPTH): two integer instructions.
__device__ __forceinline__ float mac_radius2_bits(int depth, float) {
    return __int_as_float((131 - 2 * depth) << 23);
}
__device__ __forceinline__ double mac_radius2_bits(int depth, double) {
    return __longlong_as_double((long long)(1027 - 2 * depth) << 52);
}

// ---- shared-memory barriers and one-dimensional bulk copies (TMA) ----------
//
// A copy's completion is counted on an mbarrier as transaction bytes; a wait
// is a bounded number of try_wait rounds, so a kernel whose copy or peer never
// arrives sets an error flag and ends instead of spinning.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
// an mbarrier whose phase completes after `count` arrivals (and the bytes
// announced by arrivals with expect_tx)
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count = 1) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// one arrival that also announces `bytes` of copies completing on this phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// bytes from global src to shared dst (both 16-byte aligned, bytes a multiple
// of 16), counted on bar; the caller has announced them
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// before a copy overwrites shared memory that was read through the generic proxy
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// one copy on a barrier of one arrival: announce its bytes and start it
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes,
                                            uint64_t* bar) {
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, bytes);
    bulk_copy_g2s(dst, src, bytes, bar);
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// true once the phase of the given parity has completed; false after `spin` rounds
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t spin) {
    for (uint32_t it = 0; it < spin; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

}  // namespace cagr
