// Interpolated far field: the second evaluation mode of the treecode.
//
// The reference (mayueji/CAGR CUDA-based/ext/wn_treecode/wn_treecode_cuda/
// wn_treecode_cuda_kernels.cu:556-1322) approximates an accepted node by ONE
// term at its |attr|-weighted centroid, accepted per query when
// |x - c|^2 > (4 half_w)^2 (:595).  That is first order in the node size: on
// the 100k-point torus workload its field is off the FP64 direct sum by up to
// 0.4 (field values in [-17, 2.5]).  This mode evaluates the same operators --
// the exact pair sums the reference approximates -- with a far field whose
// error falls geometrically with its degree p:
//
//  * Far field: barycentric Lagrange interpolation of the pair kernel in the
//    source position on a (p+1)^3 grid of Chebyshev points of the second kind
//    spanning the node's tight bounding box (the barycentric Lagrange
//    treecode of L. Wang, R. Krasny and S. Tlupova, Commun. Comput. Phys. 28
//    (2020) 1415-1436).  A node's proxy charges are q_m = sum_j L_m(y_j) a_j
//    over its points; a query's interaction with the node is the same pair
//    kernel summed over the proxy points.  The convection factor exp(-y_k/2)
//    is smooth in y and is interpolated with the rest of the kernel, so a
//    proxy record is exactly a point record (position, exp(-position/2),
//    charges) and far and near sources run the same inner loop.
//  * Acceptance: ONE test per warp.  The warp's 32 queries (consecutive along
//    the Hilbert / Morton curve) form a batch with bounding centre b and
//    radius r_B; a node with box centre c and radius r_C is far when
//    r_C + theta r_B < theta |b - c| -- then r_C < theta |x - c| for every
//    query x of the batch, the interpolation's accuracy condition -- and no
//    pair can lie within a query's width (|b - c| - r_B - r_C >= the batch's
//    largest width), so only the smooth outside-width branch of the kernel is
//    interpolated.  Far nodes with fewer
//    than (p+1)^3 points are summed directly (exact, and fewer terms); near
//    nodes with at most direct_max points, and near leaves, are summed
//    directly with the per-pair width test of the reference kernels.  Every
//    decision is warp-uniform: no per-lane bookkeeping, and each source
//    record is loaded once per warp (one broadcast) and used by all 32 lanes.
//  * Precision: FP32 terms, plain sums within one interaction (one proxy grid
//    or one node's points), compensated (Kahan) accumulation of the
//    interactions per query; FP64 with the double build.
//  * Proxy charges: one block per chunk of <= kChunk points of an
//    interpolation node (a node with >= (p+1)^3 points), writing chunk
//    partials that a second kernel sums in chunk order (in double), so the
//    charges are the same bits on every run.
//
// Operators: A, AT, A3, A21..A23, A2T1..A2T3, G, A2_FUSED, A2T_SUM (the three
// scalar columns of cagr_scatter3 in one walk: the proxy grid is geometric, so
// the three directions share it), A2T_SUM_SHARED, COUNT.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <string>

#include "internal.h"

namespace cagr {

constexpr int kPMax = 9;          // degree <= 8
constexpr int kChunk = 2048;      // points per proxy-charge block
// Source records (points and proxies alike) are stored in pairs: records 2b
// and 2b + 1 form block b of kBlk scalars, component c of record 2b + h at
// block[2c + h], components (y0, y1, y2, q0, e0, e1, e2, q1, q2) = 0..8 (the
// position y, the charges q, e = exp(-y/2)), block[18..19] = 0.  A block is
// 80 bytes in float: five 16-byte loads give every component as an adjacent
// pair of registers, the operands of the packed f32x2 instructions that
// evaluate two records per instruction.
constexpr int kBlk = 20;
constexpr int kComp = 9;
// The A2T sum's walk layout: blocks of kBlkES scalars, components (y0, y1, y2,
// e0 s0, e1 s1, e2 s2) -- all its pair term reads of a source (48 bytes per
// record pair in float: three 16-byte loads).
constexpr int kBlkES = 12;
constexpr unsigned kAll = 0xffffffffu;
// the pipelined walk's shape (see k_iwalk)
#ifndef CAGR_IW_SLOTS
#define CAGR_IW_SLOTS 2
#endif
#ifndef CAGR_IW_TILE
#define CAGR_IW_TILE 4096
#endif
#ifndef CAGR_IW_WARPS
#define CAGR_IW_WARPS 4
#endif
#ifndef CAGR_IW_UNROLL
#define CAGR_IW_UNROLL 8
#endif
constexpr int kSlots = CAGR_IW_SLOTS;       // tiles in flight per warp
constexpr int kTileBytes = CAGR_IW_TILE;    // per tile (4096: 51 float / 25 double record pairs)
// (measured at 1M points, A2_FUSED walk, record pairs with packed arithmetic:
// 3 slots x 3072 B 25.8 ms, 4 x 3072 26.9, 3 x 4096 26.5, 2 x 4096 23.5,
// 2 x 6144 23.8, 2 x 8192 26.2; 2-warp blocks the same as 4; later, with the
// A2T-sum records in their walk form: unroll 8 / 4 / 2 terms 23.1 / 23.5 /
// 24.8 ms (A2_FUSED) and 22.3 / 22.7 / 23.1 ms (A2T sum), 8-warp blocks 23.8 /
// 24.6, 3 slots 26.6 / 23.4)
constexpr int kPWarps = CAGR_IW_WARPS;      // warps per block
constexpr int kUnroll = CAGR_IW_UNROLL;     // pair terms per inner-loop iteration
constexpr int kUnrollB = kUnroll > 1 ? kUnroll / 2 : 1;  // blocks (two terms each) per iteration
// internal operator codes beside Op: the A2T sums of the interpolated mode
constexpr int kIOpA2TSum = 100;     // sum_k A2Tk(s_k), three scalar columns (slot 3)
constexpr int kIOpA2TShared = 101;  // sum_k A2Tk(s), one scalar column

struct Interp {
    int degree = 5, P = 6, P3 = 216;
    double theta = 0.5;
    int direct_max = 64;
    int64_t num_interp = 0, num_chunks = 0;
    void* box_c = nullptr;         // [M*4] T: bounding-box centre, radius
    void* box_h = nullptr;         // [M*4] T: half extents, 0
    int32_t* iidx = nullptr;       // [M] proxy block of the node, -1 if it has < P3 points
    int4* chunks = nullptr;        // [num_chunks] {node, first sorted point, count, proxy block}
    int32_t* chunk_first = nullptr;  // [num_interp + 1]
    void* part = nullptr;          // [num_chunks * P3 * 4] T: chunk partial charges
    void* pts[4] = {nullptr, nullptr, nullptr, nullptr};   // [N*12] T point records per slot
    void* prox[4] = {nullptr, nullptr, nullptr, nullptr};  // [num_interp*P3*12] T proxy records
    int dim[4] = {0, 0, 0, 0};     // attribute dim held by the slot (0 = empty)
    void* ptsc = nullptr;          // slot 3 in the A2T sum's walk layout: points
    void* proxc = nullptr;         //   and proxy records
    double cheb[kPMax] = {}, omega[kPMax] = {};  // Chebyshev points and barycentric weights
    int* err = nullptr;            // device flag: a walk's staging wait ran out
    uint32_t spin = 1u << 22;      // try_wait rounds before a staging wait runs out
    // Self-query walks run their groups longest first: each walk records every
    // group's cost (record pairs summed), and the groups are sorted by it for the next.
    int64_t ngroups = 0;
    uint32_t* gcost = nullptr;     // [ngroups] record pairs of each group in the last self walk
    uint32_t* gcost_sorted = nullptr;
    int32_t* giota = nullptr;      // [ngroups] 0, 1, 2, ...
    int32_t* gorder = nullptr;     // [ngroups] groups, most expensive first
    void* gsort_tmp = nullptr;
    size_t gsort_bytes = 0;
    bool gorder_valid = false;
};

namespace {

// ---- tree geometry ----------------------------------------------------------

template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(kAll, v, o));
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kAll, v, o));
    return v;
}

// One warp per node: the tight bounding box of its points (a contiguous range
// of the Morton order).  Half extents are floored at 1e-3 of the largest (a
// flat node still spans a proper interpolation box); the radius is rounded up.
template <typename T>
__global__ void k_box(const int4* __restrict__ meta, const T* __restrict__ spos, int64_t M,
                      T* __restrict__ bc, T* __restrict__ bh) {
    const int64_t node = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (node >= M) return;  // uniform per warp
    const int4 mt = meta[node];
    const int np = node_npts(mt);
    T lo[3] = {T(INFINITY), T(INFINITY), T(INFINITY)};
    T hi[3] = {-T(INFINITY), -T(INFINITY), -T(INFINITY)};
    for (int j = lane; j < np; j += 32) {
        const T* y = spos + 3 * ((int64_t)mt.y + j);
        for (int a = 0; a < 3; a++) {
            lo[a] = fmin(lo[a], y[a]);
            hi[a] = fmax(hi[a], y[a]);
        }
    }
    for (int a = 0; a < 3; a++) {
        lo[a] = warp_min(lo[a]);
        hi[a] = warp_max(hi[a]);
    }
    if (lane == 0) {
        T c[3], h[3], hmax = T(0);
        for (int a = 0; a < 3; a++) {
            if (!(lo[a] <= hi[a])) lo[a] = hi[a] = T(0);  // no finite coordinate
            c[a] = T(0.5) * (lo[a] + hi[a]);
            // the box must hold every point: half extent from the farther end
            h[a] = fmax(hi[a] - c[a], c[a] - lo[a]);
            hmax = fmax(hmax, h[a]);
        }
        const T floor_h = fmax(hmax * T(1e-3), T(1e-30));
        for (int a = 0; a < 3; a++) h[a] = fmax(h[a], floor_h);
        const T r = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]) * T(1.0 + 1.0 / 65536);
        st4<T>(bc + 4 * node, make4(c[0], c[1], c[2], r));
        st4<T>(bh + 4 * node, make4(h[0], h[1], h[2], T(0)));
    }
}

__global__ void k_iflags(const int4* __restrict__ meta, int64_t M, int P3,
                         int32_t* __restrict__ flag, int32_t* __restrict__ nch) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    const int np = node_npts(meta[i]);
    const bool f = np >= P3;
    flag[i] = f ? 1 : 0;
    nch[i] = f ? (np + kChunk - 1) / kChunk : 0;
}

// iidx = proxy block (exclusive scan of the flags) or -1; chunk descriptors
__global__ void k_ichunks(const int4* __restrict__ meta, int64_t M, const int32_t* __restrict__ flag,
                          const int32_t* __restrict__ pos, const int32_t* __restrict__ chbase,
                          int32_t* __restrict__ iidx, int4* __restrict__ chunks,
                          int32_t* __restrict__ chunk_first) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    if (!flag[i]) {
        iidx[i] = -1;
        return;
    }
    const int ii = pos[i];
    iidx[i] = ii;
    const int4 mt = meta[i];
    const int np = node_npts(mt);
    const int cb = chbase[i];
    chunk_first[ii] = cb;
    for (int c = 0; c * kChunk < np; c++)
        chunks[cb + c] = make_int4((int)i, mt.y + c * kChunk, min(kChunk, np - c * kChunk), ii);
}

// ---- records and proxy charges ------------------------------------------------

// Writes record r (position y, charges q) into the paired layout; the record
// that ends an odd-sized array also writes its partner's half as zeros.
template <typename T>
__device__ __forceinline__ void write_rec(T* base, int64_t r, int64_t nrec, T y0, T y1, T y2, T q0,
                                          T q1, T q2) {
    T* b = base + (r >> 1) * kBlk + (r & 1);
    const T v[kComp] = {y0, y1, y2, q0, exp_t(y0 * T(-0.5)), exp_t(y1 * T(-0.5)),
                        exp_t(y2 * T(-0.5)), q1, q2};
#pragma unroll
    for (int c = 0; c < kComp; c++) b[2 * c] = v[c];
    b[18] = T(0);
    if ((r & 1) == 0 && r + 1 >= nrec)
        for (int c = 0; c < 10; c++) b[2 * c + 1] = T(0);
}
template <typename T>
__device__ __forceinline__ T rec_comp(const T* base, int64_t r, int c) {
    return base[(r >> 1) * kBlk + 2 * c + (r & 1)];
}

// Point records in Morton order, the charges being the point's attribute
// (dim 3: mu; dim 1: s, 0, 0; the three scalar columns of cagr_scatter3:
// s_0, s_1, s_2).
template <typename T>
__global__ void k_ipoints(const T* __restrict__ spos, const int32_t* __restrict__ perm, int64_t n,
                          const T* __restrict__ attrs, int dim, T* __restrict__ out) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t j = perm[s];
    const T a0 = attrs[j * dim];
    const T a1 = dim == 3 ? attrs[j * 3 + 1] : T(0);
    const T a2 = dim == 3 ? attrs[j * 3 + 2] : T(0);
    write_rec(out, s, n, spos[3 * s], spos[3 * s + 1], spos[3 * s + 2], a0, a1, a2);
}

// The records of the three-column slot (sum_k A2Tk) in their walk form: the
// position and, per k, exp(-y_k/2) times the column's charge s_k -- all the
// A2T sum reads of a source (the walk multiplied the same two numbers for
// every pair; now once per record) -- in blocks of kBlkES scalars.
template <typename T>
__global__ void k_es_compact(const T* __restrict__ rec, T* __restrict__ out, int64_t nblocks) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * nblocks) return;
    const T* b = rec + (i >> 1) * kBlk + (i & 1);
    T* o = out + (i >> 1) * kBlkES + (i & 1);
    constexpr int kCharge[3] = {3, 7, 8};
#pragma unroll
    for (int c = 0; c < 3; c++) o[2 * c] = b[2 * c];
#pragma unroll
    for (int k = 0; k < 3; k++) o[2 * (3 + k)] = b[2 * (4 + k)] * b[2 * kCharge[k]];
}

template <typename T>
struct ChargeParams {
    const int4* chunks = nullptr;
    const T* bc = nullptr;
    const T* bh = nullptr;
    const T* pts = nullptr;
    T* part = nullptr;
    int P = 0, P3 = 0, P3e = 0;  // P3e: P3 rounded up to even (whole record pairs per grid)
    T cheb[kPMax] = {};
    T omega[kPMax] = {};
};

// Barycentric Lagrange basis at u (second form; an exact node hit gives the
// unit vector, as the formula's limit).
template <typename T>
__device__ __forceinline__ void lagrange(T u, int P, const T* t, const T* om, T* L) {
    int hit = -1;
    for (int k = 0; k < P; k++)
        if (u == t[k]) hit = k;
    if (hit >= 0) {
        for (int k = 0; k < P; k++) L[k] = k == hit ? T(1) : T(0);
        return;
    }
    T sum = T(0);
    for (int k = 0; k < P; k++) {
        const T v = om[k] / (u - t[k]);
        L[k] = v;
        sum += v;
    }
    const T inv = T(1) / sum;
    for (int k = 0; k < P; k++) L[k] *= inv;
}

constexpr int kChargeThreads = 256;
// points staged per tile (shared memory: Lagrange values and charges; 64 in
// double keeps the block under the 48 KB of static shared memory)
template <typename T>
constexpr int charge_tile() { return sizeof(T) == 4 ? 128 : 64; }

// Partial proxy charges of one chunk, q_abc = sum_j Lx_a(y_j) Ly_b(y_j) Lz_c(y_j)
// charges_j, as a tensor-product contraction: thread (a, b) of a slice forms
// Lx_a Ly_b charges_j once per point and adds it times every Lz_c (read from
// shared memory by all threads alike), so a point costs a thread 2 + P shared
// loads for P proxies; the kChargeThreads / P^2 slices take the tile's points
// round robin and are summed in slice order at the end (deterministic).
template <typename T>
__global__ void __launch_bounds__(kChargeThreads) k_charges(const ChargeParams<T> p) {
    constexpr int kTile = charge_tile<T>();
    __shared__ T sL[kTile][3][kPMax];
    __shared__ T sQ[kTile][4];
    __shared__ T sRed[kPMax * kPMax * kPMax][3];
    __shared__ T sCheb[kPMax], sOmega[kPMax];  // (indexed per k: not from the parameters)
    if (threadIdx.x < kPMax) {
        sCheb[threadIdx.x] = p.cheb[threadIdx.x];
        sOmega[threadIdx.x] = p.omega[threadIdx.x];
    }
    __syncthreads();
    const int4 cd = p.chunks[blockIdx.x];  // {node, first sorted point, count, proxy block}
    const T* c = p.bc + 4 * (int64_t)cd.x;
    const T* h = p.bh + 4 * (int64_t)cd.x;
    const T cen[3] = {c[0], c[1], c[2]};
    const T ih[3] = {T(1) / h[0], T(1) / h[1], T(1) / h[2]};
    const int P = p.P, P2 = P * P, P3 = p.P3;
    const int slices = kChargeThreads / P2;  // >= 3 (P <= 9)
    const int slice = (int)threadIdx.x / P2, pair = (int)threadIdx.x - slice * P2;
    const bool on = slice < slices;
    const int a = pair / P, b = pair - (pair / P) * P;
    T acc[kPMax][3];
#pragma unroll
    for (int k = 0; k < kPMax; k++) acc[k][0] = acc[k][1] = acc[k][2] = T(0);
    for (int base = 0; base < cd.z; base += kTile) {
        const int cnt = min(kTile, cd.z - base);
        for (int t = threadIdx.x; t < cnt * 3; t += kChargeThreads) {
            const int j = t / 3, ax = t - 3 * j;
            const T y = rec_comp(p.pts, (int64_t)cd.y + base + j, ax);
            // (selects, not a dynamic index into a register array)
            const T cx = ax == 0 ? cen[0] : (ax == 1 ? cen[1] : cen[2]);
            const T hx = ax == 0 ? ih[0] : (ax == 1 ? ih[1] : ih[2]);
            T u = (y - cx) * hx;
            u = fmin(fmax(u, T(-1)), T(1));
            lagrange(u, P, sCheb, sOmega, &sL[j][ax][0]);
        }
        for (int j = threadIdx.x; j < cnt; j += kChargeThreads) {
            const int64_t r = (int64_t)cd.y + base + j;
            sQ[j][0] = rec_comp(p.pts, r, 3);
            sQ[j][1] = rec_comp(p.pts, r, 7);
            sQ[j][2] = rec_comp(p.pts, r, 8);
        }
        __syncthreads();
        if (on) {
            for (int j = slice; j < cnt; j += slices) {
                const T lab = sL[j][0][a] * sL[j][1][b];
                const T t0 = lab * sQ[j][0], t1 = lab * sQ[j][1], t2 = lab * sQ[j][2];
#pragma unroll
                for (int k = 0; k < kPMax; k++) {
                    if (k < P) {
                        const T lz = sL[j][2][k];
                        acc[k][0] += t0 * lz;
                        acc[k][1] += t1 * lz;
                        acc[k][2] += t2 * lz;
                    }
                }
            }
        }
        __syncthreads();
    }
    // the slices' sums, added in slice order
    for (int sl = 0; sl < slices; sl++) {
        if (slice == sl) {
#pragma unroll
            for (int k = 0; k < kPMax; k++) {
                if (k < P) {
                    T* r = sRed[pair * P + k];
                    r[0] = sl == 0 ? acc[k][0] : r[0] + acc[k][0];
                    r[1] = sl == 0 ? acc[k][1] : r[1] + acc[k][1];
                    r[2] = sl == 0 ? acc[k][2] : r[2] + acc[k][2];
                }
            }
        }
        __syncthreads();
    }
    for (int m = threadIdx.x; m < P3; m += kChargeThreads) {
        T* o = p.part + ((int64_t)blockIdx.x * P3 + m) * 4;
        st4<T>(o, make4(sRed[m][0], sRed[m][1], sRed[m][2], T(0)));
    }
}

// Proxy records: charges = the node's chunk partials summed in chunk order
// (in double; the loads of 8 chunks are issued together, a node near the root
// having hundreds of chunks), position = the Chebyshev grid point of the
// node's box.
constexpr int kFinishBatch = 8;

template <typename T>
__global__ void k_charges_finish(const int32_t* __restrict__ chunk_first, int64_t num_interp,
                                 const int4* __restrict__ chunks, const T* __restrict__ part,
                                 const T* __restrict__ bc, const T* __restrict__ bh,
                                 const ChargeParams<T> p, T* __restrict__ prox) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int P = p.P, P3 = p.P3, P3e = p.P3e;
    const int64_t ii = idx / P3e;
    const int m = (int)(idx - ii * P3e);
    if (ii >= num_interp) return;
    const int64_t nrec = num_interp * P3e;
    if (m >= P3) {  // the padding record of an odd grid: zero charges
        write_rec(prox, idx, nrec, T(0), T(0), T(0), T(0), T(0), T(0));
        return;
    }
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    const int c0 = chunk_first[ii], c1 = chunk_first[ii + 1];
    for (int ch = c0; ch < c1; ch += kFinishBatch) {
        Vec4<T> q[kFinishBatch];
#pragma unroll
        for (int u = 0; u < kFinishBatch; u++)
            if (ch + u < c1) q[u] = ld4(part + ((int64_t)(ch + u) * P3 + m) * 4);
#pragma unroll
        for (int u = 0; u < kFinishBatch; u++) {
            if (ch + u < c1) {
                s0 += (double)q[u].x;
                s1 += (double)q[u].y;
                s2 += (double)q[u].z;
            }
        }
    }
    const int64_t node = chunks[c0].x;
    const T* c = bc + 4 * node;
    const T* h = bh + 4 * node;
    const int a = m / (P * P), b = (m / P) % P, cc = m % P;
    const T y0 = c[0] + h[0] * p.cheb[a];
    const T y1 = c[1] + h[1] * p.cheb[b];
    const T y2 = c[2] + h[2] * p.cheb[cc];
    write_rec(prox, idx, nrec, y0, y1, y2, (T)s0, (T)s1, (T)s2);
}

// ---- the walk -------------------------------------------------------------------

template <typename T>
struct IWalk {
    int64_t M = 0, nq = 0;
    const int4* meta = nullptr;
    const T* bc = nullptr;
    const int32_t* iidx = nullptr;
    const T* pts = nullptr;
    const T* prox = nullptr;
    int P3 = 0, P3e = 0;  // records per proxy grid; its stride (P3 rounded up to even)
    int direct_max = 0;
    T theta = T(0.5);
    // queries: the tree's points (grouped by qgroup), an explicit array
    // (optional processing order), or the nodes of a regular grid
    const T* spos = nullptr;
    const int32_t* perm = nullptr;
    const int32_t* qgroup = nullptr;
    const T* queries = nullptr;
    const int32_t* qorder = nullptr;
    const T* widths = nullptr;
    T width = T(0);
    int grid = 0;
    int gx = 0, gy = 0, gz = 0;
    T gox = T(0), goy = T(0), goz = T(0), gh = T(0);
    T* out = nullptr;
    int out_stride = 1;
    int accumulate = 0;
    unsigned long long* counter = nullptr;  // next group of 32 queries (persistent launch)
    const int32_t* gorder = nullptr;        // the order groups are taken in (null: their own)
    uint32_t* gcost = nullptr;              // record pairs summed per group, when non-null
    int* err = nullptr;                     // set when a staging wait runs out
    uint32_t spin = 0;                      // try_wait rounds before a wait runs out
};

template <int OP>
struct IOp {
    static constexpr bool a2 = OP == kOpA21 || OP == kOpA22 || OP == kOpA23 || OP == kOpA3 ||
                               OP == kOpA2Fused;
    static constexpr bool a2t1 = OP == kOpA2T1 || OP == kOpA2T2 || OP == kOpA2T3;
    static constexpr bool a2tsum = OP == kIOpA2TSum || OP == kIOpA2TShared;
    static constexpr int k = (OP == kOpA21 || OP == kOpA2T1)   ? 0
                             : (OP == kOpA22 || OP == kOpA2T2) ? 1
                             : (OP == kOpA23 || OP == kOpA2T3) ? 2
                                                                : -1;
    static constexpr bool s0 = k == 0 || OP == kOpA3 || OP == kOpA2Fused;
    static constexpr bool s1 = k == 1 || OP == kOpA3 || OP == kOpA2Fused;
    static constexpr bool s2 = k == 2 || OP == kOpA3 || OP == kOpA2Fused;
    static constexpr bool query_exp = a2 || a2t1 || a2tsum;
};

template <typename T>
struct IQ {
    T x, y, z;
    T tw;          // width threshold on r^2
    T iw, iw3;     // 1/w, 1/w^3 (continuous kernel inside the width)
    T ex0, ex1, ex2;  // exp(x_k / 2)
};

template <typename T>
__device__ __forceinline__ void kahan(T& s, T& c, T v) {
    const T y = v - c;
    const T t = s + y;
    c = (t - s) - y;
    s = t;
}

// ---- the pair term ------------------------------------------------------------
//
// One block = two source records; every quantity of the term is a pair, one
// value per record, computed with the packed f32x2 instructions of sm_100
// (fma/mul/add.rn.f32x2: one issue slot for two FP32 operations, the same
// rounding as the scalar ones) -- the walk is issue-bound, and this halves its
// FP32 instructions.  In double the pairs are two scalars.
template <typename T>
struct Pair;
template <>
struct Pair<float> {
    using type = float2;
};
template <>
struct Pair<double> {
    using type = double2;
};
template <typename T>
using P2 = typename Pair<T>::type;

__device__ __forceinline__ float2 pk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 pk(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ double2 fma2(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}
__device__ __forceinline__ double2 mul2(double2 a, double2 b) {
    return make_double2(a.x * b.x, a.y * b.y);
}
__device__ __forceinline__ double2 add2(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}

// The nine component pairs of a block (y0, y1, y2, q0, e0, e1, e2, q1, q2).
template <typename T>
struct Blk {
    P2<T> c[kComp];
};
__device__ __forceinline__ Blk<float> load_blk(const float* b) {
    const float4 A = ld4(b), B = ld4(b + 4), C = ld4(b + 8), D = ld4(b + 12), E = ld4(b + 16);
    Blk<float> k;
    k.c[0] = pk(A.x, A.y);
    k.c[1] = pk(A.z, A.w);
    k.c[2] = pk(B.x, B.y);
    k.c[3] = pk(B.z, B.w);
    k.c[4] = pk(C.x, C.y);
    k.c[5] = pk(C.z, C.w);
    k.c[6] = pk(D.x, D.y);
    k.c[7] = pk(D.z, D.w);
    k.c[8] = pk(E.x, E.y);
    return k;
}
__device__ __forceinline__ Blk<double> load_blk(const double* b) {
    Blk<double> k;
#pragma unroll
    for (int c = 0; c < kComp; c++) k.c[c] = *reinterpret_cast<const double2*>(b + 2 * c);
    return k;
}
// A block of the A2T sum's walk layout: positions into components 0..2, the
// e_k s_k into 4..6 (where the full layout keeps e_k).
__device__ __forceinline__ Blk<float> load_blk_es(const float* b) {
    const float4 A = ld4(b), B = ld4(b + 4), C = ld4(b + 8);
    Blk<float> k;
    k.c[0] = pk(A.x, A.y);
    k.c[1] = pk(A.z, A.w);
    k.c[2] = pk(B.x, B.y);
    k.c[4] = pk(B.z, B.w);
    k.c[5] = pk(C.x, C.y);
    k.c[6] = pk(C.z, C.w);
    k.c[3] = k.c[7] = k.c[8] = pk(0.0f, 0.0f);
    return k;
}
__device__ __forceinline__ Blk<double> load_blk_es(const double* b) {
    Blk<double> k;
#pragma unroll
    for (int c = 0; c < 3; c++) k.c[c] = *reinterpret_cast<const double2*>(b + 2 * c);
#pragma unroll
    for (int c = 0; c < 3; c++) k.c[4 + c] = *reinterpret_cast<const double2*>(b + 6 + 2 * c);
    k.c[3] = k.c[7] = k.c[8] = make_double2(0.0, 0.0);
    return k;
}

// scalars per block (record pair) in the walk of operator OP
template <int OP>
constexpr int blk_of() {
    return OP == kIOpA2TSum ? kBlkES : kBlk;
}

// The query's values as pairs (both halves equal).
template <typename T>
struct IQ2 {
    P2<T> x, y, z, ex0, ex1, ex2;
};

// One block's two pair terms into the pair sums p0..p2 (inside-width sums of
// the continuous kernel into i0..i2).  NEAR: the per-pair width test of the
// reference kernels; far sources are outside every width.  MASKED: only the
// halves in `mask` are taken (bit 0: the block's first record, bit 1: its
// second) -- a range that starts or ends inside a block.  A half not taken
// gets 1/r = 0, so its finite data contributes exactly zero.
template <typename T, int OP, bool CONT, bool NEAR, bool MASKED>
__device__ __forceinline__ void pterm(const IQ<T>& q, const IQ2<T>& q2, const T* __restrict__ b,
                                      uint32_t mask, P2<T>& p0, P2<T>& p1, P2<T>& p2, P2<T>& h0,
                                      P2<T>& h1, P2<T>& h2, T& i0, T& i1, T& i2) {
    const bool ra = !MASKED || (mask & 1u), rb = !MASKED || (mask & 2u);  // in the range
    if constexpr (OP == kOpCount) {
        p0 = add2(p0, pk(ra ? T(1) : T(0), rb ? T(1) : T(0)));
        return;
    } else {
        Blk<T> k;
        if constexpr (OP == kIOpA2TSum) k = load_blk_es(b);
        else k = load_blk(b);
        const P2<T> m1 = pk(T(-1), T(-1));
        const P2<T> dx = fma2(k.c[0], m1, q2.x);
        const P2<T> dy = fma2(k.c[1], m1, q2.y);
        const P2<T> dz = fma2(k.c[2], m1, q2.z);
        const P2<T> d2 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
        const bool oa = ra && (!NEAR || d2.x >= q.tw), ob = rb && (!NEAR || d2.y >= q.tw);
        const P2<T> r = (NEAR || MASKED) ? pk(oa ? rsqrt_t(d2.x) : T(0), ob ? rsqrt_t(d2.y) : T(0))
                                         : pk(rsqrt_t(d2.x), rsqrt_t(d2.y));
        const P2<T> r2 = mul2(r, r);
        const P2<T> r3 = mul2(r2, r);
        const P2<T> half = pk(T(0.5), T(0.5));
        // continuous kernel, inside the width: the pairs in the range that fail the test
        const bool ia = NEAR && CONT && ra && !oa, ib = NEAR && CONT && rb && !ob;
        if constexpr (OP == kOpA || OP == kOpG || IOp<OP>::a2) {
            const P2<T> dm = fma2(dz, k.c[8], fma2(dy, k.c[7], mul2(dx, k.c[3])));
            if constexpr (OP == kOpA) {
                p0 = fma2(dm, r3, p0);
                if constexpr (NEAR && CONT) {
                    if (ia) i0 += dm.x * q.iw3;
                    if (ib) i0 += dm.y * q.iw3;
                }
            } else if constexpr (OP == kOpG) {
                const P2<T> cc = mul2(mul2(pk(T(-3), T(-3)), dm), mul2(r3, r2));
                p0 = fma2(dx, cc, fma2(k.c[3], r3, p0));
                p1 = fma2(dy, cc, fma2(k.c[7], r3, p1));
                p2 = fma2(dz, cc, fma2(k.c[8], r3, p2));
            } else {
                const P2<T> t = mul2(dm, r3);
                const P2<T> hh = mul2(half, r);
                if constexpr (IOp<OP>::s0) p0 = fma2(k.c[4], fma2(hh, k.c[3], t), p0);
                if constexpr (IOp<OP>::s1) p1 = fma2(k.c[5], fma2(hh, k.c[7], t), p1);
                if constexpr (IOp<OP>::s2) p2 = fma2(k.c[6], fma2(hh, k.c[8], t), p2);
                if constexpr (NEAR && CONT) {
                    const T hi = T(0.5) * q.iw;
                    if (ia) {
                        const T ti = dm.x * q.iw3;
                        if constexpr (IOp<OP>::s0) i0 += ti + hi * k.c[3].x;
                        if constexpr (IOp<OP>::s1) i1 += ti + hi * k.c[7].x;
                        if constexpr (IOp<OP>::s2) i2 += ti + hi * k.c[8].x;
                    }
                    if (ib) {
                        const T ti = dm.y * q.iw3;
                        if constexpr (IOp<OP>::s0) i0 += ti + hi * k.c[3].y;
                        if constexpr (IOp<OP>::s1) i1 += ti + hi * k.c[7].y;
                        if constexpr (IOp<OP>::s2) i2 += ti + hi * k.c[8].y;
                    }
                }
            }
        } else if constexpr (OP == kOpAT) {
            const P2<T> c = mul2(k.c[3], r3);
            p0 = fma2(dx, c, p0);
            p1 = fma2(dy, c, p1);
            p2 = fma2(dz, c, p2);
        } else if constexpr (IOp<OP>::a2t1) {
            constexpr int K = IOp<OP>::k;
            const P2<T> gr = mul2(mul2(k.c[4 + K], k.c[3]), r);
            const P2<T> c = mul2(gr, r2);
            p0 = fma2(dx, c, p0);
            p1 = fma2(dy, c, p1);
            p2 = fma2(dz, c, p2);
            if constexpr (K == 0) p0 = fma2(half, gr, p0);
            if constexpr (K == 1) p1 = fma2(half, gr, p1);
            if constexpr (K == 2) p2 = fma2(half, gr, p2);
        } else if constexpr (IOp<OP>::a2tsum) {
            // sum_k exp(x_k/2) exp(-y_k/2) s_k (d / r^3 + e_k / (2r)); the three-column
            // slot's records hold exp(-y_k/2) s_k (k_es_form), the shared one e_k and s
            P2<T> g0, g1, g2;
            if constexpr (OP == kIOpA2TSum) {
                g0 = mul2(q2.ex0, k.c[4]);
                g1 = mul2(q2.ex1, k.c[5]);
                g2 = mul2(q2.ex2, k.c[6]);
            } else {
                g0 = mul2(q2.ex0, mul2(k.c[4], k.c[3]));
                g1 = mul2(q2.ex1, mul2(k.c[5], k.c[3]));
                g2 = mul2(q2.ex2, mul2(k.c[6], k.c[3]));
            }
            // d_k c into p_k and g_k r into h_k (the 1/2 applied once per tile)
            const P2<T> c = mul2(add2(add2(g0, g1), g2), r3);
            p0 = fma2(dx, c, p0);
            p1 = fma2(dy, c, p1);
            p2 = fma2(dz, c, p2);
            h0 = fma2(g0, r, h0);
            h1 = fma2(g1, r, h1);
            h2 = fma2(g2, r, h2);
        }
    }
}

// A tile of nb blocks into this lane's compensated sums: the first block's
// first record is skipped when sf, the last block's second when sl.  (Lanes
// outside the walking subgroup, active = false, compute and discard.)
template <typename T, int OP, bool CONT, bool NEAR>
__device__ __forceinline__ void itile(const IQ<T>& q, const IQ2<T>& q2, bool active,
                                      const T* __restrict__ b, int nb, bool sf, bool sl, T* s,
                                      T* cmp, T* in) {
    P2<T> p0 = pk(T(0), T(0)), p1 = p0, p2 = p0, h0 = p0, h1 = p0, h2 = p0;
    T i0 = T(0), i1 = T(0), i2 = T(0);
    int j0 = 0, j1 = nb;
    if (sf) {
        pterm<T, OP, CONT, NEAR, true>(q, q2, b, (nb == 1 && sl) ? 0u : 2u, p0, p1, p2, h0, h1, h2,
                                       i0, i1, i2);
        j0 = 1;
    }
    const bool last_masked = sl && nb - 1 >= j0;
    if (last_masked) j1 = nb - 1;
    int j = j0;
    for (; j + kUnrollB <= j1; j += kUnrollB) {
#pragma unroll
        for (int u = 0; u < kUnrollB; u++)
            pterm<T, OP, CONT, NEAR, false>(q, q2, b + (int64_t)(j + u) * blk_of<OP>(), 3u, p0, p1, p2, h0,
                                            h1, h2, i0, i1, i2);
    }
    for (; j < j1; j++)
        pterm<T, OP, CONT, NEAR, false>(q, q2, b + (int64_t)j * blk_of<OP>(), 3u, p0, p1, p2, h0, h1, h2,
                                        i0, i1, i2);
    if (last_masked)
        pterm<T, OP, CONT, NEAR, true>(q, q2, b + (int64_t)(nb - 1) * blk_of<OP>(), 1u, p0, p1, p2, h0, h1,
                                       h2, i0, i1, i2);
    if (!active) return;
    if constexpr (OP == kOpCount) {
        s[0] += p0.x + p0.y;
    } else if constexpr (IOp<OP>::a2tsum) {
        kahan(s[0], cmp[0], (p0.x + p0.y) + T(0.5) * (h0.x + h0.y));
        kahan(s[1], cmp[1], (p1.x + p1.y) + T(0.5) * (h1.x + h1.y));
        kahan(s[2], cmp[2], (p2.x + p2.y) + T(0.5) * (h2.x + h2.y));
    } else {
        kahan(s[0], cmp[0], p0.x + p0.y);
        kahan(s[1], cmp[1], p1.x + p1.y);
        kahan(s[2], cmp[2], p2.x + p2.y);
        if constexpr (NEAR && CONT) {
            in[0] += i0;
            in[1] += i1;
            in[2] += i2;
        }
    }
}

__device__ __forceinline__ uint32_t icompact3(uint64_t x) {
    x &= 0x1249249249249249ull;
    x = (x ^ (x >> 2)) & 0x10c30c30c30c30c3ull;
    x = (x ^ (x >> 4)) & 0x100f00f00f00f00full;
    x = (x ^ (x >> 8)) & 0x1f0000ff0000ffull;
    x = (x ^ (x >> 16)) & 0x1f00000000ffffull;
    x = (x ^ (x >> 32)) & 0x1fffffull;
    return (uint32_t)x;
}

// This lane's query (the same three sources and output rows as the
// reference-mode walks); false past the end.
template <typename T>
__device__ __forceinline__ bool iload(const IWalk<T>& p, int64_t qi, IQ<T>& q, int64_t& oidx,
                                      T& w) {
    w = p.width;
    oidx = 0;
    q.x = q.y = q.z = T(0);
    bool valid = qi < p.nq;
    if (valid && p.grid) {
        const uint32_t i = icompact3((uint64_t)qi), j = icompact3((uint64_t)qi >> 1),
                       k = icompact3((uint64_t)qi >> 2);
        valid = i < (uint32_t)p.gx && j < (uint32_t)p.gy && k < (uint32_t)p.gz;
        if (valid) {
            oidx = ((int64_t)k * p.gy + j) * p.gx + i;
            q.x = fma(T(i), p.gh, p.gox);
            q.y = fma(T(j), p.gh, p.goy);
            q.z = fma(T(k), p.gh, p.goz);
            if (p.widths) w = p.widths[oidx];
        }
    } else if (valid) {
        if (p.queries == nullptr) {
            const int64_t s = p.qgroup ? (int64_t)p.qgroup[qi] : qi;
            oidx = p.perm[s];
            q.x = p.spos[3 * s];
            q.y = p.spos[3 * s + 1];
            q.z = p.spos[3 * s + 2];
        } else {
            oidx = p.qorder ? (int64_t)p.qorder[qi] : qi;
            q.x = p.queries[3 * oidx];
            q.y = p.queries[3 * oidx + 1];
            q.z = p.queries[3 * oidx + 2];
        }
        if (p.widths) w = p.widths[oidx];
    }
    q.tw = width_threshold(w);
    q.iw = T(1) / w;
    q.iw3 = T(1) / (w * w * w);
    return valid;
}

// mode bit 0: add into the output; bit 1: write -op
template <typename T>
__device__ __forceinline__ void iput(T* o, int j, T v, int mode) {
    const T u = (mode & 2) ? -v : v;
    o[j] = (mode & 1) ? o[j] + u : u;
}

// A batch of queries: bounding centre, radius and largest width.
template <typename T>
struct Batch {
    T cx, cy, cz, r, w;
};

// Split factor of the query groups (see lane_batch).
constexpr float kSplit = 5.0f;

// The batch this lane's query walks in.  The warp's 32 queries are
// consecutive along a space-filling curve, but a group that straddles a jump
// of the curve between distant parts of the cloud has a large radius, accepts
// little as far and sums most of the cloud directly (one such warp dominated
// a launch).  So the group is split top-down in aligned halves: a group of
// 2^k lanes is split when its radius exceeds kSplit times the radius of its
// more compact half (the other half then holds the straggler), and each lane
// walks with the first group on its path that is not split.  Lanes of one
// final group reach the same decision (they share the group and its halves);
// *bits receives log2 of its size.  A compact group keeps all 32 lanes
// (measured on the 1M-point union-of-primitives cloud: ~8 % of the groups
// split at all).
template <typename T>
__device__ __forceinline__ Batch<T> lane_batch(const IQ<T>& q, bool valid, T w, int* bits) {
    T lo0 = valid ? q.x : T(INFINITY), hi0 = valid ? q.x : -T(INFINITY);
    T lo1 = valid ? q.y : T(INFINITY), hi1 = valid ? q.y : -T(INFINITY);
    T lo2 = valid ? q.z : T(INFINITY), hi2 = valid ? q.z : -T(INFINITY);
    // a NaN width admits no far node (every pair is then summed directly)
    T wm = valid ? (w == w ? w : T(INFINITY)) : T(0);
    Batch<T> b[6];
    T sib[6];  // radius of the other half of the level-k group (k >= 1)
#pragma unroll
    for (int k = 0; k < 6; k++) {
        if (k > 0) {
            const int o = 1 << (k - 1);
            sib[k] = __shfl_xor_sync(kAll, b[k - 1].r, o);
            lo0 = fmin(lo0, __shfl_xor_sync(kAll, lo0, o));
            hi0 = fmax(hi0, __shfl_xor_sync(kAll, hi0, o));
            lo1 = fmin(lo1, __shfl_xor_sync(kAll, lo1, o));
            hi1 = fmax(hi1, __shfl_xor_sync(kAll, hi1, o));
            lo2 = fmin(lo2, __shfl_xor_sync(kAll, lo2, o));
            hi2 = fmax(hi2, __shfl_xor_sync(kAll, hi2, o));
            wm = fmax(wm, __shfl_xor_sync(kAll, wm, o));
        }
        // (a group without a valid query gets the zero batch)
        const bool any = lo0 <= hi0;
        b[k].cx = any ? T(0.5) * (lo0 + hi0) : T(0);
        b[k].cy = any ? T(0.5) * (lo1 + hi1) : T(0);
        b[k].cz = any ? T(0.5) * (lo2 + hi2) : T(0);
        const T hx = any ? fmax(hi0 - b[k].cx, b[k].cx - lo0) : T(0);
        const T hy = any ? fmax(hi1 - b[k].cy, b[k].cy - lo1) : T(0);
        const T hz = any ? fmax(hi2 - b[k].cz, b[k].cz - lo2) : T(0);
        b[k].r = sqrt(hx * hx + hy * hy + hz * hz) * T(1.0 + 1.0 / 65536);
        b[k].w = any ? fmax(wm, T(0)) * T(1.0 + 1.0 / 65536) : T(0);
    }
    int k = 5;
#pragma unroll
    for (int j = 5; j > 0; j--) {
        if (k == j && b[j].r > T(kSplit) * fmin(b[j - 1].r, sib[j])) k = j - 1;
    }
    *bits = k;
    Batch<T> out = b[0];
#pragma unroll
    for (int j = 1; j < 6; j++)
        if (k == j) out = b[j];
    return out;
}

// ---- the pipelined walk ----------------------------------------------------------
//
// Every interaction is a contiguous run of source records (a node's points in
// Morton order, or a node's proxy grid), so it is staged into shared memory
// with one-dimensional TMA bulk copies (cp.async.bulk, completion counted on
// an mbarrier) and the warp's 32 lanes read each record with a broadcast
// shared-memory load.  Each warp keeps kSlots tiles in flight: the tree walk
// runs ahead of the arithmetic, issuing the copies of the next tiles while
// the current one is summed, so the L2 latency of the records (they are
// streamed: every warp reads its own interaction list) is hidden.  The launch
// is persistent: its warps take groups of 32 queries from an atomic counter,
// in curve order, so a warp that drew an expensive group does not hold back
// the others.  Every wait is bounded: a wait that runs out sets the error
// flag, waits (bounded again) for the warp's copies still in flight and ends
// the warp.
constexpr uint32_t kDrainSpin = 1u << 24;

// blocks (record pairs) per tile: 51 in float, 25 in double (the A2T sum's walk
// layout: 85, 42)
template <typename T, int OP>
constexpr int tile_blocks() {
    return kTileBytes / (blk_of<OP>() * (int)sizeof(T));
}

template <typename T>
constexpr size_t walk_smem_bytes() {
    return (size_t)kPWarps * kSlots * (kTileBytes + sizeof(uint64_t));
}

template <typename T, int OP, bool CONT>
__global__ void __launch_bounds__(kPWarps * 32) k_iwalk(const IWalk<T> p) {
    extern __shared__ __align__(128) unsigned char dsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* tiles = dsm + (size_t)warp * kSlots * kTileBytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(dsm + (size_t)kPWarps * kSlots * kTileBytes) +
                     warp * kSlots;
    if (lane == 0) {
        for (int sl = 0; sl < kSlots; sl++) mbar_init(bars + sl);
        mbar_init_fence();
    }
    __syncwarp();
    constexpr int kTB = tile_blocks<T, OP>();
    constexpr int kB = blk_of<OP>();
    static_assert(kTB < 128 && kSlots <= 6, "tile fields: 7-bit block count, 10 bits per slot");
    // warp-uniform pipeline state: next slot to consume, tiles in flight, the
    // parity of each slot's next completion, and each slot's tile in 10 bits:
    // blocks | near << 7 | skip the first record << 8 | skip the last << 9
    int head = 0, inflight = 0;
    uint32_t phase = 0;
    uint64_t tinfo = 0;
    const int M = (int)p.M;
    const int64_t ngroups = (p.nq + 31) / 32;
    for (;;) {
        unsigned long long ticket = 0;
        if (lane == 0) ticket = atomicAdd(p.counter, 1ull);
        ticket = __shfl_sync(kAll, ticket, 0);
        if ((int64_t)ticket >= ngroups) break;
        const int64_t grp = p.gorder ? (int64_t)__ldg(p.gorder + ticket) : (int64_t)ticket;
        // this group's record pairs (its cost, for the next walk's order: the same
        // measure whatever the walk's layout, so walks of different operators
        // order each other's groups alike)
        uint32_t ncost = 0;
        const int64_t qi = grp * 32 + lane;
        IQ<T> q;
        int64_t oidx;
        T w;
        const bool valid = iload(p, qi, q, oidx, w);
        if (__all_sync(kAll, !valid)) {  // grid lanes outside the grid
            if (p.gcost && lane == 0) p.gcost[grp] = 0;
            continue;
        }
        if constexpr (IOp<OP>::query_exp) {
            q.ex0 = exp_t(q.x * T(0.5));
            q.ex1 = exp_t(q.y * T(0.5));
            q.ex2 = exp_t(q.z * T(0.5));
        } else {
            q.ex0 = q.ex1 = q.ex2 = T(1);
        }
        IQ2<T> q2;
        q2.x = pk(q.x, q.x);
        q2.y = pk(q.y, q.y);
        q2.z = pk(q.z, q.z);
        q2.ex0 = pk(q.ex0, q.ex0);
        q2.ex1 = pk(q.ex1, q.ex1);
        q2.ex2 = pk(q.ex2, q.ex2);
        int bits;
        const Batch<T> mine = lane_batch(q, valid, w, &bits);
        T s[3] = {T(0), T(0), T(0)}, cmp[3] = {T(0), T(0), T(0)}, in[3] = {T(0), T(0), T(0)};
        for (int g = 0; g < 32;) {
            // the group starting at lane g (every lane of it holds the same batch)
            const int kg = __shfl_sync(kAll, bits, g);
            const bool active = valid && (lane >> kg) == (g >> kg);
            const int gnext = g + (1 << kg);
            if (!__any_sync(kAll, active)) {
                g = gnext;
                continue;
            }
            const T bcx = __shfl_sync(kAll, mine.cx, g), bcy = __shfl_sync(kAll, mine.cy, g),
                    bcz = __shfl_sync(kAll, mine.cz, g), br = __shfl_sync(kAll, mine.r, g),
                    wm = __shfl_sync(kAll, mine.w, g);
            // producer: the walk, one interaction (a run of records) at a time,
            // as a run of blocks with its first / last half skipped when the run
            // starts / ends inside a block
            int n = 0;
            int64_t blk = 0;       // next block of the current interaction
            int left = 0;          // its blocks still to issue
            int near = 0, skip_first = 0, skip_last = 0;
            const T* base = nullptr;
            bool more = true;
            for (;;) {
                while (more && inflight < kSlots) {
                    while (left == 0 && n < M) {
                        const int4 mt = __ldg(p.meta + n);
                        const Vec4<T> bx = ld4(p.bc + 4 * (int64_t)n);
                        const T dx = bcx - bx.x, dy = bcy - bx.y, dz = bcz - bx.z;
                        const T R2 = dx * dx + dy * dy + dz * dz;
                        // every query x of the batch sees the node at |x - c| >= R - r_B,
                        // so r_C + theta r_B < theta R gives r_C < theta |x - c| for each
                        const T sr = br + bx.w;
                        const T sw = sr + wm;
                        const T a = bx.w + p.theta * br;
                        const bool far = a * a < (p.theta * p.theta) * R2 && R2 >= sw * sw;
                        const int np = node_npts(mt);
                        int64_t r0 = -1, cnt = 0;
                        if (far) {
                            const int ii = __ldg(p.iidx + n);
                            if (ii >= 0) {
                                base = p.prox;
                                r0 = (int64_t)ii * p.P3e;
                                cnt = p.P3;
                            } else {
                                base = p.pts;
                                r0 = mt.y;
                                cnt = np;
                            }
                            near = 0;
                            n = mt.x;
                        } else if (node_leaf(mt) || np <= p.direct_max) {
                            base = p.pts;
                            r0 = mt.y;
                            cnt = np;
                            near = 1;
                            n = mt.x;
                        } else {
                            n = n + 1;
                        }
                        if (r0 >= 0) {
                            blk = r0 >> 1;
                            left = (int)(((r0 + cnt + 1) >> 1) - blk);
                            skip_first = (int)(r0 & 1);
                            skip_last = (int)((r0 + cnt) & 1);
                        }
                    }
                    if (left == 0) {
                        more = false;
                        break;
                    }
                    const int nb = min(left, kTB);
                    const int slot = (head + inflight) % kSlots;
                    if (lane == 0)
                        tma_load_1d(tiles + (size_t)slot * kTileBytes, base + blk * kB,
                                    (uint32_t)(nb * kB * sizeof(T)), bars + slot);
                    const uint64_t f = (uint64_t)(nb | (near << 7) | (skip_first << 8) |
                                                  ((nb == left ? skip_last : 0) << 9));
                    tinfo = (tinfo & ~(0x3ffull << (10 * slot))) | (f << (10 * slot));
                    skip_first = 0;
                    blk += nb;
                    left -= nb;
                    inflight++;
                }
                if (inflight == 0) break;
                // consumer: the oldest tile
                if (!mbar_wait(bars + head, (phase >> head) & 1u, p.spin)) {
                    // a copy did not arrive: report, let the copies in flight land, stop
                    if (lane == 0) atomicOr(p.err, 1);
                    for (int k2 = 0; k2 < inflight; k2++) {
                        const int sl = (head + k2) % kSlots;
                        mbar_wait(bars + sl, (phase >> sl) & 1u, kDrainSpin);
                    }
                    return;
                }
                phase ^= 1u << head;
                const uint32_t inf = (uint32_t)(tinfo >> (10 * head)) & 0x3ffu;
                const T* r = reinterpret_cast<const T*>(tiles + (size_t)head * kTileBytes);
                const int nbt = (int)(inf & 0x7fu);
                const bool sf = (inf >> 8) & 1u, slast = (inf >> 9) & 1u;
                if ((inf >> 7) & 1u)
                    itile<T, OP, CONT, true>(q, q2, active, r, nbt, sf, slast, s, cmp, in);
                else
                    itile<T, OP, CONT, false>(q, q2, active, r, nbt, sf, slast, s, cmp, in);
                __syncwarp();  // every lane has read the slot before it is refilled
                head = (head + 1) % kSlots;
                inflight--;
                ncost += (uint32_t)nbt;
            }
            g = gnext;
        }
        if (p.gcost && lane == 0) p.gcost[grp] = ncost;
        if (!valid) continue;
        T* o = p.out + oidx * (int64_t)p.out_stride;
        const int acc = p.accumulate;
        // the compensated sums (Kahan: cmp holds what the last additions rounded away)
        const T v0 = s[0] - cmp[0], v1 = s[1] - cmp[1], v2 = s[2] - cmp[2];
        if constexpr (IOp<OP>::a2) {
            const T ew = CONT ? exp_t(w) : T(0);
            const T u0 = q.ex0 * v0 + ew * in[0];
            const T u1 = q.ex1 * v1 + ew * in[1];
            const T u2 = q.ex2 * v2 + ew * in[2];
            if constexpr (OP == kOpA21) iput(o, 0, u0, acc);
            if constexpr (OP == kOpA22) iput(o, 0, u1, acc);
            if constexpr (OP == kOpA23) iput(o, 0, u2, acc);
            if constexpr (OP == kOpA3) iput(o, 0, (u0 + u1 + u2) / T(3), acc);
            if constexpr (OP == kOpA2Fused) {
                iput(o, 0, u0, acc);
                iput(o, 1, u1, acc);
                iput(o, 2, u2, acc);
            }
        } else if constexpr (IOp<OP>::a2t1) {
            constexpr int k = IOp<OP>::k;
            const T ek = k == 0 ? q.ex0 : (k == 1 ? q.ex1 : q.ex2);
            iput(o, 0, ek * v0, acc);
            iput(o, 1, ek * v1, acc);
            iput(o, 2, ek * v2, acc);
        } else if constexpr (OP == kOpA) {
            iput(o, 0, v0 + in[0], acc);
        } else if constexpr (OP == kOpCount) {
            iput(o, 0, v0, acc);
        } else {
            iput(o, 0, v0, acc);
            iput(o, 1, v1, acc);
            iput(o, 2, v2, acc);
        }
    }
}

template <typename T, int OP, bool CONT>
int ilaunch(IWalk<T> p, cudaStream_t s) {
    const int64_t groups = (p.nq + 31) / 32;
    if (groups == 0) return kOk;
    auto kern = k_iwalk<T, OP, CONT>;
    const size_t smem = walk_smem_bytes<T>();
    // per instantiation and device: the shared-memory limit and the resident blocks
    static int blocks_per_sm[64] = {0};
    int dev = 0, sms = 0;
    CAGR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(kErrInvalid, "device index too large");
    CAGR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (blocks_per_sm[dev] == 0) {
        CAGR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int nb = 0;
        CAGR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, kPWarps * 32, smem));
        blocks_per_sm[dev] = nb > 0 ? nb : 1;
    }
    const int64_t want = (groups + kPWarps - 1) / kPWarps;
    const int64_t blocks = std::min<int64_t>(want, (int64_t)blocks_per_sm[dev] * sms);
    void* ctr = nullptr;
    if (int rc = pool_alloc(&ctr, sizeof(unsigned long long), s)) return rc;
    int rc = kOk;
    if (cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), s) != cudaSuccess) {
        rc = set_error(kErrCuda, "walk counter");
    } else {
        p.counter = (unsigned long long*)ctr;
        kern<<<(unsigned)blocks, kPWarps * 32, smem, s>>>(p);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = set_error(kErrCuda, std::string("walk launch: ") + cudaGetErrorString(e));
    }
    pool_free(ctr, s);
    return rc;
}

template <typename T, int OP>
int ilaunch_cont(const IWalk<T>& p, int cont, cudaStream_t s) {
    return cont ? ilaunch<T, OP, true>(p, s) : ilaunch<T, OP, false>(p, s);
}

// ---- host side ----------------------------------------------------------------

template <typename F>
int cub_run(F&& f, cudaStream_t s) {
    size_t bytes = 0;
    CAGR_CUDA(f(nullptr, bytes));
    void* tmp = nullptr;
    if (int rc = pool_alloc(&tmp, bytes, s)) return rc;
    const cudaError_t e = f(tmp, bytes);
    pool_free(tmp, s);
    if (e != cudaSuccess) return set_error(kErrCuda, std::string("cub: ") + cudaGetErrorString(e));
    return kOk;
}

unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

template <typename T>
int setup_impl(Tree* t, Interp* I, cudaStream_t s) {
    const int64_t M = t->m;
    if (int rc = pool_alloc(&I->box_c, sizeof(T) * 4 * M, s)) return rc;
    if (int rc = pool_alloc(&I->box_h, sizeof(T) * 4 * M, s)) return rc;
    if (int rc = pool_alloc((void**)&I->iidx, sizeof(int32_t) * M, s)) return rc;
    if (int rc = pool_alloc((void**)&I->err, sizeof(int), s)) return rc;
    CAGR_CUDA(cudaMemsetAsync(I->err, 0, sizeof(int), s));
    k_box<T><<<blocks_for(M * 32, 128), 128, 0, s>>>(t->meta, (const T*)t->spos, M, (T*)I->box_c,
                                                     (T*)I->box_h);
    void *flag = nullptr, *nch = nullptr, *pos = nullptr, *chb = nullptr;
    int rc = pool_alloc(&flag, sizeof(int32_t) * M, s);
    if (!rc) rc = pool_alloc(&nch, sizeof(int32_t) * M, s);
    if (!rc) rc = pool_alloc(&pos, sizeof(int32_t) * M, s);
    if (!rc) rc = pool_alloc(&chb, sizeof(int32_t) * M, s);
    if (!rc) {
        k_iflags<<<blocks_for(M, 256), 256, 0, s>>>(t->meta, M, I->P3, (int32_t*)flag, (int32_t*)nch);
        rc = cub_run([&](void* tp, size_t& b) {
            return cub::DeviceScan::ExclusiveSum(tp, b, (const int32_t*)flag, (int32_t*)pos, (int)M, s);
        }, s);
    }
    if (!rc)
        rc = cub_run([&](void* tp, size_t& b) {
            return cub::DeviceScan::ExclusiveSum(tp, b, (const int32_t*)nch, (int32_t*)chb, (int)M, s);
        }, s);
    int32_t last[4] = {0, 0, 0, 0};
    if (!rc) {
        // totals = last exclusive prefix + last element
        cudaMemcpyAsync(&last[0], (int32_t*)pos + (M - 1), 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&last[1], (int32_t*)flag + (M - 1), 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&last[2], (int32_t*)chb + (M - 1), 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&last[3], (int32_t*)nch + (M - 1), 4, cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) rc = set_error(kErrCuda, "interp setup sync");
    }
    if (!rc) {
        I->num_interp = (int64_t)last[0] + last[1];
        I->num_chunks = (int64_t)last[2] + last[3];
        const int64_t ni = I->num_interp, nc = I->num_chunks;
        rc = pool_alloc((void**)&I->chunks, sizeof(int4) * (nc > 0 ? nc : 1), s);
        if (!rc) rc = pool_alloc((void**)&I->chunk_first, sizeof(int32_t) * (ni + 1), s);
        if (!rc) rc = pool_alloc(&I->part, sizeof(T) * 4 * (size_t)(nc > 0 ? nc : 1) * I->P3, s);
        if (!rc) {
            const int32_t ncl = (int32_t)nc;
            cudaMemcpyAsync(I->chunk_first + ni, &ncl, 4, cudaMemcpyHostToDevice, s);
            k_ichunks<<<blocks_for(M, 256), 256, 0, s>>>(t->meta, M, (const int32_t*)flag,
                                                         (const int32_t*)pos, (const int32_t*)chb,
                                                         I->iidx, I->chunks, I->chunk_first);
            // the copy above reads a host variable: finish it before returning
            if (cudaStreamSynchronize(s) != cudaSuccess) rc = set_error(kErrCuda, "interp setup");
        }
    }
    pool_free(flag, s);
    pool_free(nch, s);
    pool_free(pos, s);
    pool_free(chb, s);
    if (!rc && cudaGetLastError() != cudaSuccess) rc = set_error(kErrCuda, "interp setup launch");
    return rc;
}

template <typename T>
ChargeParams<T> charge_params(const Interp* I) {
    ChargeParams<T> p;
    p.P = I->P;
    p.P3 = I->P3;
    p.P3e = I->P3 + (I->P3 & 1);
    for (int k = 0; k < kPMax; k++) {
        p.cheb[k] = (T)I->cheb[k];
        p.omega[k] = (T)I->omega[k];
    }
    return p;
}

template <typename T>
int scatter_impl(Tree* t, Interp* I, int slot, const void* attrs, int dim, cudaStream_t s) {
    const int64_t N = t->n;
    const int P3e = I->P3 + (I->P3 & 1);
    if (!I->pts[slot]) {  // record pairs: ceil(N / 2) blocks
        if (int rc = pool_alloc(&I->pts[slot], sizeof(T) * kBlk * (size_t)((N + 1) / 2), s))
            return rc;
    }
    if (!I->prox[slot]) {
        const size_t np = (size_t)(I->num_interp > 0 ? I->num_interp : 1) * P3e;
        if (int rc = pool_alloc(&I->prox[slot], sizeof(T) * kBlk * (np / 2), s)) return rc;
    }
    I->dim[slot] = 0;
    k_ipoints<T><<<blocks_for(N, 256), 256, 0, s>>>((const T*)t->spos, t->perm, N, (const T*)attrs,
                                                    dim, (T*)I->pts[slot]);
    if (I->num_chunks > 0) {
        ChargeParams<T> cp = charge_params<T>(I);
        cp.chunks = I->chunks;
        cp.bc = (const T*)I->box_c;
        cp.bh = (const T*)I->box_h;
        cp.pts = (const T*)I->pts[slot];
        cp.part = (T*)I->part;
        k_charges<T><<<(unsigned)I->num_chunks, kChargeThreads, 0, s>>>(cp);
        k_charges_finish<T><<<blocks_for(I->num_interp * P3e, 256), 256, 0, s>>>(
            I->chunk_first, I->num_interp, I->chunks, (const T*)I->part, (const T*)I->box_c,
            (const T*)I->box_h, cp, (T*)I->prox[slot]);
    }
    if (slot == 3) {  // the A2T sum's slot: its walk layout
        const int64_t pb = (N + 1) / 2, xb = I->num_interp * P3e / 2;
        if (!I->ptsc)
            if (int rc = pool_alloc(&I->ptsc, sizeof(T) * kBlkES * (size_t)pb, s)) return rc;
        if (!I->proxc)
            if (int rc = pool_alloc(&I->proxc, sizeof(T) * kBlkES * (size_t)(xb > 0 ? xb : 1), s))
                return rc;
        k_es_compact<T><<<blocks_for(2 * pb, 256), 256, 0, s>>>((const T*)I->pts[slot],
                                                                 (T*)I->ptsc, pb);
        if (xb > 0)
            k_es_compact<T><<<blocks_for(2 * xb, 256), 256, 0, s>>>((const T*)I->prox[slot],
                                                                     (T*)I->proxc, xb);
    }
    CAGR_CUDA(cudaGetLastError());
    I->dim[slot] = dim;
    return kOk;
}

template <typename T>
int ensure_group_order(const Tree* t, Interp* I, cudaStream_t s);
template <typename T>
int launch_walk(const IWalk<T>& p, int op, int c, cudaStream_t s);

template <typename T>
int traverse_impl(const Tree* t, Interp* I, const TraverseArgs& a, cudaStream_t s) {
    IWalk<T> p;
    p.M = t->m;
    p.nq = a.queries ? a.nq : t->n;
    if (a.grid) {
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
    p.bc = (const T*)I->box_c;
    p.iidx = I->iidx;
    p.P3 = I->P3;
    p.P3e = I->P3 + (I->P3 & 1);
    p.direct_max = I->direct_max;
    p.theta = (T)I->theta;
    p.spos = (const T*)t->spos;
    p.perm = t->perm;
    p.qgroup = t->qgroup;   // self-queries in Hilbert groups: compact batches
    p.queries = (const T*)a.queries;
    p.qorder = a.qorder;
    p.widths = (const T*)a.widths;
    p.width = (T)a.width;
    p.out = (T*)a.out;
    p.accumulate = (a.accumulate ? 1 : 0) | (a.negate ? 2 : 0);
    p.err = I->err;
    p.spin = I->spin;
    // which slot and attribute dim the operator reads
    int op = a.op;
    if (a.op == kOpA2TFused) {
        if (a.slots == 3) op = kIOpA2TSum;
        else if (a.slots == 1) op = kIOpA2TShared;
        else return set_error(kErrInvalid, "the A2T right-hand side walk is not available with the "
                                           "interpolated far field: sum its two parts");
    }
    const int slot = op == kIOpA2TSum ? 3 : 0;
    const bool scalar_in = op == kOpAT || op == kOpA2T1 || op == kOpA2T2 || op == kOpA2T3 ||
                           op == kIOpA2TShared;
    const int need = op == kOpCount ? I->dim[0] : (op == kIOpA2TSum ? 3 : (scalar_in ? 1 : 3));
    if (I->dim[slot] == 0 || I->dim[slot] != need)
        return set_error(kErrState, "the charges of the right attribute dim are not computed "
                                    "(cagr_scatter / cagr_scatter3 first)");
    p.pts = (const T*)(slot == 3 ? I->ptsc : I->pts[slot]);
    p.prox = (const T*)(slot == 3 ? I->proxc : I->prox[slot]);
    const int out_dim = (op == kOpA || op == kOpA3 || op == kOpA21 || op == kOpA22 ||
                         op == kOpA23 || op == kOpCount) ? 1 : 3;
    p.out_stride = a.out_stride > 0 ? a.out_stride : out_dim;
    if (p.nq == 0) return kOk;
    const bool self = !a.queries && !a.grid;
    if (self) {
        if (int rc = ensure_group_order<T>(t, I, s)) return rc;
        p.gorder = I->gorder_valid ? I->gorder : nullptr;
        p.gcost = I->gcost;
    }
    const int rc = launch_walk<T>(p, op, a.continuous, s);
    if (rc || !self) return rc;
    // the next self walk takes the groups longest first (same outputs: a query's
    // sum does not depend on the warp that walks it)
    CAGR_CUDA(cub::DeviceRadixSort::SortPairsDescending(I->gsort_tmp, I->gsort_bytes, I->gcost,
                                                        I->gcost_sorted, I->giota, I->gorder,
                                                        (int)I->ngroups, 0, 32, s));
    I->gorder_valid = true;
    return kOk;
}

__global__ void k_iota(int32_t* a, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = (int32_t)i;
}

// The self-query groups' cost and order arrays (once per tree).
template <typename T>
int ensure_group_order(const Tree* t, Interp* I, cudaStream_t s) {
    if (I->gcost) return kOk;
    const int64_t G = (t->n + 31) / 32;
    if (int rc = pool_alloc((void**)&I->gcost, sizeof(uint32_t) * G, s)) return rc;
    if (int rc = pool_alloc((void**)&I->gcost_sorted, sizeof(uint32_t) * G, s)) return rc;
    if (int rc = pool_alloc((void**)&I->giota, sizeof(int32_t) * G, s)) return rc;
    if (int rc = pool_alloc((void**)&I->gorder, sizeof(int32_t) * G, s)) return rc;
    size_t bytes = 0;
    CAGR_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, I->gcost, I->gcost_sorted,
                                                        I->giota, I->gorder, (int)G, 0, 32, s));
    if (int rc = pool_alloc(&I->gsort_tmp, bytes > 0 ? bytes : 1, s)) return rc;
    I->gsort_bytes = bytes;
    k_iota<<<blocks_for(G, 256), 256, 0, s>>>(I->giota, G);
    CAGR_CUDA(cudaGetLastError());
    I->ngroups = G;
    return kOk;
}

template <typename T>
int launch_walk(const IWalk<T>& p, int op, int c, cudaStream_t s) {
    switch (op) {
        case kOpA: return ilaunch_cont<T, kOpA>(p, c, s);
        case kOpA3: return ilaunch_cont<T, kOpA3>(p, c, s);
        case kOpA21: return ilaunch_cont<T, kOpA21>(p, c, s);
        case kOpA22: return ilaunch_cont<T, kOpA22>(p, c, s);
        case kOpA23: return ilaunch_cont<T, kOpA23>(p, c, s);
        case kOpA2Fused: return ilaunch_cont<T, kOpA2Fused>(p, c, s);
        case kOpAT: return ilaunch<T, kOpAT, false>(p, s);
        case kOpA2T1: return ilaunch<T, kOpA2T1, false>(p, s);
        case kOpA2T2: return ilaunch<T, kOpA2T2, false>(p, s);
        case kOpA2T3: return ilaunch<T, kOpA2T3, false>(p, s);
        case kOpG: return ilaunch<T, kOpG, false>(p, s);
        case kIOpA2TSum: return ilaunch<T, kIOpA2TSum, false>(p, s);
        case kIOpA2TShared: return ilaunch<T, kIOpA2TShared, false>(p, s);
        case kOpCount: return ilaunch<T, kOpCount, false>(p, s);
        default:
            return set_error(kErrInvalid, "operator " + std::to_string(op) +
                                              " is not available with the interpolated far field");
    }
}

}  // namespace

void interp_free(Tree* t) {
    Interp* I = t ? t->interp : nullptr;
    if (!I) return;
    void* arrays[] = {I->box_c, I->box_h, I->iidx, I->chunks, I->chunk_first, I->part, I->err,
                      I->pts[0], I->pts[1], I->pts[2], I->pts[3],
                      I->prox[0], I->prox[1], I->prox[2], I->prox[3], I->ptsc, I->proxc,
                      I->gcost,
                      I->gcost_sorted, I->giota, I->gorder, I->gsort_tmp};
    for (void* p : arrays) pool_free(p, nullptr);
    delete I;
    t->interp = nullptr;
}

int interp_setup(Tree* t, int degree, double theta, int direct_max, cudaStream_t stream) {
    if (degree < 1 || degree > kPMax - 1) return set_error(kErrInvalid, "degree must be in [1, 8]");
    if (!(theta > 0.0 && theta < 1.0)) return set_error(kErrInvalid, "theta must be in (0, 1)");
    if (direct_max < 1 || direct_max > 65536)
        return set_error(kErrInvalid, "direct_max must be in [1, 65536]");
    if (t->m >= (int64_t(1) << 31) / 32) return set_error(kErrOverflow, "too many nodes");
    // the device may still use the previous mode's arrays
    if (t->interp) {
        if (cudaStreamSynchronize(stream) != cudaSuccess) return set_error(kErrCuda, "sync");
        interp_free(t);
    }
    Interp* I = new Interp();
    I->degree = degree;
    I->P = degree + 1;
    I->P3 = I->P * I->P * I->P;
    I->theta = theta;
    I->direct_max = direct_max;
    // Chebyshev points of the second kind t_k = cos(pi k / p) and their
    // barycentric weights (-1)^k, halved at both ends
    for (int k = 0; k <= degree; k++) {
        I->cheb[k] = std::cos(M_PI * (double)k / (double)degree);
        I->omega[k] = ((k & 1) ? -1.0 : 1.0) * ((k == 0 || k == degree) ? 0.5 : 1.0);
    }
    t->interp = I;
    const int rc = t->dtype == 0 ? setup_impl<float>(t, I, stream) : setup_impl<double>(t, I, stream);
    if (rc != kOk) {
        cudaStreamSynchronize(stream);
        interp_free(t);
    }
    return rc;
}

int interp_scatter(Tree* t, int slot, const void* attrs, int dim, cudaStream_t stream) {
    Interp* I = t->interp;
    if (!I) return set_error(kErrState, "the interpolated far field is not set up");
    if (slot < 0 || slot > 3) return set_error(kErrInvalid, "slot must be 0..2");
    if (dim != 1 && dim != 3) return set_error(kErrInvalid, "attr_dim must be 1 or 3");
    if (!attrs) return set_error(kErrInvalid, "attrs is null");
    return t->dtype == 0 ? scatter_impl<float>(t, I, slot, attrs, dim, stream)
                         : scatter_impl<double>(t, I, slot, attrs, dim, stream);
}

int interp_traverse(const Tree* t, const TraverseArgs& a, cudaStream_t stream) {
    Interp* I = t->interp;
    if (!I) return set_error(kErrState, "the interpolated far field is not set up");
    if (!a.out) return set_error(kErrInvalid, "output is null");
    if (a.queries && a.nq < 0) return set_error(kErrInvalid, "negative query count");
    if (!a.widths && !(a.width == a.width)) return set_error(kErrInvalid, "width is NaN");
    if (a.grid && (a.queries || a.qorder || a.gx <= 0 || a.gy <= 0 || a.gz <= 0 ||
                   a.gx > (1 << 20) || a.gy > (1 << 20) || a.gz > (1 << 20)))
        return set_error(kErrInvalid, "grid queries need positive dims <= 2^20 and no query array");
    if (a.qorder && !a.queries) return set_error(kErrInvalid, "a query order needs explicit queries");
    if (a.widths_hi) return set_error(kErrInvalid, "upper widths apply to the reference mode only");
    return t->dtype == 0 ? traverse_impl<float>(t, I, a, stream)
                         : traverse_impl<double>(t, I, a, stream);
}

namespace {
__global__ void k_group_order(const int32_t* __restrict__ perm, const int32_t* __restrict__ qgroup,
                              int64_t n, int32_t* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = perm[qgroup[i]];
}
}  // namespace

int query_groups(const Tree* t, int32_t* order, cudaStream_t stream) {
    k_group_order<<<blocks_for(t->n, 256), 256, 0, stream>>>(t->perm, t->qgroup, t->n, order);
    CAGR_CUDA(cudaGetLastError());
    return kOk;
}

int interp_status(const Tree* t) {
    const Interp* I = t->interp;
    if (!I) return kOk;
    int flag = 0;
    CAGR_CUDA(cudaMemcpy(&flag, I->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag)
        return set_error(kErrCuda, "a walk of the interpolated far field abandoned a staging wait "
                                   "(its outputs are incomplete)");
    return kOk;
}

int interp_set_wait_limit(Tree* t, int64_t spin) {
    Interp* I = t->interp;
    if (!I) return set_error(kErrState, "the interpolated far field is not set up");
    if (spin < 0 || spin > 0xffffffffLL) return set_error(kErrInvalid, "wait limit out of range");
    I->spin = (uint32_t)spin;
    return kOk;
}

int interp_info(const Tree* t, int* degree, double* theta, int* direct_max, int64_t* num_interp) {
    const Interp* I = t->interp;
    if (degree) *degree = I ? I->degree : 0;
    if (theta) *theta = I ? I->theta : 0.0;
    if (direct_max) *direct_max = I ? I->direct_max : 0;
    if (num_interp) *num_interp = I ? I->num_interp : 0;
    return kOk;
}

}  // namespace cagr
