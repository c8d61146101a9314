// Bottom-up node moments ("scatter point attributes to nodes").
//
// Reference: mayueji/CAGR CUDA-based/ext/wn_treecode/wn_treecode_cuda/
// wn_treecode_cuda_torch_interface.cu:41-134 launches one leaf kernel and then
// 2*tree_depth level kernels (wn_treecode_cuda_kernels.cu:419-553), each over
// all M nodes.  Here one launch does the whole reduction: one thread per leaf
// computes the leaf moments, then climbs; at every parent the last-arriving
// child (atomic arrival counter, reset by the thread that completes the node)
// computes the parent from its children in octant order.  The floating-point
// operation order is the reference's, so node sums, weights and centroids are
// bit-identical to the reference's host build:
//   leaf:     for points in node2point order  W += w;  A += a;  R += y*w;  P += y
//   internal: for children in octant order    W += Wc; A += Ac; R += Rc*Wc; P += Rc
//   centroid: W > 0 ? R * (1/W) : P * (1/npts)            (:456-461, :510-517)
// The same launch writes the Morton-ordered point records the traversal reads,
// and every record carries exp(-c/2) per axis so the traversal can form the
// convection factor exp((x-c)_k/2) as exp(x_k/2) * exp(-c_k/2) without a
// transcendental per pair.
#include <string>

#include "internal.h"

namespace cagr {
namespace {

constexpr int kBlock = 256;

template <typename T>
__device__ __forceinline__ T weight_of(const T* a, int dim) {
    if (dim == 1) return sqrt_rn(mul_rn(a[0], a[0]));
    return sqrt_rn(add_rn(add_rn(mul_rn(a[0], a[0]), mul_rn(a[1], a[1])), mul_rn(a[2], a[2])));
}

template <typename T>
__device__ __forceinline__ void write_record(T* r, const T* pos, const T* acc, int dim, T W) {
    r[REC_X] = pos[0];
    r[REC_Y] = pos[1];
    r[REC_Z] = pos[2];
    r[REC_E1] = exp_t(pos[0] * T(-0.5));
    r[REC_E2] = exp_t(pos[1] * T(-0.5));
    r[REC_E3] = exp_t(pos[2] * T(-0.5));
    r[REC_A0] = acc[0];
    r[REC_A1] = dim == 3 ? acc[1] : T(0);
    r[REC_A2] = dim == 3 ? acc[2] : T(0);
    r[REC_W] = W;
    r[10] = T(0);
    r[11] = T(0);
}

template <typename T, int DIM>
__global__ void __launch_bounds__(kBlock)
    k_moments(int64_t num_leaves, int64_t M, const int32_t* __restrict__ leaf_ids,
              const int4* __restrict__ meta, const int32_t* __restrict__ parent,
              const int32_t* __restrict__ perm, const int32_t* __restrict__ invperm,
              const int32_t* __restrict__ n2p, const int64_t* __restrict__ n2p_start,
              const T* __restrict__ spos, const T* __restrict__ attrs,
              const T* __restrict__ weights, uint32_t* __restrict__ counters, T* __restrict__ rec) {
    const int64_t li = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= num_leaves) return;
    int node = leaf_ids[li];
    const int4 lm = meta[node];
    const int pstart = lm.y, np = lm.z;

    // point records for the leaf's Morton range
    for (int j = 0; j < np; j++) {
        const int s = pstart + j;
        const int p = perm[s];
        T pos[3] = {spos[3 * s], spos[3 * s + 1], spos[3 * s + 2]};
        T a[3] = {T(0), T(0), T(0)};
        for (int c = 0; c < DIM; c++) a[c] = attrs[(int64_t)p * DIM + c];
        const T w = weights ? weights[p] : weight_of(a, DIM);
        write_record(rec + (M + s) * CAGR_REC_STRIDE, pos, a, DIM, w);
    }

    // leaf moments, points in node2point (ascending original index) order
    T W = T(0), A[3] = {T(0), T(0), T(0)}, R[3] = {T(0), T(0), T(0)}, P[3] = {T(0), T(0), T(0)};
    {
        const int64_t base = n2p_start[node];
        for (int j = 0; j < np; j++) {
            const int p = (np == 1) ? perm[pstart] : n2p[base + j];
            const int s = (np == 1) ? pstart : invperm[p];
            T a[3] = {T(0), T(0), T(0)};
            for (int c = 0; c < DIM; c++) a[c] = attrs[(int64_t)p * DIM + c];
            const T w = weights ? weights[p] : weight_of(a, DIM);
            W = add_rn(W, w);
            for (int c = 0; c < DIM; c++) A[c] = add_rn(A[c], a[c]);
            for (int d = 0; d < 3; d++) {
                const T y = spos[3 * s + d];
                R[d] = add_rn(R[d], mul_rn(y, w));
                P[d] = add_rn(P[d], y);
            }
        }
    }

    int count = np;  // points under `node`: the zero-weight centroid divides by it
    while (true) {
        T c[3];
        if (W > T(0)) {
            const T inv = div_rn(T(1), W);
            for (int d = 0; d < 3; d++) c[d] = mul_rn(R[d], inv);
        } else {
            // (wn_treecode_cuda_kernels.cu:459-460 for leaves, :515-517 for internal
            // nodes, where it divides a sum of child centroids by the point count)
            const T inv = div_rn(T(1), T(count));
            for (int d = 0; d < 3; d++) c[d] = mul_rn(P[d], inv);
        }
        write_record(rec + (int64_t)node * CAGR_REC_STRIDE, c, A, DIM, W);
        if (node == 0) return;
        // publish this node, then arrive at the parent
        __threadfence();
        const int par = parent[node];
        const int4 pm = meta[par];
        const uint32_t arrived = atomicAdd(&counters[par], 1u);
        if (arrived + 1u != (uint32_t)meta_nchild(pm.w)) return;
        counters[par] = 0u;  // every child has arrived: ready for the next pass
        __threadfence();
        node = par;
        count = pm.z;
        W = T(0);
        for (int d = 0; d < 3; d++) {
            A[d] = T(0);
            R[d] = T(0);
            P[d] = T(0);
        }
        // children of `node` in octant order = preorder: node+1, then skip pointers;
        // read through L2 (other threads wrote them during this launch)
        const int end = pm.x;
        for (int ch = node + 1; ch < end;) {
            const T* r = rec + (int64_t)ch * CAGR_REC_STRIDE;
            const T wc = __ldcg(r + REC_W);
            W = add_rn(W, wc);
            for (int cc = 0; cc < DIM; cc++) A[cc] = add_rn(A[cc], __ldcg(r + REC_A0 + cc));
            for (int d = 0; d < 3; d++) {
                const T rc = __ldcg(r + REC_X + d);
                R[d] = add_rn(R[d], mul_rn(rc, wc));
                P[d] = add_rn(P[d], rc);
            }
            ch = meta[ch].x;
        }
    }
}

template <typename T, int DIM>
__global__ void k_export_moments(const T* __restrict__ rec, int64_t M, T* __restrict__ node_attrs,
                                 T* __restrict__ reppoints, T* __restrict__ weights) {
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M) return;
    const T* r = rec + n * CAGR_REC_STRIDE;
    if (node_attrs)
        for (int c = 0; c < DIM; c++) node_attrs[n * DIM + c] = r[REC_A0 + c];
    if (reppoints)
        for (int d = 0; d < 3; d++) reppoints[n * 3 + d] = r[REC_X + d];
    if (weights) weights[n] = r[REC_W];
}

template <typename T>
int launch_moments(Tree* t, int slot, const void* attrs, int dim, const void* weights,
                   cudaStream_t s) {
    if (!t->rec[slot]) {
        cudaError_t e =
            cudaMalloc(&t->rec[slot], sizeof(T) * (size_t)(t->m + t->n) * CAGR_REC_STRIDE);
        if (e != cudaSuccess) {
            t->rec[slot] = nullptr;
            return set_error(kErrAlloc, std::string("record allocation: ") + cudaGetErrorString(e));
        }
    }
    const unsigned grid = (unsigned)((t->num_leaves + kBlock - 1) / kBlock);
    if (dim == 3)
        k_moments<T, 3><<<grid, kBlock, 0, s>>>(t->num_leaves, t->m, t->leaf_ids, t->meta,
                                                t->parent, t->perm, t->invperm, t->n2p,
                                                t->n2p_start, (const T*)t->spos, (const T*)attrs,
                                                (const T*)weights, t->counters, (T*)t->rec[slot]);
    else
        k_moments<T, 1><<<grid, kBlock, 0, s>>>(t->num_leaves, t->m, t->leaf_ids, t->meta,
                                                t->parent, t->perm, t->invperm, t->n2p,
                                                t->n2p_start, (const T*)t->spos, (const T*)attrs,
                                                (const T*)weights, t->counters, (T*)t->rec[slot]);
    CAGR_CUDA(cudaGetLastError());
    t->rec_dim[slot] = dim;
    return kOk;
}

}  // namespace

int moments(Tree* t, int slot, const void* attrs, int dim, const void* weights,
            cudaStream_t stream) {
    if (slot < 0 || slot > 2) return set_error(kErrInvalid, "moment slot must be 0, 1 or 2");
    if (dim != 1 && dim != 3) return set_error(kErrInvalid, "attribute dim must be 1 or 3");
    if (!attrs) return set_error(kErrInvalid, "attrs is null");
    return t->dtype == 0 ? launch_moments<float>(t, slot, attrs, dim, weights, stream)
                         : launch_moments<double>(t, slot, attrs, dim, weights, stream);
}

int moments_export(const Tree* t, int slot, void* node_attrs, void* reppoints, void* weights,
                   cudaStream_t stream) {
    if (slot < 0 || slot > 2 || !t->rec[slot] || t->rec_dim[slot] == 0)
        return set_error(kErrState, "no moments computed in this slot");
    const unsigned grid = (unsigned)((t->m + kBlock - 1) / kBlock);
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
