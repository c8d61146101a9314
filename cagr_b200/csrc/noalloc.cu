// Node moments without any device allocation: cagr_scatter_noalloc.
//
// Who needs it: callers that cannot call cudaMalloc at the moment they need
// node moments -- processes whose device memory is fully owned by another
// allocator (a framework's caching pool that must not be bypassed, a fixed
// memory budget) -- or host code that already holds the tree in the
// reference's layout (the seven arrays of build_tree) and has no tree handle.  The caller passes the tree arrays, the inputs and the three output
// arrays; the only scratch the computation needs -- one arrival counter per
// node -- lives in a fixed file-scope device array, so no call allocates.
//
// Limits and sharing:
//  * at most kNoallocMaxNodes nodes (2,097,152, i.e. 8 MiB of counters, about
//    1.2 million points at leaf size 1); larger trees are rejected with
//    CAGR_ERR_INVALID;
//  * every GPU that loads the library holds the 8 MiB array until the process
//    exits;
//  * all calls share the one array: calls whose kernels overlap on the GPU
//    (different streams without ordering) race on the counters and give wrong
//    results.  Order them on one stream.  Each call clears the counters it
//    uses before its kernel runs;
//  * the first call on a device looks up the array's device address (once per
//    device, with that device current).
//
// The computation is the same bottom-up pass as the tree-handle path
// (moments.cu) and the same floating-point operation order as the reference
// scatter (wn_treecode_cuda_kernels.cu:419-523), so results are identical to
// cagr_scatter + cagr_scatter_export.
#include <mutex>
#include <string>

#include "../../include/cagr.h"
#include "internal.h"

namespace {

constexpr int64_t kNoallocMaxNodes = int64_t(1) << 21;
constexpr int kMaxDevices = 64;
constexpr int kBlock = 256;

static __device__ __align__(256) uint32_t g_noalloc_counters[kNoallocMaxNodes];

std::mutex g_setup_mutex;
uint32_t* g_counters_ptr[kMaxDevices] = {};

template <typename T>
__device__ __forceinline__ T weight_of(const T* a, int dim) {
    using namespace cagr;
    if (dim == 1) return sqrt_rn(mul_rn(a[0], a[0]));
    return sqrt_rn(add_rn(add_rn(mul_rn(a[0], a[0]), mul_rn(a[1], a[1])), mul_rn(a[2], a[2])));
}

template <typename T, int DIM>
__global__ void __launch_bounds__(kBlock)
    k_scatter_noalloc(const int64_t* __restrict__ parent, const int64_t* __restrict__ children,
                      const uint8_t* __restrict__ is_leaf, const int64_t* __restrict__ npts,
                      const int64_t* __restrict__ n2p, const int64_t* __restrict__ n2p_start,
                      int64_t M, const T* __restrict__ points, const T* __restrict__ weights,
                      const T* __restrict__ attrs, T* out_attrs, T* out_rep, T* out_w,
                      uint32_t* counters) {
    using namespace cagr;
    int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= M || !is_leaf[node]) return;

    T W = T(0), A[3] = {T(0), T(0), T(0)}, R[3] = {T(0), T(0), T(0)}, P[3] = {T(0), T(0), T(0)};
    int64_t count = npts[node];
    {
        const int64_t base = n2p_start[node];
        for (int64_t j = 0; j < count; j++) {
            const int64_t p = n2p[base + j];
            T a[3] = {T(0), T(0), T(0)};
            for (int c = 0; c < DIM; c++) a[c] = attrs[p * DIM + c];
            const T w = weights ? weights[p] : weight_of(a, DIM);
            W = add_rn(W, w);
            for (int c = 0; c < DIM; c++) A[c] = add_rn(A[c], a[c]);
            for (int d = 0; d < 3; d++) {
                const T y = points[p * 3 + d];
                R[d] = add_rn(R[d], mul_rn(y, w));
                P[d] = add_rn(P[d], y);
            }
        }
    }
    while (true) {
        T c[3];
        if (W > T(0)) {
            const T inv = div_rn(T(1), W);
            for (int d = 0; d < 3; d++) c[d] = mul_rn(R[d], inv);
        } else {
            const T inv = div_rn(T(1), T(count));
            for (int d = 0; d < 3; d++) c[d] = mul_rn(P[d], inv);
        }
        for (int a = 0; a < DIM; a++) out_attrs[node * DIM + a] = A[a];
        for (int d = 0; d < 3; d++) out_rep[node * 3 + d] = c[d];
        out_w[node] = W;
        const int64_t par = parent[node];
        if (par < 0) return;
        __threadfence();
        int nch = 0;
        for (int k = 0; k < 8; k++) nch += children[par * 8 + k] >= 0 ? 1 : 0;
        const uint32_t arrived = atomicAdd(&counters[par], 1u);
        if (arrived + 1u != (uint32_t)nch) return;
        __threadfence();
        node = par;
        count = npts[par];
        W = T(0);
        for (int d = 0; d < 3; d++) A[d] = R[d] = P[d] = T(0);
        for (int k = 0; k < 8; k++) {
            const int64_t ch = children[par * 8 + k];
            if (ch < 0) continue;
            const T wc = __ldcg(out_w + ch);
            W = add_rn(W, wc);
            for (int a = 0; a < DIM; a++) A[a] = add_rn(A[a], __ldcg(out_attrs + ch * DIM + a));
            for (int d = 0; d < 3; d++) {
                const T rc = __ldcg(out_rep + ch * 3 + d);
                R[d] = add_rn(R[d], mul_rn(rc, wc));
                P[d] = add_rn(P[d], rc);
            }
        }
    }
}

// Device address of the counter array for the current device (looked up once).
int counters_for_current_device(uint32_t** out) {
    using cagr::set_error;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(CAGR_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return set_error(CAGR_ERR_INVALID, "device index too large");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_counters_ptr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_counters);
        if (e != cudaSuccess)
            return set_error(CAGR_ERR_CUDA,
                             std::string("cudaGetSymbolAddress(no-alloc counters): ") +
                                 cudaGetErrorString(e));
        g_counters_ptr[dev] = static_cast<uint32_t*>(ptr);
    }
    *out = g_counters_ptr[dev];
    return CAGR_OK;
}

template <typename T>
int launch(const int64_t* parent, const int64_t* children, const uint8_t* is_leaf,
           const int64_t* npts, const int64_t* n2p, const int64_t* n2p_start, int64_t M,
           const void* points, const void* weights, const void* attrs, int dim, void* out_attrs,
           void* out_rep, void* out_w, uint32_t* counters, cudaStream_t s) {
    const unsigned grid = (unsigned)((M + kBlock - 1) / kBlock);
    if (dim == 3)
        k_scatter_noalloc<T, 3><<<grid, kBlock, 0, s>>>(
            parent, children, is_leaf, npts, n2p, n2p_start, M, (const T*)points,
            (const T*)weights, (const T*)attrs, (T*)out_attrs, (T*)out_rep, (T*)out_w, counters);
    else
        k_scatter_noalloc<T, 1><<<grid, kBlock, 0, s>>>(
            parent, children, is_leaf, npts, n2p, n2p_start, M, (const T*)points,
            (const T*)weights, (const T*)attrs, (T*)out_attrs, (T*)out_rep, (T*)out_w, counters);
    return CAGR_OK;
}

}  // namespace

extern "C" int cagr_scatter_noalloc(const int64_t* parent_dev, const int64_t* children_dev,
                                    const uint8_t* is_leaf_dev, const int64_t* npts_dev,
                                    const int64_t* n2p_dev, const int64_t* n2p_start_dev,
                                    int64_t num_nodes, int dtype, const void* points_dev,
                                    const void* weights_dev, const void* attrs_dev, int attr_dim,
                                    void* node_attrs_dev, void* reppoints_dev,
                                    void* node_weights_dev, void* stream) {
    using cagr::set_error;
    if (num_nodes <= 0) return set_error(CAGR_ERR_INVALID, "num_nodes must be positive");
    if (num_nodes > kNoallocMaxNodes)
        return set_error(CAGR_ERR_INVALID,
                         "num_nodes " + std::to_string(num_nodes) +
                             " exceeds the no-alloc scratch capacity of " +
                             std::to_string(kNoallocMaxNodes) + " nodes");
    if (dtype != CAGR_F32 && dtype != CAGR_F64)
        return set_error(CAGR_ERR_INVALID, "dtype must be CAGR_F32 or CAGR_F64");
    if (attr_dim != 1 && attr_dim != 3) return set_error(CAGR_ERR_INVALID, "attr_dim must be 1 or 3");
    if (!parent_dev || !children_dev || !is_leaf_dev || !npts_dev || !n2p_dev || !n2p_start_dev ||
        !points_dev || !attrs_dev || !node_attrs_dev || !reppoints_dev || !node_weights_dev)
        return set_error(CAGR_ERR_INVALID, "a required pointer is null");
    uint32_t* counters = nullptr;
    if (int rc = counters_for_current_device(&counters)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // the counters of this call must start at zero (a clear, not an allocation)
    cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(uint32_t) * (size_t)num_nodes, s);
    if (e != cudaSuccess) return set_error(CAGR_ERR_CUDA, cudaGetErrorString(e));
    if (dtype == CAGR_F32)
        launch<float>(parent_dev, children_dev, is_leaf_dev, npts_dev, n2p_dev, n2p_start_dev,
                      num_nodes, points_dev, weights_dev, attrs_dev, attr_dim, node_attrs_dev,
                      reppoints_dev, node_weights_dev, counters, s);
    else
        launch<double>(parent_dev, children_dev, is_leaf_dev, npts_dev, n2p_dev, n2p_start_dev,
                       num_nodes, points_dev, weights_dev, attrs_dev, attr_dim, node_attrs_dev,
                       reppoints_dev, node_weights_dev, counters, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(CAGR_ERR_CUDA, cudaGetErrorString(e));
    return CAGR_OK;
}
