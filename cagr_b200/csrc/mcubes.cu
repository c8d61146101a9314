// Marching cubes on a regular grid of field values (the iso-surface step of the
// reconstruction).
//
// Reference role: the GaussRecon driver evaluates the field at grid corners
// and extracts the iso-surface at the median field value of the samples
// (main_GaussRecon_cuda.cu:427-494) with PoissonRecon's adaptive marching
// cubes (gaussrecon_src/Octree.cpp:852-1090).  The benchmark workloads ask for
// a regular G^3 grid, which this module handles entirely on the device.
//
// Case table: generated here, not copied.  Cube corners c = x + 2y + 4z; edge
// 4a + u + 2v runs along axis a with the other two coordinates (u, v) in
// increasing axis order.  For each of the 256 inside/outside patterns:
//  1. every face with 2 sign changes gets one segment between them; a face with
//     4 (the ambiguous pattern) gets two segments, each cutting off one INSIDE
//     corner -- a rule that depends only on that face's 4 corners, so the two
//     cells sharing a face always agree and meshes are watertight;
//  2. segments are chained into closed polygons (each crossed edge lies on two
//     faces, so every polygon is a cycle);
//  3. each polygon is oriented so that its area vector points along the sum of
//     its edges' inside-to-outside directions (outward), then fan-triangulated.
// A corner is inside when value > iso (NaN is outside).
//
// Caller-supplied tables (cagr_marching_cubes_table): the reference's layout
// (gaussrecon_src/MarchingCubes.cpp:32-324, 333-345): a case index whose bit k
// is set when corner cornerMap[k] = {0, 1, 3, 2, 4, 5, 7, 6}[k] has value < iso,
// and per case up to 5 triangles of edge ids in this file's numbering (the
// reference's Cube::EdgeIndex, Cube.cpp:86-108, is the same), -1 terminated.
// It is re-indexed on the host into the layout above with "inside" meaning
// value < iso; the device code is the same, with that predicate.
//
// Device pipeline over units of 128 consecutive grid points of one x-row:
//   count:  per unit, its points' crossed +x/+y/+z edges and its cells' triangles
//   scan:   per-unit counts -> each unit's first vertex and first triangle
//   emit:   per unit that has any, one vertex per crossed edge (the linear root
//           along it) and each cell's triangles as vertex indices (shared edges
//           share vertices); blocks skip the empty units from the scanned counts
// Output order is grid-point order for vertices (edges +x, +y, +z of a point)
// and cell order for triangles, with no per-point scratch.
#include <cub/cub.cuh>

#include <algorithm>
#include <array>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cagr.h"
#include "internal.h"

namespace cagr {
namespace {

constexpr int kMaxTri = 12;  // the generator checks the bound
constexpr int kChunk = 128;  // grid points per unit
constexpr int kEmitUnits = 256;  // units an emit block scans

struct McTable {
    int8_t tri[256][3 * kMaxTri];
    uint8_t ntri[256];
};

// corners at the two ends of edge e
inline void edge_corners(int e, int& c0, int& c1) {
    const int a = e >> 2, u = e & 1, v = (e >> 1) & 1;
    int b[3];
    // other axes in increasing order
    int o0 = a == 0 ? 1 : 0, o1 = a == 2 ? 1 : 2;
    b[a] = 0;
    b[o0] = u;
    b[o1] = v;
    c0 = b[0] + 2 * b[1] + 4 * b[2];
    b[a] = 1;
    c1 = b[0] + 2 * b[1] + 4 * b[2];
}

inline int edge_between(int ca, int cb) {
    for (int e = 0; e < 12; e++) {
        int c0, c1;
        edge_corners(e, c0, c1);
        if ((c0 == ca && c1 == cb) || (c0 == cb && c1 == ca)) return e;
    }
    return -1;
}

bool build_table(McTable& T, std::string& err) {
    std::memset(&T, 0, sizeof(T));
    // the 6 faces as corner cycles (each consecutive pair shares an edge)
    int faces[6][4];
    for (int a = 0; a < 3; a++) {
        const int o0 = a == 0 ? 1 : 0, o1 = a == 2 ? 1 : 2;
        for (int s = 0; s < 2; s++) {
            const int uv[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
            for (int q = 0; q < 4; q++) {
                int b[3];
                b[a] = s;
                b[o0] = uv[q][0];
                b[o1] = uv[q][1];
                faces[2 * a + s][q] = b[0] + 2 * b[1] + 4 * b[2];
            }
        }
    }
    for (int cfg = 0; cfg < 256; cfg++) {
        auto in = [&](int c) { return (cfg >> c) & 1; };
        // segment graph over edges: each crossed edge gets two neighbours
        std::vector<int> nb[12];
        for (int f = 0; f < 6; f++) {
            int ce[4], cc = 0;  // crossed face edges in cyclic order
            for (int q = 0; q < 4; q++) {
                const int a = faces[f][q], b = faces[f][(q + 1) & 3];
                ce[q] = in(a) != in(b) ? edge_between(a, b) : -1;
                cc += ce[q] >= 0;
            }
            if (cc == 2) {
                int x = -1, y = -1;
                for (int q = 0; q < 4; q++)
                    if (ce[q] >= 0) (x < 0 ? x : y) = ce[q];
                nb[x].push_back(y);
                nb[y].push_back(x);
            } else if (cc == 4) {
                // cut off each inside corner q: join the face edges before and after it
                for (int q = 0; q < 4; q++) {
                    if (!in(faces[f][q])) continue;
                    const int x = ce[(q + 3) & 3], y = ce[q];
                    nb[x].push_back(y);
                    nb[y].push_back(x);
                }
            } else if (cc != 0) {
                err = "odd crossing count on a face";
                return false;
            }
        }
        bool used[12] = {false};
        int nt = 0;
        for (int start = 0; start < 12; start++) {
            if (used[start] || nb[start].empty()) continue;
            if (nb[start].size() != 2) {
                err = "crossed edge without two neighbours";
                return false;
            }
            std::vector<int> cyc;
            int prev = -1, cur = start;
            while (true) {
                cyc.push_back(cur);
                used[cur] = true;
                const int nx = nb[cur][0] != prev ? nb[cur][0] : nb[cur][1];
                prev = cur;
                cur = nx;
                if (cur == start) break;
                if (used[cur] || cyc.size() > 12) {
                    err = "segments do not close";
                    return false;
                }
            }
            // orientation from edge midpoints and inside->outside directions
            double area[3] = {0, 0, 0}, g[3] = {0, 0, 0};
            std::vector<std::array<double, 3>> mid(cyc.size());
            for (size_t i = 0; i < cyc.size(); i++) {
                int c0, c1;
                edge_corners(cyc[i], c0, c1);
                const double p0[3] = {double(c0 & 1), double((c0 >> 1) & 1), double(c0 >> 2)};
                const double p1[3] = {double(c1 & 1), double((c1 >> 1) & 1), double(c1 >> 2)};
                const double sgn = in(c0) ? 1.0 : -1.0;  // inside -> outside
                for (int d = 0; d < 3; d++) {
                    mid[i][d] = 0.5 * (p0[d] + p1[d]);
                    g[d] += sgn * (p1[d] - p0[d]);
                }
            }
            for (size_t i = 0; i < cyc.size(); i++) {
                const auto& a = mid[i];
                const auto& b = mid[(i + 1) % cyc.size()];
                area[0] += a[1] * b[2] - a[2] * b[1];
                area[1] += a[2] * b[0] - a[0] * b[2];
                area[2] += a[0] * b[1] - a[1] * b[0];
            }
            if (area[0] * g[0] + area[1] * g[1] + area[2] * g[2] < 0)
                std::reverse(cyc.begin(), cyc.end());
            for (size_t i = 1; i + 1 < cyc.size(); i++) {
                if (nt >= kMaxTri) {
                    err = "too many triangles in one cell";
                    return false;
                }
                T.tri[cfg][3 * nt + 0] = (int8_t)cyc[0];
                T.tri[cfg][3 * nt + 1] = (int8_t)cyc[i];
                T.tri[cfg][3 * nt + 2] = (int8_t)cyc[i + 1];
                nt++;
            }
        }
        T.ntri[cfg] = (uint8_t)nt;
    }
    return true;
}

const McTable* host_table(std::string& err) {
    static McTable table;
    static bool ok = false;
    static std::string build_err;
    static std::once_flag once;
    std::call_once(once, [] { ok = build_table(table, build_err); });
    if (!ok) {
        err = build_err;
        return nullptr;
    }
    return &table;
}

// The case table in global memory, read through the read-only cache: lanes of
// a warp index it with different cases, which constant memory would serialise.
__device__ int8_t g_tri[256][3 * kMaxTri];
__device__ uint8_t g_ntri[256];

std::mutex g_upload_mutex;
bool g_uploaded[64] = {};

int upload_table() {
    std::string err;
    const McTable* T = host_table(err);
    if (!T) return set_error(kErrState, "marching-cubes table: " + err);
    int dev = 0;
    CAGR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(kErrInvalid, "device index too large");
    std::lock_guard<std::mutex> lock(g_upload_mutex);
    if (!g_uploaded[dev]) {
        CAGR_CUDA(cudaMemcpyToSymbol(g_tri, T->tri, sizeof(T->tri)));
        CAGR_CUDA(cudaMemcpyToSymbol(g_ntri, T->ntri, sizeof(T->ntri)));
        g_uploaded[dev] = true;
    }
    return kOk;
}

// A caller's table in the reference's layout (triangles[256][16], edge ids, -1
// terminated; case bit k = corner kCornerMap[k] below iso) re-indexed into an
// McTable whose case bit c = corner c below iso.  Rejects entries that are not
// edge ids, more than 5 triangles, and triangles on edges the case does not cross.
constexpr int kCornerMap[8] = {0, 1, 3, 2, 4, 5, 7, 6};

bool table_from_reference_layout(const int8_t* tri16, McTable& T, std::string& err) {
    std::memset(&T, 0, sizeof(T));
    for (int cs = 0; cs < 256; cs++) {
        int ci = 0;
        for (int k = 0; k < 8; k++) ci |= ((cs >> kCornerMap[k]) & 1) << k;
        const int8_t* row = tri16 + 16 * ci;
        int len = 0;
        while (len < 16 && row[len] != -1) len++;
        if (len == 16 || len % 3 != 0 || len / 3 > 5) {
            err = "case " + std::to_string(ci) + ": not a -1 terminated list of at most 5 triangles";
            return false;
        }
        for (int q = 0; q < len; q++) {
            const int e = row[q];
            int c0 = 0, c1 = 0;
            if (e >= 0 && e < 12) edge_corners(e, c0, c1);
            if (e < 0 || e >= 12 || ((cs >> c0) & 1) == ((cs >> c1) & 1)) {
                err = "case " + std::to_string(ci) + ": entry " + std::to_string(e) +
                      " is not an edge the case crosses";
                return false;
            }
            T.tri[cs][q] = (int8_t)e;
        }
        T.ntri[cs] = (uint8_t)(len / 3);
    }
    return true;
}

struct Grid {
    int nx, ny, nz, nchunks;
    int64_t units;
    float ox, oy, oz, h, iso;
};

// the inside test: value > iso (this module's table) or value < iso (a table in
// the reference's layout); NaN is outside in both
template <bool BELOW>
__device__ __forceinline__ bool inside(float v, float iso) {
    if constexpr (BELOW) return v < iso;
    return v > iso;
}

__device__ __forceinline__ int64_t gid(const Grid& g, int i, int j, int k) {
    return ((int64_t)k * g.ny + j) * g.nx + i;
}

// crossed edges owned by grid point (i, j, k): bit a = the edge toward +axis a
template <bool BELOW>
__device__ __forceinline__ uint32_t point_mask(const float* __restrict__ v, const Grid& g, int i,
                                               int j, int k) {
    const int64_t p = gid(g, i, j, k);
    const bool a = inside<BELOW>(v[p], g.iso);
    uint32_t m = 0;
    if (i + 1 < g.nx && inside<BELOW>(v[p + 1], g.iso) != a) m |= 1;
    if (j + 1 < g.ny && inside<BELOW>(v[p + g.nx], g.iso) != a) m |= 2;
    if (k + 1 < g.nz && inside<BELOW>(v[p + (int64_t)g.nx * g.ny], g.iso) != a) m |= 4;
    return m;
}

template <bool BELOW>
__device__ __forceinline__ int cell_case(const float* __restrict__ v, const Grid& g, int64_t p) {
    const int64_t sx = 1, sy = g.nx, sz = (int64_t)g.nx * g.ny;
    int c = 0;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const int64_t o = (q & 1) * sx + ((q >> 1) & 1) * sy + (q >> 2) * sz;
        c |= inside<BELOW>(v[p + o], g.iso) ? (1 << q) : 0;
    }
    return c;
}

// root position on a crossed edge: t = (iso - v0) / (v1 - v0), reference rounding
__device__ __forceinline__ float root_t(float v0, float v1, float iso) {
    return __fdiv_rn(__fsub_rn(iso, v0), __fsub_rn(v1, v0));
}

// A unit is kChunk consecutive grid points of one x-row (and the cells whose
// lowest corner they are).  Units in (row, chunk) order are in grid-point order,
// so per-unit counts scanned give each unit's first vertex and triangle.
struct Unit {
    int i0, j, k, chunk;
};

// per unit: vertices (crossed edges owned by its points), triangles (its cells).
// A warp takes kCountZ units stacked along z at one (chunk, j), kCountWarps
// warps per block at consecutive j.  A unit needs the point rows (j, k),
// (j+1, k), (j, k+1), (j+1, k+1); walking up in k, the k+1 rows of one unit are
// the k rows of the next, so each unit reads two new rows, and the rows of the
// unit after next are loaded before this one is counted (their latency overlaps
// the bit work).  Lane l holds the points x = i0 + l + 32 q (q < 4, coalesced);
// ballots turn them into inside-bit words w[q] held by every lane (w[4] bit 0:
// the next unit's first point).  A funnel shift of (w[q+1] : w[q]) by l gives
// the inside bits of x and x + 1, so a point's crossings and cell case are a
// few bit operations.
constexpr int kCountWarps = 4;
constexpr int kCountZ = 8;

struct RowVals {
    float v[5];  // x = i0 + lane + 32 q, and (lane 0) x = i0 + kChunk
};

__device__ __forceinline__ void load_row(const float* __restrict__ row, bool ok, int i0, int nx,
                                         int lane, RowVals& r) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int x = i0 + lane + 32 * q;
        r.v[q] = (ok && x < nx) ? row[x] : 0.0f;
    }
    const int x = i0 + kChunk;
    r.v[4] = (ok && lane == 0 && x < nx) ? row[x] : 0.0f;
}

template <bool BELOW>
__device__ __forceinline__ void row_bits(const RowVals& r, bool ok, int i0, int nx, int lane,
                                         float iso, uint32_t (&w)[5]) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int x = i0 + lane + 32 * q;
        w[q] = __ballot_sync(0xffffffffu, ok && x < nx && inside<BELOW>(r.v[q], iso));
    }
    const int x = i0 + kChunk;
    w[4] = __ballot_sync(0xffffffffu, ok && lane == 0 && x < nx && inside<BELOW>(r.v[4], iso));
}

template <bool BELOW>
__global__ void __launch_bounds__(32 * kCountWarps) k_mc_count(const float* __restrict__ v, Grid g,
                                                                const uint8_t* __restrict__ ntri,
                                                                int32_t* __restrict__ vcnt,
                                                                int32_t* __restrict__ tcnt) {
    const int lane = (int)threadIdx.x & 31;
    const int j = (int)blockIdx.y * kCountWarps + ((int)threadIdx.x >> 5);
    if (j >= g.ny) return;  // whole warps; no block barrier in this kernel
    const int i0 = (int)blockIdx.x * kChunk;
    const int k0 = (int)blockIdx.z * kCountZ, k1 = min(k0 + kCountZ, g.nz);
    const bool has_y = j + 1 < g.ny;
    // row (j + dy, k) starts at v + (k ny + j + dy) nx; a missing row is not read
    auto row = [&](int dy, int k) {
        return v + ((int64_t)min(k, g.nz - 1) * g.ny + min(j + dy, g.ny - 1)) * g.nx;
    };
    RowVals a0, a1, b0, b1;  // raw rows k+1 (a) and k+2 (b) in flight
    uint32_t c0[5], c1[5], n0[5], n1[5];  // bits of rows k (c) and k+1 (n)
    load_row(row(0, k0), true, i0, g.nx, lane, a0);
    load_row(row(1, k0), has_y, i0, g.nx, lane, a1);
    load_row(row(0, k0 + 1), k0 + 1 < g.nz, i0, g.nx, lane, b0);
    load_row(row(1, k0 + 1), has_y && k0 + 1 < g.nz, i0, g.nx, lane, b1);
    row_bits<BELOW>(a0, true, i0, g.nx, lane, g.iso, c0);
    row_bits<BELOW>(a1, has_y, i0, g.nx, lane, g.iso, c1);
    for (int k = k0; k < k1; k++) {
        const bool has_z = k + 1 < g.nz;
        row_bits<BELOW>(b0, has_z, i0, g.nx, lane, g.iso, n0);
        row_bits<BELOW>(b1, has_y && has_z, i0, g.nx, lane, g.iso, n1);
        if (k + 1 < k1) {  // the rows of the next unit's k + 1
            load_row(row(0, k + 2), k + 2 < g.nz, i0, g.nx, lane, b0);
            load_row(row(1, k + 2), has_y && k + 2 < g.nz, i0, g.nx, lane, b1);
        }
        uint32_t packed = 0;  // vertices + 2^16 * triangles of this lane's 4 points
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int x = i0 + lane + 32 * q;
            // bit 0: inside at x, bit 1: inside at x + 1, in rows (dy, dz) = r
            const uint32_t p0 = __funnelshift_r(c0[q], c0[q + 1], lane) & 3u;
            const uint32_t p1 = __funnelshift_r(c1[q], c1[q + 1], lane) & 3u;
            const uint32_t p2 = __funnelshift_r(n0[q], n0[q + 1], lane) & 3u;
            const uint32_t p3 = __funnelshift_r(n1[q], n1[q + 1], lane) & 3u;
            const bool has_x = x + 1 < g.nx;
            // crossings owned by x (bits past the grid and of missing rows are 0,
            // so only the +x edge of the last point and the missing rows need masks)
            packed += (has_x ? ((p0 ^ (p0 >> 1)) & 1u) : 0u) + (has_y ? ((p0 ^ p1) & 1u) : 0u) +
                      (has_z ? ((p0 ^ p2) & 1u) : 0u);
            if (has_x && has_y && has_z)
                packed += (uint32_t)__ldg(&ntri[p0 | (p1 << 2) | (p2 << 4) | (p3 << 6)]) << 16;
        }
        const uint32_t sum = __reduce_add_sync(0xffffffffu, packed);
        if (lane == 0) {
            const int64_t u = ((int64_t)k * g.ny + j) * g.nchunks + blockIdx.x;
            vcnt[u] = (int32_t)(sum & 0xffffu);
            tcnt[u] = (int32_t)(sum >> 16);
        }
#pragma unroll
        for (int q = 0; q < 5; q++) {
            c0[q] = n0[q];
            c1[q] = n1[q];
        }
    }
}

// per unit: its vertices, and its cells' triangles as vertex indices.  A cell's
// edges are owned by points in 4 point rows (dy, dz in {0, 1}) at x = i or i + 1;
// each row's in-unit vertex prefix comes from one block scan of 4 packed 16-bit
// counts, and x = i0 + kChunk (the next unit's first point) from that unit's base.
template <bool BELOW>
__global__ void __launch_bounds__(kChunk) k_mc_emit(const float* __restrict__ v, Grid g,
                                                     const int8_t* __restrict__ tri,
                                                     const uint8_t* __restrict__ ntri,
                                                     const int64_t* __restrict__ vbase,
                                                     const int64_t* __restrict__ tbase,
                                                     float* __restrict__ verts,
                                                     int32_t* __restrict__ faces,
                                                     int64_t max_verts, int64_t max_faces) {
    using ScanV = cub::BlockScan<unsigned long long, kChunk>;
    using ScanT = cub::BlockScan<int32_t, kChunk>;
    __shared__ typename ScanV::TempStorage tmp_v;
    __shared__ typename ScanT::TempStorage tmp_t;
    __shared__ uint8_t s_mask[4][kChunk + 1];
    __shared__ unsigned long long s_pre[kChunk];
    __shared__ int64_t s_base[4], s_next[4];
    __shared__ int32_t s_list[kEmitUnits];
    __shared__ int s_count;
    // the block's kEmitUnits consecutive units: the ones with vertices or
    // triangles (a small part of the grid) are listed, then emitted one by one
    // (outputs go to the scanned positions, so the list order does not matter)
    const int64_t u0 = (int64_t)blockIdx.x * kEmitUnits;
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
    for (int a = (int)threadIdx.x; a < kEmitUnits; a += kChunk) {
        const int64_t u = u0 + a;
        if (u < g.units && (vbase[u + 1] != vbase[u] || tbase[u + 1] != tbase[u]))
            s_list[atomicAdd(&s_count, 1)] = a;
    }
    __syncthreads();
    const int count = s_count;
    for (int a = 0; a < count; a++) {
        if (a > 0) __syncthreads();  // the previous unit is done with the shared arrays
        const int64_t u = u0 + s_list[a];
        Unit U;
        U.chunk = (int)(u % g.nchunks);
        const int64_t row = u / g.nchunks;
        U.j = (int)(row % g.ny);
        U.k = (int)(row / g.ny);
        U.i0 = U.chunk * kChunk;
        const int t = (int)threadIdx.x;
        const int i = U.i0 + t;
        const bool cell_row = U.j + 1 < g.ny && U.k + 1 < g.nz;
        const int rows = cell_row ? 4 : 1;
        unsigned long long c = 0;
        uint32_t own = 0;
        for (int r = 0; r < rows; r++) {
            const uint32_t m =
                i < g.nx ? point_mask<BELOW>(v, g, i, U.j + (r & 1), U.k + (r >> 1)) : 0u;
            if (r == 0) own = m;
            s_mask[r][t] = (uint8_t)m;
            c |= (unsigned long long)__popc(m) << (16 * r);
        }
        int cs = 0, nt = 0;
        if (cell_row && i + 1 < g.nx) {
            cs = cell_case<BELOW>(v, g, gid(g, i, U.j, U.k));
            nt = __ldg(&ntri[cs]);
        }
        unsigned long long cpre;
        int32_t tpre;
        ScanV(tmp_v).ExclusiveSum(c, cpre);
        ScanT(tmp_t).ExclusiveSum(nt, tpre);
        s_pre[t] = cpre;
        if (t < rows) {
            const int64_t row = (int64_t)(U.k + (t >> 1)) * g.ny + (U.j + (t & 1));
            s_base[t] = vbase[row * g.nchunks + U.chunk];
            if (U.chunk + 1 < g.nchunks) {
                s_next[t] = vbase[row * g.nchunks + U.chunk + 1];
                s_mask[t][kChunk] = (uint8_t)point_mask<BELOW>(v, g, U.i0 + kChunk, U.j + (t & 1),
                                                               U.k + (t >> 1));
            }
        }
        __syncthreads();
        if (own) {
            const float x = __fmaf_rn(float(i), g.h, g.ox), y = __fmaf_rn(float(U.j), g.h, g.oy),
                        z = __fmaf_rn(float(U.k), g.h, g.oz);
            const int64_t p = gid(g, i, U.j, U.k);
            const int64_t step[3] = {1, g.nx, (int64_t)g.nx * g.ny};
            int64_t o = s_base[0] + (int64_t)(cpre & 0xffffu);
            for (int a = 0; a < 3; a++) {
                if (!((own >> a) & 1)) continue;
                const float tt = root_t(v[p], v[p + step[a]], g.iso);
                const float d = __fmul_rn(tt, g.h);
                if (o < max_verts) {  // the host reports a mesh larger than the buffers
                    verts[3 * o + 0] = a == 0 ? __fadd_rn(x, d) : x;
                    verts[3 * o + 1] = a == 1 ? __fadd_rn(y, d) : y;
                    verts[3 * o + 2] = a == 2 ? __fadd_rn(z, d) : z;
                }
                o++;
            }
        }
        const int64_t o = tbase[u] + tpre;
        for (int q = 0; q < nt; q++) {
            for (int s = 0; s < 3; s++) {
                const int e = __ldg(&tri[cs * 3 * kMaxTri + 3 * q + s]);
                const int a = e >> 2, u = e & 1, w = (e >> 1) & 1;
                // the point owning edge e of this cell, as (dx, row r = dy + 2 dz)
                const int dx = a == 0 ? 0 : u;
                const int dy = a == 0 ? u : (a == 1 ? 0 : w);
                const int dz = a == 2 ? 0 : w;
                const int r = dy + 2 * dz, li = t + dx;
                const uint32_t below = (1u << a) - 1u;
                int64_t id;
                if (li < kChunk)
                    id = s_base[r] + (int64_t)((s_pre[li] >> (16 * r)) & 0xffffu) +
                         __popc(s_mask[r][li] & below);
                else
                    id = s_next[r] + __popc(s_mask[r][kChunk] & below);
                if (o + q < max_faces) faces[3 * (o + q) + s] = (int32_t)id;
            }
        }
    }
}

template <typename F>
int cub_scan(F&& f, cudaStream_t s) {
    size_t bytes = 0;
    CAGR_CUDA(f(nullptr, bytes));
    void* tmp = nullptr;
    if (int rc = pool_alloc(&tmp, bytes, s)) return rc;
    cudaError_t e = f(tmp, bytes);
    pool_free(tmp, s);
    if (e != cudaSuccess) return set_error(kErrCuda, cudaGetErrorString(e));
    return kOk;
}

}  // namespace

int mc_table(int8_t* tri, uint8_t* ntri) {
    std::string err;
    const McTable* T = host_table(err);
    if (!T) return set_error(kErrState, "marching-cubes table: " + err);
    if (tri) std::memcpy(tri, T->tri, sizeof(T->tri));
    if (ntri) std::memcpy(ntri, T->ntri, sizeof(T->ntri));
    return kOk;
}

int marching_cubes(const float* values, int nx, int ny, int nz, const double* origin,
                   double spacing, double iso, const int8_t* ref_table, float* verts,
                   int64_t max_verts, int32_t* faces, int64_t max_faces, int64_t* nverts,
                   int64_t* nfaces, cudaStream_t s) {
    if (!values || nx < 2 || ny < 2 || nz < 2 || !nverts || !nfaces)
        return set_error(kErrInvalid, "marching cubes needs values on a grid of at least 2^3");
    if ((int64_t)nx * ny * nz >= (int64_t(1) << 31))
        return set_error(kErrOverflow, "grid too large for 32-bit vertex indices");
    // the case table: this module's (uploaded once per device) or the caller's,
    // re-indexed and copied to the device for this call
    McTable user;
    if (ref_table) {
        std::string err;
        if (!table_from_reference_layout(ref_table, user, err))
            return set_error(kErrInvalid, "marching-cubes table: " + err);
    } else if (int rc = upload_table()) {
        return rc;
    }
    const int nchunks = (nx + kChunk - 1) / kChunk;
    const int64_t U = (int64_t)nchunks * ny * nz;
    Grid g{nx, ny, nz, nchunks, U, (float)origin[0], (float)origin[1], (float)origin[2],
           (float)spacing, (float)iso};
    // count: a warp per kCountZ units stacked in z, blocks (chunk, j / kCountWarps,
    // k / kCountZ); emit: a block per kEmitUnits consecutive units
    if (ny > 65535 || nz > 65535)
        return set_error(kErrInvalid, "marching cubes needs ny, nz <= 65535");
    const dim3 grid_c((unsigned)nchunks, (unsigned)((ny + kCountWarps - 1) / kCountWarps),
                      (unsigned)((nz + kCountZ - 1) / kCountZ)),
        grid_e((unsigned)((U + kEmitUnits - 1) / kEmitUnits));
    int32_t *vcnt = nullptr, *tcnt = nullptr;
    int64_t *vbase = nullptr, *tbase = nullptr;
    McTable* dtable = nullptr;  // the caller's table on the device
    auto cleanup = [&] {
        pool_free(vcnt, s);
        pool_free(tcnt, s);
        pool_free(vbase, s);
        pool_free(tbase, s);
        pool_free(dtable, s);
    };
    int rc = pool_alloc((void**)&vcnt, 4 * (U + 1), s);
    if (!rc) rc = pool_alloc((void**)&tcnt, 4 * (U + 1), s);
    if (!rc) rc = pool_alloc((void**)&vbase, 8 * (U + 1), s);
    if (!rc) rc = pool_alloc((void**)&tbase, 8 * (U + 1), s);
    if (!rc && ref_table) rc = pool_alloc((void**)&dtable, sizeof(McTable), s);
    const int8_t* tri = nullptr;
    const uint8_t* ntri = nullptr;
    if (!rc && ref_table) {
        // `user` outlives the copy: the stream is synchronised below
        if (cudaMemcpyAsync(dtable, &user, sizeof(McTable), cudaMemcpyHostToDevice, s) !=
            cudaSuccess)
            rc = set_error(kErrCuda, "marching-cubes table copy");
        tri = &dtable->tri[0][0];
        ntri = dtable->ntri;
    } else if (!rc) {
        void *pt = nullptr, *pn = nullptr;
        if (cudaGetSymbolAddress(&pt, g_tri) != cudaSuccess ||
            cudaGetSymbolAddress(&pn, g_ntri) != cudaSuccess)
            rc = set_error(kErrCuda, "marching-cubes table address");
        tri = (const int8_t*)pt;
        ntri = (const uint8_t*)pn;
    }
    if (rc) {
        cleanup();
        return rc;
    }
    const bool below = ref_table != nullptr;
    cudaMemsetAsync(vcnt + U, 0, 4, s);
    cudaMemsetAsync(tcnt + U, 0, 4, s);
    if (below)
        k_mc_count<true><<<grid_c, 32 * kCountWarps, 0, s>>>(values, g, ntri, vcnt, tcnt);
    else
        k_mc_count<false><<<grid_c, 32 * kCountWarps, 0, s>>>(values, g, ntri, vcnt, tcnt);
    rc = cub_scan([&](void* t, size_t& b) {
        return cub::DeviceScan::ExclusiveSum(t, b, vcnt, vbase, U + 1, s);
    }, s);
    if (!rc)
        rc = cub_scan([&](void* t, size_t& b) {
            return cub::DeviceScan::ExclusiveSum(t, b, tcnt, tbase, U + 1, s);
        }, s);
    // with output buffers, the mesh is emitted right after the one count pass
    // (writes beyond the buffers are skipped on the device) and the sizes are
    // read back once: a mesh larger than the buffers is reported with its sizes,
    // so the caller can call again with buffers of exactly those sizes
    const bool emit = verts && faces && max_verts >= 0 && max_faces >= 0;
    if (!rc && emit) {
        if (below)
            k_mc_emit<true><<<grid_e, kChunk, 0, s>>>(values, g, tri, ntri, vbase, tbase, verts,
                                                      faces, max_verts, max_faces);
        else
            k_mc_emit<false><<<grid_e, kChunk, 0, s>>>(values, g, tri, ntri, vbase, tbase, verts,
                                                       faces, max_verts, max_faces);
        if (cudaGetLastError() != cudaSuccess) rc = set_error(kErrCuda, "marching cubes launch");
    }
    int64_t nv = 0, nf = 0;
    if (!rc) {
        cudaMemcpyAsync(&nv, vbase + U, 8, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&nf, tbase + U, 8, cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) rc = set_error(kErrCuda, "marching cubes counts");
    }
    if (!rc && nv > INT32_MAX) rc = set_error(kErrOverflow, "more than 2^31 - 1 vertices");
    if (!rc) {
        *nverts = nv;
        *nfaces = nf;
        if (emit && (nv > max_verts || nf > max_faces))
            rc = set_error(kErrOverflow, "output buffers too small for the mesh (sizes returned)");
    }
    cleanup();
    return rc;
}

}  // namespace cagr
