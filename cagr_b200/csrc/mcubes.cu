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

// root position on a crossed edge: t = (iso - v0) / (v1 - v0), reference rounding
__device__ __forceinline__ float root_t(float v0, float v1, float iso) {
    return __fdiv_rn(__fsub_rn(iso, v0), __fsub_rn(v1, v0));
}

// A unit is kChunk consecutive grid points of one x-row (and the cells whose
// lowest corner they are).  Units in (row, chunk) order are in grid-point order,
// so per-unit counts scanned give each unit's first vertex and triangle.

// per unit: vertices (crossed edges owned by its points), triangles (its cells).
// A warp takes kCountZ units stacked along z at one (chunk, j), kCountWarps
// warps per block at consecutive j.  A unit needs the point rows (j, k),
// (j+1, k), (j, k+1), (j+1, k+1); walking up in k, the k+1 rows of one unit are
// the k rows of the next, so each unit reads two new rows, and the rows of the
// unit after next are loaded before this one is counted (their latency overlaps
// the work).  Lane l holds the points x = i0 + l + 32 q (q < 4, coalesced) and
// lane 0 also x = i0 + kChunk (the next unit's first point).
//
// Most units lie away from the surface: every point of their 4 rows is on the
// same side.  Each row keeps, per lane, the minimum and maximum of its points
// (a point outside the grid or in a missing row loads as NaN, which fmin and
// fmax ignore; a NaN value of the field, which is outside, loads as -inf, or
// +inf when inside means below the iso-value); two warp votes on the 4 rows'
// extremes then settle such a unit with no bit work.  The others are counted
// from ballots: inside-bit words w[q] held by every lane, where a funnel shift of
// (w[q+1] : w[q]) by l gives the inside bits of x and x + 1, so a point's
// crossings and cell case are a few bit operations.
constexpr int kCountWarps = 4;
constexpr int kCountZ = 8;

struct RowVals {
    float v[5];  // x = i0 + lane + 32 q, and (lane 0) x = i0 + kChunk
    float lo, hi;  // their minimum and maximum (points that do not exist ignored)
};

// The field value as the early-out compares it: NaN (outside) as the side
// that is never inside.
template <bool BELOW>
__device__ __forceinline__ float sided(float x) {
    return x == x ? x : (BELOW ? INFINITY : -INFINITY);
}

// The row's values at this lane's points (the row's pointer is only formed
// for rows inside the grid); a point that does not exist (ok = false: a
// missing row) loads as NaN.
template <bool BELOW>
__device__ __forceinline__ void load_row(const float* __restrict__ v, const Grid& g, int j, int k,
                                         bool ok, int i0, int lane, RowVals& r) {
    const float* row = v + ((int64_t)min(k, g.nz - 1) * g.ny + min(j, g.ny - 1)) * g.nx;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int x = i0 + lane + 32 * q;
        r.v[q] = (ok && x < g.nx) ? sided<BELOW>(row[x]) : NAN;
    }
    const int x = i0 + kChunk;
    r.v[4] = (ok && lane == 0 && x < g.nx) ? sided<BELOW>(row[x]) : NAN;
}

__device__ __forceinline__ void row_flags(RowVals& r) {
    r.lo = fminf(fminf(fminf(r.v[0], r.v[1]), fminf(r.v[2], r.v[3])), r.v[4]);
    r.hi = fmaxf(fmaxf(fmaxf(r.v[0], r.v[1]), fmaxf(r.v[2], r.v[3])), r.v[4]);
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
                                                                int32_t* __restrict__ tcnt,
                                                                int32_t* __restrict__ active,
                                                                uint32_t* __restrict__ nactive) {
    const int lane = (int)threadIdx.x & 31;
    const int j = (int)blockIdx.y * kCountWarps + ((int)threadIdx.x >> 5);
    if (j >= g.ny) return;  // whole warps; no block barrier in this kernel
    const int i0 = (int)blockIdx.x * kChunk;
    const int k0 = (int)blockIdx.z * kCountZ, k1 = min(k0 + kCountZ, g.nz);
    const bool has_y = j + 1 < g.ny;
    // rows (j, k) and (j+1, k) in slot (k - k0) % 3: the unit's k, its k + 1,
    // and k + 2 in flight (the loop is unrolled, so slots are registers)
    RowVals ra[3], rb[3];
    load_row<BELOW>(v, g, j, k0, true, i0, lane, ra[0]);
    load_row<BELOW>(v, g, j + 1, k0, has_y, i0, lane, rb[0]);
    load_row<BELOW>(v, g, j, k0 + 1, k0 + 1 < g.nz, i0, lane, ra[1]);
    load_row<BELOW>(v, g, j + 1, k0 + 1, has_y && k0 + 1 < g.nz, i0, lane, rb[1]);
    row_flags(ra[0]);
    row_flags(rb[0]);
#pragma unroll
    for (int kk = 0; kk < kCountZ; kk++) {
        const int k = k0 + kk;
        if (k >= k1) break;
        const int s0 = kk % 3, s1 = (kk + 1) % 3, s2 = (kk + 2) % 3;
        const bool has_z = k + 1 < g.nz;
        if (kk + 1 < kCountZ && k + 1 < k1) {  // the rows of the next unit's k + 1
            load_row<BELOW>(v, g, j, k + 2, k + 2 < g.nz, i0, lane, ra[s2]);
            load_row<BELOW>(v, g, j + 1, k + 2, has_y && k + 2 < g.nz, i0, lane, rb[s2]);
        }
        row_flags(ra[s1]);
        row_flags(rb[s1]);
        // (every lane: NaN extremes, no point, compare false and vote neither way)
        const float lo = fminf(fminf(ra[s0].lo, rb[s0].lo), fminf(ra[s1].lo, rb[s1].lo));
        const float hi = fmaxf(fmaxf(ra[s0].hi, rb[s0].hi), fmaxf(ra[s1].hi, rb[s1].hi));
        const bool lane_all = BELOW ? !(hi >= g.iso) : !(lo <= g.iso);  // every point inside
        const bool lane_any = BELOW ? lo < g.iso : hi > g.iso;           // some point inside
        const bool all_in = __all_sync(0xffffffffu, lane_all);
        const bool any_in = __any_sync(0xffffffffu, lane_any);
        uint32_t sum = 0;  // vertices + 2^16 * triangles of the unit
        if (any_in && !all_in) {
            uint32_t w0[5], w1[5], w2[5], w3[5];
            row_bits<BELOW>(ra[s0], true, i0, g.nx, lane, g.iso, w0);
            row_bits<BELOW>(rb[s0], has_y, i0, g.nx, lane, g.iso, w1);
            row_bits<BELOW>(ra[s1], has_z, i0, g.nx, lane, g.iso, w2);
            row_bits<BELOW>(rb[s1], has_y && has_z, i0, g.nx, lane, g.iso, w3);
            uint32_t packed = 0;  // this lane's 4 points
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int x = i0 + lane + 32 * q;
                // bit 0: inside at x, bit 1: inside at x + 1, in rows (dy, dz)
                const uint32_t b0 = __funnelshift_r(w0[q], w0[q + 1], lane) & 3u;
                const uint32_t b1 = __funnelshift_r(w1[q], w1[q + 1], lane) & 3u;
                const uint32_t b2 = __funnelshift_r(w2[q], w2[q + 1], lane) & 3u;
                const uint32_t b3 = __funnelshift_r(w3[q], w3[q + 1], lane) & 3u;
                const bool has_x = x + 1 < g.nx;
                // crossings owned by x (bits past the grid and of missing rows are 0,
                // so only the +x edge of the last point and the missing rows need masks)
                packed += (has_x ? ((b0 ^ (b0 >> 1)) & 1u) : 0u) +
                          (has_y ? ((b0 ^ b1) & 1u) : 0u) + (has_z ? ((b0 ^ b2) & 1u) : 0u);
                if (has_x && has_y && has_z)
                    packed += (uint32_t)__ldg(&ntri[b0 | (b1 << 2) | (b2 << 4) | (b3 << 6)]) << 16;
            }
            sum = __reduce_add_sync(0xffffffffu, packed);
        }
        if (lane == 0) {
            const int64_t u = ((int64_t)k * g.ny + j) * g.nchunks + blockIdx.x;
            vcnt[u] = (int32_t)(sum & 0xffffu);
            tcnt[u] = (int32_t)(sum >> 16);
            if (sum != 0u) active[atomicAdd(nactive, 1u)] = (int32_t)u;  // order is free
        }
    }
}

// per unit with output: its vertices, and its cells' triangles as vertex
// indices.  One warp per listed unit (grid-stride over the count kernel's
// list; the outputs go to the scanned positions, so the list order does not
// matter).  A cell's edges are owned by points of the 4 point rows R = dy +
// 2 dz (dy, dz in {0, 1}) at x or x + 1; a point's crossed edges need its +y
// and +z neighbour rows too, so the warp reads 8 rows: (j + dy, k + dz) for
// the 4 point rows and (j + 2, k), (j + 2, k + 1), (j, k + 2), (j + 1, k + 2);
// lanes 0 and 1 also read x = i0 + 128 and i0 + 129.
// From the rows' inside-bit words (ballots) every lane forms, per point row,
// the crossed-edge words and their prefix counts, and writes each of its
// points' edge mask and in-unit vertex prefix to per-warp shared memory; a
// triangle's vertex is then that point's unit base + prefix + the edge's rank
// among the point's crossed edges (the next unit's base for x = i0 + 128).
constexpr int kEmitWarps = 4;

template <bool BELOW>
__global__ void __launch_bounds__(32 * kEmitWarps, 5) k_mc_emit(const float* __restrict__ v, Grid g,
                                                              const int8_t* __restrict__ tri,
                                                              const uint8_t* __restrict__ ntri,
                                                              const int64_t* __restrict__ vbase,
                                                              const int64_t* __restrict__ tbase,
                                                              const int32_t* __restrict__ active,
                                                              const uint32_t* __restrict__ nactive,
                                                              float* __restrict__ verts,
                                                              int32_t* __restrict__ faces,
                                                              int64_t max_verts, int64_t max_faces) {
    __shared__ uint8_t s_m[kEmitWarps][4][kChunk + 1];     // crossed edges (bit a: +axis a)
    __shared__ uint16_t s_pre[kEmitWarps][4][kChunk];      // in-unit vertex prefix
    __shared__ int64_t s_base[kEmitWarps][8];              // R: unit base; 4 + R: next unit's
    __shared__ int8_t s_tri[256 * 3 * kMaxTri];            // the case table, per block
    __shared__ uint8_t s_ntri[256];
    for (int i = (int)threadIdx.x; i < 256 * 3 * kMaxTri; i += 32 * kEmitWarps) s_tri[i] = tri[i];
    for (int i = (int)threadIdx.x; i < 256; i += 32 * kEmitWarps) s_ntri[i] = ntri[i];
    __syncthreads();
    const int lane = (int)threadIdx.x & 31, wid = (int)threadIdx.x >> 5;
    const uint32_t n_act = *nactive;
    for (uint32_t a = blockIdx.x * kEmitWarps + wid; a < n_act; a += gridDim.x * kEmitWarps) {
        const int64_t u = active[a];
        const int chunk = (int)(u % g.nchunks);
        const int64_t rowid = u / g.nchunks;
        const int j = (int)(rowid % g.ny), k = (int)(rowid / g.ny);
        const int i0 = chunk * kChunk;
        // the unit bases, issued with the rows' loads: lane R < 4 the unit of point
        // row R, lane 4 + R the next unit of that row, lane 8 this unit's triangles
        int64_t base = 0;
        {
            const int R = lane & 3, dy = R & 1, dz = R >> 1;
            const int64_t uR = ((int64_t)(k + dz) * g.ny + (j + dy)) * g.nchunks + chunk;
            const bool rok = j + dy < g.ny && k + dz < g.nz;
            if (lane < 4 && rok) base = vbase[uR];
            else if (lane < 8 && rok && chunk + 1 < g.nchunks) base = vbase[uR + 1];
            else if (lane == 8) base = tbase[u];
        }
        // rows: 0..3 = point rows (dy, dz) = (R & 1, R >> 1); 4, 5 = (2, 0), (2, 1);
        // 6, 7 = (0, 2), (1, 2)
        constexpr int kDy[8] = {0, 1, 0, 1, 2, 2, 0, 1}, kDz[8] = {0, 0, 1, 1, 0, 1, 2, 2};
        uint32_t w[8][5];
        float val[3][5];  // raw values of point rows 0, 1, 2 (the vertex roots)
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int jj = j + kDy[r], kz = k + kDz[r];
            const bool ok = jj < g.ny && kz < g.nz;
            const float* row = v + ((int64_t)min(kz, g.nz - 1) * g.ny + min(jj, g.ny - 1)) * g.nx;
            float x5[5];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int x = i0 + lane + 32 * q;
                x5[q] = (ok && x < g.nx) ? row[x] : 0.0f;
            }
            const int xe = i0 + kChunk + lane;  // lanes 0, 1: x = i0 + 128, i0 + 129
            x5[4] = (ok && lane < 2 && xe < g.nx) ? row[xe] : 0.0f;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int x = i0 + lane + 32 * q;
                w[r][q] = __ballot_sync(0xffffffffu, ok && x < g.nx && inside<BELOW>(x5[q], g.iso));
            }
            w[r][4] = __ballot_sync(0xffffffffu,
                                    ok && lane < 2 && xe < g.nx && inside<BELOW>(x5[4], g.iso));
            if (r < 3)
#pragma unroll
                for (int q = 0; q < 5; q++) val[r][q] = x5[q];
        }
        // per point row: crossed-edge words, each lane's points' masks and prefixes
        const bool row_ok[4] = {true, j + 1 < g.ny, k + 1 < g.nz, j + 1 < g.ny && k + 1 < g.nz};
        const int ny_of[4] = {1, 4, 3, 5};  // the row one step +y of point row R
        const int nz_of[4] = {2, 3, 6, 7};  // the row one step +z of point row R
        uint32_t m0[4];  // this lane's points' crossed edges in row 0
#pragma unroll
        for (int R = 0; R < 4; R++) {
            const int dy = R & 1, dz = R >> 1;
            const bool yok = row_ok[R] && j + dy + 1 < g.ny;
            const bool zok = row_ok[R] && k + dz + 1 < g.nz;
            uint32_t cum = 0;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int xl = g.nx - 1 - (i0 + 32 * q);  // bits whose point has x + 1 < nx
                const uint32_t X = (w[R][q] ^ __funnelshift_r(w[R][q], w[R][q + 1], 1)) &
                                   (xl >= 32 ? 0xffffffffu : (xl <= 0 ? 0u : (1u << xl) - 1u));
                const uint32_t Y = yok ? (w[R][q] ^ w[ny_of[R]][q]) : 0u;
                const uint32_t Z = zok ? (w[R][q] ^ w[nz_of[R]][q]) : 0u;
                const uint32_t lo = (1u << lane) - 1u;
                const uint32_t m = ((X >> lane) & 1u) | (((Y >> lane) & 1u) << 1) |
                                   (((Z >> lane) & 1u) << 2);
                if (R == 0) m0[q] = m;
                // (a word without crossings owns no vertex: no triangle reads its entries)
                if ((X | Y | Z) != 0u) {
                    s_m[wid][R][lane + 32 * q] = (uint8_t)m;
                    s_pre[wid][R][lane + 32 * q] =
                        (uint16_t)(cum + __popc(X & lo) + __popc(Y & lo) + __popc(Z & lo));
                    cum += __popc(X) + __popc(Y) + __popc(Z);
                }
            }
            if (lane == R) {  // the next unit's first point, x = i0 + 128, in this row
                const int x = i0 + kChunk;
                uint32_t m = 0;
                if (x < g.nx) {
                    const uint32_t b = w[R][4];
                    if (x + 1 < g.nx) m |= (b ^ (b >> 1)) & 1u;
                    if (yok) m |= ((b ^ w[ny_of[R]][4]) & 1u) << 1;
                    if (zok) m |= ((b ^ w[nz_of[R]][4]) & 1u) << 2;
                }
                s_m[wid][R][kChunk] = (uint8_t)m;
            }
        }
        if (lane < 8) s_base[wid][lane] = base;
        const int64_t tb = __shfl_sync(0xffffffffu, base, 8);
        __syncwarp();
        // vertices of this unit's points (row 0)
        const int64_t vb = s_base[wid][0];
        float vx1[4];  // the +x neighbours: the next lane's value (lane 31: lane 0's of
                       // the next word, or the next unit's first point)
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const float wrap = __shfl_sync(0xffffffffu, q < 3 ? val[0][q + 1] : val[0][4], 0);
            const float down = __shfl_down_sync(0xffffffffu, val[0][q], 1);
            vx1[q] = lane == 31 ? wrap : down;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t m = m0[q];
            if (!m) continue;
            const int i = i0 + lane + 32 * q;
            const float x = __fmaf_rn(float(i), g.h, g.ox), y = __fmaf_rn(float(j), g.h, g.oy),
                        z = __fmaf_rn(float(k), g.h, g.oz);
            const float v0 = val[0][q];
            const float nbr[3] = {vx1[q], val[1][q], val[2][q]};
            int64_t o = vb + s_pre[wid][0][lane + 32 * q];
#pragma unroll
            for (int ax = 0; ax < 3; ax++) {
                if (!((m >> ax) & 1u)) continue;
                const float d = __fmul_rn(root_t(v0, nbr[ax], g.iso), g.h);
                if (o < max_verts) {  // the host reports a mesh larger than the buffers
                    verts[3 * o + 0] = ax == 0 ? __fadd_rn(x, d) : x;
                    verts[3 * o + 1] = ax == 1 ? __fadd_rn(y, d) : y;
                    verts[3 * o + 2] = ax == 2 ? __fadd_rn(z, d) : z;
                }
                o++;
            }
        }
        // triangles of this unit's cells, in x order
        if (j + 1 < g.ny && k + 1 < g.nz) {
            // the 4 words' cases and counts, then their 4 scans side by side
            int cs[4], nt[4], incl[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int x = i0 + lane + 32 * q;
                cs[q] = 0;
                nt[q] = 0;
                if (x + 1 < g.nx) {
#pragma unroll
                    for (int R = 0; R < 4; R++)
                        cs[q] |=
                            (int)((__funnelshift_r(w[R][q], w[R][q + 1], lane) & 3u) << (2 * R));
                    nt[q] = s_ntri[cs[q]];
                }
                incl[q] = nt[q];
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {  // warp inclusive scans of the counts
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int t = __shfl_up_sync(0xffffffffu, incl[q], o);
                    if (lane >= o) incl[q] += t;
                }
            }
            int64_t fo = tb;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int64_t first = fo + (incl[q] - nt[q]);
                fo += __shfl_sync(0xffffffffu, incl[q], 31);
                for (int t3 = 0; t3 < nt[q]; t3++) {
#pragma unroll
                    for (int sv = 0; sv < 3; sv++) {
                        const int e = s_tri[cs[q] * 3 * kMaxTri + 3 * t3 + sv];
                        const int ax = e >> 2, eu = e & 1, ew = (e >> 1) & 1;
                        // the point owning edge e of this cell: (dx, row R = dy + 2 dz)
                        const int dx = ax == 0 ? 0 : eu;
                        const int dy = ax == 0 ? eu : (ax == 1 ? 0 : ew);
                        const int dz = ax == 2 ? 0 : ew;
                        const int R = dy + 2 * dz, xi = lane + 32 * q + dx;
                        const uint32_t below = (1u << ax) - 1u;
                        const int64_t id =
                            xi < kChunk ? s_base[wid][R] + s_pre[wid][R][xi] +
                                              __popc(s_m[wid][R][xi] & below)
                                        : s_base[wid][4 + R] + __popc(s_m[wid][R][kChunk] & below);
                        if (first + t3 < max_faces) faces[3 * (first + t3) + sv] = (int32_t)id;
                    }
                }
            }
        }
        __syncwarp();  // the shared rows are rewritten by the warp's next unit
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
    // k / kCountZ); emit: a persistent grid whose warps take the listed units
    if (ny > 65535 || nz > 65535)
        return set_error(kErrInvalid, "marching cubes needs ny, nz <= 65535");
    const dim3 grid_c((unsigned)nchunks, (unsigned)((ny + kCountWarps - 1) / kCountWarps),
                      (unsigned)((nz + kCountZ - 1) / kCountZ)),
        grid_e(148u * 5u);  // persistent (5 blocks per SM): warps stride over the
                            // listed units
    int32_t *vcnt = nullptr, *tcnt = nullptr, *act = nullptr;
    uint32_t* nact = nullptr;
    int64_t *vbase = nullptr, *tbase = nullptr;
    McTable* dtable = nullptr;  // the caller's table on the device
    auto cleanup = [&] {
        pool_free(vcnt, s);
        pool_free(tcnt, s);
        pool_free(vbase, s);
        pool_free(tbase, s);
        pool_free(act, s);
        pool_free(nact, s);
        pool_free(dtable, s);
    };
    int rc = pool_alloc((void**)&vcnt, 4 * (U + 1), s);
    if (!rc) rc = pool_alloc((void**)&act, 4 * U, s);  // units with output, any order
    if (!rc) rc = pool_alloc((void**)&nact, 4, s);
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
    cudaMemsetAsync(nact, 0, 4, s);
    if (below)
        k_mc_count<true><<<grid_c, 32 * kCountWarps, 0, s>>>(values, g, ntri, vcnt, tcnt, act,
                                                              nact);
    else
        k_mc_count<false><<<grid_c, 32 * kCountWarps, 0, s>>>(values, g, ntri, vcnt, tcnt, act,
                                                               nact);
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
            k_mc_emit<true><<<grid_e, 32 * kEmitWarps, 0, s>>>(
                values, g, tri, ntri, vbase, tbase, act, nact, verts, faces, max_verts, max_faces);
        else
            k_mc_emit<false><<<grid_e, 32 * kEmitWarps, 0, s>>>(
                values, g, tri, ntri, vbase, tbase, act, nact, verts, faces, max_verts, max_faces);
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
