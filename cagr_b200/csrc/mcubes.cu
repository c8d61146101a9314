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

constexpr int kMaxTri = 12;   // triangles a case row of the exported table has room for
constexpr int kCellTris = 5;  // triangles a case has (the generator and the reference-layout
                              // check enforce it)
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
                if (nt >= kCellTris) {
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
        if (len == 16 || len % 3 != 0 || len / 3 > kCellTris) {
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
// This kernel takes rows that need not start on a 16-byte boundary; rows that
// do go to k_mc_count_bulk below, which shares its per-unit steps.
// A warp takes kCountZ units stacked along z at one (chunk, j), kCountWarps
// warps per block at consecutive j.  A unit needs the point rows (j, k),
// (j+1, k), (j, k+1), (j+1, k+1); walking up in k, the k+1 rows of one unit are
// the k rows of the next, so each unit reads two new rows, and the rows of the
// next kCountAhead units are in flight while one is counted (their latency
// overlaps the work).  Lane l holds x = i0 + l + 32 q (q < 4, coalesced scalar
// loads) and x = i0 + kChunk (the next unit's first point, one broadcast
// load).  (The bulk kernel's lanes hold x = i0 + 4 l + q instead: VEC below.)
//
// Coordinates past the grid are clamped to the row's last point and a missing
// row (j + 1 = ny, k + 1 = nz) is read as the unit's own row j or plane k: the
// copies are points of the same unit, so its extremes do not change, and every
// load is of a point inside the grid.  Most units lie away from the surface:
// every point of their 4 rows is on the same side.  Per lane, a unit keeps two
// extremes of its points: one that propagates NaN (min for inside = above the
// iso-value, max for below: "every point inside" is this extreme inside, and a
// NaN, which is outside, makes it false) and one that ignores NaN (the other
// of max / min: "some point inside").  Two warp votes settle such a unit with
// no bit work.  The others are counted from per-point inside bits, masked to
// the points and rows that exist.
constexpr int kCountWarps = 4;
constexpr int kCountZ = 8;
constexpr int kCountAhead = 1;  // planes in flight beyond the unit's k + 1
constexpr int kCountSlots = kCountAhead + 2;
constexpr unsigned kFull = 0xffffffffu;

// minimum and maximum that give NaN when either operand is NaN
__device__ __forceinline__ float min_nan(float a, float b) {
    float d;
    asm("min.NaN.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float max_nan(float a, float b) {
    float d;
    asm("max.NaN.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
// the extreme for "every point inside" (propagates NaN) and for "some point
// inside" (ignores NaN)
template <bool BELOW>
__device__ __forceinline__ float ext_all(float a, float b) {
    return BELOW ? max_nan(a, b) : min_nan(a, b);
}
template <bool BELOW>
__device__ __forceinline__ float ext_any(float a, float b) {
    return BELOW ? fminf(a, b) : fmaxf(a, b);
}

struct RowVals {
    float v[4];  // x = i0 + lane + 32 q (VEC: x = i0 + 4 lane + q)
    float e;     // x = i0 + kChunk
    float xa, xn;  // the row's two extremes (ext_all, ext_any) at this lane
};

__device__ __forceinline__ const float* row_ptr(const float* __restrict__ v, const Grid& g, int j,
                                                int k) {
    return v + ((int64_t)min(k, g.nz - 1) * g.ny + j) * g.nx;
}

__device__ __forceinline__ void load_row(const float* __restrict__ row, int i0, int nx, int lane,
                                         RowVals& r) {
#pragma unroll
    for (int q = 0; q < 4; q++) r.v[q] = __ldg(row + min(i0 + lane + 32 * q, nx - 1));
    r.e = __ldg(row + min(i0 + kChunk, nx - 1));
}

template <bool BELOW>
__device__ __forceinline__ void row_ext(RowVals& r) {
    r.xa = ext_all<BELOW>(ext_all<BELOW>(ext_all<BELOW>(r.v[0], r.v[1]),
                                         ext_all<BELOW>(r.v[2], r.v[3])), r.e);
    r.xn = ext_any<BELOW>(ext_any<BELOW>(ext_any<BELOW>(r.v[0], r.v[1]),
                                         ext_any<BELOW>(r.v[2], r.v[3])), r.e);
}

// VEC: a lane's fixed facts about its points x0 + q (x0 = i0 + 4 lane), set
// once per warp: xin bit q = the point exists (x0 + q < nx), xm bit q = it has
// a +x neighbour (x0 + q + 1 < nx), e_ok = x = i0 + kChunk exists, last = lane 31
struct LaneVec {
    uint32_t xin = 0, xm = 0;
    bool e_ok = false, last = false;
};

__device__ __forceinline__ LaneVec lane_vec(int i0, int nx, int lane) {
    LaneVec l;
    const int x0 = i0 + 4 * lane;
    const int have = nx - x0, room = nx - 1 - x0;
    l.xin = have >= 4 ? 0xfu : have > 0 ? (1u << have) - 1u : 0u;
    l.xm = room >= 4 ? 0xfu : room > 0 ? (1u << room) - 1u : 0u;
    l.e_ok = i0 + kChunk < nx;
    l.last = lane == 31;
    return l;
}

// VEC: the inside bits of this lane's points x0 + q (bit q) and of x0 + 4 (bit
// 4: the next lane's first point, or x = i0 + kChunk for lane 31); 0 for a
// point past the grid or a missing row (ok = false)
template <bool BELOW>
__device__ __forceinline__ uint32_t row_nibble(const RowVals& r, bool ok, const LaneVec& l,
                                               float iso) {
    uint32_t b = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) b |= inside<BELOW>(r.v[q], iso) ? 1u << q : 0u;
    b = ok ? b & l.xin : 0u;
    const uint32_t nb = __shfl_down_sync(kFull, b, 1) & 1u;
    const uint32_t eb = (ok && l.e_ok && inside<BELOW>(r.e, iso)) ? 1u : 0u;
    return b | ((l.last ? eb : nb) << 4);
}

// scalar layout: ballot words, bit l of w[q] = inside at x = i0 + l + 32 q,
// w[4] bit 0 = inside at x = i0 + kChunk
template <bool BELOW>
__device__ __forceinline__ void row_words(const RowVals& r, bool ok, int i0, int nx, int lane,
                                          float iso, uint32_t (&w)[5]) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int x = i0 + lane + 32 * q;
        w[q] = __ballot_sync(kFull, ok && x < nx && inside<BELOW>(r.v[q], iso));
    }
    w[4] = __ballot_sync(kFull, ok && lane == 0 && i0 + kChunk < nx && inside<BELOW>(r.e, iso));
}

// vertices + 2^16 * triangles of a unit the surface may cross (warp-uniform
// call; ntri: the case table's triangle counts, in shared memory for VEC,
// global for the scalar layout, whose short blocks gain nothing from staging
// it: 302 -> 325 us on a 513^3 field when they did)
template <bool BELOW, bool VEC>
__device__ __forceinline__ uint32_t unit_sum(const RowVals& r0, const RowVals& r1,
                                             const RowVals& r2, const RowVals& r3, bool has_y,
                                             bool has_z, int i0, const Grid& g, int lane,
                                             const uint8_t* __restrict__ ntri, const LaneVec& lv) {
    uint32_t packed = 0;  // this lane's 4 points
    if constexpr (VEC) {
        const uint32_t e0 = row_nibble<BELOW>(r0, true, lv, g.iso);
        const uint32_t e1 = row_nibble<BELOW>(r1, has_y, lv, g.iso);
        const uint32_t e2 = row_nibble<BELOW>(r2, has_z, lv, g.iso);
        const uint32_t e3 = row_nibble<BELOW>(r3, has_y && has_z, lv, g.iso);
        const uint32_t xm = lv.xm;  // points of this lane with a +x neighbour
        packed = __popc((e0 ^ (e0 >> 1)) & xm);
        if (has_y) packed += __popc((e0 ^ e1) & 0xfu);
        if (has_z) packed += __popc((e0 ^ e2) & 0xfu);
        if (has_y && has_z) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t cs = ((e0 >> q) & 3u) | (((e1 >> q) & 3u) << 2) |
                                    (((e2 >> q) & 3u) << 4) | (((e3 >> q) & 3u) << 6);
                if ((xm >> q) & 1u) packed += (uint32_t)ntri[cs] << 16;
            }
        }
    } else {
        uint32_t w0[5], w1[5], w2[5], w3[5];
        row_words<BELOW>(r0, true, i0, g.nx, lane, g.iso, w0);
        row_words<BELOW>(r1, has_y, i0, g.nx, lane, g.iso, w1);
        row_words<BELOW>(r2, has_z, i0, g.nx, lane, g.iso, w2);
        row_words<BELOW>(r3, has_y && has_z, i0, g.nx, lane, g.iso, w3);
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
            packed += (has_x ? ((b0 ^ (b0 >> 1)) & 1u) : 0u) + (has_y ? ((b0 ^ b1) & 1u) : 0u) +
                      (has_z ? ((b0 ^ b2) & 1u) : 0u);
            if (has_x && has_y && has_z)
                packed += (uint32_t)__ldg(&ntri[b0 | (b1 << 2) | (b2 << 4) | (b3 << 6)]) << 16;
        }
    }
    return __reduce_add_sync(kFull, packed);
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
    const int jb = has_y ? j + 1 : j;
    // rows (j, k) and (j+1, k) of plane k in slot (k - k0) % kCountSlots (the
    // loop is unrolled, so slots are registers); planes k0 .. k0 + kCountAhead first
    RowVals ra[kCountSlots], rb[kCountSlots];
#pragma unroll
    for (int p = 0; p <= kCountAhead; p++) {
        load_row(row_ptr(v, g, j, k0 + p), i0, g.nx, lane, ra[p]);
        load_row(row_ptr(v, g, jb, k0 + p), i0, g.nx, lane, rb[p]);
    }
    row_ext<BELOW>(ra[0]);
    row_ext<BELOW>(rb[0]);
#pragma unroll
    for (int kk = 0; kk < kCountZ; kk++) {
        const int k = k0 + kk;
        if (k >= k1) break;
        const int s0 = kk % kCountSlots, s1 = (kk + 1) % kCountSlots;
        // the plane the unit kCountAhead further up needs as its k + 1, into the
        // slot of plane k - 1 (its unit is done)
        constexpr int kA = kCountAhead + 1;
        if (kk + kA <= kCountZ && k + kA <= k1) {
            const int sn = (kk + kA) % kCountSlots;
            load_row(row_ptr(v, g, j, k + kA), i0, g.nx, lane, ra[sn]);
            load_row(row_ptr(v, g, jb, k + kA), i0, g.nx, lane, rb[sn]);
        }
        row_ext<BELOW>(ra[s1]);
        row_ext<BELOW>(rb[s1]);
        const float xa = ext_all<BELOW>(ext_all<BELOW>(ra[s0].xa, rb[s0].xa),
                                        ext_all<BELOW>(ra[s1].xa, rb[s1].xa));
        const float xn = ext_any<BELOW>(ext_any<BELOW>(ra[s0].xn, rb[s0].xn),
                                        ext_any<BELOW>(ra[s1].xn, rb[s1].xn));
        const bool all_in = __all_sync(kFull, inside<BELOW>(xa, g.iso));
        const bool any_in = __any_sync(kFull, inside<BELOW>(xn, g.iso));
        uint32_t sum = 0;  // vertices + 2^16 * triangles of the unit
        if (any_in && !all_in)
            sum = unit_sum<BELOW, false>(ra[s0], rb[s0], ra[s1], rb[s1], has_y, k + 1 < g.nz, i0, g,
                                         lane, ntri, LaneVec{});
        if (lane == 0) {
            const int64_t u = ((int64_t)k * g.ny + j) * g.nchunks + blockIdx.x;
            vcnt[u] = (int32_t)(sum & 0xffffu);
            tcnt[u] = (int32_t)(sum >> 16);
            if (sum != 0u) active[atomicAdd(nactive, 1u)] = (int32_t)u;  // order is free
        }
    }
}

// The count pass for rows that start on 16-byte boundaries (nx a multiple of
// 4), with the rows staged in shared memory by bulk copies.  A block takes one
// x-tile of kTileChunks units (and the next tile's first 4 points) of the row
// pair (j, j + 1) for kBulkZ planes: a producer warp copies each plane's two
// tile rows (one cp.async.bulk per row, completion counted on the slot's full
// barrier) into a ring of kBulkSlots plane slots, and consumer warp c counts
// the units of chunk c from the slots with the count kernel's per-unit steps
// (the same clamped points and extremes; lane l holds x = i0 + 4 l + q, read
// as one 16-byte word, and counts with the VEC bit path of unit_sum).  A
// consumer copies a plane's values to registers as soon as it has
// arrived and releases the slot on its empty barrier, so the producer keeps up
// to kBulkSlots planes in flight per block without holding registers for
// them.  Every wait is bounded: a wait that runs out sets *err and ends the
// warp (the producer first waits, bounded again, for its copies in flight).
constexpr int kTileChunks = 4;                      // consumer warps per block
constexpr int kTileX = kTileChunks * kChunk + 4;    // floats of a staged tile row
constexpr int kBulkZ = 16;                          // units per warp, stacked in z
constexpr int kBulkSlots = 4;                       // planes staged at once
constexpr uint32_t kBulkSpin = 1u << 22;            // try_wait rounds before a wait gives up

constexpr size_t bulk_smem_bytes() {
    return sizeof(float) * 2 * kTileX * kBulkSlots + 2 * kBulkSlots * sizeof(uint64_t);
}

// a row of this lane's values from a staged tile row (off4: the lane's 4
// points, a multiple of 4; offe: the unit's x = i0 + kChunk, both clamped to the
// staged points)
__device__ __forceinline__ void load_srow(const float* srow, int off4, int offe, RowVals& r) {
    const float4 q = *reinterpret_cast<const float4*>(srow + off4);
    r.v[0] = q.x;
    r.v[1] = q.y;
    r.v[2] = q.z;
    r.v[3] = q.w;
    r.e = srow[offe];
}

// plane p's two rows (row ry stands for row j + 1) into registers once the
// plane has arrived, then the slot is released; false when the wait ran out
__device__ __forceinline__ bool take_plane(const float* stage, uint64_t* full, uint64_t* empty,
                                           int p, int ry, int off4, int offe, int lane,
                                           RowVals& a, RowVals& b) {
    const int s = p % kBulkSlots;
    if (!mbar_wait(full + s, (uint32_t)(p / kBulkSlots) & 1u, kBulkSpin)) return false;
    load_srow(stage + (size_t)(2 * s) * kTileX, off4, offe, a);
    load_srow(stage + (size_t)(2 * s + ry) * kTileX, off4, offe, b);
    __syncwarp();
    if (lane == 0) mbar_arrive(empty + s);
    return true;
}

template <bool BELOW>
__global__ void __launch_bounds__(32 * (kTileChunks + 1), 8) k_mc_count_bulk(
    const float* __restrict__ v, Grid g, const uint8_t* __restrict__ ntri,
    int32_t* __restrict__ vcnt, int32_t* __restrict__ tcnt, int32_t* __restrict__ active,
    uint32_t* __restrict__ nactive, uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char dsm[];
    float* stage = reinterpret_cast<float*>(dsm);  // slot s, row r: stage + (2 s + r) kTileX
    uint64_t* full = reinterpret_cast<uint64_t*>(dsm + sizeof(float) * 2 * kTileX * kBulkSlots);
    uint64_t* empty = full + kBulkSlots;
    const int warp = (int)threadIdx.x >> 5, lane = (int)threadIdx.x & 31;
    const int x0 = (int)blockIdx.x * (kTileChunks * kChunk);
    const int j = (int)blockIdx.y;
    const int k0 = (int)blockIdx.z * kBulkZ, k1 = min(k0 + kBulkZ, g.nz);
    const int nvalid = min(kTileX, g.nx - x0);                           // staged floats per row
    const int nw = min(kTileChunks, (g.nx - x0 + kChunk - 1) / kChunk);  // chunks in the tile
    const bool has_y = j + 1 < g.ny;
    const int nplanes = k1 - k0 + 1;  // planes k0 .. k1 (k1 = nz: the last plane again)
    __shared__ uint8_t s_ntri[256];  // the case table's triangle counts
    for (int i = (int)threadIdx.x; i < 256; i += (int)blockDim.x) s_ntri[i] = ntri[i];
    if (threadIdx.x == 0) {
        for (int s = 0; s < kBulkSlots; s++) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, (uint32_t)nw);
        }
        mbar_init_fence();
    }
    __syncthreads();
    if (warp == kTileChunks) {  // the producer
        if (lane != 0) return;
        const uint32_t bytes = (uint32_t)nvalid * 4u;
        int issued = 0;
        bool ok = true;
        for (int p = 0; p < nplanes; p++) {
            const int s = p % kBulkSlots;
            // the slot's previous plane released by every consumer
            if (p >= kBulkSlots && !mbar_wait(empty + s, (uint32_t)((p / kBulkSlots) - 1) & 1u,
                                             kBulkSpin)) {
                ok = false;
                break;
            }
            const float* src = v + ((int64_t)min(k0 + p, g.nz - 1) * g.ny + j) * g.nx + x0;
            float* dst = stage + (size_t)(2 * s) * kTileX;
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(full + s, has_y ? 2u * bytes : bytes);
            bulk_copy_g2s(dst, src, bytes, full + s);
            if (has_y) bulk_copy_g2s(dst + kTileX, src + g.nx, bytes, full + s);
            issued = p + 1;
        }
        if (!ok) {
            atomicOr(err, 1u);
            // the copies still in flight: the last plane issued into each slot
            for (int p = max(0, issued - kBulkSlots); p < issued; p++)
                mbar_wait(full + p % kBulkSlots, (uint32_t)(p / kBulkSlots) & 1u, kBulkSpin);
        }
        return;
    }
    if (warp >= nw) return;  // no chunk of the grid (its barriers count nw consumers)
    const int lx = warp * kChunk;  // the chunk's offset in the tile
    const int i0 = x0 + lx;
    const int64_t chunk = (int64_t)blockIdx.x * kTileChunks + warp;
    const int off4 = min(lx + 4 * lane, nvalid - 4), offe = min(lx + kChunk, nvalid - 1);
    const int ry = has_y ? 1 : 0;  // a missing row j + 1 is read as row j
    RowVals ra0, rb0;
    if (!take_plane(stage, full, empty, 0, ry, off4, offe, lane, ra0, rb0)) {
        if (lane == 0) atomicOr(err, 1u);
        return;
    }
    row_ext<BELOW>(ra0);
    row_ext<BELOW>(rb0);
    const LaneVec lv = lane_vec(i0, g.nx, lane);
    // (unrolled by two: the compiler renames the rows instead of copying them)
#pragma unroll 2
    for (int k = k0; k < k1; k++) {
        RowVals ra1, rb1;
        if (!take_plane(stage, full, empty, k - k0 + 1, ry, off4, offe, lane, ra1, rb1)) {
            if (lane == 0) atomicOr(err, 1u);
            return;
        }
        row_ext<BELOW>(ra1);
        row_ext<BELOW>(rb1);
        const float xa = ext_all<BELOW>(ext_all<BELOW>(ra0.xa, rb0.xa), ext_all<BELOW>(ra1.xa, rb1.xa));
        const float xn = ext_any<BELOW>(ext_any<BELOW>(ra0.xn, rb0.xn), ext_any<BELOW>(ra1.xn, rb1.xn));
        const bool all_in = __all_sync(kFull, inside<BELOW>(xa, g.iso));
        const bool any_in = __any_sync(kFull, inside<BELOW>(xn, g.iso));
        uint32_t sum = 0;  // vertices + 2^16 * triangles of the unit
        if (any_in && !all_in)
            sum = unit_sum<BELOW, true>(ra0, rb0, ra1, rb1, has_y, k + 1 < g.nz, i0, g, lane,
                                        s_ntri, lv);
        if (lane == 0) {
            const int64_t u = ((int64_t)k * g.ny + j) * g.nchunks + chunk;
            vcnt[u] = (int32_t)(sum & 0xffffu);
            tcnt[u] = (int32_t)(sum >> 16);
            if (sum != 0u) active[atomicAdd(nactive, 1u)] = (int32_t)u;  // order is free
        }
        ra0 = ra1;
        rb0 = rb1;
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
// The output is written from two lists in per-warp shared memory, so that the
// work is spread over the lanes whichever cells the surface crosses: the
// unit's vertices (point, axis) in vertex order, and its triangles (cell,
// triangle of the cell's case) in triangle order, with each cell's case.  Lane l takes entries l,
// l + 32, ...: a vertex each, and of the triangles a face's vertex id each
// (3 per triangle), so consecutive lanes write consecutive words.
constexpr int kEmitWarps = 4;
constexpr int kEmitBlocksPerSM = 8;              // resident blocks the launch bound asks for
constexpr int kUnitVerts = 3 * kChunk;          // a point owns at most 3 edges
constexpr int kUnitTris = kCellTris * kChunk;  // a cell has at most kCellTris triangles

template <bool BELOW>
__global__ void __launch_bounds__(32 * kEmitWarps, kEmitBlocksPerSM) k_mc_emit(const float* __restrict__ v, Grid g,
                                                              const int8_t* __restrict__ tri,
                                                              const uint8_t* __restrict__ ntri,
                                                              const int64_t* __restrict__ vbase,
                                                              const int64_t* __restrict__ tbase,
                                                              const int32_t* __restrict__ active,
                                                              const uint32_t* __restrict__ nactive,
                                                              float* __restrict__ verts,
                                                              int32_t* __restrict__ faces,
                                                              int64_t max_verts, int64_t max_faces) {
    __shared__ uint8_t s_m[kEmitWarps][4][kChunk + 1];  // crossed edges (bit a: +axis a)
    __shared__ uint16_t s_pre[kEmitWarps][4][kChunk];   // in-unit vertex prefix
    __shared__ float s_val[kEmitWarps][3][kChunk + 1];  // point row 0 (with x = i0 + 128),
                                                        // rows 1 (+y) and 2 (+z)
    __shared__ uint16_t s_vl[kEmitWarps][kUnitVerts];   // vertices: point | axis << 8
    __shared__ uint16_t s_tl[kEmitWarps][kUnitTris];    // triangles: cell | t << 7
    __shared__ uint8_t s_case[kEmitWarps][kChunk];      // each cell's case
    __shared__ int64_t s_base[kEmitWarps][8];           // R: unit base; 4 + R: next unit's
    __shared__ uint32_t s_w[kEmitWarps][8][5];          // the rows' inside-bit words
    __shared__ int8_t s_tri[256 * 3 * kCellTris];       // the case table, per block
    __shared__ uint8_t s_ntri[256];
    for (int i = (int)threadIdx.x; i < 256 * 3 * kCellTris; i += 32 * kEmitWarps)
        s_tri[i] = tri[(i / (3 * kCellTris)) * 3 * kMaxTri + i % (3 * kCellTris)];
    for (int i = (int)threadIdx.x; i < 256; i += 32 * kEmitWarps) s_ntri[i] = ntri[i];
    __syncthreads();
    const int lane = (int)threadIdx.x & 31, wid = (int)threadIdx.x >> 5;
    const uint32_t n_act = *nactive;
    const uint32_t stride = gridDim.x * kEmitWarps;
    uint32_t a = blockIdx.x * kEmitWarps + wid;
    int64_t u_next = a < n_act ? active[a] : 0;  // the warp's next unit, read a unit ahead
    for (; a < n_act; a += stride) {
        const int64_t u = u_next;
        if (a + stride < n_act) u_next = active[a + stride];
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
        // (the words go to shared memory: every lane reads them as broadcasts, and
        // the registers they would hold go to more resident warps)
        uint32_t(&w)[8][5] = s_w[wid];
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
                const uint32_t b =
                    __ballot_sync(kFull, ok && x < g.nx && inside<BELOW>(x5[q], g.iso));
                if (lane == 0) w[r][q] = b;
            }
            const uint32_t b4 =
                __ballot_sync(kFull, ok && lane < 2 && xe < g.nx && inside<BELOW>(x5[4], g.iso));
            if (lane == 0) w[r][4] = b4;
            if (r < 3) {  // the values the unit's vertices interpolate
#pragma unroll
                for (int q = 0; q < 4; q++) s_val[wid][r][lane + 32 * q] = x5[q];
                if (r == 0 && lane == 0) s_val[wid][0][kChunk] = x5[4];
            }
        }
        __syncwarp();
        // per point row: crossed-edge words, each lane's points' masks and prefixes;
        // row 0's crossed edges are the unit's vertices, listed in vertex order
        const bool row_ok[4] = {true, j + 1 < g.ny, k + 1 < g.nz, j + 1 < g.ny && k + 1 < g.nz};
        const int ny_of[4] = {1, 4, 3, 5};  // the row one step +y of point row R
        const int nz_of[4] = {2, 3, 6, 7};  // the row one step +z of point row R
        uint32_t nverts = 0;
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
                                   (xl >= 32 ? kFull : (xl <= 0 ? 0u : (1u << xl) - 1u));
                const uint32_t Y = yok ? (w[R][q] ^ w[ny_of[R]][q]) : 0u;
                const uint32_t Z = zok ? (w[R][q] ^ w[nz_of[R]][q]) : 0u;
                const uint32_t lo = (1u << lane) - 1u;
                const uint32_t m = ((X >> lane) & 1u) | (((Y >> lane) & 1u) << 1) |
                                   (((Z >> lane) & 1u) << 2);
                // (a word without crossings owns no vertex: no triangle reads its entries)
                if ((X | Y | Z) != 0u) {
                    const uint32_t pre = cum + __popc(X & lo) + __popc(Y & lo) + __popc(Z & lo);
                    s_m[wid][R][lane + 32 * q] = (uint8_t)m;
                    s_pre[wid][R][lane + 32 * q] = (uint16_t)pre;
                    if (R == 0) {
                        uint32_t o = pre;
#pragma unroll
                        for (int ax = 0; ax < 3; ax++)
                            if ((m >> ax) & 1u)
                                s_vl[wid][o++] = (uint16_t)((lane + 32 * q) | (ax << 8));
                    }
                    cum += __popc(X) + __popc(Y) + __popc(Z);
                }
            }
            if (R == 0) nverts = cum;
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
        const int64_t tb = __shfl_sync(kFull, base, 8);
        // the triangles of this unit's cells, listed in x order
        uint32_t ntris = 0;
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
                if (nt[q]) s_case[wid][lane + 32 * q] = (uint8_t)cs[q];
                incl[q] = nt[q];
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {  // warp inclusive scans of the counts
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int t = __shfl_up_sync(kFull, incl[q], o);
                    if (lane >= o) incl[q] += t;
                }
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t first = ntris + (uint32_t)(incl[q] - nt[q]);
                for (int t3 = 0; t3 < nt[q]; t3++)
                    s_tl[wid][first + t3] = (uint16_t)((lane + 32 * q) | (t3 << 7));
                ntris += (uint32_t)__shfl_sync(kFull, incl[q], 31);
            }
        }
        __syncwarp();
        // vertices
        {
            const int64_t vb = s_base[wid][0];
            const float y = __fmaf_rn(float(j), g.h, g.oy), z = __fmaf_rn(float(k), g.h, g.oz);
            for (uint32_t e = lane; e < nverts; e += 32) {
                const uint32_t ent = s_vl[wid][e];
                const int xi = (int)(ent & 0xffu), ax = (int)(ent >> 8);
                const float v0 = s_val[wid][0][xi];
                const float v1 = ax == 0 ? s_val[wid][0][xi + 1] : s_val[wid][ax][xi];
                const float x = __fmaf_rn(float(i0 + xi), g.h, g.ox);
                const float d = __fmul_rn(root_t(v0, v1, g.iso), g.h);
                const int64_t o = vb + e;
                if (o < max_verts) {  // the host reports a mesh larger than the buffers
                    verts[3 * o + 0] = ax == 0 ? __fadd_rn(x, d) : x;
                    verts[3 * o + 1] = ax == 1 ? __fadd_rn(y, d) : y;
                    verts[3 * o + 2] = ax == 2 ? __fadd_rn(z, d) : z;
                }
            }
        }
        // faces: entry e is vertex e % 3 of the unit's triangle e / 3
        for (uint32_t e = lane; e < 3 * ntris; e += 32) {
            const uint32_t t = e / 3, sv = e - 3 * t;
            const uint32_t ent = s_tl[wid][t];
            const int xc = (int)(ent & 127u), t3 = (int)(ent >> 7), c = s_case[wid][xc];
            const int ed = s_tri[c * 3 * kCellTris + 3 * t3 + (int)sv];
            const int ax = ed >> 2, eu = ed & 1, ew = (ed >> 1) & 1;
            // the point owning edge ed of this cell: (dx, row R = dy + 2 dz)
            const int dx = ax == 0 ? 0 : eu;
            const int dy = ax == 0 ? eu : (ax == 1 ? 0 : ew);
            const int dz = ax == 2 ? 0 : ew;
            const int R = dy + 2 * dz, xi = xc + dx;
            const uint32_t below = (1u << ax) - 1u;
            const int64_t id = xi < kChunk ? s_base[wid][R] + s_pre[wid][R][xi] +
                                                 __popc(s_m[wid][R][xi] & below)
                                           : s_base[wid][4 + R] + __popc(s_m[wid][R][kChunk] & below);
            if (tb + (int64_t)t < max_faces) faces[3 * tb + e] = (int32_t)id;
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
    int dev = 0, sms = 0;
    CAGR_CUDA(cudaGetDevice(&dev));
    CAGR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const dim3 grid_c((unsigned)nchunks, (unsigned)((ny + kCountWarps - 1) / kCountWarps),
                      (unsigned)((nz + kCountZ - 1) / kCountZ)),
        grid_e((unsigned)(sms * kEmitBlocksPerSM));  // persistent: warps stride over the
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
    if (!rc) rc = pool_alloc((void**)&nact, 8, s);  // listed units, then the error flag
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
    cudaMemsetAsync(nact, 0, 8, s);
    uint32_t* nerr = nact + 1;
    // rows staged by bulk copies when every row starts on a 16-byte boundary
    const bool vec = nx % 4 == 0 && ((uintptr_t)values & 15u) == 0;
    const dim3 grid_b((unsigned)((nx + kTileChunks * kChunk - 1) / (kTileChunks * kChunk)),
                      (unsigned)ny, (unsigned)((nz + kBulkZ - 1) / kBulkZ));
    if (below && vec)
        k_mc_count_bulk<true><<<grid_b, 32 * (kTileChunks + 1), bulk_smem_bytes(), s>>>(
            values, g, ntri, vcnt, tcnt, act, nact, nerr);
    else if (vec)
        k_mc_count_bulk<false><<<grid_b, 32 * (kTileChunks + 1), bulk_smem_bytes(), s>>>(
            values, g, ntri, vcnt, tcnt, act, nact, nerr);
    else if (below)
        k_mc_count<true><<<grid_c, 32 * kCountWarps, 0, s>>>(values, g, ntri, vcnt, tcnt,
                                                                     act, nact);
    else
        k_mc_count<false><<<grid_c, 32 * kCountWarps, 0, s>>>(values, g, ntri, vcnt, tcnt,
                                                                      act, nact);
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
    uint32_t herr = 0;
    if (!rc) {
        cudaMemcpyAsync(&nv, vbase + U, 8, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&nf, tbase + U, 8, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&herr, nerr, 4, cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) rc = set_error(kErrCuda, "marching cubes counts");
    }
    if (!rc && herr) rc = set_error(kErrCuda, "marching cubes: a staging wait ran out");
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
