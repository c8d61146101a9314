// main_GaussReconCUDA on libcagr_b200: the reconstruction driver of the
// reference (mayueji/CAGR CUDA-based/ext/gaussrecon_src/main_GaussRecon_cuda.cu:
// 225-500) rebuilt on the library's C ABI (include/cagr.h).
//
//   main_GaussReconCUDA -i oriented.xyz -o out.ply [-w 0.01] [-m 1] [-d 10]
//
// Same command line (:238-245), input (x y z nx ny nz per line,
// gaussrecon_src/Octree.cpp:212), normalisation, field and output:
//   * points into PGR's unit cube: scale = 1.1 x the largest bounding-box
//     extent, corner = (max + min - scale) / 2 (Octree.cpp:244-261), then to
//     the treecode's [-1, 1]^3 as 2 p - 1 (:270-272);
//   * normals n / |n| * 1e-5 with weights 1e-5 (fixed area, :276-288);
//   * grid value = -A3 with the continuous kernel and width -w at the grid
//     nodes (:427-445, :478); iso-value = -(median of A3 at the samples)
//     (:448-486);
//   * the mesh in the input's coordinates as a binary PLY (float x, y, z;
//     uchar-counted int faces; Octree.cpp:1259-1267).
// The grid: PGR's adaptive octree is replaced by the regular grid of depth -d
// ((2^d + 1)^3 nodes over the unit cube), evaluated and contoured on the GPU
// (cagr_field_grid, cagr_marching_cubes); -m (PGR's minimum depth) has no
// meaning for a regular grid and is accepted for compatibility.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "cagr.h"

namespace {

const char* kUsage =
    "usage: main_GaussReconCUDA -i <input.xyz> -o <output.ply> [-w width=0.01] [-m minDepth=1] "
    "[-d maxDepth=10]\n";

struct Args {
    std::string in, out;
    float width = 0.01f;
    int min_depth = 1, max_depth = 10;
};

bool parse(int argc, char** argv, Args* a) {
    for (int i = 1; i < argc; i++) {
        const std::string k = argv[i];
        if (i + 1 >= argc) return false;
        const char* v = argv[++i];
        char* end = nullptr;
        if (k == "-i") a->in = v;
        else if (k == "-o") a->out = v;
        else if (k == "-w") a->width = std::strtof(v, &end);
        else if (k == "-m") a->min_depth = (int)std::strtol(v, &end, 10);
        else if (k == "-d") a->max_depth = (int)std::strtol(v, &end, 10);
        else return false;
        if (end && *end) return false;
    }
    return !a->in.empty() && !a->out.empty();
}

int fail(const char* what, int rc) {
    std::fprintf(stderr, "[main_GaussReconCUDA] %s: %s (%s)\n", what, cagr_status_string(rc),
                 cagr_last_error());
    return 1;
}

int cuda_fail(const char* what, cudaError_t e) {
    std::fprintf(stderr, "[main_GaussReconCUDA] %s: %s\n", what, cudaGetErrorString(e));
    return 1;
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Device buffer freed on scope exit.
struct Dev {
    void* p = nullptr;
    ~Dev() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes > 0 ? bytes : 1); }
};

struct TreeGuard {
    cagr_tree* t = nullptr;
    ~TreeGuard() {
        if (t) cagr_tree_destroy(t);
    }
};

bool write_ply(const std::string& path, const std::vector<float>& v, const std::vector<int32_t>& f) {
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) return false;
    const size_t nv = v.size() / 3, nf = f.size() / 3;
    std::fprintf(fp,
                 "ply\nformat binary_little_endian 1.0\nelement vertex %zu\nproperty float x\n"
                 "property float y\nproperty float z\nelement face %zu\n"
                 "property list uchar int vertex_indices\nend_header\n",
                 nv, nf);
    bool ok = std::fwrite(v.data(), sizeof(float), v.size(), fp) == v.size();
    unsigned char rec[13];
    for (size_t i = 0; ok && i < nf; i++) {
        rec[0] = 3;
        std::memcpy(rec + 1, f.data() + 3 * i, 12);
        ok = std::fwrite(rec, 1, 13, fp) == 13;
    }
    return std::fclose(fp) == 0 && ok;
}

}  // namespace

int main(int argc, char** argv) {
    Args a;
    if (!parse(argc, argv, &a)) {
        std::fputs(kUsage, stderr);
        return 2;
    }
    if (a.max_depth < a.min_depth)
        std::printf("[main_GaussReconCUDA] WARNING: minDepth %d larger than maxDepth %d, "
                    "ignoring the given minDepth\n", a.min_depth, a.max_depth);
    if (a.max_depth < 1 || a.max_depth > 10) {
        std::fprintf(stderr, "[main_GaussReconCUDA] -d must be in [1, 10]\n");
        return 2;
    }
    const auto t_start = std::chrono::steady_clock::now();

    // ---- input: x y z nx ny nz per line (Octree.cpp:211-224) ----
    FILE* fp = std::fopen(a.in.c_str(), "r");
    if (!fp) {
        std::fprintf(stderr, "[main_GaussReconCUDA] cannot open %s\n", a.in.c_str());
        return 1;
    }
    std::vector<float> xyz, nml;
    float r[6];
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    while (std::fscanf(fp, "%f %f %f %f %f %f", r, r + 1, r + 2, r + 3, r + 4, r + 5) == 6) {
        for (int d = 0; d < 3; d++) {
            if (xyz.empty() || r[d] > hi[d]) hi[d] = r[d];
            if (xyz.empty() || r[d] < lo[d]) lo[d] = r[d];
        }
        xyz.insert(xyz.end(), r, r + 3);
        nml.insert(nml.end(), r + 3, r + 6);
    }
    std::fclose(fp);
    const int64_t n = (int64_t)xyz.size() / 3;
    if (n == 0) {
        std::fprintf(stderr, "[main_GaussReconCUDA] no points in %s\n", a.in.c_str());
        return 1;
    }
    // ---- normalisation (Octree.cpp:244-261, main_GaussRecon_cuda.cu:270-288) ----
    const float scale = std::max(std::max(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]) * 1.1f;
    float corner[3];
    for (int d = 0; d < 3; d++) corner[d] = (hi[d] + lo[d] - scale) / 2;
    const float area = 1e-5f;
    std::vector<float> pts(3 * n), attrs(3 * n), weights(n, area);
    for (int64_t j = 0; j < n; j++) {
        for (int d = 0; d < 3; d++) pts[3 * j + d] = 2 * ((xyz[3 * j + d] - corner[d]) / scale) - 1;
        const float nx = nml[3 * j], ny = nml[3 * j + 1], nz = nml[3 * j + 2];
        const float len = std::max(std::sqrt(nx * nx + ny * ny + nz * nz), 1e-12f);
        attrs[3 * j] = nx / len * area;
        attrs[3 * j + 1] = ny / len * area;
        attrs[3 * j + 2] = nz / len * area;
    }
    std::printf("[main_GaussReconCUDA] %lld points, grid depth %d, width %g\n", (long long)n,
                a.max_depth, a.width);

    // ---- treecode field at the samples and at the grid nodes ----
    cudaStream_t st = nullptr;
    cudaError_t ce;
    Dev d_pts, d_attrs, d_w, d_samples;
    if ((ce = d_pts.alloc(sizeof(float) * 3 * n)) || (ce = d_attrs.alloc(sizeof(float) * 3 * n)) ||
        (ce = d_w.alloc(sizeof(float) * n)) || (ce = d_samples.alloc(sizeof(float) * n)))
        return cuda_fail("cudaMalloc", ce);
    if ((ce = cudaMemcpy(d_pts.p, pts.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice)) ||
        (ce = cudaMemcpy(d_attrs.p, attrs.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice)) ||
        (ce = cudaMemcpy(d_w.p, weights.data(), sizeof(float) * n, cudaMemcpyHostToDevice)))
        return cuda_fail("cudaMemcpy", ce);
    TreeGuard tree;
    int rc = cagr_tree_build(d_pts.p, n, CAGR_F32, 15, 1, st, &tree.t);
    if (rc) return fail("cagr_tree_build", rc);
    if ((rc = cagr_scatter(tree.t, 0, d_attrs.p, 3, d_w.p, st))) return fail("cagr_scatter", rc);
    if ((rc = cagr_multiply(tree.t, CAGR_OP_A3, nullptr, nullptr, n, nullptr, a.width,
                            CAGR_FLAG_CONTINUOUS, d_samples.p, 0, st)))
        return fail("cagr_multiply(A3)", rc);
    std::vector<float> samples(n);
    if ((ce = cudaMemcpy(samples.data(), d_samples.p, sizeof(float) * n, cudaMemcpyDeviceToHost)))
        return cuda_fail("cudaMemcpy", ce);
    std::nth_element(samples.begin(), samples.begin() + n / 2, samples.end());
    const float iso = -samples[n / 2];

    const int g = (1 << a.max_depth) + 1;
    const double spacing = 2.0 / (double)(g - 1);
    const double origin[3] = {-1.0, -1.0, -1.0};
    const size_t nodes = (size_t)g * g * g;
    Dev d_field;
    if ((ce = d_field.alloc(sizeof(float) * nodes))) return cuda_fail("cudaMalloc(field)", ce);
    // grid value = -A3 (main_GaussRecon_cuda.cu:478)
    if ((rc = cagr_field_grid(tree.t, CAGR_OP_A3, g, g, g, origin, spacing, nullptr, a.width,
                              CAGR_FLAG_CONTINUOUS | CAGR_FLAG_NEGATE, d_field.p, st)))
        return fail("cagr_field_grid", rc);
    int64_t nv = 0, nf = 0;
    if ((rc = cagr_marching_cubes((const float*)d_field.p, g, g, g, origin, spacing, iso, nullptr,
                                  0, nullptr, 0, &nv, &nf, st)))
        return fail("cagr_marching_cubes", rc);
    Dev d_v, d_f;
    if ((ce = d_v.alloc(sizeof(float) * 3 * nv)) || (ce = d_f.alloc(sizeof(int32_t) * 3 * nf)))
        return cuda_fail("cudaMalloc(mesh)", ce);
    if ((rc = cagr_marching_cubes((const float*)d_field.p, g, g, g, origin, spacing, iso,
                                  (float*)d_v.p, nv, (int32_t*)d_f.p, nf, &nv, &nf, st)))
        return fail("cagr_marching_cubes", rc);
    std::vector<float> verts(3 * nv);
    std::vector<int32_t> faces(3 * nf);
    if ((ce = cudaMemcpy(verts.data(), d_v.p, sizeof(float) * 3 * nv, cudaMemcpyDeviceToHost)) ||
        (ce = cudaMemcpy(faces.data(), d_f.p, sizeof(int32_t) * 3 * nf, cudaMemcpyDeviceToHost)))
        return cuda_fail("cudaMemcpy", ce);
    // back to the input's coordinates (Octree.cpp:1262-1266, 1285-1287)
    for (int64_t i = 0; i < nv; i++)
        for (int d = 0; d < 3; d++)
            verts[3 * i + d] = (verts[3 * i + d] + 1.0f) * 0.5f * scale + corner[d];
    if (!write_ply(a.out, verts, faces)) {
        std::fprintf(stderr, "[main_GaussReconCUDA] cannot write %s\n", a.out.c_str());
        return 1;
    }
    std::printf("[main_GaussReconCUDA] iso-value %g, %lld vertices, %lld faces -> %s (%.3f s)\n",
                iso, (long long)nv, (long long)nf, a.out.c_str(), seconds_since(t_start));
    return 0;
}
