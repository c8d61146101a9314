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
// --op A selects the operator of the reference's CPU driver
// (main_GaussRecon_cpu.cpp:280-318: multiply_by_A, continuous kernel) instead
// of the CUDA driver's A3.  The run prints its phases: input parsing, device
// set-up (context and uploads), the device work, output.
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
    "[-d maxDepth=10] [--op A3|A]\n";

struct Args {
    std::string in, out;
    float width = 0.01f;
    int min_depth = 1, max_depth = 10;
    int op = CAGR_OP_A3;
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
        else if (k == "--op" && std::strcmp(v, "A3") == 0) a->op = CAGR_OP_A3;
        else if (k == "--op" && std::strcmp(v, "A") == 0) a->op = CAGR_OP_A;
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

// Whole-file read of "x y z nx ny nz" records (whitespace separated; a
// trailing incomplete record is ignored, as fscanf's loop would).
bool read_xyz(const std::string& path, std::vector<float>& xyz, std::vector<float>& nml) {
    FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) return false;
    std::vector<char> buf;
    char chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof(chunk), fp)) > 0) buf.insert(buf.end(), chunk, chunk + got);
    std::fclose(fp);
    buf.push_back('\0');
    const char* p = buf.data();
    float r[6];
    for (;;) {
        int k = 0;
        for (; k < 6; k++) {
            char* end = nullptr;
            r[k] = std::strtof(p, &end);
            if (end == p) break;
            p = end;
        }
        if (k < 6) break;
        xyz.insert(xyz.end(), r, r + 3);
        nml.insert(nml.end(), r + 3, r + 6);
    }
    return true;
}

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
    std::vector<float> xyz, nml;
    if (!read_xyz(a.in, xyz, nml)) {
        std::fprintf(stderr, "[main_GaussReconCUDA] cannot open %s\n", a.in.c_str());
        return 1;
    }
    const int64_t n = (int64_t)xyz.size() / 3;
    if (n == 0) {
        std::fprintf(stderr, "[main_GaussReconCUDA] no points in %s\n", a.in.c_str());
        return 1;
    }
    float lo[3], hi[3];
    for (int d = 0; d < 3; d++) lo[d] = hi[d] = xyz[d];
    for (int64_t j = 1; j < n; j++)
        for (int d = 0; d < 3; d++) {
            hi[d] = std::max(hi[d], xyz[3 * j + d]);
            lo[d] = std::min(lo[d], xyz[3 * j + d]);
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
    std::printf("[main_GaussReconCUDA] %lld points, grid depth %d, width %g, operator %s\n",
                (long long)n, a.max_depth, a.width, a.op == CAGR_OP_A ? "A" : "A3");
    const double t_read = seconds_since(t_start);

    // ---- treecode field at the samples and at the grid nodes ----
    const auto t_dev0 = std::chrono::steady_clock::now();
    cudaStream_t st = nullptr;
    cudaError_t ce;
    if ((ce = cudaFree(nullptr))) return cuda_fail("CUDA context", ce);
    Dev d_pts, d_attrs, d_w, d_samples;
    if ((ce = d_pts.alloc(sizeof(float) * 3 * n)) || (ce = d_attrs.alloc(sizeof(float) * 3 * n)) ||
        (ce = d_w.alloc(sizeof(float) * n)) || (ce = d_samples.alloc(sizeof(float) * n)))
        return cuda_fail("cudaMalloc", ce);
    if ((ce = cudaMemcpy(d_pts.p, pts.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice)) ||
        (ce = cudaMemcpy(d_attrs.p, attrs.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice)) ||
        (ce = cudaMemcpy(d_w.p, weights.data(), sizeof(float) * n, cudaMemcpyHostToDevice)))
        return cuda_fail("cudaMemcpy", ce);
    const double t_setup = seconds_since(t_dev0);
    const auto t_gpu0 = std::chrono::steady_clock::now();
    const char* opname = a.op == CAGR_OP_A ? "cagr_multiply(A)" : "cagr_multiply(A3)";
    TreeGuard tree;
    int rc = cagr_tree_build(d_pts.p, n, CAGR_F32, 15, 1, st, &tree.t);
    if (rc) return fail("cagr_tree_build", rc);
    if ((rc = cagr_scatter(tree.t, 0, d_attrs.p, 3, d_w.p, st))) return fail("cagr_scatter", rc);
    if ((rc = cagr_multiply(tree.t, a.op, nullptr, nullptr, n, nullptr, a.width,
                            CAGR_FLAG_CONTINUOUS, d_samples.p, 0, st)))
        return fail(opname, rc);
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
    // grid value = -A3 (main_GaussRecon_cuda.cu:478; -A in main_GaussRecon_cpu.cpp)
    if ((rc = cagr_field_grid(tree.t, a.op, g, g, g, origin, spacing, nullptr, a.width,
                              CAGR_FLAG_CONTINUOUS | CAGR_FLAG_NEGATE, d_field.p, st)))
        return fail("cagr_field_grid", rc);
    // one pass over the grid into buffers of an estimated size (a surface
    // crossing every layer: 8 vertices per cell column of a face), again with
    // the exact sizes if the mesh is larger
    int64_t nv = 8 * (int64_t)g * g, nf = 2 * nv + 1024;
    Dev d_v, d_f;
    for (int attempt = 0;; attempt++) {
        if ((ce = d_v.alloc(sizeof(float) * 3 * nv)) || (ce = d_f.alloc(sizeof(int32_t) * 3 * nf)))
            return cuda_fail("cudaMalloc(mesh)", ce);
        const int64_t cap_v = nv, cap_f = nf;
        rc = cagr_marching_cubes((const float*)d_field.p, g, g, g, origin, spacing, iso,
                                 (float*)d_v.p, cap_v, (int32_t*)d_f.p, cap_f, &nv, &nf, st);
        if (rc == CAGR_ERR_OVERFLOW && attempt == 0 && (nv > cap_v || nf > cap_f)) {
            cudaFree(d_v.p);
            cudaFree(d_f.p);
            d_v.p = d_f.p = nullptr;
            continue;
        }
        if (rc) return fail("cagr_marching_cubes", rc);
        break;
    }
    std::vector<float> verts(3 * nv);
    std::vector<int32_t> faces(3 * nf);
    if ((ce = cudaMemcpy(verts.data(), d_v.p, sizeof(float) * 3 * nv, cudaMemcpyDeviceToHost)) ||
        (ce = cudaMemcpy(faces.data(), d_f.p, sizeof(int32_t) * 3 * nf, cudaMemcpyDeviceToHost)))
        return cuda_fail("cudaMemcpy", ce);
    const double t_gpu = seconds_since(t_gpu0);
    const auto t_out0 = std::chrono::steady_clock::now();
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
    std::printf("[main_GaussReconCUDA] phases: input %.3f s, device set-up %.3f s, device work "
                "(tree, moments, field, marching cubes, mesh copy) %.3f s, output %.3f s\n",
                t_read, t_setup, t_gpu, seconds_since(t_out0));
    return 0;
}
