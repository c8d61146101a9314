// TEST INFRASTRUCTURE.  A C entry point over the reference's own marching-cubes
// case logic (gaussrecon_src/MarchingCubes.cpp, compiled where it lies by
// `make -C oracle ref-mc`): its tables and its per-cube triangle lists, used to
// pin the oracle's classic-table restatement and to write the table fixture.
#include "MarchingCubes.h"

extern "C" {

// edge_mask[256] and triangles[256 * 16] exactly as the reference defines them
void ref_mc_tables(int* edge_mask, int* triangles) {
    for (int c = 0; c < 256; c++) {
        edge_mask[c] = MarchingCubes::edgeMask[c];
        for (int q = 0; q < 16; q++) triangles[16 * c + q] = MarchingCubes::triangles[c][q];
    }
}

// the reference's case index of one cube (values in corner order x + 2y + 4z)
int ref_mc_index(const float* v8, float iso) { return MarchingCubes::GetIndex(v8, iso); }

// the reference's triangles of one cube: edge ids into idx[0 .. 3 n), returns n
int ref_mc_cell(const float* v8, float iso, int* idx) {
    return MarchingCubes::AddTriangleIndices(v8, iso, idx);
}
}
