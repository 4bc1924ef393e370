// mc.cuh -- marching cubes on a regular grid (two passes, cell-ordered output).
#pragma once

#include "common.cuh"

namespace dwg {

struct McGrid {
    int res[3];
    float origin[3];
    float spacing;
    const float* positions = nullptr;  // optional materialised sample positions
    int zoff = 0;                      // z index of the first sample (a slab of a larger grid)
};

struct McWorkspace {
    DevBuf<unsigned int> block_counts;
    DevBuf<unsigned int> block_offsets;
    DevBuf<unsigned char> scratch;
};

// host copies of the case tables: edge masks from the cube geometry, the
// reference's triangles per case; false if the triangles of a case do not
// close into the polygons the geometry gives
bool mc_tables_host(int* edge_table, signed char* tri_table);
int mc_upload_tables();

// count -> scan -> emit.  *num_tris_dev receives the full count (may exceed cap).
int mc_run(const float* field, const McGrid& g, float iso, const float* iso_dev, float* tris,
           float* centroids, float* normals, long long cap, unsigned long long* num_tris_dev,
           McWorkspace& ws, cudaStream_t s);

}  // namespace dwg
