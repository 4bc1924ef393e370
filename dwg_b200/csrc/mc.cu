// mc.cu -- marching cubes, two passes with cell-ordered (deterministic) output.
//
// The reference (src/TurboMC.cu:383-478) launches one 12-thread block per cell
// and appends triangles at atomicAdd slots.  Here pass 1 classifies 256 cells
// per block and reduces the triangle counts; a scan over blocks gives every
// block its output offset; pass 2 re-classifies, scans counts inside the block
// and writes each triangle at its final position, so the triangle order is
// the cell order (x fastest) -- identical from run to run.
//
// Conventions kept from the reference: corner c of cell (x,y,z) sits at
// (x + (b0 != b1), y + b1, z + !b2) (src/TurboMC.cu:408-413); bit c of the case
// index is set when the corner value is above the iso value (:418-425); edge e
// joins corners (e & 7, e<4 ? (e+1)&3 : e<8 ? 4+((e-3)&3) : e-4) (:433-434);
// vertex = P1 - l (P2 - P1), l = (v1 - iso)/(v2 - v1 + 1e-10) (:373-381);
// centroid = mean of the vertices; normal = -cross/(|cross| + 1e-8) (:453-470);
// the triangles of each case are the reference's (kTriangles below), checked
// against the polygons the cube geometry gives (mc_tables_host).
#include <cub/cub.cuh>

#include <mutex>

#include "mc.cuh"

namespace dwg {

__constant__ signed char c_tri[256][16];
__constant__ unsigned char c_ntri[256];
__constant__ unsigned short c_edges[256];

static const int kCorner[8][3] = {{0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1},
                                  {0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}};
static int edge_a(int e) { return e & 7; }
static int edge_b(int e) { return e < 4 ? ((e + 1) & 3) : (e < 8 ? 4 + ((e - 3) & 3) : e - 4); }

// Triangles of each of the 256 cases, as edge-index triples: the reference's
// per-case triangle lists (src/TurboMC.cu:57-314), kept equal on purpose.
// The DWG iteration pushes every triangle's unit normal onto the 15 nearest
// points of its centroid, so splitting a 4-7-gon along other diagonals changes
// the reconstruction, not only the mesh (measured on BASELINE config 1 with
// the FP64 oracle: 0.965 leaf-orientation agreement between the two splits).
static const signed char kTriangles[256][16] = {
    {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 8, 3, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 1, 9, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {1, 8, 3, 9, 8, 1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {1, 2, 10, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 8, 3, 1, 2, 10, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {9, 2, 10, 0, 2, 9, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {2, 8, 3, 2, 10, 8, 10, 9, 8, -1, -1, -1, -1, -1, -1, -1},
    {3, 11, 2, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 11, 2, 8, 11, 0, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {1, 9, 0, 2, 3, 11, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {1, 11, 2, 1, 9, 11, 9, 8, 11, -1, -1, -1, -1, -1, -1, -1},
    {3, 10, 1, 11, 10, 3, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 10, 1, 0, 8, 10, 8, 11, 10, -1, -1, -1, -1, -1, -1, -1},
    {3, 9, 0, 3, 11, 9, 11, 10, 9, -1, -1, -1, -1, -1, -1, -1},
    {9, 8, 10, 10, 8, 11, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {4, 7, 8, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {4, 3, 0, 7, 3, 4, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 1, 9, 8, 4, 7, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {4, 1, 9, 4, 7, 1, 7, 3, 1, -1, -1, -1, -1, -1, -1, -1},
    {1, 2, 10, 8, 4, 7, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {3, 4, 7, 3, 0, 4, 1, 2, 10, -1, -1, -1, -1, -1, -1, -1},
    {9, 2, 10, 9, 0, 2, 8, 4, 7, -1, -1, -1, -1, -1, -1, -1},
    {2, 10, 9, 2, 9, 7, 2, 7, 3, 7, 9, 4, -1, -1, -1, -1},
    {8, 4, 7, 3, 11, 2, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {11, 4, 7, 11, 2, 4, 2, 0, 4, -1, -1, -1, -1, -1, -1, -1},
    {9, 0, 1, 8, 4, 7, 2, 3, 11, -1, -1, -1, -1, -1, -1, -1},
    {4, 7, 11, 9, 4, 11, 9, 11, 2, 9, 2, 1, -1, -1, -1, -1},
    {3, 10, 1, 3, 11, 10, 7, 8, 4, -1, -1, -1, -1, -1, -1, -1},
    {1, 11, 10, 1, 4, 11, 1, 0, 4, 7, 11, 4, -1, -1, -1, -1},
    {4, 7, 8, 9, 0, 11, 9, 11, 10, 11, 0, 3, -1, -1, -1, -1},
    {4, 7, 11, 4, 11, 9, 9, 11, 10, -1, -1, -1, -1, -1, -1, -1},
    {9, 5, 4, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {9, 5, 4, 0, 8, 3, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 5, 4, 1, 5, 0, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {8, 5, 4, 8, 3, 5, 3, 1, 5, -1, -1, -1, -1, -1, -1, -1},
    {1, 2, 10, 9, 5, 4, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {3, 0, 8, 1, 2, 10, 4, 9, 5, -1, -1, -1, -1, -1, -1, -1},
    {5, 2, 10, 5, 4, 2, 4, 0, 2, -1, -1, -1, -1, -1, -1, -1},
    {2, 10, 5, 3, 2, 5, 3, 5, 4, 3, 4, 8, -1, -1, -1, -1},
    {9, 5, 4, 2, 3, 11, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 11, 2, 0, 8, 11, 4, 9, 5, -1, -1, -1, -1, -1, -1, -1},
    {0, 5, 4, 0, 1, 5, 2, 3, 11, -1, -1, -1, -1, -1, -1, -1},
    {2, 1, 5, 2, 5, 8, 2, 8, 11, 4, 8, 5, -1, -1, -1, -1},
    {10, 3, 11, 10, 1, 3, 9, 5, 4, -1, -1, -1, -1, -1, -1, -1},
    {4, 9, 5, 0, 8, 1, 8, 10, 1, 8, 11, 10, -1, -1, -1, -1},
    {5, 4, 0, 5, 0, 11, 5, 11, 10, 11, 0, 3, -1, -1, -1, -1},
    {5, 4, 8, 5, 8, 10, 10, 8, 11, -1, -1, -1, -1, -1, -1, -1},
    {9, 7, 8, 5, 7, 9, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {9, 3, 0, 9, 5, 3, 5, 7, 3, -1, -1, -1, -1, -1, -1, -1},
    {0, 7, 8, 0, 1, 7, 1, 5, 7, -1, -1, -1, -1, -1, -1, -1},
    {1, 5, 3, 3, 5, 7, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {9, 7, 8, 9, 5, 7, 10, 1, 2, -1, -1, -1, -1, -1, -1, -1},
    {10, 1, 2, 9, 5, 0, 5, 3, 0, 5, 7, 3, -1, -1, -1, -1},
    {8, 0, 2, 8, 2, 5, 8, 5, 7, 10, 5, 2, -1, -1, -1, -1},
    {2, 10, 5, 2, 5, 3, 3, 5, 7, -1, -1, -1, -1, -1, -1, -1},
    {7, 9, 5, 7, 8, 9, 3, 11, 2, -1, -1, -1, -1, -1, -1, -1},
    {9, 5, 7, 9, 7, 2, 9, 2, 0, 2, 7, 11, -1, -1, -1, -1},
    {2, 3, 11, 0, 1, 8, 1, 7, 8, 1, 5, 7, -1, -1, -1, -1},
    {11, 2, 1, 11, 1, 7, 7, 1, 5, -1, -1, -1, -1, -1, -1, -1},
    {9, 5, 8, 8, 5, 7, 10, 1, 3, 10, 3, 11, -1, -1, -1, -1},
    {5, 7, 0, 5, 0, 9, 7, 11, 0, 1, 0, 10, 11, 10, 0, -1},
    {11, 10, 0, 11, 0, 3, 10, 5, 0, 8, 0, 7, 5, 7, 0, -1},
    {11, 10, 5, 7, 11, 5, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {10, 6, 5, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 8, 3, 5, 10, 6, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {9, 0, 1, 5, 10, 6, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {1, 8, 3, 1, 9, 8, 5, 10, 6, -1, -1, -1, -1, -1, -1, -1},
    {1, 6, 5, 2, 6, 1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {1, 6, 5, 1, 2, 6, 3, 0, 8, -1, -1, -1, -1, -1, -1, -1},
    {9, 6, 5, 9, 0, 6, 0, 2, 6, -1, -1, -1, -1, -1, -1, -1},
    {5, 9, 8, 5, 8, 2, 5, 2, 6, 3, 2, 8, -1, -1, -1, -1},
    {2, 3, 11, 10, 6, 5, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {11, 0, 8, 11, 2, 0, 10, 6, 5, -1, -1, -1, -1, -1, -1, -1},
    {0, 1, 9, 2, 3, 11, 5, 10, 6, -1, -1, -1, -1, -1, -1, -1},
    {5, 10, 6, 1, 9, 2, 9, 11, 2, 9, 8, 11, -1, -1, -1, -1},
    {6, 3, 11, 6, 5, 3, 5, 1, 3, -1, -1, -1, -1, -1, -1, -1},
    {0, 8, 11, 0, 11, 5, 0, 5, 1, 5, 11, 6, -1, -1, -1, -1},
    {3, 11, 6, 0, 3, 6, 0, 6, 5, 0, 5, 9, -1, -1, -1, -1},
    {6, 5, 9, 6, 9, 11, 11, 9, 8, -1, -1, -1, -1, -1, -1, -1},
    {5, 10, 6, 4, 7, 8, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {4, 3, 0, 4, 7, 3, 6, 5, 10, -1, -1, -1, -1, -1, -1, -1},
    {1, 9, 0, 5, 10, 6, 8, 4, 7, -1, -1, -1, -1, -1, -1, -1},
    {10, 6, 5, 1, 9, 7, 1, 7, 3, 7, 9, 4, -1, -1, -1, -1},
    {6, 1, 2, 6, 5, 1, 4, 7, 8, -1, -1, -1, -1, -1, -1, -1},
    {1, 2, 5, 5, 2, 6, 3, 0, 4, 3, 4, 7, -1, -1, -1, -1},
    {8, 4, 7, 9, 0, 5, 0, 6, 5, 0, 2, 6, -1, -1, -1, -1},
    {7, 3, 9, 7, 9, 4, 3, 2, 9, 5, 9, 6, 2, 6, 9, -1},
    {3, 11, 2, 7, 8, 4, 10, 6, 5, -1, -1, -1, -1, -1, -1, -1},
    {5, 10, 6, 4, 7, 2, 4, 2, 0, 2, 7, 11, -1, -1, -1, -1},
    {0, 1, 9, 4, 7, 8, 2, 3, 11, 5, 10, 6, -1, -1, -1, -1},
    {9, 2, 1, 9, 11, 2, 9, 4, 11, 7, 11, 4, 5, 10, 6, -1},
    {8, 4, 7, 3, 11, 5, 3, 5, 1, 5, 11, 6, -1, -1, -1, -1},
    {5, 1, 11, 5, 11, 6, 1, 0, 11, 7, 11, 4, 0, 4, 11, -1},
    {0, 5, 9, 0, 6, 5, 0, 3, 6, 11, 6, 3, 8, 4, 7, -1},
    {6, 5, 9, 6, 9, 11, 4, 7, 9, 7, 11, 9, -1, -1, -1, -1},
    {10, 4, 9, 6, 4, 10, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {4, 10, 6, 4, 9, 10, 0, 8, 3, -1, -1, -1, -1, -1, -1, -1},
    {10, 0, 1, 10, 6, 0, 6, 4, 0, -1, -1, -1, -1, -1, -1, -1},
    {8, 3, 1, 8, 1, 6, 8, 6, 4, 6, 1, 10, -1, -1, -1, -1},
    {1, 4, 9, 1, 2, 4, 2, 6, 4, -1, -1, -1, -1, -1, -1, -1},
    {3, 0, 8, 1, 2, 9, 2, 4, 9, 2, 6, 4, -1, -1, -1, -1},
    {0, 2, 4, 4, 2, 6, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {8, 3, 2, 8, 2, 4, 4, 2, 6, -1, -1, -1, -1, -1, -1, -1},
    {10, 4, 9, 10, 6, 4, 11, 2, 3, -1, -1, -1, -1, -1, -1, -1},
    {0, 8, 2, 2, 8, 11, 4, 9, 10, 4, 10, 6, -1, -1, -1, -1},
    {3, 11, 2, 0, 1, 6, 0, 6, 4, 6, 1, 10, -1, -1, -1, -1},
    {6, 4, 1, 6, 1, 10, 4, 8, 1, 2, 1, 11, 8, 11, 1, -1},
    {9, 6, 4, 9, 3, 6, 9, 1, 3, 11, 6, 3, -1, -1, -1, -1},
    {8, 11, 1, 8, 1, 0, 11, 6, 1, 9, 1, 4, 6, 4, 1, -1},
    {3, 11, 6, 3, 6, 0, 0, 6, 4, -1, -1, -1, -1, -1, -1, -1},
    {6, 4, 8, 11, 6, 8, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {7, 10, 6, 7, 8, 10, 8, 9, 10, -1, -1, -1, -1, -1, -1, -1},
    {0, 7, 3, 0, 10, 7, 0, 9, 10, 6, 7, 10, -1, -1, -1, -1},
    {10, 6, 7, 1, 10, 7, 1, 7, 8, 1, 8, 0, -1, -1, -1, -1},
    {10, 6, 7, 10, 7, 1, 1, 7, 3, -1, -1, -1, -1, -1, -1, -1},
    {1, 2, 6, 1, 6, 8, 1, 8, 9, 8, 6, 7, -1, -1, -1, -1},
    {2, 6, 9, 2, 9, 1, 6, 7, 9, 0, 9, 3, 7, 3, 9, -1},
    {7, 8, 0, 7, 0, 6, 6, 0, 2, -1, -1, -1, -1, -1, -1, -1},
    {7, 3, 2, 6, 7, 2, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {2, 3, 11, 10, 6, 8, 10, 8, 9, 8, 6, 7, -1, -1, -1, -1},
    {2, 0, 7, 2, 7, 11, 0, 9, 7, 6, 7, 10, 9, 10, 7, -1},
    {1, 8, 0, 1, 7, 8, 1, 10, 7, 6, 7, 10, 2, 3, 11, -1},
    {11, 2, 1, 11, 1, 7, 10, 6, 1, 6, 7, 1, -1, -1, -1, -1},
    {8, 9, 6, 8, 6, 7, 9, 1, 6, 11, 6, 3, 1, 3, 6, -1},
    {0, 9, 1, 11, 6, 7, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {7, 8, 0, 7, 0, 6, 3, 11, 0, 11, 6, 0, -1, -1, -1, -1},
    {7, 11, 6, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {7, 6, 11, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {3, 0, 8, 11, 7, 6, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 1, 9, 11, 7, 6, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {8, 1, 9, 8, 3, 1, 11, 7, 6, -1, -1, -1, -1, -1, -1, -1},
    {10, 1, 2, 6, 11, 7, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {1, 2, 10, 3, 0, 8, 6, 11, 7, -1, -1, -1, -1, -1, -1, -1},
    {2, 9, 0, 2, 10, 9, 6, 11, 7, -1, -1, -1, -1, -1, -1, -1},
    {6, 11, 7, 2, 10, 3, 10, 8, 3, 10, 9, 8, -1, -1, -1, -1},
    {7, 2, 3, 6, 2, 7, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {7, 0, 8, 7, 6, 0, 6, 2, 0, -1, -1, -1, -1, -1, -1, -1},
    {2, 7, 6, 2, 3, 7, 0, 1, 9, -1, -1, -1, -1, -1, -1, -1},
    {1, 6, 2, 1, 8, 6, 1, 9, 8, 8, 7, 6, -1, -1, -1, -1},
    {10, 7, 6, 10, 1, 7, 1, 3, 7, -1, -1, -1, -1, -1, -1, -1},
    {10, 7, 6, 1, 7, 10, 1, 8, 7, 1, 0, 8, -1, -1, -1, -1},
    {0, 3, 7, 0, 7, 10, 0, 10, 9, 6, 10, 7, -1, -1, -1, -1},
    {7, 6, 10, 7, 10, 8, 8, 10, 9, -1, -1, -1, -1, -1, -1, -1},
    {6, 8, 4, 11, 8, 6, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {3, 6, 11, 3, 0, 6, 0, 4, 6, -1, -1, -1, -1, -1, -1, -1},
    {8, 6, 11, 8, 4, 6, 9, 0, 1, -1, -1, -1, -1, -1, -1, -1},
    {9, 4, 6, 9, 6, 3, 9, 3, 1, 11, 3, 6, -1, -1, -1, -1},
    {6, 8, 4, 6, 11, 8, 2, 10, 1, -1, -1, -1, -1, -1, -1, -1},
    {1, 2, 10, 3, 0, 11, 0, 6, 11, 0, 4, 6, -1, -1, -1, -1},
    {4, 11, 8, 4, 6, 11, 0, 2, 9, 2, 10, 9, -1, -1, -1, -1},
    {10, 9, 3, 10, 3, 2, 9, 4, 3, 11, 3, 6, 4, 6, 3, -1},
    {8, 2, 3, 8, 4, 2, 4, 6, 2, -1, -1, -1, -1, -1, -1, -1},
    {0, 4, 2, 4, 6, 2, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {1, 9, 0, 2, 3, 4, 2, 4, 6, 4, 3, 8, -1, -1, -1, -1},
    {1, 9, 4, 1, 4, 2, 2, 4, 6, -1, -1, -1, -1, -1, -1, -1},
    {8, 1, 3, 8, 6, 1, 8, 4, 6, 6, 10, 1, -1, -1, -1, -1},
    {10, 1, 0, 10, 0, 6, 6, 0, 4, -1, -1, -1, -1, -1, -1, -1},
    {4, 6, 3, 4, 3, 8, 6, 10, 3, 0, 3, 9, 10, 9, 3, -1},
    {10, 9, 4, 6, 10, 4, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {4, 9, 5, 7, 6, 11, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 8, 3, 4, 9, 5, 11, 7, 6, -1, -1, -1, -1, -1, -1, -1},
    {5, 0, 1, 5, 4, 0, 7, 6, 11, -1, -1, -1, -1, -1, -1, -1},
    {11, 7, 6, 8, 3, 4, 3, 5, 4, 3, 1, 5, -1, -1, -1, -1},
    {9, 5, 4, 10, 1, 2, 7, 6, 11, -1, -1, -1, -1, -1, -1, -1},
    {6, 11, 7, 1, 2, 10, 0, 8, 3, 4, 9, 5, -1, -1, -1, -1},
    {7, 6, 11, 5, 4, 10, 4, 2, 10, 4, 0, 2, -1, -1, -1, -1},
    {3, 4, 8, 3, 5, 4, 3, 2, 5, 10, 5, 2, 11, 7, 6, -1},
    {7, 2, 3, 7, 6, 2, 5, 4, 9, -1, -1, -1, -1, -1, -1, -1},
    {9, 5, 4, 0, 8, 6, 0, 6, 2, 6, 8, 7, -1, -1, -1, -1},
    {3, 6, 2, 3, 7, 6, 1, 5, 0, 5, 4, 0, -1, -1, -1, -1},
    {6, 2, 8, 6, 8, 7, 2, 1, 8, 4, 8, 5, 1, 5, 8, -1},
    {9, 5, 4, 10, 1, 6, 1, 7, 6, 1, 3, 7, -1, -1, -1, -1},
    {1, 6, 10, 1, 7, 6, 1, 0, 7, 8, 7, 0, 9, 5, 4, -1},
    {4, 0, 10, 4, 10, 5, 0, 3, 10, 6, 10, 7, 3, 7, 10, -1},
    {7, 6, 10, 7, 10, 8, 5, 4, 10, 4, 8, 10, -1, -1, -1, -1},
    {6, 9, 5, 6, 11, 9, 11, 8, 9, -1, -1, -1, -1, -1, -1, -1},
    {3, 6, 11, 0, 6, 3, 0, 5, 6, 0, 9, 5, -1, -1, -1, -1},
    {0, 11, 8, 0, 5, 11, 0, 1, 5, 5, 6, 11, -1, -1, -1, -1},
    {6, 11, 3, 6, 3, 5, 5, 3, 1, -1, -1, -1, -1, -1, -1, -1},
    {1, 2, 10, 9, 5, 11, 9, 11, 8, 11, 5, 6, -1, -1, -1, -1},
    {0, 11, 3, 0, 6, 11, 0, 9, 6, 5, 6, 9, 1, 2, 10, -1},
    {11, 8, 5, 11, 5, 6, 8, 0, 5, 10, 5, 2, 0, 2, 5, -1},
    {6, 11, 3, 6, 3, 5, 2, 10, 3, 10, 5, 3, -1, -1, -1, -1},
    {5, 8, 9, 5, 2, 8, 5, 6, 2, 3, 8, 2, -1, -1, -1, -1},
    {9, 5, 6, 9, 6, 0, 0, 6, 2, -1, -1, -1, -1, -1, -1, -1},
    {1, 5, 8, 1, 8, 0, 5, 6, 8, 3, 8, 2, 6, 2, 8, -1},
    {1, 5, 6, 2, 1, 6, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {1, 3, 6, 1, 6, 10, 3, 8, 6, 5, 6, 9, 8, 9, 6, -1},
    {10, 1, 0, 10, 0, 6, 9, 5, 0, 5, 6, 0, -1, -1, -1, -1},
    {0, 3, 8, 5, 6, 10, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {10, 5, 6, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {11, 5, 10, 7, 5, 11, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {11, 5, 10, 11, 7, 5, 8, 3, 0, -1, -1, -1, -1, -1, -1, -1},
    {5, 11, 7, 5, 10, 11, 1, 9, 0, -1, -1, -1, -1, -1, -1, -1},
    {10, 7, 5, 10, 11, 7, 9, 8, 1, 8, 3, 1, -1, -1, -1, -1},
    {11, 1, 2, 11, 7, 1, 7, 5, 1, -1, -1, -1, -1, -1, -1, -1},
    {0, 8, 3, 1, 2, 7, 1, 7, 5, 7, 2, 11, -1, -1, -1, -1},
    {9, 7, 5, 9, 2, 7, 9, 0, 2, 2, 11, 7, -1, -1, -1, -1},
    {7, 5, 2, 7, 2, 11, 5, 9, 2, 3, 2, 8, 9, 8, 2, -1},
    {2, 5, 10, 2, 3, 5, 3, 7, 5, -1, -1, -1, -1, -1, -1, -1},
    {8, 2, 0, 8, 5, 2, 8, 7, 5, 10, 2, 5, -1, -1, -1, -1},
    {9, 0, 1, 5, 10, 3, 5, 3, 7, 3, 10, 2, -1, -1, -1, -1},
    {9, 8, 2, 9, 2, 1, 8, 7, 2, 10, 2, 5, 7, 5, 2, -1},
    {1, 3, 5, 3, 7, 5, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 8, 7, 0, 7, 1, 1, 7, 5, -1, -1, -1, -1, -1, -1, -1},
    {9, 0, 3, 9, 3, 5, 5, 3, 7, -1, -1, -1, -1, -1, -1, -1},
    {9, 8, 7, 5, 9, 7, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {5, 8, 4, 5, 10, 8, 10, 11, 8, -1, -1, -1, -1, -1, -1, -1},
    {5, 0, 4, 5, 11, 0, 5, 10, 11, 11, 3, 0, -1, -1, -1, -1},
    {0, 1, 9, 8, 4, 10, 8, 10, 11, 10, 4, 5, -1, -1, -1, -1},
    {10, 11, 4, 10, 4, 5, 11, 3, 4, 9, 4, 1, 3, 1, 4, -1},
    {2, 5, 1, 2, 8, 5, 2, 11, 8, 4, 5, 8, -1, -1, -1, -1},
    {0, 4, 11, 0, 11, 3, 4, 5, 11, 2, 11, 1, 5, 1, 11, -1},
    {0, 2, 5, 0, 5, 9, 2, 11, 5, 4, 5, 8, 11, 8, 5, -1},
    {9, 4, 5, 2, 11, 3, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {2, 5, 10, 3, 5, 2, 3, 4, 5, 3, 8, 4, -1, -1, -1, -1},
    {5, 10, 2, 5, 2, 4, 4, 2, 0, -1, -1, -1, -1, -1, -1, -1},
    {3, 10, 2, 3, 5, 10, 3, 8, 5, 4, 5, 8, 0, 1, 9, -1},
    {5, 10, 2, 5, 2, 4, 1, 9, 2, 9, 4, 2, -1, -1, -1, -1},
    {8, 4, 5, 8, 5, 3, 3, 5, 1, -1, -1, -1, -1, -1, -1, -1},
    {0, 4, 5, 1, 0, 5, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {8, 4, 5, 8, 5, 3, 9, 0, 5, 0, 3, 5, -1, -1, -1, -1},
    {9, 4, 5, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {4, 11, 7, 4, 9, 11, 9, 10, 11, -1, -1, -1, -1, -1, -1, -1},
    {0, 8, 3, 4, 9, 7, 9, 11, 7, 9, 10, 11, -1, -1, -1, -1},
    {1, 10, 11, 1, 11, 4, 1, 4, 0, 7, 4, 11, -1, -1, -1, -1},
    {3, 1, 4, 3, 4, 8, 1, 10, 4, 7, 4, 11, 10, 11, 4, -1},
    {4, 11, 7, 9, 11, 4, 9, 2, 11, 9, 1, 2, -1, -1, -1, -1},
    {9, 7, 4, 9, 11, 7, 9, 1, 11, 2, 11, 1, 0, 8, 3, -1},
    {11, 7, 4, 11, 4, 2, 2, 4, 0, -1, -1, -1, -1, -1, -1, -1},
    {11, 7, 4, 11, 4, 2, 8, 3, 4, 3, 2, 4, -1, -1, -1, -1},
    {2, 9, 10, 2, 7, 9, 2, 3, 7, 7, 4, 9, -1, -1, -1, -1},
    {9, 10, 7, 9, 7, 4, 10, 2, 7, 8, 7, 0, 2, 0, 7, -1},
    {3, 7, 10, 3, 10, 2, 7, 4, 10, 1, 10, 0, 4, 0, 10, -1},
    {1, 10, 2, 8, 7, 4, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {4, 9, 1, 4, 1, 7, 7, 1, 3, -1, -1, -1, -1, -1, -1, -1},
    {4, 9, 1, 4, 1, 7, 0, 8, 1, 8, 7, 1, -1, -1, -1, -1},
    {4, 0, 3, 7, 4, 3, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {4, 8, 7, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {9, 10, 8, 10, 11, 8, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {3, 0, 9, 3, 9, 11, 11, 9, 10, -1, -1, -1, -1, -1, -1, -1},
    {0, 1, 10, 0, 10, 8, 8, 10, 11, -1, -1, -1, -1, -1, -1, -1},
    {3, 1, 10, 11, 3, 10, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {1, 2, 11, 1, 11, 9, 9, 11, 8, -1, -1, -1, -1, -1, -1, -1},
    {3, 0, 9, 3, 9, 11, 1, 2, 9, 2, 11, 9, -1, -1, -1, -1},
    {0, 2, 11, 8, 0, 11, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {3, 2, 11, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {2, 3, 8, 2, 8, 10, 10, 8, 9, -1, -1, -1, -1, -1, -1, -1},
    {9, 10, 2, 0, 9, 2, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {2, 3, 8, 2, 8, 10, 0, 1, 8, 1, 10, 8, -1, -1, -1, -1},
    {1, 10, 2, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {1, 3, 8, 9, 1, 8, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 9, 1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {0, 3, 8, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
    {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
};

// The polygons of every case from the cube geometry, checked against the
// triangle lists above.  On each face the crossing edges pair up into
// segments (an ambiguous face cuts off its two corners above the iso value);
// segments are oriented so that, looking at the face from outside with its
// corners counter-clockwise, a segment starts at the crossing entered from a
// corner below the iso value.  The triangles of a case must cover exactly the
// polygons these segments close into, with the same orientation: their
// directed boundary edges (those whose reverse is not an edge of another
// triangle) are the segments.  Returns false if any case disagrees.
bool mc_tables_host(int* edge_table, signed char* tri_table) {
    int face[6][4];
    int nf = 0;
    for (int axis = 0; axis < 3; ++axis)
        for (int val = 0; val < 2; ++val) {
            int cs[4], k = 0;
            for (int c = 0; c < 8; ++c)
                if (kCorner[c][axis] == val) cs[k++] = c;
            int o[4] = {cs[0], -1, -1, -1};
            for (int i = 1; i < 4; ++i)
                for (int j = 0; j < 4; ++j) {
                    int c = cs[j];
                    bool used = false;
                    for (int u = 0; u < i; ++u) used |= (o[u] == c);
                    int dist = 0;
                    for (int d = 0; d < 3; ++d) dist += abs(kCorner[c][d] - kCorner[o[i - 1]][d]);
                    if (!used && dist == 1) {
                        o[i] = c;
                        break;
                    }
                }
            // (o1 - o0) x (o2 - o1) must point along the outward normal
            int a[3], b[3];
            for (int d = 0; d < 3; ++d) {
                a[d] = kCorner[o[1]][d] - kCorner[o[0]][d];
                b[d] = kCorner[o[2]][d] - kCorner[o[1]][d];
            }
            int cr[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
            if (cr[axis] * (val ? 1 : -1) < 0) {
                int tmp = o[1];
                o[1] = o[3];
                o[3] = tmp;
            }
            for (int i = 0; i < 4; ++i) face[nf][i] = o[i];
            ++nf;
        }
    auto edge_of = [](int p, int q) {
        for (int e = 0; e < 12; ++e)
            if ((edge_a(e) == p && edge_b(e) == q) || (edge_a(e) == q && edge_b(e) == p)) return e;
        return -1;
    };
    bool ok = true;
    for (int ci = 0; ci < 256; ++ci) {
        int above[8];
        for (int c = 0; c < 8; ++c) above[c] = (ci >> c) & 1;
        int mask = 0;
        for (int e = 0; e < 12; ++e)
            if (above[edge_a(e)] != above[edge_b(e)]) mask |= 1 << e;
        edge_table[ci] = mask;
        int next[12];
        for (int e = 0; e < 12; ++e) next[e] = -1;
        for (int f = 0; f < 6; ++f) {
            int ce[4], from_above[4], n = 0;
            for (int k = 0; k < 4; ++k) {
                int p = face[f][k], q = face[f][(k + 1) & 3];
                if (above[p] != above[q]) {
                    ce[n] = edge_of(p, q);
                    from_above[n] = above[p];
                    ++n;
                }
            }
            int seg[2][2], ns = 0;
            if (n == 2) {
                seg[0][0] = 0;
                seg[0][1] = 1;
                ns = 1;
            } else if (n == 4) {
                if (above[face[f][0]]) {
                    seg[0][0] = 3; seg[0][1] = 0;
                    seg[1][0] = 1; seg[1][1] = 2;
                } else {
                    seg[0][0] = 0; seg[0][1] = 1;
                    seg[1][0] = 2; seg[1][1] = 3;
                }
                ns = 2;
            }
            for (int k = 0; k < ns; ++k) {
                int x = seg[k][0], y = seg[k][1];
                if (!from_above[x])
                    next[ce[x]] = ce[y];
                else
                    next[ce[y]] = ce[x];
            }
        }
        // directed edge counts of the case's triangles
        int de[12][12] = {};
        int w = 0;
        for (; w < 16 && kTriangles[ci][w] >= 0; w += 3)
            for (int k = 0; k < 3; ++k) {
                const int p = kTriangles[ci][w + k], q = kTriangles[ci][w + (k + 1) % 3];
                if (p < 0 || p > 11 || q < 0 || q > 11 || !(mask >> p & 1)) ok = false;
                else ++de[p][q];
            }
        for (int p = 0; p < 12; ++p)
            for (int q = 0; q < 12; ++q) {
                const bool boundary = de[p][q] == 1 && de[q][p] == 0;
                const bool interior = de[p][q] == 1 && de[q][p] == 1;
                if (de[p][q] > 1 || (de[p][q] == 1 && !boundary && !interior)) ok = false;
                if (boundary != (next[p] == q)) ok = false;
            }
        for (int k = 0; k < 16; ++k) tri_table[ci * 16 + k] = kTriangles[ci][k];
    }
    return ok;
}

int mc_upload_tables() {
    // once per device; the lock makes concurrent first calls from several host
    // threads upload once and return only after the upload
    static std::mutex mu;
    static bool done[64] = {false};
    int dev = 0;
    DWG_CHECK_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && done[dev]) return DWG_OK;
    int et[256];
    signed char tt[256 * 16];
    DWG_REQUIRE(mc_tables_host(et, tt), "marching cubes: a case's triangles do not match its polygons");
    unsigned char nt[256];
    unsigned short es[256];
    for (int i = 0; i < 256; ++i) {
        int k = 0;
        while (k < 16 && tt[i * 16 + k] >= 0) k += 3;
        nt[i] = (unsigned char)(k / 3);
        es[i] = (unsigned short)et[i];
    }
    DWG_CHECK_CUDA(cudaMemcpyToSymbol(c_tri, tt, sizeof(tt)));
    DWG_CHECK_CUDA(cudaMemcpyToSymbol(c_ntri, nt, sizeof(nt)));
    DWG_CHECK_CUDA(cudaMemcpyToSymbol(c_edges, es, sizeof(es)));
    if (dev >= 0 && dev < 64) done[dev] = true;
    return DWG_OK;
}

constexpr int kMcThreads = 256;

struct McArgs {
    const float* __restrict__ field;
    const float* __restrict__ pos;
    int rx, ry, rz;
    long long ncell;
    float ox, oy, oz, h;
    int zoff;  // global z index of local sample 0
    float iso;
    const float* iso_dev;
};

__device__ __forceinline__ int mc_case(const McArgs& a, long long cell, int& x, int& y, int& z,
                                       float v[8], float iso) {
    const long long cx = a.rx - 1, cy = a.ry - 1;
    x = (int)(cell % cx);
    long long t = cell / cx;
    y = (int)(t % cy);
    z = (int)(t / cy);
    int ci = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int ox = ((c & 1) != ((c >> 1) & 1)) ? 1 : 0;
        const int oy = (c >> 1) & 1;
        const int oz = (c & 4) ? 0 : 1;
        v[c] = a.field[(long long)(x + ox) + (long long)a.rx * ((long long)(y + oy) + (long long)a.ry * (z + oz))];
        if (v[c] > iso) ci |= 1 << c;
    }
    return ci;
}

__global__ void __launch_bounds__(kMcThreads) k_mc_count(McArgs a, unsigned int* __restrict__ counts) {
    const float iso = a.iso_dev ? *a.iso_dev : a.iso;
    long long cell = (long long)blockIdx.x * kMcThreads + threadIdx.x;
    unsigned n = 0;
    if (cell < a.ncell) {
        int x, y, z;
        float v[8];
        n = c_ntri[mc_case(a, cell, x, y, z, v, iso)];
    }
    typedef cub::BlockReduce<unsigned, kMcThreads> BR;
    __shared__ typename BR::TempStorage tmp;
    unsigned tot = BR(tmp).Sum(n);
    if (threadIdx.x == 0) counts[blockIdx.x] = tot;
}

__global__ void k_mc_total(const unsigned int* __restrict__ counts, const unsigned int* __restrict__ offs,
                           long long nb, unsigned long long* __restrict__ total) {
    *total = (unsigned long long)offs[nb - 1] + counts[nb - 1];
}

__global__ void __launch_bounds__(kMcThreads)
    k_mc_emit(McArgs a, const unsigned int* __restrict__ offs, long long cap, float* __restrict__ tris,
              float* __restrict__ cen, float* __restrict__ nrm) {
    const float iso = a.iso_dev ? *a.iso_dev : a.iso;
    long long cell = (long long)blockIdx.x * kMcThreads + threadIdx.x;
    int x = 0, y = 0, z = 0, ci = 0;
    float v[8];
    unsigned n = 0;
    if (cell < a.ncell) {
        ci = mc_case(a, cell, x, y, z, v, iso);
        n = c_ntri[ci];
    }
    typedef cub::BlockScan<unsigned, kMcThreads> BS;
    __shared__ typename BS::TempStorage tmp;
    unsigned local;
    BS(tmp).ExclusiveSum(n, local);
    if (!n) return;
    unsigned long long base = (unsigned long long)offs[blockIdx.x] + local;
    float p[8][3];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int ox = ((c & 1) != ((c >> 1) & 1)) ? 1 : 0;
        const int oy = (c >> 1) & 1;
        const int oz = (c & 4) ? 0 : 1;
        const int gx = x + ox, gy = y + oy, gz = z + oz;
        if (a.pos) {
            long long gi = (long long)gx + (long long)a.rx * ((long long)gy + (long long)a.ry * gz);
            p[c][0] = a.pos[gi * 3];
            p[c][1] = a.pos[gi * 3 + 1];
            p[c][2] = a.pos[gi * 3 + 2];
        } else {
            p[c][0] = __fadd_rn(a.ox, __fmul_rn((float)gx, a.h));
            p[c][1] = __fadd_rn(a.oy, __fmul_rn((float)gy, a.h));
            p[c][2] = __fadd_rn(a.oz, __fmul_rn((float)(gz + a.zoff), a.h));
        }
    }
    const unsigned emask = c_edges[ci];
    float vl[12][3];
#pragma unroll
    for (int e = 0; e < 12; ++e) {
        if (!(emask & (1u << e))) continue;
        const int ia = e & 7;
        const int ib = e < 4 ? ((e + 1) & 3) : (e < 8 ? 4 + ((e - 3) & 3) : e - 4);
        float num = __fsub_rn(v[ia], iso);
        float den = __double2float_rn(__dadd_rn((double)__fsub_rn(v[ib], v[ia]), 1e-10));
        float ell = __fdiv_rn(num, den);
#pragma unroll
        for (int d = 0; d < 3; ++d) vl[e][d] = __fsub_rn(p[ia][d], __fmul_rn(ell, __fsub_rn(p[ib][d], p[ia][d])));
    }
    for (unsigned k = 0; k < n; ++k) {
        unsigned long long t = base + k;
        if ((long long)t >= cap) break;
        const int e0 = c_tri[ci][3 * k], e1 = c_tri[ci][3 * k + 1], e2 = c_tri[ci][3 * k + 2];
        float P0[3], P1[3], P2[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            P0[d] = vl[e0][d];
            P1[d] = vl[e1][d];
            P2[d] = vl[e2][d];
        }
        if (tris) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                tris[t * 9 + d] = P0[d];
                tris[t * 9 + 3 + d] = P1[d];
                tris[t * 9 + 6 + d] = P2[d];
            }
        }
        if (cen) {
#pragma unroll
            for (int d = 0; d < 3; ++d) cen[t * 3 + d] = __fdiv_rn(__fadd_rn(__fadd_rn(P0[d], P1[d]), P2[d]), 3.0f);
        }
        if (nrm) {
            float u[3], w[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                u[d] = __fsub_rn(P1[d], P0[d]);
                w[d] = __fsub_rn(P2[d], P0[d]);
            }
            float cx = __fsub_rn(__fmul_rn(u[1], w[2]), __fmul_rn(u[2], w[1]));
            float cy = __fsub_rn(__fmul_rn(u[2], w[0]), __fmul_rn(u[0], w[2]));
            float cz = __fsub_rn(__fmul_rn(u[0], w[1]), __fmul_rn(u[1], w[0]));
            float sc = -inv_len_eps(__fsqrt_rn(sq3_rn(cx, cy, cz)));
            nrm[t * 3] = __fmul_rn(cx, sc);
            nrm[t * 3 + 1] = __fmul_rn(cy, sc);
            nrm[t * 3 + 2] = __fmul_rn(cz, sc);
        }
    }
}

int mc_run(const float* field, const McGrid& g, float iso, const float* iso_dev, float* tris,
           float* centroids, float* normals, long long cap, unsigned long long* num_tris_dev,
           McWorkspace& ws, cudaStream_t s) {
    DWG_REQUIRE(field && num_tris_dev, "marching cubes: null field or count pointer");
    DWG_REQUIRE(g.res[0] >= 2 && g.res[1] >= 2 && g.res[2] >= 2, "marching cubes: resolution must be >= 2");
    DWG_TRY(mc_upload_tables());
    McArgs a;
    a.field = field;
    a.pos = g.positions;
    a.rx = g.res[0];
    a.ry = g.res[1];
    a.rz = g.res[2];
    a.ncell = (long long)(g.res[0] - 1) * (g.res[1] - 1) * (g.res[2] - 1);
    a.ox = g.origin[0];
    a.oy = g.origin[1];
    a.oz = g.origin[2];
    a.zoff = g.zoff;
    a.h = g.spacing;
    a.iso = iso;
    a.iso_dev = iso_dev;
    long long nb = (a.ncell + kMcThreads - 1) / kMcThreads;
    DWG_REQUIRE(nb < (1ll << 31), "marching cubes: grid too large");
    DWG_TRY(ws.block_counts.reserve(nb));
    DWG_TRY(ws.block_offsets.reserve(nb));
    k_mc_count<<<(unsigned)nb, kMcThreads, 0, s>>>(a, ws.block_counts.ptr);
    DWG_CHECK_LAUNCH();
    size_t bytes = 0;
    unsigned* cin = ws.block_counts.ptr;
    unsigned* cout = ws.block_offsets.ptr;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cin, cout, (int)nb, s));
    DWG_TRY(ws.scratch.reserve(bytes + 256));
    bytes = ws.scratch.n;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(ws.scratch.ptr, bytes, cin, cout, (int)nb, s));
    k_mc_total<<<1, 1, 0, s>>>(cin, cout, nb, num_tris_dev);
    k_mc_emit<<<(unsigned)nb, kMcThreads, 0, s>>>(a, cout, cap, tris, centroids, normals);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

}  // namespace dwg

// ----------------------------------------------------------------------------
// Marching cubes without any device allocation.
//
// Some callers cannot call cudaMalloc when they mesh: a real-time loop that
// must not allocate after start-up (cudaMalloc and cudaFree can wait for the
// whole device), or an application whose device memory is a fixed budget
// handed out by its own pool.  dwg_marching_cubes_noalloc serves them with the
// same two kernels as dwg_marching_cubes; its scratch (per-block triangle
// counts, their offsets and the total) lives in the file-scope device array
// below, which every GPU that loads this library holds until the process
// exits.  The scan writes every offset and the total it later reads, so
// nothing has to be cleared between calls.
// ----------------------------------------------------------------------------
namespace dwg {

// 2^19 blocks of 256 cells: grids up to 134,217,728 cells (e.g. 512^3)
constexpr long long kMcNoAllocMaxBlocks = 1ll << 19;
constexpr long long kMcNoAllocMaxCells = kMcNoAllocMaxBlocks * kMcThreads;
// [0, max) block counts, [max, 2 max) block offsets, then the 64-bit total
static __device__ __align__(256) unsigned int g_mc_noalloc_scratch[2 * kMcNoAllocMaxBlocks + 64];

// exclusive scan of the block counts by one block, in chunks, with a carry;
// writes every offset and the total, so no slot has to start at zero
constexpr int kMcScanThreads = 1024;
__global__ void __launch_bounds__(kMcScanThreads)
    k_mc_noalloc_scan(const unsigned int* __restrict__ counts, unsigned int* __restrict__ offs, long long nb,
                      unsigned long long* __restrict__ total) {
    typedef cub::BlockScan<unsigned long long, kMcScanThreads> BS;
    __shared__ typename BS::TempStorage tmp;
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < nb; base += kMcScanThreads) {
        const long long i = base + threadIdx.x;
        const unsigned long long v = i < nb ? counts[i] : 0ull;
        unsigned long long ex, agg;
        BS(tmp).ExclusiveSum(v, ex, agg);
        if (i < nb) offs[i] = (unsigned int)(carry + ex);
        __syncthreads();
        if (threadIdx.x == 0) carry += agg;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// device address of the scratch array, looked up once per device with that
// device current (the host-side symbol is not a device address)
static int mc_noalloc_scratch(unsigned int** out) {
    static std::mutex mu;
    static unsigned int* addr[64] = {nullptr};
    int dev = 0;
    DWG_CHECK_CUDA(cudaGetDevice(&dev));
    DWG_REQUIRE(dev >= 0 && dev < 64, "marching_cubes_noalloc: device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_mc_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error("marching_cubes_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return DWG_ERR_CUDA;
        }
        addr[dev] = (unsigned int*)p;
    }
    *out = addr[dev];
    return DWG_OK;
}

}  // namespace dwg

extern "C" int dwg_marching_cubes_noalloc(const float* field_dev, const int res[3], const float* positions_dev,
                                          const float origin[3], float spacing, float iso, float* tris_dev,
                                          float* centroids_dev, float* normals_dev, long long capacity,
                                          long long* num_tris_host, void* stream) {
    using namespace dwg;
    DWG_REQUIRE(field_dev && res && num_tris_host, "marching_cubes_noalloc: null field, resolution or count");
    DWG_REQUIRE(origin || positions_dev, "marching_cubes_noalloc: grid undefined (no origin, no positions)");
    DWG_REQUIRE(res[0] >= 2 && res[1] >= 2 && res[2] >= 2, "marching_cubes_noalloc: resolution must be >= 2");
    DWG_REQUIRE(capacity >= 0, "marching_cubes_noalloc: negative capacity");
    const long long ncell = (long long)(res[0] - 1) * (res[1] - 1) * (res[2] - 1);
    DWG_REQUIRE(ncell <= kMcNoAllocMaxCells,
                "marching_cubes_noalloc: %lld cells exceed the allocation-free limit of %lld cells; use "
                "dwg_marching_cubes",
                ncell, kMcNoAllocMaxCells);
    DWG_TRY(mc_upload_tables());
    unsigned int* scratch = nullptr;
    DWG_TRY(mc_noalloc_scratch(&scratch));
    unsigned int* counts = scratch;
    unsigned int* offs = scratch + kMcNoAllocMaxBlocks;
    unsigned long long* total = reinterpret_cast<unsigned long long*>(scratch + 2 * kMcNoAllocMaxBlocks);
    cudaStream_t s = (cudaStream_t)stream;
    McArgs a;
    a.field = field_dev;
    a.pos = positions_dev;
    a.rx = res[0];
    a.ry = res[1];
    a.rz = res[2];
    a.ncell = ncell;
    a.ox = origin ? origin[0] : 0.f;
    a.oy = origin ? origin[1] : 0.f;
    a.oz = origin ? origin[2] : 0.f;
    a.zoff = 0;
    a.h = spacing;
    a.iso = iso;
    a.iso_dev = nullptr;
    const long long nb = (ncell + kMcThreads - 1) / kMcThreads;
    k_mc_count<<<(unsigned)nb, kMcThreads, 0, s>>>(a, counts);
    k_mc_noalloc_scan<<<1, kMcScanThreads, 0, s>>>(counts, offs, nb, total);
    k_mc_emit<<<(unsigned)nb, kMcThreads, 0, s>>>(a, offs, capacity, tris_dev, centroids_dev, normals_dev);
    DWG_CHECK_LAUNCH();
    unsigned long long T = 0;
    DWG_CHECK_CUDA(cudaMemcpyAsync(&T, total, sizeof(T), cudaMemcpyDeviceToHost, s));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    *num_tris_host = (long long)T;
    if ((long long)T > capacity) {
        set_error("marching_cubes_noalloc: %llu triangles exceed capacity %lld", T, capacity);
        return DWG_ERR_OVERFLOW;
    }
    return DWG_OK;
}
