// octree.cuh -- GPU octree with the topology of igl::octreeDWG
// (deps/libigl/include/igl/octree.cpp:171-335).
//
// Layout in HBM (structure of arrays):
//   points, sorted by their octant path (a 3*max_depth-bit key, stable):
//     pa[i] = (x, y, z, area)  float4      nr[i] = (nx, ny, nz, radius) float4
//     perm[i] = input index of sorted point i
//   nodes, numbered v in depth-first pre-order (a node's subtree is
//   contiguous and its first child, if any, is the next node):
//     info[v] = (pt_start, pt_count, skip, depth | LEAF)   int4
//     skip[v] = index of the first node after v's subtree, so the children of
//     v are v+1, skip[v+1], ... while < skip[v]
//     cm_d, r_d, ec_d: FP64 moments, pre-order
//   traversal records, numbered p in level order (by depth, then pre-order),
//   where the children of a node are consecutive:
//     node_a[p] = (cm.x, cm.y, cm.z, open threshold | leaf point count)  float4
//     node_b[p] = (sum A n .x, .y, .z, meta)                             float4
//     node_r[p] = R (max |p - cm|, rounded from FP64)                    float
//     level_nodes[p] = v,  lvl_of[v] = p
//   meta of an internal node: first child p (bits 0-27) | (children - 1) << 28;
//   of a leaf: LEAF (bit 31) | SINGLE (bit 30, one point) | pt_start (bits 0-27).
//   The open threshold is the largest float T with sqrt_rn(d2) > beta*R <=>
//   d2 > T for every float d2 != T; its sign bit is set when d2 == T needs the
//   exact test.
// Empty octants are not stored (the reference skips them at
// src/TurboLibiGWN.cu:630).
#pragma once

#include "common.cuh"

namespace dwg {

constexpr int kLeafFlag = 1 << 8;
constexpr int kMaxDepth = 21;
constexpr int kMetaIndex = (1 << 28) - 1;
constexpr int kMetaSingle = 1 << 30;
constexpr unsigned kMetaLeafBit = 1u << 31;

struct Octree {
    int n = 0;
    int max_depth = 0;
    int M = 0;
    double root[4] = {0, 0, 0, 0};  // centre xyz, width (host copy)
    DevBuf<double> root_dev;        // same on the device
    DevBuf<unsigned long long> keys;  // sorted keys
    DevBuf<int> perm;                 // sorted -> input
    DevBuf<int> inv_perm;             // input -> sorted
    DevBuf<float4> pa, nr;
    DevBuf<int4> info;
    DevBuf<float4> node_a, node_b;
    DevBuf<float> node_r;
    float thr_beta = -1.f;  // beta the open thresholds were computed for (-1: none)
    DevBuf<double> cm_d, r_d, ec_d;
    // far-field expansion coefficients of orders 1 and 2 about each node's
    // centre of mass (igl::fast_winding_number precompute,
    // deps/libigl/include/igl/fast_winding_number.cpp:87-105): 9 + 27 per node,
    // FP64 in pre-order (ho_d); their FP32 contraction for evaluation in level
    // order (node_h, 8 float4: m1, trace m1, the linear part of order 2, the
    // 18 distinct sums of the order-2 tensor symmetric in its first two indices)
    DevBuf<double> ho_d;
    DevBuf<float4> node_h;
    // level order: level d = positions level_off[d] .. level_off[d+1]
    DevBuf<int> level_nodes, lvl_of, node_meta;
    int level_off[kMaxDepth + 2] = {0};
    DevBuf<unsigned char> scratch;  // CUB temporary storage
    mutable DevBuf<unsigned int> work;  // [0] work counter of the persistent GWN kernel, [1] error flag
};

int octree_build(Octree& t, const float* points_dev, int n, int max_depth, const float* areas_dev,
                 cudaStream_t s);
// gather per-point arrays (input order) into sorted order; any may be null
int octree_set_point_data(Octree& t, const float* normals_dev, const float* areas_dev,
                          const float* radii_dev, cudaStream_t s);
// the same from arrays already in sorted order (internal pipeline use)
int octree_set_sorted_normals(Octree& t, const float* normals_sorted_dev, cudaStream_t s);
// FP64 moments: sum A p / sum A, max |p - CM|, from pa (positions, areas)
int octree_update_centres(Octree& t, cudaStream_t s);
// FP64 sum A n from pa.w and nr.xyz
int octree_update_normals(Octree& t, cudaStream_t s);
// expansion coefficients of orders 1..order (1 or 2) from the current
// centres, areas and normals (after octree_update_normals)
int octree_update_expansion(Octree& t, int order, cudaStream_t s);
// open thresholds for the opening ratio beta (no-op when already current)
int octree_set_beta(Octree& t, float beta, cudaStream_t s);
// node centre of every node at the octreeDWG recursion (FP64), for leaf extraction
int octree_leaf_centres(Octree& t, int min_count, DevBuf<float>& out_xyz, DevBuf<int>& out_node,
                        int* num_leaves, cudaStream_t s);

// DWG_ERR_INVALID when x[0..m) holds a NaN or an infinity (synchronises s)
int require_finite(const float* x, long long m, const char* what, cudaStream_t s);

// bounding box of float3 points: out[0..2] = min, out[3..5] = max (device)
int bbox_device(const float* points_dev, long long n, float* out_dev, cudaStream_t s);

}  // namespace dwg
