// knn.cuh -- exact k nearest neighbours over a uniform cell grid.
#pragma once

#include "common.cuh"

namespace dwg {

struct KnnIndex {
    int n = 0;
    int G[3] = {1, 1, 1};
    float lo[3] = {0, 0, 0};
    float h = 1.f, inv_h = 1.f;
    DevBuf<float4> pts;       // grouped by cell: (x, y, z, input index as int bits)
    DevBuf<int> cell_start;   // G0*G1*G2 + 1
    DevBuf<int> cell_fill;
    DevBuf<float> bbox;
    DevBuf<unsigned char> scratch;
    // occupancy pyramid: level l >= 1 halves the grid (rounding up) and flags
    // the cells whose 2x2x2 children hold a point; top level is 1x1x1
    static constexpr int kMaxLevels = 16;
    int levels = 0;  // top level index (0: no pyramid)
    int ldim[kMaxLevels][3] = {};
    long long loff[kMaxLevels] = {};
    DevBuf<unsigned char> occ;
    // kb[c] >= distance from the centre of cell c to its kKnnBoundK-th
    // nearest point: over the whole grid on the first cell-grouped query, or
    // (kb_per_query, indexes rebuilt between queries) for the cells holding
    // queries only, at every query
    mutable DevBuf<float> kb, kb_tmp;
    mutable bool kb_ready = false;
    bool kb_per_query = false;
    // workspace of the cell-grouped queries
    mutable DevBuf<int> c_count, c_start, c_fill, c_active, c_misc, c_fb, c_deep;
    mutable DevBuf<unsigned int> c_m;
    mutable DevBuf<unsigned int> c_s;  // per cell: largest |q - x_c| + seed radius (seeded queries)
    mutable DevBuf<float> c_deep_bound;
    mutable DevBuf<unsigned char> c_scratch;
    // query bucketing workspace (grown on demand; not thread safe)
    int morton_shift = 0;
    mutable DevBuf<int> q_key, q_order, q_hist, q_fill;
    mutable DevBuf<unsigned char> q_scratch;
};

int knn_build(KnnIndex& ix, const float* points_dev, int n, cudaStream_t s);

constexpr int kKnnBoundK = 16;  // queries with k <= 16 and no exclusion use cell grouping

struct KnnQuery {
    const float* q = nullptr;              // packed xyz, or ...
    const int* q_index = nullptr;          // ... indices into q_source (packed xyz)
    const float* q_source = nullptr;
    long long nq = 0;                      // host count, or
    const unsigned long long* nq_dev = nullptr;  // device count (clamped to nq)
    const int* nq_dev_i32 = nullptr;       // device count as int (clamped to nq)
    const unsigned char* exclude = nullptr;  // skip candidates with exclude[idx] != 0
    const int* gate_count = nullptr;       // run only when *gate_count > gate_min
    int gate_min = 0;
    bool use_cells = true;                 // allow the cell-grouped search (k <= 16)
    // per query (null: none): a key above the key of its k-th nearest point
    // (squared distance bits << 32 | index), ~0 where there is none; the
    // searches start from it instead of their own bounds where it is lower
    const unsigned long long* seed = nullptr;
};

// out[j*k + i] = index of the i-th nearest; -1 when fewer than k candidates
int knn_query(const KnnIndex& ix, const KnnQuery& q, int k, int* out, cudaStream_t s);

// sub = the points of `full` with exclude[id] == 0, on the same grid (no
// host synchronisation: capturable once sub's buffers exist); indices stay
// those of full
int knn_build_subset(const KnnIndex& full, const unsigned char* exclude, KnnIndex& sub, cudaStream_t s);

}  // namespace dwg
