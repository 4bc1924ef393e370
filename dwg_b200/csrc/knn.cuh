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
    // query bucketing workspace (grown on demand; not thread safe)
    int morton_shift = 0;
    mutable DevBuf<int> q_key, q_order, q_hist, q_fill;
    mutable DevBuf<unsigned char> q_scratch;
};

int knn_build(KnnIndex& ix, const float* points_dev, int n, cudaStream_t s);

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
};

// out[j*k + i] = index of the i-th nearest; -1 when fewer than k candidates
int knn_query(const KnnIndex& ix, const KnnQuery& q, int k, int* out, cudaStream_t s);

}  // namespace dwg
