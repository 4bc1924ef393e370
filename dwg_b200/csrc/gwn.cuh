// gwn.cuh -- generalised winding number sums over the octree.
#pragma once

#include "octree.cuh"

namespace dwg {

struct GwnQuery {
    // point queries (packed xyz) ...
    const float* q = nullptr;
    long long nq = 0;
    // ... or a regular grid (q == nullptr)
    int res[3] = {0, 0, 0};
    float origin[3] = {0, 0, 0};
    float spacing = 0;
};

// out[i] = w(q_i); terms_total (nullable) += number of evaluated terms;
// per_query_terms (nullable) receives the count per query.
// sigma_dev (nullable) overrides p.sigma with a device value (graph replay).
int gwn_eval(const Octree& t, const GwnQuery& q, const dwg_gwn_params& p, float* out,
             unsigned long long* terms_total, int* per_query_terms, cudaStream_t s,
             const float* sigma_dev = nullptr);

}  // namespace dwg
