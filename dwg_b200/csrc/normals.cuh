// normals.cuh -- normal initialisation, diffusion and repair kernels.
#pragma once

#include "common.cuh"
#include "knn.cuh"

namespace dwg {

int gauss_map(const float* P, int n, float* normals, cudaStream_t s);

// tri -> k nearest points scatter into 2^-40 fixed-point accumulators (acc,
// 3*L int64, must be zero on entry), then normalise; acc is cleared again on
// exit.  The triangle count is min(num_tris, *num_tris_dev) when num_tris_dev
// is given.
int diffuse_normals(const int* knn, const float* tri_normals, long long num_tris,
                    const unsigned long long* num_tris_dev, int k, int L, float* normals,
                    long long* acc, unsigned char* is_zero, int* zero_count, cudaStream_t s);
// the two halves of diffuse_normals: the scatter into acc, and the
// normalisation that reads and clears it; between them the accumulators of
// several ranks can be summed (integers: the sum is exact in any order)
int diffuse_scatter(const int* knn, const float* tri_normals, long long num_tris,
                    const unsigned long long* num_tris_dev, int k, int L, long long* acc, cudaStream_t s);
int diffuse_finish(int L, float* normals, long long* acc, unsigned char* is_zero, int* zero_count, cudaStream_t s);

struct ZeroRepairWs {
    KnnIndex sub;  // the unflagged points, rebuilt per call
    DevBuf<int> list;
    DevBuf<int> count;
    DevBuf<int> nb;
    DevBuf<unsigned char> scratch;
    // per point, its k neighbours of the last call that queried it (-1:
    // none), and per query of this call the key they bound its k-th nearest by
    DevBuf<int> prev;
    DevBuf<unsigned long long> seed;
    int prev_k = 0;
};
int zero_repair(const KnnIndex& ix, const float* positions, int L, float* normals, const unsigned char* is_zero,
                int k, int min_zero, ZeroRepairWs& ws, cudaStream_t s);

// OutlierFilter + AsFiltertoZero (src/TurboDWG.cu:991-1009, :442-454): the
// ceil(n * thr) largest areas are divided by 1000; equal areas are taken in
// index order (a stable descending sort)
int outlier_filter(float* areas, int n, float thr, cudaStream_t s);

int load_normals(const int* knn, int k, long long nq, const float* leaf_normals, float* out, cudaStream_t s);
int radii(const float* P, int n, const int* knn, int k, float* out, cudaStream_t s);

// Deterministic FP64 mean of x[0..n) -> *mean_dev (float).  When half_dev is
// non-null and *half_dev != 0 the value is halved (src/TurboDWG.cu:547-550).
// iso_hist (nullable) receives the value at index *iter_dev.
int mean_to_iso(const float* x, long long n, float* mean_dev, const int* half_dev, float* iso_hist,
                const int* iter_dev, DevBuf<double>& partial, cudaStream_t s);

}  // namespace dwg
