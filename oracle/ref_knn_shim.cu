// C entry points over the reference's GPU kNN (src/KNN_GWN.cu of DWGTech/DWG,
// cudaKDTree builder + cct kNN), compiled from the reference sources by
// oracle/ref_knn.mk into oracle/_ref/libref_knn.so.  TEST INFRASTRUCTURE ONLY:
// the tests compare the product's kNN with the reference's on the GPU.
#include <cuda_runtime.h>

// declared in the reference (include/TurboDWG.h:14-27)
void GenerateKDTreeForDWG(float3* d_points, float3* d_normals, int points_size, float3* bound_upper,
                          float3* bound_lower);
void CudaKNNWithKDTreeforDWG(float3* d_points, int numPoints, float3* d_queries, int numQueries,
                             float3* bound_upper, float3* bound_lower, int* d_results, int k);

extern "C" {

// Builds the reference kd-tree in place on points_dev (n float3, reordered),
// normals_dev is co-permuted; bounds (6 floats, lower then upper) to bounds_host.
int refknn_build(float* points_dev, float* normals_dev, int n, float* bounds_host) {
    float3 *up = nullptr, *lo = nullptr;
    if (cudaMallocManaged(&up, sizeof(float3)) != cudaSuccess) return -1;
    if (cudaMallocManaged(&lo, sizeof(float3)) != cudaSuccess) return -1;
    GenerateKDTreeForDWG((float3*)points_dev, (float3*)normals_dev, n, up, lo);
    cudaDeviceSynchronize();
    bounds_host[0] = lo->x; bounds_host[1] = lo->y; bounds_host[2] = lo->z;
    bounds_host[3] = up->x; bounds_host[4] = up->y; bounds_host[5] = up->z;
    cudaFree(up);
    cudaFree(lo);
    return (int)cudaGetLastError();
}

// k nearest (indices into the reordered tree array) of queries_dev.
int refknn_query(float* tree_dev, int n, float* queries_dev, int nq, const float* bounds_host, int* out_dev, int k) {
    float3 *up = nullptr, *lo = nullptr;
    if (cudaMallocManaged(&up, sizeof(float3)) != cudaSuccess) return -1;
    if (cudaMallocManaged(&lo, sizeof(float3)) != cudaSuccess) return -1;
    *lo = make_float3(bounds_host[0], bounds_host[1], bounds_host[2]);
    *up = make_float3(bounds_host[3], bounds_host[4], bounds_host[5]);
    CudaKNNWithKDTreeforDWG((float3*)tree_dev, n, (float3*)queries_dev, nq, up, lo, out_dev, k);
    cudaDeviceSynchronize();
    cudaFree(up);
    cudaFree(lo);
    return (int)cudaGetLastError();
}
}
