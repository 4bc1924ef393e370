// dwg_turbo.hpp -- C++ mirror of the reference's operator classes over the C ABI.
//
// Class and method names follow DWGTech/DWG so that code written against
// include/TurboNormalInit.h, include/Turbo_GWN_l.h, include/MarchingCubeCuda.h
// and include/TurboDWG.h ports by renaming types:
//   * Eigen matrices become float device arrays (n x 3, row-major) and the CPU
//     octree arguments (O_PI, O_CH, O_CM, O_R, O_EC) become a GPU octree built
//     from the points;
//   * pointers are device pointers from cudaMalloc (the reference uses
//     cudaMallocManaged and reads them on the host);
//   * errors throw dwg::Error (the reference exit()s on CUDA errors,
//     src/TurboDWG.cu:3-12) -- the C ABI underneath returns status codes.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "dwg_b200.h"

namespace dwg {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != DWG_OK) throw Error(rc, std::string("dwg_b200: ") + dwg_last_error());
}

// include/TurboNormalInit.h:9-14
class TurboNormalInitialization {
   public:
    // The bounds are those of the points; the reference passes its kd-tree
    // bounds (the same box), here they are computed on the device.
    void GaussMapInit(const float* point_pos, float* point_normal, int point_num, void* stream = nullptr) {
        check(dwg_gauss_map_init(point_pos, point_num, point_normal, stream));
    }
};

// include/Turbo_GWN_l.h:24-69
class TurboLibiGWN {
   public:
    TurboLibiGWN() = default;
    TurboLibiGWN(const float* point_cloud, int n, int max_depth = 10, const float* areas = nullptr,
                 void* stream = nullptr) {
        PreLibiGWN(point_cloud, n, max_depth, areas, stream);
    }
    TurboLibiGWN(const TurboLibiGWN&) = delete;
    TurboLibiGWN& operator=(const TurboLibiGWN&) = delete;
    ~TurboLibiGWN() { EarseMemory(); }

    void PreLibiGWN(const float* point_cloud, int n, int max_depth = 10, const float* areas = nullptr,
                    void* stream = nullptr) {
        EarseMemory();
        check(dwg_octree_build(point_cloud, n, max_depth, areas, stream, &tree_));
    }
    void UpdateMassNormals(const float* i_Normals, const float* i_As, void* stream = nullptr) {
        check(dwg_octree_update_normals(tree_, i_Normals, i_As, stream));
    }
    void UpdateGWNInfo(const float* i_Normals, const float* i_As, void* stream = nullptr) {
        check(dwg_octree_update_info(tree_, i_Normals, i_As, stream));
    }
    // plain GWN (src/TurboLibiGWN.cu:899-910); expansion_order 1 or 2 adds
    // igl::fast_winding_number's far-field terms
    void TurboLibiGWNLaunch(const float* query_points, int query_size, float beta, float* out_gwn,
                            void* stream = nullptr, int expansion_order = 0) {
        dwg_gwn_params p{beta, 0.f, 0.0015f, 0, 0, 1, 0, expansion_order};
        check(dwg_gwn_points(tree_, nullptr, nullptr, nullptr, query_points, query_size, &p, out_gwn, nullptr,
                             stream));
    }
    // screened GWN (src/TurboLibiGWN.cu:912-922)
    void TurboLibiScreenedGWNLaunch(const float* query_points, int query_size, const float* i_radii, float beta,
                                    float sigma, float* out_gwn, bool use_radii, void* stream = nullptr) {
        dwg_gwn_params p{beta, sigma, 0.0015f, 1, use_radii ? 1 : 0, 1};
        check(dwg_gwn_points(tree_, nullptr, nullptr, use_radii ? i_radii : nullptr, query_points, query_size, &p,
                             out_gwn, nullptr, stream));
    }
    void EarseMemory() {
        if (tree_) dwg_octree_destroy(tree_);
        tree_ = nullptr;
    }
    dwg_octree* handle() const { return tree_; }

   private:
    dwg_octree* tree_ = nullptr;
};

// include/MarchingCubeCuda.h:35-44; returns the triangle count.  Writes a
// binary STL when iterations == 123456 (mesh_full_path + ".stl") or when
// test_iter != 999999 and iterations % test_iter == 0, like the reference.
class TurboMC {
   public:
    int TurboMarchingCubes(const float* voxel_values, const float* voxel_poses, int res_x, int res_y, int res_z,
                           float threshold, int iterations, const std::string& mesh_path,
                           const std::string& mesh_full_path, float* mid_points, float* mid_normals,
                           int test_iter = 999999, void* stream = nullptr, const float* origin = nullptr,
                           float spacing = 0.f) {
        const int res[3] = {res_x, res_y, res_z};
        long long cap = (long long)res_x * res_y * res_z / 2;
        if (cap < 1000000) cap = 1000000;
        const bool stl = (test_iter != 999999 && iterations % test_iter == 0) || iterations == 123456;
        float* tris = nullptr;
        if (stl && cudaMalloc_(&tris, cap * 9 * sizeof(float)) != 0) throw Error(DWG_ERR_NOMEM, "cudaMalloc failed");
        long long T = 0;
        int rc = dwg_marching_cubes(voxel_values, res, voxel_poses, origin, spacing, threshold, tris, mid_points,
                                    mid_normals, cap, nullptr, &T, stream);
        if (rc == DWG_OK && stl) {
            std::string path = iterations == 123456 ? mesh_full_path + ".stl"
                                                    : mesh_path + std::to_string(iterations) + "iter.stl";
            rc = dwg_write_stl_device(path.c_str(), tris, T, stream);
        }
        if (tris) cudaFree_(tris);
        check(rc);
        return (int)T;
    }

   private:
    static int cudaMalloc_(float** p, size_t bytes);
    static void cudaFree_(float* p);
};

// include/TurboDWG.h:14-27: GenerateKDTreeForDWG + CudaKNNWithKDTreeforDWG
class KnnIndex {
   public:
    KnnIndex(const float* d_points, int n, void* stream = nullptr) { check(dwg_knn_build(d_points, n, stream, &ix_)); }
    KnnIndex(const KnnIndex&) = delete;
    KnnIndex& operator=(const KnnIndex&) = delete;
    ~KnnIndex() {
        if (ix_) dwg_knn_destroy(ix_);
    }
    void query(const float* d_queries, long long num_queries, int k, int* d_results, void* stream = nullptr) {
        check(dwg_knn_query(ix_, d_queries, num_queries, k, d_results, stream));
    }

   private:
    dwg_knn_index* ix_ = nullptr;
};

// include/TurboDWG.h:29-74: the iteration and meshing driver
class TurboDWG {
   public:
    TurboDWG(const float* d_points, const float* d_normals, int n, const dwg_params& prm, void* stream = nullptr) {
        check(dwg_pipeline_create(d_points, d_normals, n, &prm, stream, &p_));
    }
    TurboDWG(const TurboDWG&) = delete;
    TurboDWG& operator=(const TurboDWG&) = delete;
    ~TurboDWG() {
        if (p_) dwg_pipeline_destroy(p_);
    }
    void TurboScreenedDWGLaunch(int total_iters) { check(dwg_pipeline_iterate(p_, total_iters)); }
    void GenerateMesh() { check(dwg_pipeline_finalize(p_)); }
    long long size(const char* what) {
        long long v = 0;
        check(dwg_pipeline_size(p_, what, &v));
        return v;
    }
    template <typename T>
    std::vector<T> get(const char* what, size_t count) {
        std::vector<T> v(count);
        if (count) check(dwg_pipeline_get(p_, what, v.data()));
        return v;
    }
    dwg_pipeline* handle() const { return p_; }

   private:
    dwg_pipeline* p_ = nullptr;
};

}  // namespace dwg

inline int dwg::TurboMC::cudaMalloc_(float** p, size_t bytes) { return (int)::cudaMalloc((void**)p, bytes); }
inline void dwg::TurboMC::cudaFree_(float* p) { ::cudaFree(p); }
