// DWG_CUDA -- command line front end with the reference's flags and defaults
// (src/main.cpp:17-166 of DWGTech/DWG), running the B200 pipeline.
//
//   DWG_CUDA --in_path DIR --in_name cloud.xyz --out_path DIR [flags]
//
// Output naming follows the reference: <out_path>/<name>_md_<max_depth>_gr_
// <grid_reso>_iter_<total_iter>.stl (--output_mode 1, default) and .xyz with
// normals (2), or both (3).  Extra flags: --seed (random normals of
// --in_normal 0), --precision (0 FP32, 1 FP32 compensated, 2 accurate terms),
// --use_graph (0/1).  --com_As 1 computes PCA normals and point areas on the
// GPU (the reference's PCL NormalEstimation and CGAL point_areas).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "dwg_turbo.hpp"

static void help() {
    const char* lines[][2] = {
        {"--in_path", "The absolute path of the input point cloud"},
        {"--in_name", "The file name of the input point cloud (only supports .xyz currently)"},
        {"--out_path", "The absolute path of the output mesh/point cloud with normals"},
        {"--output_mode", "Output mode: 1 Mesh(.stl) (default)   2 Point cloud with normals(.xyz)   3 Both 1 and 2"},
        {"--in_normal", "Initialization mode: 0 Random   1 Input   2 Random leaves (--com_As 1)   3 Gauss map (default)"},
        {"--lambda", "Screening Coefficient"},
        {"--max_depth", "The max depth of octree"},
        {"--use_radii", "Turn on screening mode or not (0 turn off   1 turn on)"},
        {"--kw", "The number of nearest neighbors for the iteration (default 10)"},
        {"--final_kw", "The number of nearest neighbors for the final output (default 10)"},
        {"--grid_reso", "The resolution of Marching Cubes for the iteration"},
        {"--final_reso", "The resolution of Marching Cubes for the final output"},
        {"--total_iter", "The number of iteration"},
        {"--test_iter", "Output the result each [test_iter] iterations (off by default)"},
        {"--com_As", "Computing area weight or not (0 or 1)"},
        {"--use_leaves_generate", "Mesh from the octree leaves (0 turn off   1 turn on)"},
        {"--seed", "Seed of the random initial normals (--in_normal 0)"},
        {"--precision", "0 FP32, 1 FP32 compensated (default), 2 accurate terms"},
    };
    for (auto& l : lines) printf("%s   %s\n", l[0], l[1]);
}

int main(int argc, char** argv) {
    if (argc < 2 || std::strcmp(argv[1], "--help") == 0) {
        help();
        return argc < 2 ? 1 : 0;
    }
    std::string in_path = " ", in_name = " ", out_path = " ";
    dwg_params prm;
    dwg_params_default(&prm);
    int output_mode = 1, com_As = 0, test_iter = 999999;
    unsigned long long seed = 0;
    for (int i = 1; i + 1 < argc; i += 2) {
        const std::string k = argv[i];
        const char* v = argv[i + 1];
        if (k == "--in_path") in_path = v;
        else if (k == "--in_name") in_name = v;
        else if (k == "--out_path") out_path = v;
        else if (k == "--in_normal") prm.in_normal = std::atoi(v);
        else if (k == "--grid_reso") prm.grid_reso = std::atoi(v);
        else if (k == "--final_reso") prm.final_reso = std::atoi(v);
        else if (k == "--max_depth") prm.max_depth = std::atoi(v);
        else if (k == "--kw") prm.kw = std::atoi(v);
        else if (k == "--final_kw") prm.final_kw = std::atoi(v);
        else if (k == "--normal_kw") prm.normal_kw = std::atoi(v);
        else if (k == "--lambda") prm.lambda = (float)std::atof(v);
        else if (k == "--min_num") prm.min_num = std::atoi(v);
        else if (k == "--total_iter") prm.total_iter = std::atoi(v);
        else if (k == "--output_mode") output_mode = std::atoi(v);
        else if (k == "--use_leaves_generate") prm.use_leaves_generate = std::atoi(v);
        else if (k == "--use_radii") prm.use_radii = std::atoi(v);
        else if (k == "--com_As") com_As = prm.com_as = std::atoi(v);
        else if (k == "--As_thres") prm.as_thres = (float)std::atof(v);
        else if (k == "--offset_1") prm.offset_1 = (float)std::atof(v);
        else if (k == "--offset_2") prm.offset_2 = (float)std::atof(v);
        else if (k == "--test_iter") test_iter = std::atoi(v);
        else if (k == "--seed") seed = std::strtoull(v, nullptr, 10);
        else if (k == "--precision") prm.precision = std::atoi(v);
        else if (k == "--use_graph") prm.use_graph = std::atoi(v);
        else {
            fprintf(stderr, "unknown flag %s\n", k.c_str());
            return 2;
        }
    }
    if (com_As != 0 && com_As != 1) {
        fprintf(stderr, "--com_As should be 0 or 1\n");  // include/DWGProcess.h:801-806
        return 2;
    }
    if (test_iter != 999999) fprintf(stderr, "note: --test_iter intermediate meshes are not written\n");
    const std::string full = in_path + "/" + in_name;
    const std::string pure = in_name.size() > 4 ? in_name.substr(0, in_name.size() - 4) : in_name;
    const std::string out_full = out_path + "/" + pure + "_md_" + std::to_string(prm.max_depth) + "_gr_" +
                                 std::to_string(prm.grid_reso) + "_iter_" + std::to_string(prm.total_iter);
    try {
        float *P = nullptr, *N = nullptr;
        int n = 0;
        dwg::check(dwg_read_xyz(full.c_str(), 1, &P, &N, &n));
        std::vector<float> normals(N, N + (size_t)n * 3);
        if (prm.in_normal == 0 || (prm.in_normal == 2 && !prm.com_as)) {
            // GetRandomNs (include/DWGProcess.h:264-281), seeded
            std::mt19937_64 gen(seed);
            std::uniform_real_distribution<double> dis(0.0, 2.0 * M_PI);
            for (int i = 0; i < n; ++i) {
                double u = dis(gen), v = dis(gen);
                normals[(size_t)i * 3] = (float)(std::sin(u) * std::cos(v));
                normals[(size_t)i * 3 + 1] = (float)(std::sin(u) * std::sin(v));
                normals[(size_t)i * 3 + 2] = (float)std::cos(u);
            }
        }
        auto t0 = std::chrono::high_resolution_clock::now();
        float *dP = nullptr, *dN = nullptr;
        if (cudaMalloc(&dP, sizeof(float) * 3 * n) != cudaSuccess || cudaMalloc(&dN, sizeof(float) * 3 * n) != cudaSuccess)
            throw dwg::Error(DWG_ERR_NOMEM, "cudaMalloc failed");
        cudaMemcpy(dP, P, sizeof(float) * 3 * n, cudaMemcpyHostToDevice);
        cudaMemcpy(dN, normals.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice);
        {
            dwg::TurboDWG dwg(dP, prm.in_normal == 3 ? nullptr : dN, n, prm);
            dwg.TurboScreenedDWGLaunch(prm.total_iter);
            dwg.GenerateMesh();
            long long T = dwg.size("triangles");
            printf("Num triangles: %lld\n", T);
            if (output_mode == 1 || output_mode == 3) {
                void* tris = nullptr;
                dwg::check(dwg_pipeline_device_ptr(dwg.handle(), "tris", &tris));
                dwg::check(dwg_write_stl_device((out_full + ".stl").c_str(), (const float*)tris, T, nullptr));
                printf("Mesh saved to %s.stl (%lld triangle(s)).\n", out_full.c_str(), T);
            }
            if ((output_mode == 2 || output_mode == 3) && !prm.use_leaves_generate) {
                auto pn = dwg.get<float>("point_nrm", (size_t)n * 3);
                dwg::check(dwg_write_xyz((out_full + ".xyz").c_str(), P, pn.data(), n));
            }
        }
        auto t1 = std::chrono::high_resolution_clock::now();
        printf("Total Time (Wall time) = %.3f s\n", std::chrono::duration<double>(t1 - t0).count());
        cudaFree(dP);
        cudaFree(dN);
        dwg_free_host(P);
        dwg_free_host(N);
    } catch (const dwg::Error& e) {
        fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
