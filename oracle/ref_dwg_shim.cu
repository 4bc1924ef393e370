// C entry points over the reference's own GPU code of DWGTech/DWG, compiled
// unchanged from its sources by oracle/ref_dwg.mk into oracle/_ref/libref_dwg.so:
//   TurboLibiGWN  (src/TurboLibiGWN.cu)  PreLibiGWN, UpdateMassNormals,
//                 UpdateGWNInfo, TurboLibiScreenedGWNLaunch, TurboLibiGWNLaunch
//   TurboMC       (src/TurboMC.cu)       TurboMarchingCubes
//   TurboDWG      (src/TurboDWG.cu)      constructor, TurboScreenedDWGLaunch,
//                 GenerateMesh (the final pass on the points)
//   GenerateKDTreeForGWN (src/KNN_GWN.cu) the kd-tree order of a point set
// TEST INFRASTRUCTURE ONLY: the tests compare the product with these on the
// GPU.  Every array crosses this boundary as a HOST array; the shim copies it
// into managed memory, as the reference's own host code expects (it reads
// some of its buffers on the host, e.g. src/TurboLibiGWN.cu:906).
// The reference's CPU preparation (libigl octree, FP64 moments, voxel grid)
// needs Eigen and is supplied by the caller from the oracle's restatement.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <fcntl.h>
#include <iostream>
#include <string>
#include <unistd.h>
#include <unordered_map>
#include <vector>

#include "TurboDWG.h"

extern "C" void GenerateKDTreeForGWN(std::vector<float>& points_pos_x, std::vector<float>& points_pos_y,
                                     std::vector<float>& points_pos_z, std::vector<float>& new_points_pos_x,
                                     std::vector<float>& new_points_pos_y, std::vector<float>& new_points_pos_z,
                                     std::vector<float>& bound_upper, std::vector<float>& bound_lower,
                                     bool out_index_map,
                                     std::unordered_map<geometrycentral::Vector3, int>& points_indices_map);

namespace {

// Redirects the reference's std::cout / printf output (fd 1) into a file for
// the duration of a call, so that a caller can read the per-iteration values it
// prints (W_mean, triangle and zero counts) without changing its sources.
struct StdoutToFile {
    int saved = -1;
    explicit StdoutToFile(const char* path) {
        if (!path || !*path) return;
        std::cout.flush();
        fflush(stdout);
        int fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
        if (fd < 0) return;
        saved = dup(1);
        dup2(fd, 1);
        close(fd);
    }
    ~StdoutToFile() {
        if (saved < 0) return;
        std::cout.flush();
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};

template <typename T>
T* managed_copy(const T* host, size_t n) {
    T* p = nullptr;
    if (cudaMallocManaged((void**)&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) return nullptr;
    if (host && n) memcpy(p, host, n * sizeof(T));
    return p;
}

// The igl octree arrays (O_PI, O_CH, O_CM, O_R, O_EC) from flat host arrays.
struct IglOctree {
    std::vector<std::vector<int>> PI;
    Eigen::MatrixXi CH;
    Eigen::MatrixXd CM, EC;
    Eigen::VectorXd R;
    IglOctree(int M, const int* ch, const long long* pi_off, const int* pi_flat, const double* cm,
              const double* r, const double* ec) {
        PI.resize(M);
        CH.resize(M, 8);
        CM.resize(M, 3);
        EC.resize(M, 3);
        R.resize(M);
        for (int i = 0; i < M; i++) {
            PI[i].assign(pi_flat + pi_off[i], pi_flat + pi_off[i + 1]);
            for (int j = 0; j < 8; j++) CH(i, j) = ch[(size_t)i * 8 + j];
            for (int d = 0; d < 3; d++) {
                CM(i, d) = cm[(size_t)i * 3 + d];
                EC(i, d) = ec[(size_t)i * 3 + d];
            }
            R[i] = r[i];
        }
    }
};

Eigen::MatrixXf rows3(const float* a, int n) {
    Eigen::MatrixXf m(n, 3);
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) m(i, d) = a[(size_t)i * 3 + d];
    return m;
}

Eigen::VectorXf vec(const float* a, int n) {
    Eigen::VectorXf v(n);
    for (int i = 0; i < n; i++) v[i] = a[i];
    return v;
}

// TurboDWG keeps its device state protected; this view reads it after a run.
struct DWGView : public TurboDWG {
    using TurboDWG::TurboDWG;
    float3* normals() { return m_Normals_GPU; }
    float3* points() { return m_Point_Cloud_GPU; }
    int size() { return m_Point_Cloud_size; }
};

struct GwnHandle {
    TurboLibiGWN gwn;
    float3* pc = nullptr;  // managed copy of the octree's points
    int n = 0;
};

}  // namespace

extern "C" {

// Kd-tree order of a point set by the reference's builder (GenerateKDTreeForGWN,
// src/KNN_GWN.cu:68-140): out_xyz = the reordered points, perm[i] = the input
// index of out_xyz[i] (the reference's position -> index map), bounds =
// lower xyz then upper xyz.  Returns 0, or -1 if a position was duplicated.
int refdwg_kd_sort(const float* xyz, int n, float* out_xyz, int* perm, float* bounds) {
    std::vector<float> x(n), y(n), z(n), nx(n), ny(n), nz(n), up(3), lo(3);
    for (int i = 0; i < n; i++) {
        x[i] = xyz[(size_t)i * 3];
        y[i] = xyz[(size_t)i * 3 + 1];
        z[i] = xyz[(size_t)i * 3 + 2];
    }
    std::unordered_map<geometrycentral::Vector3, int> map;
    {
        StdoutToFile quiet("/dev/null");
        GenerateKDTreeForGWN(x, y, z, nx, ny, nz, up, lo, true, map);
    }
    if ((int)map.size() != n) return -1;
    for (int i = 0; i < n; i++) {
        out_xyz[(size_t)i * 3] = nx[i];
        out_xyz[(size_t)i * 3 + 1] = ny[i];
        out_xyz[(size_t)i * 3 + 2] = nz[i];
        geometrycentral::Vector3 c;
        c.x = nx[i];
        c.y = ny[i];
        c.z = nz[i];
        perm[i] = map[c];
    }
    for (int d = 0; d < 3; d++) {
        bounds[d] = lo[d];
        bounds[3 + d] = up[d];
    }
    return (int)cudaGetLastError();
}

// TurboLibiGWN::PreLibiGWN (src/TurboLibiGWN.cu:132-231) on an igl octree of
// the points P (n x 3): children M x 8 (-1 = none), per-node point lists
// (pi_off[M+1], pi_flat), FP64 centres of mass, radii and Σ A n.
void* refgwn_create(const float* P, int n, int M, const int* ch, const long long* pi_off, const int* pi_flat,
                    const double* cm, const double* r, const double* ec) {
    auto* h = new GwnHandle();
    IglOctree t(M, ch, pi_off, pi_flat, cm, r, ec);
    h->gwn.PreLibiGWN(t.PI, t.CH, t.CM, t.R, t.EC);
    h->pc = managed_copy(reinterpret_cast<const float3*>(P), (size_t)n);
    h->n = n;
    cudaDeviceSynchronize();
    return h;
}

void refgwn_free(void* hv) {
    auto* h = static_cast<GwnHandle*>(hv);
    if (!h) return;
    h->gwn.EarseMemory();
    cudaFree(h->pc);
    delete h;
}

// UpdateMassNormals (src/TurboLibiGWN.cu:1039-1046), or with info != 0
// UpdateGWNInfo (:1048-1055), then the screened (screened != 0,
// TurboLibiScreenedGWNLaunch :912-922) or plain (TurboLibiGWNLaunch :898-910)
// sums at the nq queries Q; out = nq floats.
int refgwn_eval(void* hv, const float* N, const float* A, const float* radii, int info, const float* Q, int nq,
                int screened, float beta, float sigma, int use_radii, float* out) {
    auto* h = static_cast<GwnHandle*>(hv);
    float3* Nd = managed_copy(reinterpret_cast<const float3*>(N), (size_t)h->n);
    float* Ad = managed_copy(A, (size_t)h->n);
    float* Rd = managed_copy(radii, (size_t)h->n);
    float3* Qd = managed_copy(reinterpret_cast<const float3*>(Q), (size_t)nq);
    // the plain launcher prints out_gwn[666] from the host
    float* Od = managed_copy<float>(nullptr, (size_t)(nq > 667 ? nq : 667));
    if (!Nd || !Ad || !Rd || !Qd || !Od) return -1;
    {
        StdoutToFile quiet("/dev/null");
        if (info) h->gwn.UpdateGWNInfo(Nd, h->pc, Ad);
        else h->gwn.UpdateMassNormals(Nd, Ad);
        if (screened)
            h->gwn.TurboLibiScreenedGWNLaunch(Qd, h->pc, nq, Nd, Ad, Rd, beta, sigma, Od, use_radii != 0);
        else
            h->gwn.TurboLibiGWNLaunch(Qd, h->pc, nq, Nd, Ad, beta, Od);
    }
    cudaDeviceSynchronize();
    memcpy(out, Od, (size_t)nq * sizeof(float));
    cudaFree(Nd);
    cudaFree(Ad);
    cudaFree(Rd);
    cudaFree(Qd);
    cudaFree(Od);
    return (int)cudaGetLastError();
}

// TurboMC::TurboMarchingCubes (src/TurboMC.cu:572-638) on a field of rx*ry*rz
// values (x fastest) with per-sample positions; writes the triangles'
// centroids and normals (capacity max(R^3/2, 1e6) each, as the reference's
// callers allocate) and returns the triangle count.  With stl_base set, the
// reference also writes its triangles to <stl_base>.stl (the final-mesh mode,
// iterations == 123456); otherwise no file is written.
long long refmc_run(const float* values, const float* poses, int rx, int ry, int rz, float iso, float* centroids,
                    float* normals, long long cap, const char* stl_base) {
    const size_t G = (size_t)rx * ry * rz;
    long long buf = std::max<long long>((long long)G / 2, 1000000);
    float* Vd = managed_copy(values, G);
    float3* Pd = managed_copy(reinterpret_cast<const float3*>(poses), G);
    float3* Cd = managed_copy<float3>(nullptr, (size_t)buf);
    float3* Nd = managed_copy<float3>(nullptr, (size_t)buf);
    if (!Vd || !Pd || !Cd || !Nd) return -1;
    int T;
    {
        StdoutToFile quiet("/dev/null");
        TurboMC mc;
        const bool stl = stl_base && *stl_base;
        T = mc.TurboMarchingCubes(Vd, Pd, rx, ry, rz, iso, stl ? 123456 : 0, "nothing", stl ? stl_base : "nothing",
                                  Cd, Nd, 999999);
    }
    cudaDeviceSynchronize();
    const long long m = std::min<long long>(T, cap);
    memcpy(centroids, Cd, (size_t)m * sizeof(float3));
    memcpy(normals, Nd, (size_t)m * sizeof(float3));
    cudaFree(Vd);
    cudaFree(Pd);
    cudaFree(Cd);
    cudaFree(Nd);
    return cudaGetLastError() == cudaSuccess ? (long long)T : -1;
}

// The reference's DWG run (include/DWGProcess.h:651-689 from TurboDWG's
// constructor on): leaves (L x 3, in kd-tree order) with their normals, areas
// and radii, the iteration grid (G x 3 positions, res), the leaves' kd bounds
// (lower, upper), the igl octree of the leaves; TurboScreenedDWGLaunch with
// beta 2.3 (src/TurboDWG.cu:456-672); then GenerateMesh on the points
// (src/TurboDWG.cu:808-924, output mode 3): points (N x 3, kd order), their
// areas, the final grid, the igl octree of the points, the points' kd bounds.
// Writes <mesh_base>.stl and <mesh_base>.xyz, the reference's printed output to
// log_path, the leaf normals after the iterations to leaf_normals_out (L x 3)
// and the device seconds of the iterations and of the final pass to secs[2].
int refdwg_run(int L, const float* leaves, const float* leaf_normals, const float* leaf_areas,
               const float* leaf_radii, int G, const float* grid, const int* res, const float* leaf_bounds,
               int M2, const int* ch2, const long long* pi_off2, const int* pi_flat2, const double* cm2,
               const double* r2, const double* ec2, float sigma, int total_iter, int use_radii, float as_thres,
               int in_normal, int N, const float* points, const float* point_areas, int G2, const float* grid2,
               const int* res2, const float* point_bounds, int M1, const int* ch1, const long long* pi_off1,
               const int* pi_flat1, const double* cm1, const double* r1, const double* ec1, int final_kw,
               int normal_kw, const char* mesh_base, const char* log_path, float* leaf_normals_out, double* secs) {
    StdoutToFile redirect(log_path);
    Eigen::MatrixXf Lf = rows3(leaves, L), LNf = rows3(leaf_normals, L), Gf = rows3(grid, G);
    Eigen::VectorXf LAf = vec(leaf_areas, L), LRf = vec(leaf_radii, L);
    std::vector<float> lup = {leaf_bounds[3], leaf_bounds[4], leaf_bounds[5]};
    std::vector<float> llo = {leaf_bounds[0], leaf_bounds[1], leaf_bounds[2]};
    IglOctree t2(M2, ch2, pi_off2, pi_flat2, cm2, r2, ec2);
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    DWGView dwg(Lf, LNf, LAf, LRf, Gf, res[0], res[1], res[2], lup, llo);
    cudaDeviceSynchronize();
    cudaEventRecord(e0);
    dwg.TurboScreenedDWGLaunch(t2.PI, t2.CH, t2.CM, t2.R, t2.EC, 2.3f, sigma, total_iter, use_radii != 0, as_thres,
                               in_normal, clock(), "nothing", 999999);
    cudaEventRecord(e1);
    cudaDeviceSynchronize();
    memcpy(leaf_normals_out, dwg.normals(), (size_t)L * sizeof(float3));
    Eigen::MatrixXf Pf = rows3(points, N), G2f = rows3(grid2, G2);
    Eigen::VectorXf PAf = vec(point_areas, N);
    std::vector<float> pup = {point_bounds[3], point_bounds[4], point_bounds[5]};
    std::vector<float> plo = {point_bounds[0], point_bounds[1], point_bounds[2]};
    IglOctree t1(M1, ch1, pi_off1, pi_flat1, cm1, r1, ec1);
    dwg.GenerateMesh(Pf, PAf, G2f, t1.PI, t1.CH, t1.CM, t1.R, t1.EC, res2[0], res2[1], res2[2], pup, plo, 2.3f,
                     sigma, final_kw, normal_kw, use_radii != 0, as_thres, mesh_base, 0, clock(), 3);
    cudaEventRecord(e2);
    cudaDeviceSynchronize();
    float ms01 = 0, ms12 = 0;
    cudaEventElapsedTime(&ms01, e0, e1);
    cudaEventElapsedTime(&ms12, e1, e2);
    secs[0] = ms01 * 1e-3;
    secs[1] = ms12 * 1e-3;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    return (int)cudaGetLastError();
}
}
