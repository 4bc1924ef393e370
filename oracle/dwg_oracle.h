/*
 * dwg_oracle.h -- CPU restatement of the DWG reconstruction hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * is compared against: tests, the smoke check and the CPU-baseline leg of the
 * benchmark may load it; the product (dwg_b200) never does.
 *
 * Every function restates one step of the reference (DWGTech/DWG) and cites the
 * file:line it follows.  Sums are carried in FP64; the discrete decisions that
 * the GPU makes in FP32 (Barnes-Hut opening test, kNN distance keys, marching
 * cubes interpolation) are evaluated here with the same IEEE single-precision
 * operations in the same order, so that both sides take identical decisions.
 *
 * Parity pins: the marching-cubes polygon loops and per-case triangle counts
 * are checked against a fixture derived from the reference's own table
 * (tests/golden/mc_reference_loops.json).  The reference ships no tests or
 * golden vectors for the sums, so the GWN sums are pinned by analytic
 * known answers (closed-sphere winding number, exact all-pairs vs Barnes-Hut).
 */
#ifndef DWG_ORACLE_H
#define DWG_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- octree (igl::octreeDWG, deps/libigl/include/igl/octree.cpp:171-335) ---- */
typedef struct dwgo_octree dwgo_octree;
dwgo_octree* dwgo_octree_build(const double* P, int n, int max_depth);
void dwgo_octree_free(dwgo_octree* t);
int dwgo_octree_num_nodes(const dwgo_octree* t);
/* children [M*8] (-1 = leaf), centers [M*3], widths [M], counts [M], depth [M] */
void dwgo_octree_export(const dwgo_octree* t, int* children, double* centers,
                        double* widths, int* counts, int* depth);
/* concatenated point lists in node order; list_off [M+1] */
void dwgo_octree_lists(const dwgo_octree* t, long long* list_off, int* lists);
/* Morton order (depth-first leaf order, stable): perm[i] = input index of the
 * i-th point in that order. */
void dwgo_octree_dfs_order(const dwgo_octree* t, int* perm);
/* position in that order of the first point of every node (empty nodes:
 * where their points would start) */
void dwgo_octree_dfs_starts(const dwgo_octree* t, int* start);

/* ---- moments (igl::fast_winding_number precompute, order 0,
 *      deps/libigl/include/igl/fast_winding_number.cpp:9-120) ---- */
void dwgo_moments(const dwgo_octree* t, const float* P, const float* N,
                  const float* A, double* CM, double* R, double* EC);

/* ---- generalised winding number, Barnes-Hut (src/TurboLibiGWN.cu:328-836) ---- */
void dwgo_gwn_bh(const dwgo_octree* t, const float* P, const float* N,
                 const float* A, const float* radii, const double* CM,
                 const double* R, const double* EC, const float* Q, long long nq,
                 float beta, float sigma, int screened, int use_radii,
                 float screen, int nthreads, double* out, long long* terms);
/* the same sums and their analytic gradients with respect to the query
 * (grad_out: nq x 3), same decisions; order-0 far field */
void dwgo_gwn_bh_grad(const dwgo_octree* t, const float* P, const float* N,
                      const float* A, const float* radii, const double* CM,
                      const double* R, const double* EC, const float* Q, long long nq,
                      float beta, float sigma, int screened, int use_radii,
                      float screen, int nthreads, double* out, double* grad_out);
/* igl::fast_winding_number's expansion coefficients of orders 1 and 2
 * (deps/libigl/include/igl/fast_winding_number.cpp:87-105), 36 per node:
 * m1[u + 3v] = sum A a_u n_v, m2[9i + u + 3v] = sum 0.5 a_i A a_u n_v with
 * a = p - CM, summed directly over each node's points */
void dwgo_expansion(const dwgo_octree* t, const float* P, const float* N, const float* A,
                    const double* CM, double* HO);
/* plain Barnes-Hut sum with far-field expansions of the given order (0-2):
 * the DWG traversal and opening test, far internal nodes evaluated by
 * expansion_eval (fast_winding_number.cpp:187-241) */
void dwgo_fwn(const dwgo_octree* t, const float* P, const float* N, const float* A,
              const double* CM, const double* R, const double* EC, const double* HO, int order,
              const float* Q, long long nq, float beta, int nthreads, double* out, long long* terms);
/* exact all-pairs sum of the same kernel (no far field) */
void dwgo_gwn_exact(const float* P, const float* N, const float* A,
                    const float* radii, int n, const float* Q, long long nq,
                    float sigma, int screened, int use_radii, float screen,
                    int nthreads, double* out);

/* ---- voxel grid (igl::voxel_grid, deps/libigl/include/igl/voxel_grid.cpp:11-87) ---- */
void dwgo_voxel_grid(const float* P, int n, float offset, int s, int res[3],
                     float origin[3], float* spacing);
void dwgo_grid_points(const int res[3], const float origin[3], float spacing,
                      float* out);

/* ---- marching cubes (src/TurboMC.cu:373-478) ---- */
/* the reference's triangles per case (256 x 16 edge indices, -1 padded); must
 * be set before any marching-cubes call */
void dwgo_mc_set_triangles(const signed char* tri_table);
/* edge masks and the set triangles */
void dwgo_mc_tables(int* edge_table, signed char* tri_table);
/* edge masks and the polygons of the cube geometry, fanned from their lowest
 * edge (tri_table may be NULL) */
void dwgo_mc_polygons(int* edge_table, signed char* tri_table);
long long dwgo_marching_cubes(const float* field, const int res[3],
                              const float origin[3], float spacing, float iso,
                              float* tris, float* centroids, float* normals,
                              long long cap, unsigned char* cases);

/* ---- kNN (cukd FixedCandidateList order, include/cudaKDTree/cukd/knn.h) ---- */
void dwgo_knn(const float* P, int n, const float* Q, long long nq, int k,
              int nthreads, int* out);

/* ---- normal diffusion (src/TurboDWG.cu:134-266,322-359) ---- */
int dwgo_diffuse_normals(const int* knn, const float* tri_normals,
                         long long T, int k, int L, float* normals,
                         unsigned char* is_zero);
void dwgo_zero_repair(const float* Lpos, int L, float* normals,
                      const unsigned char* is_zero, int k, int nthreads);
void dwgo_gauss_map(const float* P, int n, float* normals);
void dwgo_load_normals(const int* knn, int k, long long nq,
                       const float* leaf_normals, float* out);
void dwgo_radii(const float* P, int n, const int* knn, int k, float* radii);

/* NormalEstimation (include/DWGProcess.h:152-200, PCL): the eigenvector of
 * the smallest eigenvalue of the covariance of the k neighbours (knn, self
 * included), flipped towards `view`; eigenvectors by cyclic Jacobi
 * rotations in FP64 */
void dwgo_pca_normals(const float* P, int n, const int* knn, int k, const float view[3], float* normals);
/* igl::copyleft::cgal::point_areas (deps/libigl/include/igl/copyleft/cgal/
 * point_areas.cpp:39-210) with the 2-D Delaunay triangulation restated by
 * its definition (a triangle is Delaunay when no other point lies inside
 * its circumcircle); knn rows start with the point itself */
void dwgo_point_areas(const float* P, int n, const int* knn, int k, const float* normals, float* areas);
/* seeded stand-in for the reference's unseeded random leaf normals of the
 * --com_As 1 --in_normal 2 start (include/DWGProcess.h:643-657) */
void dwgo_random_normals(int n, float* normals);

/* ---- full reconstruction (include/DWGProcess.h:474-797 + src/TurboDWG.cu:456-924) ---- */
typedef struct {
    int in_normal;       /* 0 random(seeded, given as input), 1 input, 2 random leaves
                            (com_as 1), 3 Gauss map */
    int grid_reso, final_reso, kw, final_kw, normal_kw, max_depth;
    float lambda;        /* --lambda (sigma) */
    int min_num, use_radii;
    float offset_1, offset_2;
    int use_leaves_generate, total_iter;
    float beta, area, screen;
    int knn_tri;         /* 15 */
    int knn_zero;        /* 10 */
    float as_thres;      /* --As_thres (0) */
    int com_as;          /* --com_As (0) */
} dwgo_params;

/* OutlierFilter + AsFiltertoZero (src/TurboDWG.cu:991-1009, :442-454): the
 * ceil(n * thr) largest areas divided by 1000, equal areas in index order */
void dwgo_outlier_filter(float* A, int n, float thr);

typedef struct dwgo_run dwgo_run;
dwgo_run* dwgo_reconstruct(const float* P, int n, const float* N_in,
                           const dwgo_params* prm, int nthreads);
void dwgo_run_free(dwgo_run* r);
/* sizes: 0 leaves, 1 final points, 2 final triangles, 3 iterations,
 *        4..6 final grid res, 7..9 iteration grid res */
long long dwgo_run_size(const dwgo_run* r, int what);
/* arrays: "leaf_pos", "leaf_nrm", "point_nrm", "tris", "iso", "tri_count",
 *         "final_field", "zero_count" */
int dwgo_run_get(const dwgo_run* r, const char* name, void* dst);

#ifdef __cplusplus
}
#endif
#endif
