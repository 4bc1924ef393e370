/*
 * dwg_b200.h -- C ABI of the B200-native DWG reconstruction hot path.
 *
 * Conventions
 *   - Pointers named *_dev are device pointers (cudaMalloc'd by the caller,
 *     not managed memory); *_host are host pointers.  Point arrays are packed
 *     xyz float triples (n * 3 floats).
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *     Calls enqueue work on it; results are valid once the stream has
 *     completed, unless a function says it synchronises.
 *   - Every function returns DWG_OK (0) or a negative status; the message of
 *     the last error of the calling thread is available from dwg_last_error().
 *   - Objects (octree, kNN index, pipeline) are owned by the library and freed
 *     with their *_destroy function.  A handle must not be used from two host
 *     threads at once.
 *   - The library keeps per-device state for the life of the process, keyed by
 *     the device ordinal: recycled streams, events and graph executables, one
 *     allocation stream per device, the marching-cubes tables in constant
 *     memory, kernel occupancy figures and the allocation-free scratch
 *     address.  None of it survives a cudaDeviceReset: reset a device only
 *     after the last call into the library.
 */
#ifndef DWG_B200_H
#define DWG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DWG_OK 0
#define DWG_ERR_INVALID (-1)   /* bad argument (null pointer, size, k > n ...) */
#define DWG_ERR_CUDA (-2)      /* a CUDA runtime call failed */
#define DWG_ERR_OVERFLOW (-3)  /* an output capacity was exceeded */
#define DWG_ERR_NOMEM (-4)     /* device allocation failed */
#define DWG_ERR_DEVICE (-5)    /* a kernel reported an error status */

const char* dwg_last_error(void);
/* library version string */
const char* dwg_version(void);

/* ------------------------------------------------------------------------
 * Gauss-map initial normals: n_i = (p_i - c) / (|p_i - c| + 1e-8), with c the
 * centre of the points' bounding box (computed on the device).
 * Replaces TurboNormalInitialization::GaussMapInit
 * (include/TurboNormalInit.h:13, src/TurboNormalInit.cu:29-44); the reference
 * takes the bounds from its kd-tree build instead of computing them.
 * ------------------------------------------------------------------------ */
int dwg_gauss_map_init(const float* points_dev, int n, float* normals_dev, void* stream);

/* ------------------------------------------------------------------------
 * Octree over a point set, rebuilt on the GPU.  Topology follows
 * igl::octreeDWG (deps/libigl/include/igl/octree.cpp:171-335): a cube around
 * the bounding box, a cell splits while it holds more than one point and its
 * depth is below max_depth (1..21).  The CPU octree + TurboLibiGWN::PreLibiGWN
 * flattening (src/TurboLibiGWN.cu:132-231) are replaced by this build.
 * `areas_dev` fixes the mass centres / radii (fast_winding_number.cpp:9-120,
 * computed in FP64); NULL means unit areas.
 * ------------------------------------------------------------------------ */
typedef struct dwg_octree dwg_octree;
int dwg_octree_build(const float* points_dev, int n, int max_depth, const float* areas_dev,
                     void* stream, dwg_octree** out);
int dwg_octree_destroy(dwg_octree* tree);
/* number of nodes (host query; synchronises the build stream once) */
int dwg_octree_num_nodes(const dwg_octree* tree, int* num_nodes);
/* Recompute the dipole moments sum(A_i n_i) per node, FP64.
 * Replaces TurboLibiGWN::UpdateMassNormals (src/TurboLibiGWN.cu:924-952,1044-1052). */
int dwg_octree_update_normals(dwg_octree* tree, const float* normals_dev, const float* areas_dev,
                              void* stream);
/* Recompute centres, radii and moments from new areas.
 * Replaces TurboLibiGWN::UpdateGWNInfo (src/TurboLibiGWN.cu:954-1017,1054-1062). */
int dwg_octree_update_info(dwg_octree* tree, const float* normals_dev, const float* areas_dev,
                           void* stream);
/* Sticky error word of the traversal kernels of this tree (synchronises):
 * 0 = none; bit 0 stack overflow, bit 1 malformed node links, bit 2 leaf
 * range outside the point array, bit 3 an opening threshold that failed its
 * self-check, bit 4 a bulk copy of the kept-weight reader that did not land
 * within its bounded wait.  Any set bit makes the call return DWG_ERR_DEVICE. */
int dwg_octree_status(const dwg_octree* tree, unsigned int* flags);
/* Size of the interaction list dwg_gwn_grid keeps (params->lists >= 1): its
 * entries (16 bytes each) and the weight slots it holds (8 bytes per entry
 * and lane each); 0 and 0 when none is kept.  No reference counterpart: the
 * lists are this library's own cache of the Barnes-Hut decisions. */
int dwg_octree_list_size(const dwg_octree* tree, long long* entries, int* weight_slots);
/* Copy the node table to host memory (for checking).  Arrays may be NULL.
 * Nodes are in depth-first pre-order; points are in the octree's sorted
 * order, perm_host[i] = input index of sorted point i.
 *   depth[M], pt_start[M], pt_count[M], skip[M] (index after the subtree),
 *   cm[M*3] (FP64), radius[M] (FP64), ec[M*3] (FP64), perm[n] */
int dwg_octree_export(const dwg_octree* tree, int* depth_host, int* pt_start_host,
                      int* pt_count_host, int* skip_host, double* cm_host, double* radius_host,
                      double* ec_host, int* perm_host);

/* ------------------------------------------------------------------------
 * Generalised winding number at query points, Barnes-Hut over `tree`.
 * w(q) = sum over terms of A (sigma rho + 1) ((p - q).n) / (e^{sigma rho} 4 pi rho^3 + 1e-7)
 * (screened, rho = max(|p-q|, s)), or A ((p - q).n) / (4 pi |p-q|^3 + 1e-8)
 * (plain); far nodes (|CM - q| > beta R) contribute one dipole term.
 * The opening decisions are the reference's, per query.
 * Replaces TurboLibiGWN::TurboLibiScreenedGWNLaunch / TurboLibiGWNLaunch
 * (include/Turbo_GWN_l.h:38-56, src/TurboLibiGWN.cu:814-922).
 * normals/areas/radii are indexed like the points the tree was built from.
 * ------------------------------------------------------------------------ */
typedef struct {
    float beta;      /* opening ratio, reference 2.3 */
    float sigma;     /* screening coefficient (--lambda) */
    float screen;    /* screen radius s when use_radii == 0, reference 0.0015 */
    int screened;    /* 1 screened kernel, 0 plain kernel */
    int use_radii;   /* 1: s = radii[i] for point terms (far field keeps `screen`) */
    int precision;   /* terms in FP32; 0 FP32 accumulation, 1 FP64 accumulation
                        (default), 2 FP64 accumulation with correctly rounded
                        sqrt / exp / division in the terms, 3 FP32
                        accumulation compensated per query (Neumaier: every
                        addition's rounding error kept in a second FP32
                        word); 0, 1 and 3 use the MUFU approximations of
                        rsqrt / exp2 / rcp in the terms */
    int tile;        /* grid samples per warp: 0 4x4x2 (default), 1 8x4x1,
                        2 2x4x4, 3 8x2x2 (point queries ignore it) */
    int order;       /* far-field expansion order of the plain sum: 0 (the DWG
                        kernels), 1 or 2 (igl::fast_winding_number's
                        expansion_order, deps/libigl/include/igl/
                        fast_winding_number.cpp:9-120,187-241); screened sums
                        take 0 only */
    int lists;       /* screened grid sums (dwg_gwn_grid): 1 records the
                        Barnes-Hut interaction lists of the grid on the first
                        call (synchronises) and replays them on later calls
                        with the same grid, beta and tile until the centres
                        change (dwg_octree_update_info): bit-identical values,
                        no traversal; 2 also keeps the terms' screening
                        weights for two (sigma, screen) values (precision 0,
                        1 and 3): later calls with one of them read the weights
                        instead of evaluating them, same bits (the calls of
                        one octree must then follow each other on one
                        stream); 0 traverses every call */
} dwg_gwn_params;

int dwg_gwn_points(dwg_octree* tree, const float* normals_dev, const float* areas_dev,
                   const float* radii_dev, const float* queries_dev, long long num_queries,
                   const dwg_gwn_params* params, float* out_dev, unsigned long long* terms_dev,
                   void* stream);

/* Same as dwg_gwn_points, writing the number of terms of every query to
 * per_query_terms_dev (int32) -- a check that the opening decisions match
 * a CPU restatement of the traversal, query by query. */
int dwg_gwn_points_counted(dwg_octree* tree, const float* normals_dev, const float* areas_dev,
                           const float* radii_dev, const float* queries_dev, long long num_queries,
                           const dwg_gwn_params* params, float* out_dev, int* per_query_terms_dev,
                           void* stream);

/* Far-field expansion coefficients of orders 1 and 2 (FP64, node order of
 * dwg_octree_export, 36 per node: m1[u + 3v] = sum A a_u n_v and
 * m2[9i + u + 3v] = sum 0.5 a_i A a_u n_v with a = p - CM), computed from the
 * tree's current normals and areas.  The coefficients of
 * igl::fast_winding_number's precompute with expansion_order 2
 * (deps/libigl/include/igl/fast_winding_number.cpp:87-105, EC columns 3..38). */
int dwg_octree_expansion(dwg_octree* tree, double* out_host, void* stream);

/* Same sum at the samples of a regular grid: q(x,y,z) = origin + (x,y,z) * spacing,
 * x fastest; out has res[0]*res[1]*res[2] values.  The reference materialises
 * the grid positions (igl::voxel_grid + H2D copy); here they are closed-form. */
int dwg_gwn_grid(dwg_octree* tree, const float* normals_dev, const float* areas_dev,
                 const float* radii_dev, const int res[3], const float origin[3], float spacing,
                 const dwg_gwn_params* params, float* out_dev, unsigned long long* terms_dev,
                 void* stream);

/* Values and gradients of the same sums.  The reference has no gradient
 * (its sums are ScreenedGWNLibiPStoQ / GWNLibiPStoQ, src/TurboLibiGWN.cu:
 * 328-812); grad_dev (3 floats per query, nullable) receives the analytic
 * derivative of each term with respect to the query -- of the point terms
 * and of the far nodes' order-0 dipoles, with the opening decisions of
 * dwg_gwn_points -- and out_dev (nullable) the values.  FP32 terms summed in
 * FP64, one thread per query (slower than dwg_gwn_points, which the DWG loop
 * uses); params->order must be 0; lists, tile and precision are ignored. */
int dwg_gwn_points_grad(dwg_octree* tree, const float* normals_dev, const float* areas_dev,
                        const float* radii_dev, const float* queries_dev, long long num_queries,
                        const dwg_gwn_params* params, float* out_dev, float* grad_dev, void* stream);
int dwg_gwn_grid_grad(dwg_octree* tree, const float* normals_dev, const float* areas_dev,
                      const float* radii_dev, const int res[3], const float origin[3], float spacing,
                      const dwg_gwn_params* params, float* out_dev, float* grad_dev, void* stream);

/* The same sums (and, with grad_dev, gradients) in FP64: terms and sums in
 * double from the tree's FP64 moments, with the opening decisions of the
 * FP32 kernels -- the yardstick for checking FP32 fields on the GPU (as the
 * FP64 CPU restatement does on the host).  No counterpart in the reference. */
int dwg_gwn_points_fp64(dwg_octree* tree, const float* normals_dev, const float* areas_dev,
                        const float* radii_dev, const float* queries_dev, long long num_queries,
                        const dwg_gwn_params* params, double* out_dev, double* grad_dev, void* stream);
int dwg_gwn_grid_fp64(dwg_octree* tree, const float* normals_dev, const float* areas_dev,
                      const float* radii_dev, const int res[3], const float origin[3], float spacing,
                      const dwg_gwn_params* params, double* out_dev, double* grad_dev, void* stream);

/* Closed-form igl::voxel_grid(V, offset, s, 1) (deps/libigl/include/igl/voxel_grid.cpp:11-87):
 * resolution, origin and spacing of the padded grid around points_dev.
 * Synchronises `stream` (the bounding box is read back). */
int dwg_voxel_grid(const float* points_dev, int n, float offset, int s, void* stream, int res[3],
                   float origin[3], float* spacing);

/* ------------------------------------------------------------------------
 * Marching cubes on a scalar grid (x fastest).  Corner, edge and case
 * conventions of TurboMC::TurboMarchingCubes (src/TurboMC.cu:383-478,572-638);
 * triangles are written in cell order (deterministic), each as 3 vertices
 * (9 floats), plus centroid (3) and unit normal -cross/(|cross|+1e-8) (3).
 * positions_dev (R^3 * 3 floats) may be NULL: then q = origin + idx*spacing.
 * Output arrays may be NULL; at most `capacity` triangles are written.
 * *num_tris_dev (device, unsigned long long) receives the full count T; when
 * num_tris_host is non-NULL the call synchronises and stores T there, and
 * returns DWG_ERR_OVERFLOW if T > capacity.
 * ------------------------------------------------------------------------ */
int dwg_marching_cubes(const float* field_dev, const int res[3], const float* positions_dev,
                       const float origin[3], float spacing, float iso, float* tris_dev,
                       float* centroids_dev, float* normals_dev, long long capacity,
                       unsigned long long* num_tris_dev, long long* num_tris_host, void* stream);
/* The generated case tables (edge mask [256], triangle edges [256*16], -1 padded). */
int dwg_mc_tables(int* edge_table_host, signed char* tri_table_host);

/* Marching cubes that allocates no device memory.  No counterpart in the
 * reference.  It is for callers that cannot call cudaMalloc while they mesh:
 * a real-time loop that must not allocate after start-up (cudaMalloc and
 * cudaFree can wait for the whole device and take unbounded time), and an
 * application whose device memory is a fixed budget handed out by its own
 * pool, where a library allocation could fail or take memory the pool
 * counts on.  Same arguments, kernels and output as dwg_marching_cubes; the
 * count is returned in *num_tris_host (required), and the call synchronises
 * `stream` to read it.  With T > capacity it writes the first `capacity`
 * triangles, sets *num_tris_host = T and returns DWG_ERR_OVERFLOW.
 * Its scratch is a static device array of the library (about 4 MB, held by
 * every GPU that loads the library until the process exits), which limits the
 * grid to 134,217,728 cells (e.g. 512^3); larger grids are rejected with
 * DWG_ERR_INVALID before any GPU work.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress) and uploads the case
 * tables.  Every call reuses
 * the array (the scan rewrites each slot it reads), so calls that overlap on
 * the GPU (different streams or threads at once) race.  The looked-up
 * address and the tables are cached per device ordinal and do not survive a
 * cudaDeviceReset. */
int dwg_marching_cubes_noalloc(const float* field_dev, const int res[3], const float* positions_dev,
                               const float origin[3], float spacing, float iso, float* tris_dev,
                               float* centroids_dev, float* normals_dev, long long capacity,
                               long long* num_tris_host, void* stream);

/* ------------------------------------------------------------------------
 * k nearest neighbours.  Results ascend by the cukd candidate key
 * (float bits of |p-q|^2) << 32 | index (include/cudaKDTree/cukd/knn.h:279-282),
 * self included.  Replaces GenerateKDTreeForDWG + CudaKNNWithKDTreeforDWG
 * (include/TurboDWG.h:14-27, src/KNN_GWN.cu:183-212,490-715) and the GWN
 * variants (include/DWGProcess.h:20-30).  1 <= k <= 64, k <= n.
 * ------------------------------------------------------------------------ */
typedef struct dwg_knn_index dwg_knn_index;
int dwg_knn_build(const float* points_dev, int n, void* stream, dwg_knn_index** out);
int dwg_knn_destroy(dwg_knn_index* index);
int dwg_knn_query(dwg_knn_index* index, const float* queries_dev, long long num_queries, int k,
                  int* out_dev, void* stream);
/* one-shot convenience: build, query, destroy */
int dwg_knn(const float* points_dev, int n, const float* queries_dev, long long num_queries, int k,
            int* out_dev, void* stream);

/* ------------------------------------------------------------------------
 * Normal diffusion step: every triangle adds its normal to its k nearest
 * points, sums are normalised; points whose sum has length < 1e-10 keep
 * their normal and are flagged (is_zero_dev, may be NULL); *zero_count_dev
 * receives their number.  Replaces ResetZero + UpdateNormals +
 * NormalizeNormals (src/TurboDWG.cu:134-143,179-204,238-266,571-583).
 * Sums are accumulated in 2^-40 fixed point so the result is independent of
 * the order of the atomics.
 * ------------------------------------------------------------------------ */
int dwg_diffuse_normals(const int* knn_dev, const float* tri_normals_dev, long long num_tris, int k,
                        int num_points, float* normals_dev, unsigned char* is_zero_dev,
                        int* zero_count_dev, void* stream);
/* Zero-normal repair: each flagged point gets the normalised sum of the
 * normals of its k nearest unflagged points.  Replaces LoadZeroData +
 * GenerateKDTreeForDWG + kNN + SimpleUpdateNonzeroNormals
 * (src/TurboDWG.cu:145-177,322-359,585-644).  `index` must be built on the
 * same points.  Runs only when the flagged count exceeds `min_zero` (10 in
 * the reference), decided on the device.  The index keeps each flagged
 * point's neighbours: a later repair on the same index starts that point's
 * search from them where they are still unflagged (same results, less
 * search), so repairs on one index are not thread safe. */
int dwg_zero_repair(dwg_knn_index* index, float* normals_dev, const unsigned char* is_zero_dev,
                    const int* zero_count_dev, int k, int min_zero, void* stream);
/* Point normals = normalised mean of the normals of the k nearest leaves.
 * Replaces LoadNormals (src/TurboDWG.cu:206-236,834-853). */
int dwg_load_normals(const int* knn_dev, int k, long long num_queries,
                     const float* leaf_normals_dev, float* out_dev, void* stream);
/* r_i = clamp(sqrt(mean_j |p_i - p_j|^2), 0.0015, 0.015) over the k nearest
 * (self included).  Replaces SimpleUpdateRadii / TurboDWG::UpdateRadii
 * (src/TurboDWG.cu:361-391,674-691), with its per-neighbour offset initialised. */
int dwg_radii(const float* points_dev, int n, const int* knn_dev, int k, float* radii_dev,
              void* stream);

/* ------------------------------------------------------------------------
 * --com_As 1 inputs: normals and areas from the points themselves.
 * ------------------------------------------------------------------------ */
/* PCA normals: the eigenvector of the smallest eigenvalue of the covariance
 * of the k nearest points (knn_dev rows, self included), flipped so that
 * (view - p) . n >= 0.  view_host: 3 floats in host memory.  Replaces
 * pcl::NormalEstimation with setKSearch(10) and the bounding-box centre as
 * viewpoint (include/DWGProcess.h:152-200). */
int dwg_pca_normals(const float* points_dev, int n, const int* knn_dev, int k, const float* view_host,
                    float* normals_dev, void* stream);
/* Point areas: for point i, the neighbours of its knn_dev row (self first,
 * k <= 32) whose normal has a positive dot product with n_i are projected
 * on their PCA plane; the share of point i of every Delaunay triangle of
 * that 2-D set around it (half, quarter or Voronoi share by the obtuse
 * rules) is summed; 0 when fewer than 3 neighbours are kept.  Replaces
 * igl::copyleft::cgal::point_areas (include/DWGProcess.h:345-378,789-790;
 * deps/libigl/include/igl/copyleft/cgal/point_areas.cpp:39-210). */
int dwg_point_areas(const float* points_dev, int n, const int* knn_dev, int k, const float* normals_dev,
                    float* areas_dev, void* stream);

/* ------------------------------------------------------------------------
 * Full reconstruction (TurboIterative + TurboDWG::TurboScreenedDWGLaunch +
 * TurboDWG::GenerateMesh, include/DWGProcess.h:474-797,
 * src/TurboDWG.cu:456-924).  Parameters mirror the DWG_CUDA flags
 * (src/main.cpp:19-39).
 * ------------------------------------------------------------------------ */
typedef struct {
    int in_normal;          /* 0 random, 1 input, 2 random leaf normals (com_as 1), 3 Gauss map
                               (default), 4 learned (dwg_pipeline_create_learned) */
    int grid_reso;          /* --grid_reso (400) */
    int final_reso;         /* --final_reso (500) */
    int kw, final_kw, normal_kw; /* 10, 10, 10 */
    int max_depth;          /* --max_depth (10) */
    float lambda;           /* --lambda (10) */
    int min_num;            /* --min_num (0) */
    int use_radii;          /* --use_radii (0) */
    float offset_1, offset_2; /* 0.05, 0.01 */
    int use_leaves_generate; /* --use_leaves_generate (0) */
    int total_iter;         /* --total_iter (40) */
    float beta;             /* 2.3 */
    float area;             /* 2e-6 */
    float screen;           /* 0.0015 */
    int knn_tri;            /* 15 */
    int knn_zero;           /* 10 */
    int precision;          /* dwg_gwn_params.precision */
    int use_graph;          /* capture one iteration in a CUDA graph and replay it */
    int tile;               /* dwg_gwn_params.tile of the grid sums */
    float as_thres;         /* --As_thres (0): the ceil(n * as_thres) largest areas are divided by 1000 */
    int com_as;             /* --com_As (0): 1 = areas by dwg_point_areas (leaves, then points in the
                               final pass) and, unless in_normal is 1, PCA normals (k = 10) as the
                               input normals; in_normal 2 then starts from random leaf normals */
    int grid_lists;         /* 1: record the iteration grid's Barnes-Hut interaction lists in the
                               first iteration and replay them afterwards (the same terms in the
                               same order: bit-identical fields, no traversal); 2 (default): also
                               keep each term's screening weight for every sigma of the schedule
                               and read it back in later iterations with that sigma (the same
                               bits; 8 bytes per list entry and lane per sigma, dropped when it
                               does not fit in a third of the free memory); 0: traverse in every
                               iteration */
} dwg_params;

void dwg_params_default(dwg_params* p);

typedef struct dwg_pipeline dwg_pipeline;
/* points_dev: n normalised points; normals_dev: input normals (in_normal 0/1) or NULL. */
int dwg_pipeline_create(const float* points_dev, const float* normals_dev, int n,
                        const dwg_params* params, void* stream, dwg_pipeline** out);
/* Waits for the pipeline's own stream and returns its device memory to the
 * pool without waiting for other streams: work that the caller queued on
 * another stream and that reads the pipeline's buffers (dwg_pipeline_device_ptr)
 * must be finished first. */
int dwg_pipeline_destroy(dwg_pipeline* p);
/* run `n_iters` diffusion iterations (continuing the count) */
int dwg_pipeline_iterate(dwg_pipeline* p, int n_iters);
/* final meshing pass; the mesh stays on the device */
int dwg_pipeline_finalize(dwg_pipeline* p);
/* sizes: "leaves", "points", "triangles" (final mesh; synchronises),
 * "iterations", "grid" (iteration grid samples), "final_grid",
 * "grid_list_entries" (interaction-list entries the iteration grid keeps,
 * 16 bytes each; 0 when it is traversed) and "grid_weight_slots" (sigmas
 * whose screening weights it keeps, 256 bytes per entry each) */
int dwg_pipeline_size(dwg_pipeline* p, const char* what, long long* value);
/* copy a result to host memory (synchronises): "leaf_pos" [L*3], "leaf_nrm" [L*3],
 * "point_nrm" [N*3], "tris" [T*9], "iso" [iters], "tri_count" [iters] (int64),
 * "zero_count" [iters] (int32), "field" [iteration grid], "final_field",
 * "final_iso" [1], "terms" [iters] (uint64 pair evaluations per iteration),
 * "grid_res" [3] (int32), "final_res" [3] (int32) */
int dwg_pipeline_get(dwg_pipeline* p, const char* what, void* dst_host);
/* device pointer of a pipeline array (no copy): "leaf_pos", "leaf_nrm",
 * "point_nrm", "tris", "field", "final_field" */
int dwg_pipeline_device_ptr(dwg_pipeline* p, const char* what, void** ptr);

/* ------------------------------------------------------------------------
 * One cloud on several GPUs: z-slab sharding (one process per GPU).  The
 * reference runs one cloud on one GPU; here rank r of `world` evaluates the
 * winding number and marching cubes only on its run of z-cells of each grid
 * (the samples of the run and the shared boundary layer) and finds the
 * neighbours of its own triangles; octrees, leaves, the leaf sums, the iso
 * value and the zero repair are replicated.  Once per iteration the 3 L
 * fixed-point normal sums and the triangle count (3 L + 1 int64) are summed
 * over the ranks by `exchange`; integer sums are exact in any order, so every
 * rank ends each iteration with the leaf normals of a one-GPU run, bit for
 * bit, and the ranks' meshes concatenated in rank order are the one-GPU mesh.
 * `exchange` is called on every rank in the same order with no pipeline work
 * in flight; it must replace buf_dev[0..count) by the element-wise sum over
 * the ranks before it returns (e.g. ncclAllReduce + stream synchronise) and
 * return 0.  Iterations run without a CUDA graph.  Sizes and arrays of the
 * pipeline ("grid", "field", "final_grid", "final_field", "triangles",
 * "tris") are this rank's; "slab" (int32[4]: first z-sample and count of the
 * iteration grid, then of the final grid) locates them; "tri_count" is the
 * total. */
typedef int (*dwg_exchange_fn)(void* user, long long* buf_dev, long long count, void* stream);
int dwg_pipeline_create_sharded(const float* points_dev, const float* normals_dev, int n,
                                const dwg_params* params, int rank, int world, dwg_exchange_fn exchange,
                                void* user, void* stream, dwg_pipeline** out);
/* the slab of rank `rank`: z-samples z0 .. z0 + nz - 1 of a grid of `samples`
 * z-samples (the samples - 1 cells split into `world` contiguous runs) */
int dwg_slab_range(int samples, int rank, int world, int* z0, int* nz);

/* ------------------------------------------------------------------------
 * Batched reconstruction of many clouds (no counterpart in the reference,
 * which reconstructs one cloud per DWG_CUDA run).  Each cloud is a pipeline
 * with its own flags (params[i]; in_normal 3, one tile and one precision for
 * all); one iteration of all clouds is one CUDA graph.  The first iteration
 * records every cloud's grid interaction lists while they fit (a quarter of
 * the free memory stays reserved), then screening weights go to the largest
 * lists first while they fit; clouds whose lists did not fit have their
 * grids summed by a single persistent launch over their bricks.  The lists
 * and weights are released by dwg_batch_finalize.
 * ------------------------------------------------------------------------ */
typedef struct dwg_batch dwg_batch;
int dwg_batch_create(const float* const* points_dev, const int* counts, int num_clouds, const dwg_params* params,
                     void* stream, dwg_batch** out);
int dwg_batch_destroy(dwg_batch* b);
int dwg_batch_iterate(dwg_batch* b, int n_iters);
int dwg_batch_finalize(dwg_batch* b);
/* borrowed handle of cloud `index` for the dwg_pipeline_size / _get /
 * _device_ptr getters; valid until dwg_batch_destroy, never destroyed by the
 * caller */
int dwg_batch_cloud(dwg_batch* b, int index, dwg_pipeline** cloud);

/* ------------------------------------------------------------------------
 * Autotuner of the grid sums (no counterpart in the reference, which fixes
 * beta = 2.3 in src/TurboLibiGWN.cu and one thread per query).  For one
 * cloud it runs `warm_iters` DWG iterations, measures the RMS error of the
 * Barnes-Hut sums against exact sums at `samples` seeded grid samples for
 * candidate opening ratios beta in [1.5, 4.5], times a full grid evaluation
 * for those within `tol` (absolute RMS; tol <= 0: no larger than the error
 * of the reference's beta = 2.3), and then the four brick shapes at the
 * fastest.
 * ------------------------------------------------------------------------ */
typedef struct {
    float beta;     /* chosen opening ratio */
    int tile;       /* chosen brick shape (dwg_gwn_params.tile) */
    float rms_err;  /* RMS |w_beta - w_exact| at the samples */
    float max_err;  /* max  |w_beta - w_exact| at the samples */
    float grid_ms;  /* one grid evaluation at (beta, tile) */
    float ref_ms;   /* one grid evaluation at beta 2.3, tile 0 */
    float ref_rms_err; /* RMS error at beta 2.3 */
    float field_rms;   /* RMS of the exact sums at the samples */
} dwg_tune_result;
int dwg_autotune(const float* points_dev, int n, const dwg_params* params, float tol, int samples,
                 int warm_iters, void* stream, dwg_tune_result* out);

/* ------------------------------------------------------------------------
 * Learned normal initialiser (no counterpart in the reference: it replaces
 * TurboNormalInitialization::GaussMapInit, include/TurboNormalInit.h:13, as
 * the source of the leaves' initial normals).  A point-wise MLP
 * 12 -> 128 -> 128 -> 128 -> 3 (GELU) over covariance features of the 16
 * nearest points, BF16 weights and activations, FP32 accumulation, trained
 * with the library's own forward / backward / Adam kernels on DWG-converged
 * normals.  A handle is used by one thread at a time.
 * Parameters (host arrays, files): for each layer W [din x dout] row-major
 * then b [dout], with din = 16, 128, 128, 128 and dout = 128, 128, 128, 8
 * (inputs padded from 12 to 16, outputs from 3 to 8; padding entries zero).
 * ------------------------------------------------------------------------ */
typedef struct dwg_mlp dwg_mlp;
#define DWG_MLP_FEATURES 12
long long dwg_mlp_param_count(void);
/* random initialisation (uniform, fan-in scaled) from `seed` */
int dwg_mlp_create(unsigned long long seed, void* stream, dwg_mlp** out);
int dwg_mlp_destroy(dwg_mlp* m);
int dwg_mlp_set_params(dwg_mlp* m, const float* params_host, long long count);
int dwg_mlp_get_params(dwg_mlp* m, float* params_host, long long count);
/* file: 8 bytes "DWGMLP01", int64 count, count little-endian float32 */
int dwg_mlp_load(dwg_mlp* m, const char* path);
int dwg_mlp_save(dwg_mlp* m, const char* path);
/* features_dev [n x 12]: eigenvalues of the covariance of the 16 nearest
 * points (self included) over their sum, the smallest and the largest
 * eigenvector turned away from the bounding-box centre, and the offset to the
 * neighbourhood centroid over the RMS spread */
int dwg_mlp_features(const float* points_dev, int n, float* features_dev, void* stream);
/* raw outputs out_dev [n x 3] */
int dwg_mlp_forward(dwg_mlp* m, const float* features_dev, long long n, float* out_dev, void* stream);
/* loss = mean(1 - <y/|y|, t>) over the batch; gradients of the flat
 * parameters into grads_host (count = dwg_mlp_param_count()); no update */
int dwg_mlp_gradients(dwg_mlp* m, const float* features_dev, const float* targets_dev, long long n,
                      float* loss_host, float* grads_host, long long count, void* stream);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on one batch */
int dwg_mlp_train_step(dwg_mlp* m, const float* features_dev, const float* targets_dev, long long n,
                       float lr, float* loss_host, void* stream);
/* unit initial normals of n points (features, forward, normalise; the Gauss
 * map where the output is degenerate) */
int dwg_mlp_init_normals(dwg_mlp* m, const float* points_dev, int n, float* normals_dev, void* stream);
/* dwg_pipeline_create with the leaves' initial normals from `init`
 * (params->in_normal must be 4); `init` is used during the call only */
int dwg_pipeline_create_learned(const float* points_dev, int n, const dwg_params* params, dwg_mlp* init,
                                void* stream, dwg_pipeline** out);

/* One call from host memory to host memory: create + iterate(total_iter) +
 * finalize + copy of the mesh and point normals.  tris_host holds up to
 * tri_capacity triangles; *num_tris receives the full count. */
int dwg_reconstruct_host(const float* points_host, const float* normals_host, int n,
                         const dwg_params* params, float* point_normals_host, float* tris_host,
                         long long tri_capacity, long long* num_tris, void* stream);

/* ------------------------------------------------------------------------
 * Host IO helpers (include/DWGProcess.h:53-97, src/TurboMC.cu:344-371,
 * src/TurboDWG.cu:903-923).
 * ------------------------------------------------------------------------ */
/* Read "x y z [nx ny nz]" lines; returns the count in *n and malloc'd arrays
 * (free with dwg_free_host).  When `normalize` is set, centre on the mean and
 * divide by max 2|x| (FP64), as the reference reader does.  Blank lines are
 * skipped; a line with 1-2 numbers or a non-finite coordinate is an error
 * naming the line.  Parsed on all host cores, with the doubles of %lf. */
int dwg_read_xyz(const char* path, int normalize, float** points, float** normals, int* n);
void dwg_free_host(void* p);
int dwg_write_stl(const char* path, const float* tris_host, long long num_tris);
/* The same STL file from triangles in device memory (9 floats each, e.g.
 * dwg_pipeline_device_ptr "tris"): the 50-byte records are packed on the GPU
 * in chunks of 2^20 triangles and written while the next chunk is packed.
 * Synchronises `stream`. */
int dwg_write_stl_device(const char* path, const float* tris_dev, long long num_tris, void* stream);
int dwg_write_xyz(const char* path, const float* points_host, const float* normals_host, int n);

#ifdef __cplusplus
}
#endif
#endif /* DWG_B200_H */
