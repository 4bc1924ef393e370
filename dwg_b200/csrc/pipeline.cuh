// pipeline.cuh -- the DWG reconstruction driver on one GPU.
#pragma once

#include "areas.cuh"
#include "gwn.cuh"
#include "knn.cuh"
#include "mc.cuh"
#include "mlp.cuh"
#include "normals.cuh"
#include "octree.cuh"

namespace dwg {

// element-wise int64 sum over the ranks of a sharded reconstruction, in place
// (the same call on every rank, in the same order); 0 on success
typedef int (*ExchangeFn)(void* user, long long* buf_dev, long long count, void* stream);

// the z-slab of rank `rank` of `world` in a grid of `samples` z-samples: the
// samples - 1 cells are split into contiguous runs, a run of cells c0 .. c1-1
// needs samples c0 .. c1 (one shared boundary layer)
void slab_range(int samples, int rank, int world, int* z0, int* nz);

struct Pipeline {
    dwg_params prm;
    Mlp* init_mlp = nullptr;        // learned initialiser of in_normal 4 (used during setup only)
    cudaStream_t s = nullptr;       // the pipeline's own non-blocking stream
    cudaStream_t caller = nullptr;  // the stream the caller passed
    cudaEvent_t ev = nullptr;
    int n = 0;  // points
    int L = 0;  // leaves
    DevBuf<float> P, Nin, area_pts;
    Octree t1, t2;
    KnnIndex kidx;  // on the leaves (canonical order)
    // leaves, canonical order (depth-first order of the octree on the leaves)
    DevBuf<float> leaf_pos, leaf_nrm, leaf_area, leaf_rad;
    // iteration grid
    int gres[3] = {0, 0, 0};
    float gorg[3] = {0, 0, 0};
    float gh = 0;
    DevBuf<float> field, wleaf;
    GwnList glist;               // interaction lists of the iteration grid (fixed leaves, fixed grid)
    GwnList llist;               // interaction lists of the sums at the leaves (fixed leaves)
    bool grid_batched = false;   // a batch sums the grid after the first iteration: no grid lists
    int weight_slots() const;    // sigmas of the schedule whose screening weights are kept
    size_t glist_budget = 0;     // largest list kept, bytes
    long long cap = 0;
    DevBuf<float> cent, tnrm;
    DevBuf<unsigned long long> ntri;
    McWorkspace mcws;
    DevBuf<int> knn_buf;
    DevBuf<long long> acc;
    DevBuf<unsigned char> is_zero;
    DevBuf<int> zero_count;
    ZeroRepairWs zws;
    DevBuf<double> partial;
    // per-iteration state on the device
    DevBuf<int> iter_dev, half_tab, cur_half;
    DevBuf<float> sigma_tab, cur_sigma, iso_dev;
    DevBuf<unsigned long long> terms_cur;
    DevBuf<float> iso_hist;
    DevBuf<long long> tri_hist;
    DevBuf<int> zero_hist;
    DevBuf<unsigned long long> terms_hist;
    int iter = 0;
    int hist_cap = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    // final pass
    bool finalized = false;
    int fres[3] = {0, 0, 0};
    // z-slab sharding: this rank evaluates and meshes the z-samples gz0 ..
    // gz0 + gnz - 1 of the iteration grid (fz0, fnz: the final grid); the
    // normal accumulators and the triangle count are summed over the ranks
    // once per iteration, everything else is replicated
    int rank = 0, world = 1;
    ExchangeFn exchange = nullptr;
    void* exchange_user = nullptr;
    int gz0 = 0, gnz = 0, fz0 = 0, fnz = 0;
    float forg[3] = {0, 0, 0};
    float fh = 0;
    DevBuf<float> final_field, point_nrm, tris, wfin, p_sorted, pt_rad;
    DevBuf<int> nb_final;
    DevBuf<unsigned long long> final_ntri;
    DevBuf<float> final_iso;
    long long final_cap = 0;

    ~Pipeline();
    int setup(const float* points_dev, const float* normals_dev, int n_points, const dwg_params& p,
              cudaStream_t stream);
    int iterate(int n_iters);
    int iterate_once();
    // the phases of one iteration on stream s (graph-capturable)
    int iterate_pre();
    int iterate_grid();
    int iterate_post();
    int exchange_sums();
    dwg_gwn_params gwn_params() const;
    int finalize();
    int ensure_hist(int total);
    // order the pipeline stream after the caller's work, and back
    int join_in();
    int join_out();
};

int voxel_grid_host(const float* points_dev, int n, float offset, int s_res, cudaStream_t st, int res[3],
                    float origin[3], float* spacing);

}  // namespace dwg
