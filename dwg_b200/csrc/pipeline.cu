// pipeline.cu -- DWG reconstruction on one GPU, every step on the device.
//
// Reference flow (include/DWGProcess.h:99-262,474-797; src/TurboDWG.cu:456-924):
// CPU octree on the points, octree-leaf cell centres as the iteration's point
// set, CPU moment precompute, then per iteration: mass-normal update,
// screened GWN at the leaves and at the grid, mean iso value, marching cubes,
// kNN of the triangle centroids, normal scatter / normalise, zero-normal
// repair; finally a pass over all points at the final resolution.
//
// Here both octrees, their moments, the grids and the kNN structure are built
// on the GPU once; one iteration is a fixed sequence of fixed-size launches
// whose varying values (sigma, iso halving, triangle count, zero count) live
// in device memory, so it can be captured once as a CUDA graph and replayed.
#include <cub/cub.cuh>

#include <cmath>
#include <utility>
#include <vector>

#include "pipeline.cuh"

namespace dwg {

constexpr int kPcaK = 10;   // ne.setKSearch(10), include/DWGProcess.h:178
constexpr int kAreaK = 15;  // point_areas neighbourhoods, include/DWGProcess.h:232,357

// Closed form of igl::voxel_grid(V, offset, s, 1) (deps/libigl/include/igl/voxel_grid.cpp:11-87)
// in single precision; samples at origin + index * spacing.
int voxel_grid_host(const float* P, int n, float offset, int s_res, cudaStream_t st, int res[3], float origin[3],
                    float* spacing) {
    DWG_REQUIRE(P && n >= 1, "voxel_grid: need points");
    DWG_REQUIRE(s_res >= 4, "voxel_grid: resolution must be >= 4 (got %d)", s_res);
    DevBuf<float> bb;
    DWG_TRY(bb.reserve(6));
    DWG_TRY(bbox_device(P, n, bb.ptr, st));
    float b[6];
    DWG_CHECK_CUDA(cudaMemcpyAsync(b, bb.ptr, sizeof(b), cudaMemcpyDeviceToHost, st));
    DWG_CHECK_CUDA(cudaStreamSynchronize(st));
    volatile float mn[3], mx[3], diag[3];
    for (int d = 0; d < 3; ++d) {
        mn[d] = b[d] - offset;
        mx[d] = b[3 + d] + offset;
        diag[d] = mx[d] - mn[d];
    }
    int si = 0;
    for (int d = 1; d < 3; ++d)
        if (diag[d] > diag[si]) si = d;
    const float s_len = diag[si];
    const float sf = (float)(s_res - 2);
    for (int d = 0; d < 3; ++d) {
        if (d == si) {
            res[d] = s_res - 2;
        } else {
            volatile float v = sf * diag[d];
            v = v / s_len;
            res[d] = (int)std::ceil((float)v);
        }
        res[d] += 2;
    }
    volatile float Aa[3];
    for (int d = 0; d < 3; ++d) {
        volatile float ps = 1.0f / ((float)res[d] - 1.0f);
        volatile float den = 1.0f - 2.0f * ps;
        Aa[d] = diag[d] / den;
    }
    int ai = 0;
    for (int d = 1; d < 3; ++d)
        if (Aa[d] > Aa[ai]) ai = d;
    volatile float h = Aa[ai] / ((float)res[ai] - 1.0f);
    for (int d = 0; d < 3; ++d) {
        volatile float c = (mn[d] + mx[d]) / 2.0f;
        volatile float half = 0.5f * ((float)res[d] - 1.0f);
        volatile float ext = half * h;
        origin[d] = c - ext;
    }
    *spacing = h;
    return DWG_OK;
}

// ---------------------------------------------------------------- kernels --
__global__ void k_gather_xyz(const float* __restrict__ src, const int* __restrict__ perm, int n,
                             float* __restrict__ dst) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int i = perm[j];
    dst[(size_t)j * 3] = src[(size_t)i * 3];
    dst[(size_t)j * 3 + 1] = src[(size_t)i * 3 + 1];
    dst[(size_t)j * 3 + 2] = src[(size_t)i * 3 + 2];
}

// area of canonical leaf i into the octree record of sorted point i (the two orders coincide for t2)
__global__ void k_set_area(float4* __restrict__ pa, const float* __restrict__ area, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pa[i].w = area[i];
}

__global__ void k_fill(float* __restrict__ x, long long n, float v) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) x[i] = v;
}

__global__ void k_sorted_xyz(const float4* __restrict__ pa, int n, float* __restrict__ out) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    float4 p = pa[j];
    out[(size_t)j * 3] = p.x;
    out[(size_t)j * 3 + 1] = p.y;
    out[(size_t)j * 3 + 2] = p.z;
}

__global__ void k_set_nr(float4* __restrict__ nr, const float* __restrict__ N, const float* __restrict__ R, int n) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    float4 v = nr[j];
    if (N) {
        v.x = N[(size_t)j * 3];
        v.y = N[(size_t)j * 3 + 1];
        v.z = N[(size_t)j * 3 + 2];
    }
    if (R) v.w = R[j];
    nr[j] = v;
}

// SmoothNormalstoOctreeLeaves (include/DWGProcess.h:430-472): per leaf cell,
// per component sum_j exp(-((p_jk - c_k)/W)^2 / 4) n_jk, FP64
__global__ void k_smooth_leaves(const int4* __restrict__ info, const int* __restrict__ leaf_node, int L,
                                const unsigned long long* __restrict__ keys, const double* __restrict__ root, int D,
                                const float4* __restrict__ pa, const float4* __restrict__ nr,
                                double* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L) return;
    int4 iv = info[leaf_node[i]];
    int depth = iv.w & 0xff;
    unsigned long long key = keys[iv.x];
    double c[3] = {root[0], root[1], root[2]}, w = root[3];
    for (int d = 0; d < depth; ++d) {
        int o = (int)((key >> (3 * (D - 1 - d))) & 7ull);
        double h = w / 2.0, hh = h / 2.0;
        c[0] += (o & 1) ? hh : -hh;
        c[1] += (o & 2) ? hh : -hh;
        c[2] += (o & 4) ? hh : -hh;
        w = h;
    }
    double acc[3] = {0, 0, 0};
    for (int j = iv.x; j < iv.x + iv.y; ++j) {
        float4 p = pa[j];
        float4 q = nr[j];
        const double pv[3] = {p.x, p.y, p.z}, nv[3] = {q.x, q.y, q.z};
        for (int k = 0; k < 3; ++k) {
            double x = (pv[k] - c[k]) / w;
            acc[k] += exp(-(x * x) / 4.0) * nv[k];
        }
    }
    for (int k = 0; k < 3; ++k) out[(size_t)i * 3 + k] = acc[k];
}

__global__ void k_sumsq(const double* __restrict__ x, long long n, double* __restrict__ part) {
    long long chunk = (n + 255) / 256;
    long long b0 = blockIdx.x * chunk, b1 = b0 + chunk < n ? b0 + chunk : n;
    double acc = 0;
    for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) acc += x[i] * x[i];
    typedef cub::BlockReduce<double, 256> BR;
    __shared__ typename BR::TempStorage tmp;
    double t = BR(tmp).Sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// Eigen's normalized() over the whole L x 3 matrix (include/DWGProcess.h:537)
__global__ void k_frobenius_apply(const double* __restrict__ part, const double* __restrict__ x, long long n,
                                  const int* __restrict__ perm, float* __restrict__ out) {
    __shared__ double norm;
    if (threadIdx.x == 0) {
        double t = 0;
        for (int b = 0; b < 256; ++b) t += part[b];
        norm = sqrt(t);
    }
    __syncthreads();
    long long L = n / 3;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < L; j += (long long)gridDim.x * blockDim.x) {
        long long i = perm[j];
        for (int k = 0; k < 3; ++k) {
            double v = x[i * 3 + k];
            out[j * 3 + k] = (float)(norm > 0 ? v / norm : v);
        }
    }
}

// sigma schedule and iso halving (src/TurboDWG.cu:526-550), per iteration
__global__ void k_iter_begin(const int* __restrict__ iter, const float* __restrict__ sigma_tab,
                             const int* __restrict__ half_tab, float* __restrict__ cur_sigma,
                             int* __restrict__ cur_half, unsigned long long* __restrict__ terms) {
    int t = *iter;
    *cur_sigma = sigma_tab[t];
    *cur_half = half_tab[t];
    *terms = 0;
}

__global__ void k_iter_end(int* __restrict__ iter, const unsigned long long* __restrict__ ntri, long long cap,
                           const int* __restrict__ zc, const unsigned long long* __restrict__ terms,
                           long long* __restrict__ tri_hist, int* __restrict__ zero_hist,
                           unsigned long long* __restrict__ terms_hist) {
    int t = *iter;
    unsigned long long T = *ntri;
    tri_hist[t] = (long long)T;
    zero_hist[t] = *zc;
    terms_hist[t] = *terms;
    *iter = t + 1;
}

__global__ void k_put_count(const unsigned long long* __restrict__ ntri, long long* __restrict__ slot) {
    *slot = (long long)*ntri;
}

__global__ void k_get_count(long long* __restrict__ slot, unsigned long long* __restrict__ ntri) {
    *ntri = (unsigned long long)*slot;
    *slot = 0;
}

void slab_range(int samples, int rank, int world, int* z0, int* nz) {
    const long long cells = samples - 1;
    const long long c0 = cells * rank / world, c1 = cells * (rank + 1) / world;
    *z0 = (int)c0;
    *nz = (int)(c1 - c0 + 1);
}

// ------------------------------------------------------------------ setup --
Pipeline::~Pipeline() {
    if (s) cudaStreamSynchronize(s);
    graph_exec_release(graph_exec);  // idle: the stream was drained
    if (graph) cudaGraphDestroy(graph);
    event_release(ev);
    stream_release(s);
}

int Pipeline::join_in() {
    DWG_CHECK_CUDA(cudaEventRecord(ev, caller));
    DWG_CHECK_CUDA(cudaStreamWaitEvent(s, ev, 0));
    return DWG_OK;
}

int Pipeline::join_out() {
    DWG_CHECK_CUDA(cudaEventRecord(ev, s));
    DWG_CHECK_CUDA(cudaStreamWaitEvent(caller, ev, 0));
    return DWG_OK;
}

static float sigma_at(int t, float lambda) {
    float s = lambda;
    if (t < 4) s = 20.0f;
    if (t > 0 && t % 7 == 0) s = 10.0f;
    return s;
}

int Pipeline::ensure_hist(int total) {
    if (total <= hist_cap) return DWG_OK;
    int cap2 = total + 16;
    std::vector<float> st(cap2);
    std::vector<int> ht(cap2);
    for (int t = 0; t < cap2; ++t) {
        st[t] = sigma_at(t, prm.lambda);
        ht[t] = (t % 5 == 0 && t != 0) ? 1 : 0;
    }
    // keep the history already recorded
    std::vector<float> ih(hist_cap);
    std::vector<long long> th(hist_cap);
    std::vector<int> zh(hist_cap);
    std::vector<unsigned long long> mh(hist_cap);
    if (hist_cap) {
        DWG_CHECK_CUDA(cudaMemcpyAsync(ih.data(), iso_hist.ptr, sizeof(float) * hist_cap, cudaMemcpyDeviceToHost, s));
        DWG_CHECK_CUDA(cudaMemcpyAsync(th.data(), tri_hist.ptr, sizeof(long long) * hist_cap, cudaMemcpyDeviceToHost, s));
        DWG_CHECK_CUDA(cudaMemcpyAsync(zh.data(), zero_hist.ptr, sizeof(int) * hist_cap, cudaMemcpyDeviceToHost, s));
        DWG_CHECK_CUDA(cudaMemcpyAsync(mh.data(), terms_hist.ptr, sizeof(unsigned long long) * hist_cap,
                                       cudaMemcpyDeviceToHost, s));
        DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    }
    // the captured graph holds the old table pointers
    if (graph_exec) {
        cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
    }
    if (graph) {
        cudaGraphDestroy(graph);
        graph = nullptr;
    }
    DWG_TRY(sigma_tab.reserve(cap2));
    DWG_TRY(half_tab.reserve(cap2));
    DWG_TRY(iso_hist.reserve(cap2));
    DWG_TRY(tri_hist.reserve(cap2));
    DWG_TRY(zero_hist.reserve(cap2));
    DWG_TRY(terms_hist.reserve(cap2));
    DWG_CHECK_CUDA(cudaMemcpyAsync(sigma_tab.ptr, st.data(), sizeof(float) * cap2, cudaMemcpyHostToDevice, s));
    DWG_CHECK_CUDA(cudaMemcpyAsync(half_tab.ptr, ht.data(), sizeof(int) * cap2, cudaMemcpyHostToDevice, s));
    DWG_CHECK_CUDA(cudaMemsetAsync(iso_hist.ptr, 0, sizeof(float) * cap2, s));
    DWG_CHECK_CUDA(cudaMemsetAsync(tri_hist.ptr, 0, sizeof(long long) * cap2, s));
    DWG_CHECK_CUDA(cudaMemsetAsync(zero_hist.ptr, 0, sizeof(int) * cap2, s));
    DWG_CHECK_CUDA(cudaMemsetAsync(terms_hist.ptr, 0, sizeof(unsigned long long) * cap2, s));
    if (hist_cap) {
        DWG_CHECK_CUDA(cudaMemcpyAsync(iso_hist.ptr, ih.data(), sizeof(float) * hist_cap, cudaMemcpyHostToDevice, s));
        DWG_CHECK_CUDA(cudaMemcpyAsync(tri_hist.ptr, th.data(), sizeof(long long) * hist_cap, cudaMemcpyHostToDevice, s));
        DWG_CHECK_CUDA(cudaMemcpyAsync(zero_hist.ptr, zh.data(), sizeof(int) * hist_cap, cudaMemcpyHostToDevice, s));
        DWG_CHECK_CUDA(cudaMemcpyAsync(terms_hist.ptr, mh.data(), sizeof(unsigned long long) * hist_cap,
                                       cudaMemcpyHostToDevice, s));
    }
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    hist_cap = cap2;
    return DWG_OK;
}

int Pipeline::setup(const float* points_dev, const float* normals_dev, int n_points, const dwg_params& p,
                    cudaStream_t stream) {
    DWG_REQUIRE(points_dev && n_points >= 2, "pipeline: need at least 2 points (n=%d)", n_points);
    DWG_REQUIRE(p.max_depth >= 1 && p.max_depth <= kMaxDepth, "pipeline: max_depth must be in [1, %d]", kMaxDepth);
    DWG_REQUIRE(p.grid_reso >= 4 && p.final_reso >= 4, "pipeline: grid resolutions must be >= 4");
    DWG_REQUIRE(p.knn_tri >= 1 && p.knn_tri <= 64 && p.knn_zero >= 1 && p.knn_zero <= 64 && p.kw >= 1 &&
                    p.kw <= 64 && p.final_kw >= 1 && p.final_kw <= 64 && p.normal_kw >= 1 && p.normal_kw <= 64,
                "pipeline: k values must be in [1, 64]");
    DWG_REQUIRE(p.in_normal >= 0 && p.in_normal <= 4, "pipeline: in_normal must be in [0, 4]");
    DWG_REQUIRE(p.com_as == 0 || p.com_as == 1, "pipeline: com_as must be 0 or 1");
    // --com_As 1 replaces the input normals by PCA normals unless in_normal is 1
    // (include/DWGProcess.h:152-200, :494-495)
    const bool pca = p.com_as && p.in_normal != 1;
    DWG_REQUIRE(p.in_normal >= 3 || pca || normals_dev, "pipeline: in_normal %d needs input normals", p.in_normal);
    DWG_REQUIRE(p.in_normal != 4 || init_mlp, "pipeline: in_normal 4 needs a learned initialiser");
    DWG_REQUIRE(world >= 1 && rank >= 0 && rank < world, "pipeline: bad rank %d of %d", rank, world);
    DWG_REQUIRE(world == 1 || exchange, "pipeline: a sharded pipeline needs an exchange function");
    prm = p;
    caller = stream;
    s = stream_acquire();
    ev = event_acquire();
    DWG_REQUIRE(s && ev, "pipeline: no CUDA stream or event");
    // setup's work, its temporaries included, runs on s alone: releases are
    // ordered there instead of waiting for the device
    FreeScope on_s(s, false);
    DWG_TRY(join_in());
    n = n_points;
    DWG_TRY(mc_upload_tables());
    DWG_TRY(P.reserve((size_t)n * 3));
    DWG_CHECK_CUDA(cudaMemcpyAsync(P.ptr, points_dev, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s));
    DWG_TRY(area_pts.reserve(n));
    k_fill<<<div_up(n, 256), 256, 0, s>>>(area_pts.ptr, n, p.area);
    DWG_CHECK_LAUNCH();
    if (normals_dev && !pca) {
        DWG_TRY(Nin.reserve((size_t)n * 3));
        DWG_CHECK_CUDA(cudaMemcpyAsync(Nin.ptr, normals_dev, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s));
    }
    if (pca) {
        // NormalEstimation, 10 nearest points, viewpoint at the box centre
        DWG_TRY(Nin.reserve((size_t)n * 3));
        const int kp = n < kPcaK ? n : kPcaK;
        KnnIndex pix;
        DWG_TRY(knn_build(pix, P.ptr, n, s));
        DevBuf<int> nb;
        DWG_TRY(nb.reserve((size_t)n * kp));
        KnnQuery q;
        q.q = P.ptr;
        q.nq = n;
        DWG_TRY(knn_query(pix, q, kp, nb.ptr, s));
        DevBuf<float> box;
        DWG_TRY(box.reserve(9));
        DWG_TRY(box_centre(P.ptr, n, box.ptr, box.ptr + 6, s));
        DWG_TRY(pca_normals(P.ptr, n, nb.ptr, kp, box.ptr + 6, Nin.ptr, s));
        DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    }
    // octree on the points (include/DWGProcess.h:227)
    DWG_TRY(octree_build(t1, P.ptr, n, p.max_depth, area_pts.ptr, s));
    // leaf cell centres with more than min_num points (GetOctreeLeaves, :383-428)
    DevBuf<float> raw_pos;
    DevBuf<int> raw_node;
    DWG_TRY(octree_leaf_centres(t1, p.min_num, raw_pos, raw_node, &L, s));
    DWG_REQUIRE(L >= 2, "pipeline: fewer than 2 octree leaves (%d)", L);
    // every neighbour query needs at least k leaves (points for the final radii)
    {
        int kmax = p.knn_tri > p.knn_zero ? p.knn_tri : p.knn_zero;
        if (!p.use_leaves_generate && p.normal_kw > kmax) kmax = p.normal_kw;
        if (p.use_radii && p.kw > kmax) kmax = p.kw;
        DWG_REQUIRE(L >= kmax, "pipeline: %d octree leaves, fewer than the %d neighbours a query needs", L, kmax);
        DWG_REQUIRE(!p.use_radii || p.use_leaves_generate || n >= p.final_kw,
                    "pipeline: %d points, fewer than final_kw = %d", n, p.final_kw);
    }
    // octree on the leaves; its sorted order is the canonical leaf order
    DWG_TRY(leaf_area.reserve(L));
    k_fill<<<div_up(L, 256), 256, 0, s>>>(leaf_area.ptr, L, p.area);
    DevBuf<float> raw_area;
    DWG_TRY(raw_area.reserve(L));
    k_fill<<<div_up(L, 256), 256, 0, s>>>(raw_area.ptr, L, p.area);
    DWG_TRY(octree_build(t2, raw_pos.ptr, L, p.max_depth, raw_area.ptr, s));
    DWG_TRY(leaf_pos.reserve((size_t)L * 3));
    DWG_TRY(leaf_nrm.reserve((size_t)L * 3));
    DWG_TRY(leaf_rad.reserve(L));
    k_gather_xyz<<<div_up(L, 256), 256, 0, s>>>(raw_pos.ptr, t2.perm.ptr, L, leaf_pos.ptr);
    k_fill<<<div_up(L, 256), 256, 0, s>>>(leaf_rad.ptr, L, p.screen);
    DWG_CHECK_LAUNCH();
    // leaf normals smoothed from the point normals: the start of in_normal
    // 0-2, and the normals of the --com_As areas
    if (p.in_normal < 3 || p.com_as) {
        DWG_TRY(octree_set_point_data(t1, Nin.ptr, nullptr, nullptr, s));
        DevBuf<double> sm, part;
        DWG_TRY(sm.reserve((size_t)L * 3));
        DWG_TRY(part.reserve(256));
        k_smooth_leaves<<<div_up(L, 128), 128, 0, s>>>(t1.info.ptr, raw_node.ptr, L, t1.keys.ptr, t1.root_dev.ptr,
                                                       t1.max_depth, t1.pa.ptr, t1.nr.ptr, sm.ptr);
        k_sumsq<<<256, 256, 0, s>>>(sm.ptr, (long long)L * 3, part.ptr);
        k_frobenius_apply<<<div_up(L, 256), 256, 0, s>>>(part.ptr, sm.ptr, (long long)L * 3, t2.perm.ptr,
                                                         leaf_nrm.ptr);
        DWG_CHECK_LAUNCH();
        DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    }
    // kNN structure over the leaves, radii (GetRadiiandAs, include/DWGProcess.h:283-343)
    DWG_TRY(knn_build(kidx, leaf_pos.ptr, L, s));
    if (p.use_radii) {
        DevBuf<int> nb;
        DWG_TRY(nb.reserve((size_t)L * p.kw));
        KnnQuery q;
        q.q = leaf_pos.ptr;
        q.nq = L;
        DWG_TRY(knn_query(kidx, q, p.kw, nb.ptr, s));
        DWG_TRY(radii(leaf_pos.ptr, L, nb.ptr, p.kw, leaf_rad.ptr, s));
        DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    }
    if (p.com_as) {
        // leaf areas from the 15 nearest leaves (GetRadiiandAs,
        // include/DWGProcess.h:345-378), before the moments (:680)
        const int ka = L < kAreaK ? L : kAreaK;
        DevBuf<int> nb;
        DWG_TRY(nb.reserve((size_t)L * ka));
        KnnQuery q;
        q.q = leaf_pos.ptr;
        q.nq = L;
        DWG_TRY(knn_query(kidx, q, ka, nb.ptr, s));
        DWG_TRY(point_areas(leaf_pos.ptr, L, nb.ptr, ka, leaf_nrm.ptr, leaf_area.ptr, s));
        k_set_area<<<div_up(L, 256), 256, 0, s>>>(t2.pa.ptr, leaf_area.ptr, L);
        DWG_CHECK_LAUNCH();
        DWG_TRY(octree_update_centres(t2, s));
        DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    }
    if (p.as_thres > 0.f) {
        // OutlierFilter on the leaves' areas (src/TurboDWG.cu:512), canonical
        // order; the centres of mass keep the unfiltered areas
        DWG_TRY(outlier_filter(leaf_area.ptr, L, p.as_thres, s));
        k_set_area<<<div_up(L, 256), 256, 0, s>>>(t2.pa.ptr, leaf_area.ptr, L);
        DWG_CHECK_LAUNCH();
    }
    if (p.in_normal == 2 && p.com_as) DWG_TRY(random_normals(leaf_nrm.ptr, L, s));
    // iteration grid around the points (include/DWGProcess.h:672)
    DWG_TRY(voxel_grid_host(P.ptr, n, p.offset_1, p.grid_reso, s, gres, gorg, &gh));
    if (p.in_normal == 3) DWG_TRY(gauss_map(leaf_pos.ptr, L, leaf_nrm.ptr, s));
    // learned initialiser in place of the Gauss map (falls back to it per leaf
    // where the network output is degenerate)
    if (p.in_normal == 4) DWG_TRY(mlp_init_normals(*init_mlp, kidx, leaf_pos.ptr, L, leaf_nrm.ptr, s));
    k_set_nr<<<div_up(L, 256), 256, 0, s>>>(t2.nr.ptr, leaf_nrm.ptr, leaf_rad.ptr, L);
    DWG_CHECK_LAUNCH();
    // this rank's z-slab of the grid (the whole grid on one GPU)
    DWG_REQUIRE(world <= gres[2] - 1, "pipeline: %d ranks for %d grid cells in z", world, gres[2] - 1);
    if (world > 1) {
        slab_range(gres[2], rank, world, &gz0, &gnz);
    } else {
        gz0 = 0;
        gnz = gres[2];
    }
    // buffers of one iteration
    long long ng = (long long)gres[0] * gres[1] * gres[2];
    cap = ng / 2 > 1000000 ? ng / 2 : 1000000;  // src/TurboDWG.cu:466
    DWG_TRY(field.reserve((size_t)gres[0] * gres[1] * gnz));
    {
        // the grid's interaction lists may take a quarter of the free memory, at most 16 GB
        const size_t fr = device_free_bytes();
        glist_budget = fr / 4 < ((size_t)16 << 30) ? fr / 4 : ((size_t)16 << 30);
    }
    {
        // when fewer weight slots fit than the schedule has sigmas, the slots
        // go to the sigmas of the most iterations (lambda before the first
        // iterations' 20)
        const int iters = p.total_iter > 0 ? p.total_iter : 1;
        float sg[kGwnWeightSlots] = {};
        int cnt[kGwnWeightSlots] = {}, m = 0;
        for (int t = 0; t < iters; ++t) {
            const float v = sigma_at(t, p.lambda);
            int c = 0;
            while (c < m && sg[c] != v) ++c;
            if (c == m) {
                if (m == kGwnWeightSlots) continue;
                sg[m++] = v;
            }
            ++cnt[c];
        }
        for (int a = 0; a < m; ++a)  // most iterations first, first use breaking ties
            for (int b = a + 1; b < m; ++b)
                if (cnt[b] > cnt[a]) {
                    std::swap(cnt[a], cnt[b]);
                    std::swap(sg[a], sg[b]);
                }
        for (int c = 0; c < kGwnWeightSlots; ++c) glist.pref[c] = llist.pref[c] = c < m ? sg[c] : 0.f;
    }
    DWG_TRY(wleaf.reserve(L));
    DWG_TRY(cent.reserve((size_t)cap * 3));
    DWG_TRY(tnrm.reserve((size_t)cap * 3));
    DWG_TRY(ntri.reserve(1));
    DWG_TRY(knn_buf.reserve((size_t)cap * p.knn_tri));
    // 3 L fixed-point normal sums and, for the exchange, one triangle count
    DWG_TRY(acc.reserve((size_t)L * 3 + 1));
    DWG_CHECK_CUDA(cudaMemsetAsync(acc.ptr, 0, sizeof(long long) * (3 * (size_t)L + 1), s));
    DWG_TRY(is_zero.reserve(L));
    DWG_TRY(zero_count.reserve(1));
    DWG_CHECK_CUDA(cudaMemsetAsync(zero_count.ptr, 0, sizeof(int), s));
    DWG_TRY(iter_dev.reserve(1));
    DWG_TRY(cur_half.reserve(1));
    DWG_TRY(cur_sigma.reserve(1));
    DWG_TRY(iso_dev.reserve(1));
    DWG_TRY(terms_cur.reserve(1));
    DWG_CHECK_CUDA(cudaMemsetAsync(iter_dev.ptr, 0, sizeof(int), s));
    DWG_TRY(ensure_hist(p.total_iter > 0 ? p.total_iter : 1));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    return join_out();
}

// one DWG iteration, src/TurboDWG.cu:516-657, in three phases so that a
// batch of clouds can share one launch for the grid sums
dwg_gwn_params Pipeline::gwn_params() const {
    dwg_gwn_params gp{};
    gp.tile = prm.tile;
    gp.beta = prm.beta;
    gp.sigma = prm.lambda;
    gp.screen = prm.screen;
    gp.screened = 1;
    gp.use_radii = prm.use_radii;
    gp.precision = prm.precision;
    return gp;
}

// grid_lists 2 also keeps the screening weights of every sigma of the
// schedule's first total_iter iterations (20, then lambda and 10)
int Pipeline::weight_slots() const {
    int n = 0;
    if (prm.grid_lists >= 2) {
        float seen[kGwnWeightSlots];
        const int iters = prm.total_iter > 0 ? prm.total_iter : 1;
        for (int t = 0; t < iters && n < kGwnWeightSlots; ++t) {
            const float sg = sigma_at(t, prm.lambda);
            bool dup = false;
            for (int c = 0; c < n; ++c) dup = dup || seen[c] == sg;
            if (!dup) seen[n++] = sg;
        }
    }
    return n;
}

// moments, GWN at the leaves, mean iso
int Pipeline::iterate_pre() {
    k_iter_begin<<<1, 1, 0, s>>>(iter_dev.ptr, sigma_tab.ptr, half_tab.ptr, cur_sigma.ptr, cur_half.ptr,
                                 terms_cur.ptr);
    DWG_CHECK_LAUNCH();
    // UpdateMassNormals (:535)
    k_set_nr<<<div_up(L, 256), 256, 0, s>>>(t2.nr.ptr, leaf_nrm.ptr, nullptr, L);
    DWG_TRY(octree_update_normals(t2, s));
    // screened GWN at the leaves (:536)
    const dwg_gwn_params gp = gwn_params();
    GwnQuery ql;
    ql.q = leaf_pos.ptr;
    ql.nq = L;
    if (prm.grid_lists)
        DWG_TRY(gwn_eval_listed(t2, ql, gp, llist, wleaf.ptr, terms_cur.ptr, s, cur_sigma.ptr, glist_budget,
                                weight_slots()));
    else
        DWG_TRY(gwn_eval(t2, ql, gp, wleaf.ptr, terms_cur.ptr, nullptr, s, cur_sigma.ptr));
    // mean iso value, halved every 5th iteration (:541-550)
    return mean_to_iso(wleaf.ptr, L, iso_dev.ptr, cur_half.ptr, iso_hist.ptr, iter_dev.ptr, partial, s);
}

// screened GWN at the grid (:537)
int Pipeline::iterate_grid() {
    GwnQuery qg;
    for (int d = 0; d < 3; ++d) {
        qg.res[d] = gres[d];
        qg.origin[d] = gorg[d];
    }
    qg.res[2] = gnz;
    qg.zoff = gz0;
    qg.spacing = gh;
    if (prm.grid_lists && !grid_batched)
        return gwn_eval_listed(t2, qg, gwn_params(), glist, field.ptr, terms_cur.ptr, s, cur_sigma.ptr, glist_budget,
                               weight_slots());
    return gwn_eval(t2, qg, gwn_params(), field.ptr, terms_cur.ptr, nullptr, s, cur_sigma.ptr);
}

// marching cubes, kNN, normal update, zero repair
int Pipeline::iterate_post() {
    // marching cubes at the iso value (:554)
    McGrid g;
    for (int d = 0; d < 3; ++d) {
        g.res[d] = gres[d];
        g.origin[d] = gorg[d];
    }
    g.res[2] = gnz;
    g.zoff = gz0;
    g.spacing = gh;
    DWG_TRY(mc_run(field.ptr, g, 0.f, iso_dev.ptr, nullptr, cent.ptr, tnrm.ptr, cap, ntri.ptr, mcws, s));
    // k nearest leaves of every triangle centroid (:560-569)
    KnnQuery q;
    q.q = cent.ptr;
    q.nq = cap;
    q.nq_dev = ntri.ptr;
    DWG_TRY(knn_query(kidx, q, prm.knn_tri, knn_buf.ptr, s));
    // normal scatter + normalise (:571-583); sharded: the scatter of this
    // rank's triangles, the sums of all ranks, then the normalisation
    if (world > 1) {
        DWG_TRY(diffuse_scatter(knn_buf.ptr, tnrm.ptr, cap, ntri.ptr, prm.knn_tri, L, acc.ptr, s));
        DWG_TRY(exchange_sums());
        DWG_TRY(diffuse_finish(L, leaf_nrm.ptr, acc.ptr, is_zero.ptr, zero_count.ptr, s));
    } else {
        DWG_TRY(diffuse_normals(knn_buf.ptr, tnrm.ptr, cap, ntri.ptr, prm.knn_tri, L, leaf_nrm.ptr, acc.ptr,
                                is_zero.ptr, zero_count.ptr, s));
    }
    // zero-normal repair when more than knn_zero points are zero (:585-644)
    DWG_TRY(zero_repair(kidx, leaf_pos.ptr, L, leaf_nrm.ptr, is_zero.ptr, prm.knn_zero, prm.knn_zero, zws, s));
    k_iter_end<<<1, 1, 0, s>>>(iter_dev.ptr, ntri.ptr, cap, zero_count.ptr, terms_cur.ptr, tri_hist.ptr,
                               zero_hist.ptr, terms_hist.ptr);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

// the fixed-point normal sums and the triangle count of all ranks: acc[3L]
// carries this rank's count out and the total back (the exchange is a host
// call, so the stream is drained first)
int Pipeline::exchange_sums() {
    long long* slot = acc.ptr + 3 * (size_t)L;
    k_put_count<<<1, 1, 0, s>>>(ntri.ptr, slot);
    DWG_CHECK_LAUNCH();
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    const int rc = exchange(exchange_user, acc.ptr, 3 * (long long)L + 1, (void*)s);
    DWG_REQUIRE(rc == 0, "pipeline: the exchange of rank %d failed (%d)", rank, rc);
    k_get_count<<<1, 1, 0, s>>>(slot, ntri.ptr);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

int Pipeline::iterate_once() {
    DWG_TRY(iterate_pre());
    DWG_TRY(iterate_grid());
    return iterate_post();
}

int Pipeline::iterate(int n_iters) {
    DWG_REQUIRE(!finalized, "pipeline: already finalized");
    if (n_iters <= 0) return DWG_OK;
    DWG_TRY(ensure_hist(iter + n_iters));
    DWG_TRY(join_in());
    for (int k = 0; k < n_iters; ++k) {
        // a sharded iteration calls the host exchange: no graph
        if (prm.use_graph && iter > 0 && world == 1) {
            if (!graph_exec) {
                DWG_CHECK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                int st = iterate_once();
                cudaGraph_t gr = nullptr;
                cudaError_t e = cudaStreamEndCapture(s, &gr);
                if (st != DWG_OK) {
                    if (gr) cudaGraphDestroy(gr);
                    return st;
                }
                DWG_CHECK_CUDA(e);
                graph = gr;
                DWG_TRY(graph_exec_acquire(graph, &graph_exec));
            }
            DWG_CHECK_CUDA(cudaGraphLaunch(graph_exec, s));
        } else {
            DWG_TRY(iterate_once());
        }
        ++iter;
    }
    return join_out();
}

// final pass, src/TurboDWG.cu:768-924
int Pipeline::finalize() {
    DWG_REQUIRE(!finalized, "pipeline: already finalized");
    DWG_TRY(join_in());
    dwg_gwn_params gp{};
    gp.tile = prm.tile;
    gp.beta = prm.beta;
    gp.sigma = prm.lambda;
    gp.screen = prm.screen;
    gp.screened = 1;
    gp.use_radii = prm.use_radii;
    gp.precision = prm.precision;
    DWG_TRY(final_iso.reserve(1));
    DWG_TRY(final_ntri.reserve(1));
    Octree* tree = nullptr;
    const float* qpts = nullptr;
    long long nqp = 0;
    if (prm.use_leaves_generate == 1) {
        // GenerateMesh(grid_points, ...) from the leaves (src/TurboDWG.cu:768-806)
        DWG_TRY(voxel_grid_host(leaf_pos.ptr, L, 0.01f, prm.final_reso, s, fres, forg, &fh));
        if (prm.use_radii) {
            DevBuf<int> nb;
            DWG_TRY(nb.reserve((size_t)L * prm.final_kw));
            KnnQuery q;
            q.q = leaf_pos.ptr;
            q.nq = L;
            DWG_TRY(knn_query(kidx, q, prm.final_kw, nb.ptr, s));
            DWG_TRY(radii(leaf_pos.ptr, L, nb.ptr, prm.final_kw, leaf_rad.ptr, s));
            DWG_CHECK_CUDA(cudaStreamSynchronize(s));
        }
        k_set_nr<<<div_up(L, 256), 256, 0, s>>>(t2.nr.ptr, leaf_nrm.ptr, leaf_rad.ptr, L);
        DWG_CHECK_LAUNCH();
        tree = &t2;
        qpts = leaf_pos.ptr;
        nqp = L;
        DWG_TRY(point_nrm.reserve((size_t)n * 3));
        DWG_CHECK_CUDA(cudaMemsetAsync(point_nrm.ptr, 0, sizeof(float) * 3 * n, s));
    } else {
        // GenerateMesh(cloud_points, ...) (src/TurboDWG.cu:808-924)
        DWG_TRY(voxel_grid_host(P.ptr, n, prm.offset_2, prm.final_reso, s, fres, forg, &fh));
        DWG_TRY(point_nrm.reserve((size_t)n * 3));
        DWG_TRY(nb_final.reserve((size_t)n * prm.normal_kw));
        KnnQuery q;
        q.q = P.ptr;
        q.nq = n;
        DWG_TRY(knn_query(kidx, q, prm.normal_kw, nb_final.ptr, s));
        DWG_TRY(load_normals(nb_final.ptr, prm.normal_kw, n, leaf_nrm.ptr, point_nrm.ptr, s));
        DWG_TRY(pt_rad.reserve(n));
        k_fill<<<div_up(n, 256), 256, 0, s>>>(pt_rad.ptr, n, prm.screen);
        DWG_CHECK_LAUNCH();
        KnnIndex pix;
        if (prm.use_radii || prm.com_as) DWG_TRY(knn_build(pix, P.ptr, n, s));
        if (prm.com_as) {
            // point areas from the 15 nearest points and the loaded normals
            // (include/DWGProcess.h:783-792), then the moments with these
            // areas (UpdateGWNInfo, src/TurboDWG.cu:931)
            const int ka = n < kAreaK ? n : kAreaK;
            DevBuf<int> nb;
            DWG_TRY(nb.reserve((size_t)n * ka));
            KnnQuery q2;
            q2.q = P.ptr;
            q2.nq = n;
            DWG_TRY(knn_query(pix, q2, ka, nb.ptr, s));
            DWG_TRY(point_areas(P.ptr, n, nb.ptr, ka, point_nrm.ptr, area_pts.ptr, s));
            DWG_TRY(octree_set_point_data(t1, nullptr, area_pts.ptr, nullptr, s));
            DWG_TRY(octree_update_centres(t1, s));
            DWG_CHECK_CUDA(cudaStreamSynchronize(s));
        }
        if (prm.use_radii) {
            DevBuf<int> nb;
            DWG_TRY(nb.reserve((size_t)n * prm.final_kw));
            KnnQuery q2;
            q2.q = P.ptr;
            q2.nq = n;
            DWG_TRY(knn_query(pix, q2, prm.final_kw, nb.ptr, s));
            DWG_TRY(radii(P.ptr, n, nb.ptr, prm.final_kw, pt_rad.ptr, s));
            DWG_CHECK_CUDA(cudaStreamSynchronize(s));
        }
        // OutlierFilter on the points' areas (src/TurboDWG.cu:876, :935), input order
        if (prm.as_thres > 0.f) DWG_TRY(outlier_filter(area_pts.ptr, n, prm.as_thres, s));
        DWG_TRY(octree_set_point_data(t1, point_nrm.ptr, prm.as_thres > 0.f || prm.com_as ? area_pts.ptr : nullptr,
                                      pt_rad.ptr, s));
        DWG_TRY(p_sorted.reserve((size_t)n * 3));
        k_sorted_xyz<<<div_up(n, 256), 256, 0, s>>>(t1.pa.ptr, n, p_sorted.ptr);
        DWG_CHECK_LAUNCH();
        tree = &t1;
        qpts = p_sorted.ptr;
        nqp = n;
    }
    DWG_TRY(octree_update_normals(*tree, s));
    DWG_TRY(wfin.reserve(nqp));
    GwnQuery ql;
    ql.q = qpts;
    ql.nq = nqp;
    DWG_TRY(gwn_eval(*tree, ql, gp, wfin.ptr, nullptr, nullptr, s));
    long long ng = (long long)fres[0] * fres[1] * fres[2];
    DWG_REQUIRE(world <= fres[2] - 1, "pipeline: %d ranks for %d final grid cells in z", world, fres[2] - 1);
    if (world > 1) {
        slab_range(fres[2], rank, world, &fz0, &fnz);
    } else {
        fz0 = 0;
        fnz = fres[2];
    }
    DWG_TRY(final_field.reserve((size_t)fres[0] * fres[1] * fnz));
    GwnQuery qg;
    for (int d = 0; d < 3; ++d) {
        qg.res[d] = fres[d];
        qg.origin[d] = forg[d];
    }
    qg.res[2] = fnz;
    qg.zoff = fz0;
    qg.spacing = fh;
    DWG_TRY(gwn_eval(*tree, qg, gp, final_field.ptr, nullptr, nullptr, s));
    DWG_TRY(mean_to_iso(wfin.ptr, nqp, final_iso.ptr, nullptr, nullptr, nullptr, partial, s));
    final_cap = ng / 2 > 1000000 ? ng / 2 : 1000000;
    DWG_TRY(tris.reserve((size_t)final_cap * 9));
    McGrid g;
    for (int d = 0; d < 3; ++d) {
        g.res[d] = fres[d];
        g.origin[d] = forg[d];
    }
    g.res[2] = fnz;
    g.zoff = fz0;
    g.spacing = fh;
    DWG_TRY(mc_run(final_field.ptr, g, 0.f, final_iso.ptr, tris.ptr, nullptr, nullptr, final_cap, final_ntri.ptr,
                   mcws, s));
    finalized = true;
    return join_out();
}

}  // namespace dwg
