// capi.cu -- extern "C" entry points of libdwg_b200.so (see include/dwg_b200.h).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "batch.cuh"
#include "tune.cuh"

namespace dwg {

static thread_local char g_err[1024] = {0};

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

namespace {
// bytes this library holds per device (pool blocks it has not freed), and
// the memory it could count on when first asked: free then + held then
std::mutex g_mem_mu;
size_t g_live[64] = {0};
size_t g_base[64] = {0};
bool g_have_base[64] = {false};
std::unordered_map<void*, std::pair<int, size_t>> g_sizes;
}  // namespace

size_t device_free_bytes() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    std::lock_guard<std::mutex> lock(g_mem_mu);
    if (!g_have_base[dev]) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) g_base[dev] = fr + g_live[dev];
        g_have_base[dev] = true;
    }
    return g_base[dev] > g_live[dev] ? g_base[dev] - g_live[dev] : 0;
}

namespace {
std::mutex g_recycle_mu;
std::vector<std::pair<int, cudaStream_t>> g_streams;
std::vector<std::pair<int, cudaEvent_t>> g_events;
}  // namespace

cudaStream_t stream_acquire() {
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lock(g_recycle_mu);
        for (size_t i = 0; i < g_streams.size(); ++i)
            if (g_streams[i].first == dev) {
                cudaStream_t s = g_streams[i].second;
                g_streams.erase(g_streams.begin() + (long)i);
                return s;
            }
    }
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    return s;
}

void stream_release(cudaStream_t s) {
    if (!s) return;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(g_recycle_mu);
    if (g_streams.size() < 64) g_streams.emplace_back(dev, s);
    else cudaStreamDestroy(s);
}

cudaEvent_t event_acquire() {
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lock(g_recycle_mu);
        for (size_t i = 0; i < g_events.size(); ++i)
            if (g_events[i].first == dev) {
                cudaEvent_t e = g_events[i].second;
                g_events.erase(g_events.begin() + (long)i);
                return e;
            }
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
    return e;
}

void event_release(cudaEvent_t e) {
    if (!e) return;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(g_recycle_mu);
    if (g_events.size() < 64) g_events.emplace_back(dev, e);
    else cudaEventDestroy(e);
}

namespace {
std::vector<std::pair<int, cudaGraphExec_t>> g_execs;  // guarded by g_recycle_mu
}  // namespace

int graph_exec_acquire(cudaGraph_t g, cudaGraphExec_t* out) {
    int dev = 0;
    DWG_CHECK_CUDA(cudaGetDevice(&dev));
    cudaGraphExec_t e = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_recycle_mu);
        for (size_t i = 0; i < g_execs.size(); ++i)
            if (g_execs[i].first == dev) {
                e = g_execs[i].second;
                g_execs.erase(g_execs.begin() + (long)i);
                break;
            }
    }
    if (e) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(e, g, &info) == cudaSuccess) {
            *out = e;
            return DWG_OK;
        }
        cudaGetLastError();  // another shape: that executable is not reused
        cudaGraphExecDestroy(e);
    }
    DWG_CHECK_CUDA(cudaGraphInstantiate(out, g, 0));
    return DWG_OK;
}

void graph_exec_release(cudaGraphExec_t e) {
    if (!e) return;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(g_recycle_mu);
    if (g_execs.size() < 8) g_execs.emplace_back(dev, e);
    else cudaGraphExecDestroy(e);
}

namespace {
struct FreeState {
    bool active = false, idle = false;
    cudaStream_t stream = nullptr;
};
thread_local FreeState t_free;
std::mutex g_side_mu;
cudaStream_t g_side[64] = {};  // per device: allocations and idle releases (never destroyed)

cudaStream_t side_stream(int dev) {
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_side_mu);
    if (!g_side[dev]) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            unsigned long long keep = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaStream_t s = nullptr;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
        g_side[dev] = s;
    }
    return g_side[dev];
}
}  // namespace

FreeScope::FreeScope(cudaStream_t stream, bool idle)
    : prev_active_(t_free.active), prev_idle_(t_free.idle), prev_stream_(t_free.stream) {
    t_free.active = true;
    t_free.idle = idle;
    t_free.stream = stream;
}

FreeScope::~FreeScope() {
    t_free.active = prev_active_;
    t_free.idle = prev_idle_;
    t_free.stream = prev_stream_;
}

int pool_alloc(void** p, size_t bytes) {
    int dev = 0;
    DWG_CHECK_CUDA(cudaGetDevice(&dev));
    cudaStream_t side = side_stream(dev);
    DWG_REQUIRE(side, "device allocation: no allocation stream on device %d", dev);
    cudaError_t e = cudaMallocAsync(p, bytes, side);
    if (e == cudaSuccess) e = cudaStreamSynchronize(side);  // complete before any stream uses it
    if (e != cudaSuccess) {
        // the code is returned; a failed allocation must not stay behind as
        // the runtime's last error (callers that fall back would meet it at
        // their next launch check)
        if (e == cudaErrorMemoryAllocation) cudaGetLastError();
        set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
        *p = nullptr;
        return e == cudaErrorMemoryAllocation ? DWG_ERR_NOMEM : DWG_ERR_CUDA;
    }
    if (dev >= 0 && dev < 64) {
        std::lock_guard<std::mutex> lock(g_mem_mu);
        g_live[dev] += bytes;
        g_sizes[*p] = {dev, bytes};
    }
    return DWG_OK;
}

void pool_free(void* p) {
    if (!p) return;
    int dev = -1;
    {
        std::lock_guard<std::mutex> lock(g_mem_mu);
        auto it = g_sizes.find(p);
        if (it != g_sizes.end()) {
            dev = it->second.first;
            g_live[dev] -= std::min(g_live[dev], it->second.second);
            g_sizes.erase(it);
        }
    }
    if (t_free.active) {
        cudaStream_t s = t_free.stream;
        if (t_free.idle) {
            if (dev < 0) cudaGetDevice(&dev);
            s = side_stream(dev);
        }
        if (s && cudaFreeAsync(p, s) == cudaSuccess) return;
        cudaGetLastError();
    }
    // wait for every stream's use of the block, then return it to the pool
    if (cudaDeviceSynchronize() != cudaSuccess) return;
    cudaFreeAsync(p, cudaStreamLegacy);
}

}  // namespace dwg

using namespace dwg;

struct dwg_octree {
    Octree t;
    GwnList list;  // interaction lists of dwg_gwn_grid with params->lists
};
struct dwg_knn_index {
    KnnIndex ix;
    // the zero repair's workspace: repairs on the same index start each
    // flagged point's search from its neighbours of the previous repair
    ZeroRepairWs zws;
    DevBuf<float> zpos;  // the points in input order
    bool zpos_ready = false;
};
struct dwg_batch {
    Batch b;
};
struct dwg_mlp {
    Mlp m;
};

#define S(stream) ((cudaStream_t)(stream))

#define API_GUARD(...)                                           \
    try {                                                        \
        __VA_ARGS__                                              \
    } catch (const std::bad_alloc&) {                            \
        set_error("host allocation failed");                     \
        return DWG_ERR_NOMEM;                                    \
    } catch (...) {                                              \
        set_error("unexpected exception");                       \
        return DWG_ERR_INVALID;                                  \
    }

extern "C" {

const char* dwg_last_error(void) { return g_err; }
const char* dwg_version(void) { return "dwg_b200 0.1 (sm_100a)"; }

int dwg_gauss_map_init(const float* points_dev, int n, float* normals_dev, void* stream) {
    API_GUARD(return gauss_map(points_dev, n, normals_dev, S(stream));)
}

int dwg_octree_build(const float* points_dev, int n, int max_depth, const float* areas_dev, void* stream,
                     dwg_octree** out) {
    API_GUARD({
        DWG_REQUIRE(out != nullptr, "octree_build: out is null");
        DWG_REQUIRE(points_dev != nullptr, "octree_build: points are null");
        *out = nullptr;
        dwg_octree* o = new dwg_octree();
        int st = octree_build(o->t, points_dev, n, max_depth, areas_dev, S(stream));
        if (st != DWG_OK) {
            delete o;
            return st;
        }
        *out = o;
        return DWG_OK;
    })
}

int dwg_octree_destroy(dwg_octree* tree) {
    delete tree;
    return DWG_OK;
}

int dwg_octree_num_nodes(const dwg_octree* tree, int* num_nodes) {
    DWG_REQUIRE(tree && num_nodes, "octree_num_nodes: null argument");
    *num_nodes = tree->t.M;
    return DWG_OK;
}

int dwg_octree_update_normals(dwg_octree* tree, const float* normals_dev, const float* areas_dev, void* stream) {
    API_GUARD({
        DWG_REQUIRE(tree && normals_dev, "octree_update_normals: null argument");
        DWG_TRY(octree_set_point_data(tree->t, normals_dev, areas_dev, nullptr, S(stream)));
        return octree_update_normals(tree->t, S(stream));
    })
}

int dwg_octree_update_info(dwg_octree* tree, const float* normals_dev, const float* areas_dev, void* stream) {
    API_GUARD({
        DWG_REQUIRE(tree, "octree_update_info: null tree");
        DWG_TRY(octree_set_point_data(tree->t, normals_dev, areas_dev, nullptr, S(stream)));
        DWG_TRY(octree_update_centres(tree->t, S(stream)));
        tree->list.valid = false;  // new centres: new decisions
        return octree_update_normals(tree->t, S(stream));
    })
}

int dwg_octree_list_size(const dwg_octree* tree, long long* entries, int* weight_slots) {
    API_GUARD({
        DWG_REQUIRE(tree && entries && weight_slots, "octree_list_size: null argument");
        const bool kept = tree->list.valid && !tree->list.too_big;
        *entries = kept ? (long long)tree->list.entries : 0;
        *weight_slots = kept ? tree->list.nslots : 0;
        return DWG_OK;
    });
}

int dwg_octree_status(const dwg_octree* tree, unsigned int* flags) {
    API_GUARD({
        DWG_REQUIRE(tree && flags, "octree_status: null argument");
        DWG_CHECK_CUDA(cudaDeviceSynchronize());
        unsigned int w[2] = {0, 0};
        DWG_CHECK_CUDA(cudaMemcpy(w, tree->t.work.ptr, sizeof(w), cudaMemcpyDeviceToHost));
        *flags = w[1];
        if (w[1]) {
            set_error("octree traversal reported error flags 0x%x", w[1]);
            return DWG_ERR_DEVICE;
        }
        return DWG_OK;
    })
}

int dwg_octree_export(const dwg_octree* tree, int* depth, int* pt_start, int* pt_count, int* skip, double* cm,
                      double* radius, double* ec, int* perm) {
    API_GUARD({
        DWG_REQUIRE(tree, "octree_export: null tree");
        const Octree& t = tree->t;
        DWG_CHECK_CUDA(cudaDeviceSynchronize());
        std::vector<int4> info(t.M);
        DWG_CHECK_CUDA(cudaMemcpy(info.data(), t.info.ptr, sizeof(int4) * t.M, cudaMemcpyDeviceToHost));
        for (int v = 0; v < t.M; ++v) {
            if (depth) depth[v] = info[v].w & 0xff;
            if (pt_start) pt_start[v] = info[v].x;
            if (pt_count) pt_count[v] = info[v].y;
            if (skip) skip[v] = info[v].z;
        }
        if (cm) DWG_CHECK_CUDA(cudaMemcpy(cm, t.cm_d.ptr, sizeof(double) * 3 * t.M, cudaMemcpyDeviceToHost));
        if (radius) DWG_CHECK_CUDA(cudaMemcpy(radius, t.r_d.ptr, sizeof(double) * t.M, cudaMemcpyDeviceToHost));
        if (ec) DWG_CHECK_CUDA(cudaMemcpy(ec, t.ec_d.ptr, sizeof(double) * 3 * t.M, cudaMemcpyDeviceToHost));
        if (perm) DWG_CHECK_CUDA(cudaMemcpy(perm, t.perm.ptr, sizeof(int) * t.n, cudaMemcpyDeviceToHost));
        return DWG_OK;
    })
}

int dwg_octree_expansion(dwg_octree* tree, double* out_host, void* stream) {
    API_GUARD({
        DWG_REQUIRE(tree && out_host, "octree_expansion: null argument");
        Octree& t = tree->t;
        DWG_TRY(octree_update_expansion(t, 2, S(stream)));
        DWG_CHECK_CUDA(cudaMemcpyAsync(out_host, t.ho_d.ptr, sizeof(double) * 36 * t.M, cudaMemcpyDeviceToHost,
                                       S(stream)));
        DWG_CHECK_CUDA(cudaStreamSynchronize(S(stream)));
        return DWG_OK;
    })
}

static int gwn_common(dwg_octree* tree, const float* normals_dev, const float* areas_dev, const float* radii_dev,
                      const GwnQuery& q, const dwg_gwn_params* params, float* out_dev,
                      unsigned long long* terms_dev, int* per_query, void* stream) {
    DWG_REQUIRE(tree && params && out_dev, "gwn: null argument");
    DWG_REQUIRE(params->beta >= 0.f, "gwn: beta must be >= 0");
    DWG_TRY(octree_set_point_data(tree->t, normals_dev, areas_dev, radii_dev, S(stream)));
    if (normals_dev || areas_dev) DWG_TRY(octree_update_normals(tree->t, S(stream)));
    return gwn_eval(tree->t, q, *params, out_dev, terms_dev, per_query, S(stream));
}

int dwg_gwn_points(dwg_octree* tree, const float* normals_dev, const float* areas_dev, const float* radii_dev,
                   const float* queries_dev, long long num_queries, const dwg_gwn_params* params, float* out_dev,
                   unsigned long long* terms_dev, void* stream) {
    API_GUARD({
        DWG_REQUIRE(tree && params && num_queries >= 0 && (queries_dev || num_queries == 0), "gwn_points: bad queries");
        if (num_queries == 0) return DWG_OK;  // an empty query set (its pointers may be null)
        GwnQuery q;
        q.q = queries_dev;
        q.nq = num_queries;
        return gwn_common(tree, normals_dev, areas_dev, radii_dev, q, params, out_dev, terms_dev, nullptr, stream);
    })
}

// per-query term counts (checking the opening decisions)
int dwg_gwn_points_counted(dwg_octree* tree, const float* normals_dev, const float* areas_dev,
                           const float* radii_dev, const float* queries_dev, long long num_queries,
                           const dwg_gwn_params* params, float* out_dev, int* per_query_terms_dev, void* stream) {
    API_GUARD({
        DWG_REQUIRE(tree && params && num_queries >= 0 && (queries_dev || num_queries == 0), "gwn_points: bad queries");
        if (num_queries == 0) return DWG_OK;
        GwnQuery q;
        q.q = queries_dev;
        q.nq = num_queries;
        return gwn_common(tree, normals_dev, areas_dev, radii_dev, q, params, out_dev, nullptr, per_query_terms_dev,
                          stream);
    })
}

int dwg_gwn_grid(dwg_octree* tree, const float* normals_dev, const float* areas_dev, const float* radii_dev,
                 const int res[3], const float origin[3], float spacing, const dwg_gwn_params* params,
                 float* out_dev, unsigned long long* terms_dev, void* stream) {
    API_GUARD({
        DWG_REQUIRE(res && origin, "gwn_grid: null grid");
        GwnQuery q;
        for (int d = 0; d < 3; ++d) {
            q.res[d] = res[d];
            q.origin[d] = origin[d];
        }
        q.spacing = spacing;
        if (params && params->lists && params->screened && params->order == 0) {
            DWG_REQUIRE(tree && out_dev, "gwn_grid: null argument");
            DWG_TRY(octree_set_point_data(tree->t, normals_dev, areas_dev, radii_dev, S(stream)));
            // kept screening weights use the points' radii (use_radii): new
            // radii make them stale
            if (radii_dev) DWG_TRY(gwn_list_drop_weights(tree->list, S(stream)));
            if (normals_dev || areas_dev) DWG_TRY(octree_update_normals(tree->t, S(stream)));
            return gwn_eval_listed(tree->t, q, *params, tree->list, out_dev, terms_dev, S(stream), nullptr, 0,
                                   params->lists >= 2 ? 2 : 0);
        }
        return gwn_common(tree, normals_dev, areas_dev, radii_dev, q, params, out_dev, terms_dev, nullptr, stream);
    })
}

static int gwn_thread_common(dwg_octree* tree, const float* normals_dev, const float* areas_dev,
                             const float* radii_dev, const GwnQuery& q, const dwg_gwn_params* params, bool fp64,
                             void* out_w, void* out_g, void* stream) {
    DWG_REQUIRE(tree && params && (out_w || out_g), "gwn: null argument");
    DWG_TRY(octree_set_point_data(tree->t, normals_dev, areas_dev, radii_dev, S(stream)));
    if (normals_dev || areas_dev) DWG_TRY(octree_update_normals(tree->t, S(stream)));
    return gwn_eval_thread(tree->t, q, *params, fp64, out_w, out_g, S(stream));
}

int dwg_gwn_points_grad(dwg_octree* tree, const float* normals_dev, const float* areas_dev, const float* radii_dev,
                        const float* queries_dev, long long num_queries, const dwg_gwn_params* params,
                        float* out_dev, float* grad_dev, void* stream) {
    API_GUARD({
        DWG_REQUIRE(num_queries >= 0 && (queries_dev || num_queries == 0), "gwn_points_grad: bad queries");
        if (num_queries == 0) return DWG_OK;
        GwnQuery q;
        q.q = queries_dev;
        q.nq = num_queries;
        return gwn_thread_common(tree, normals_dev, areas_dev, radii_dev, q, params, false, out_dev, grad_dev, stream);
    })
}

int dwg_gwn_points_fp64(dwg_octree* tree, const float* normals_dev, const float* areas_dev, const float* radii_dev,
                        const float* queries_dev, long long num_queries, const dwg_gwn_params* params,
                        double* out_dev, double* grad_dev, void* stream) {
    API_GUARD({
        DWG_REQUIRE(num_queries >= 0 && (queries_dev || num_queries == 0), "gwn_points_fp64: bad queries");
        if (num_queries == 0) return DWG_OK;
        GwnQuery q;
        q.q = queries_dev;
        q.nq = num_queries;
        return gwn_thread_common(tree, normals_dev, areas_dev, radii_dev, q, params, true, out_dev, grad_dev, stream);
    })
}

static int grid_query(const int res[3], const float origin[3], float spacing, GwnQuery& q) {
    DWG_REQUIRE(res && origin, "gwn_grid: null grid");
    for (int d = 0; d < 3; ++d) {
        q.res[d] = res[d];
        q.origin[d] = origin[d];
    }
    q.spacing = spacing;
    return DWG_OK;
}

int dwg_gwn_grid_grad(dwg_octree* tree, const float* normals_dev, const float* areas_dev, const float* radii_dev,
                      const int res[3], const float origin[3], float spacing, const dwg_gwn_params* params,
                      float* out_dev, float* grad_dev, void* stream) {
    API_GUARD({
        GwnQuery q;
        DWG_TRY(grid_query(res, origin, spacing, q));
        return gwn_thread_common(tree, normals_dev, areas_dev, radii_dev, q, params, false, out_dev, grad_dev, stream);
    })
}

int dwg_gwn_grid_fp64(dwg_octree* tree, const float* normals_dev, const float* areas_dev, const float* radii_dev,
                      const int res[3], const float origin[3], float spacing, const dwg_gwn_params* params,
                      double* out_dev, double* grad_dev, void* stream) {
    API_GUARD({
        GwnQuery q;
        DWG_TRY(grid_query(res, origin, spacing, q));
        return gwn_thread_common(tree, normals_dev, areas_dev, radii_dev, q, params, true, out_dev, grad_dev, stream);
    })
}

int dwg_voxel_grid(const float* points_dev, int n, float offset, int s, void* stream, int res[3], float origin[3],
                   float* spacing) {
    API_GUARD({
        DWG_REQUIRE(res && origin && spacing, "voxel_grid: null output");
        return voxel_grid_host(points_dev, n, offset, s, S(stream), res, origin, spacing);
    })
}

int dwg_marching_cubes(const float* field_dev, const int res[3], const float* positions_dev, const float origin[3],
                       float spacing, float iso, float* tris_dev, float* centroids_dev, float* normals_dev,
                       long long capacity, unsigned long long* num_tris_dev, long long* num_tris_host, void* stream) {
    API_GUARD({
        DWG_REQUIRE(res && (origin || positions_dev), "marching_cubes: grid undefined");
        DWG_REQUIRE(capacity >= 0, "marching_cubes: negative capacity");
        McGrid g;
        for (int d = 0; d < 3; ++d) {
            g.res[d] = res[d];
            g.origin[d] = origin ? origin[d] : 0.f;
        }
        g.spacing = spacing;
        g.positions = positions_dev;
        static thread_local McWorkspace ws;
        DevBuf<unsigned long long> own;
        unsigned long long* cnt = num_tris_dev;
        if (!cnt) {
            DWG_TRY(own.reserve(1));
            cnt = own.ptr;
        }
        DWG_TRY(mc_run(field_dev, g, iso, nullptr, tris_dev, centroids_dev, normals_dev, capacity, cnt, ws,
                       S(stream)));
        if (num_tris_host || !num_tris_dev) {
            unsigned long long T = 0;
            DWG_CHECK_CUDA(cudaMemcpyAsync(&T, cnt, sizeof(T), cudaMemcpyDeviceToHost, S(stream)));
            DWG_CHECK_CUDA(cudaStreamSynchronize(S(stream)));
            if (num_tris_host) *num_tris_host = (long long)T;
            if ((long long)T > capacity) {
                set_error("marching_cubes: %llu triangles exceed capacity %lld", T, capacity);
                return DWG_ERR_OVERFLOW;
            }
        }
        return DWG_OK;
    })
}

int dwg_mc_tables(int* edge_table_host, signed char* tri_table_host) {
    DWG_REQUIRE(edge_table_host && tri_table_host, "mc_tables: null output");
    DWG_REQUIRE(mc_tables_host(edge_table_host, tri_table_host), "mc_tables: a case's triangles do not match its polygons");
    return DWG_OK;
}

int dwg_knn_build(const float* points_dev, int n, void* stream, dwg_knn_index** out) {
    API_GUARD({
        DWG_REQUIRE(out, "knn_build: out is null");
        *out = nullptr;
        dwg_knn_index* o = new dwg_knn_index();
        int st = knn_build(o->ix, points_dev, n, S(stream));
        if (st != DWG_OK) {
            delete o;
            return st;
        }
        *out = o;
        return DWG_OK;
    })
}

int dwg_knn_destroy(dwg_knn_index* index) {
    delete index;
    return DWG_OK;
}

int dwg_knn_query(dwg_knn_index* index, const float* queries_dev, long long num_queries, int k, int* out_dev,
                  void* stream) {
    API_GUARD({
        DWG_REQUIRE(index && num_queries >= 0 && ((queries_dev && out_dev) || num_queries == 0),
                    "knn_query: null argument");
        DWG_REQUIRE(k >= 1 && k <= index->ix.n, "knn_query: k=%d outside [1, %d points]", k, index->ix.n);
        if (num_queries == 0) return DWG_OK;  // an empty query set (its pointers may be null)
        KnnQuery q;
        q.q = queries_dev;
        q.nq = num_queries;
        return knn_query(index->ix, q, k, out_dev, S(stream));
    })
}

int dwg_knn(const float* points_dev, int n, const float* queries_dev, long long num_queries, int k, int* out_dev,
            void* stream) {
    API_GUARD({
        DWG_REQUIRE(k >= 1 && k <= n, "knn: k=%d must be in [1, n=%d]", k, n);
        KnnIndex ix;
        DWG_TRY(knn_build(ix, points_dev, n, S(stream)));
        KnnQuery q;
        q.q = queries_dev;
        q.nq = num_queries;
        DWG_TRY(knn_query(ix, q, k, out_dev, S(stream)));
        DWG_CHECK_CUDA(cudaStreamSynchronize(S(stream)));
        return DWG_OK;
    })
}

int dwg_diffuse_normals(const int* knn_dev, const float* tri_normals_dev, long long num_tris, int k, int num_points,
                        float* normals_dev, unsigned char* is_zero_dev, int* zero_count_dev, void* stream) {
    API_GUARD({
        DevBuf<long long> acc;
        DWG_TRY(acc.reserve((size_t)num_points * 3));
        DWG_CHECK_CUDA(cudaMemsetAsync(acc.ptr, 0, sizeof(long long) * 3 * num_points, S(stream)));
        DWG_TRY(diffuse_normals(knn_dev, tri_normals_dev, num_tris, nullptr, k, num_points, normals_dev, acc.ptr,
                                is_zero_dev, zero_count_dev, S(stream)));
        DWG_CHECK_CUDA(cudaStreamSynchronize(S(stream)));
        return DWG_OK;
    })
}

int dwg_zero_repair(dwg_knn_index* index, float* normals_dev, const unsigned char* is_zero_dev,
                    const int* zero_count_dev, int k, int min_zero, void* stream) {
    API_GUARD({
        DWG_REQUIRE(index, "zero_repair: null index");
        (void)zero_count_dev;
        // positions in input order are needed for the query side (once per
        // index: an index's points do not change)
        DevBuf<float>& pos = index->zpos;
        if (!index->zpos_ready) {
            DWG_TRY(pos.reserve((size_t)index->ix.n * 3));
            std::vector<float4> h(index->ix.n);
            std::vector<float> hp((size_t)index->ix.n * 3);
            DWG_CHECK_CUDA(cudaMemcpyAsync(h.data(), index->ix.pts.ptr, sizeof(float4) * index->ix.n,
                                           cudaMemcpyDeviceToHost, S(stream)));
            DWG_CHECK_CUDA(cudaStreamSynchronize(S(stream)));
            for (int j = 0; j < index->ix.n; ++j) {
                int id;
                memcpy(&id, &h[j].w, 4);
                hp[(size_t)id * 3] = h[j].x;
                hp[(size_t)id * 3 + 1] = h[j].y;
                hp[(size_t)id * 3 + 2] = h[j].z;
            }
            DWG_CHECK_CUDA(cudaMemcpyAsync(pos.ptr, hp.data(), sizeof(float) * hp.size(), cudaMemcpyHostToDevice,
                                           S(stream)));
            DWG_CHECK_CUDA(cudaStreamSynchronize(S(stream)));
            index->zpos_ready = true;
        }
        DWG_TRY(zero_repair(index->ix, pos.ptr, index->ix.n, normals_dev, is_zero_dev, k, min_zero, index->zws,
                            S(stream)));
        DWG_CHECK_CUDA(cudaStreamSynchronize(S(stream)));
        return DWG_OK;
    })
}

int dwg_load_normals(const int* knn_dev, int k, long long num_queries, const float* leaf_normals_dev, float* out_dev,
                     void* stream) {
    API_GUARD(return load_normals(knn_dev, k, num_queries, leaf_normals_dev, out_dev, S(stream));)
}

int dwg_radii(const float* points_dev, int n, const int* knn_dev, int k, float* radii_dev, void* stream) {
    API_GUARD(return radii(points_dev, n, knn_dev, k, radii_dev, S(stream));)
}

int dwg_pca_normals(const float* points_dev, int n, const int* knn_dev, int k, const float* view_host,
                    float* normals_dev, void* stream) {
    API_GUARD({
        DWG_REQUIRE(view_host, "pca_normals: null viewpoint");
        DevBuf<float> view;
        DWG_TRY(view.reserve(3));
        DWG_CHECK_CUDA(cudaMemcpyAsync(view.ptr, view_host, sizeof(float) * 3, cudaMemcpyHostToDevice, S(stream)));
        DWG_TRY(pca_normals(points_dev, n, knn_dev, k, view.ptr, normals_dev, S(stream)));
        DWG_CHECK_CUDA(cudaStreamSynchronize(S(stream)));
        return DWG_OK;
    })
}

int dwg_point_areas(const float* points_dev, int n, const int* knn_dev, int k, const float* normals_dev,
                    float* areas_dev, void* stream) {
    API_GUARD(return point_areas(points_dev, n, knn_dev, k, normals_dev, areas_dev, S(stream));)
}

void dwg_params_default(dwg_params* p) {
    if (!p) return;
    p->in_normal = 3;
    p->grid_reso = 400;
    p->final_reso = 500;
    p->kw = 10;
    p->final_kw = 10;
    p->normal_kw = 10;
    p->max_depth = 10;
    p->lambda = 10.f;
    p->min_num = 0;
    p->use_radii = 0;
    p->offset_1 = 0.05f;
    p->offset_2 = 0.01f;
    p->use_leaves_generate = 0;
    p->total_iter = 40;
    p->beta = 2.3f;
    p->area = 2e-6f;
    p->screen = 0.0015f;
    p->knn_tri = 15;
    p->knn_zero = 10;
    p->precision = 1;
    p->use_graph = 1;
    p->tile = 0;
    p->as_thres = 0.f;
    p->com_as = 0;
    p->grid_lists = 2;
}

int dwg_pipeline_create(const float* points_dev, const float* normals_dev, int n, const dwg_params* params,
                        void* stream, dwg_pipeline** out) {
    API_GUARD({
        DWG_REQUIRE(out && params, "pipeline_create: null argument");
        *out = nullptr;
        dwg_pipeline* o = new dwg_pipeline();
        int st = o->p.setup(points_dev, normals_dev, n, *params, S(stream));
        if (st != DWG_OK) {
            delete o;
            return st;
        }
        *out = o;
        return DWG_OK;
    })
}

int dwg_pipeline_create_sharded(const float* points_dev, const float* normals_dev, int n, const dwg_params* params,
                                int rank, int world, dwg_exchange_fn exchange, void* user, void* stream,
                                dwg_pipeline** out) {
    API_GUARD({
        DWG_REQUIRE(out && params, "pipeline_create_sharded: null argument");
        DWG_REQUIRE(world >= 1 && rank >= 0 && rank < world, "pipeline_create_sharded: bad rank %d of %d", rank,
                    world);
        *out = nullptr;
        dwg_pipeline* o = new dwg_pipeline();
        o->p.rank = rank;
        o->p.world = world;
        o->p.exchange = exchange;
        o->p.exchange_user = user;
        int st = o->p.setup(points_dev, normals_dev, n, *params, S(stream));
        if (st != DWG_OK) {
            delete o;
            return st;
        }
        *out = o;
        return DWG_OK;
    })
}

int dwg_slab_range(int samples, int rank, int world, int* z0, int* nz) {
    API_GUARD({
        DWG_REQUIRE(z0 && nz && world >= 1 && rank >= 0 && rank < world && samples - 1 >= world,
                    "slab_range: bad arguments (samples %d, rank %d of %d)", samples, rank, world);
        slab_range(samples, rank, world, z0, nz);
        return DWG_OK;
    })
}

int dwg_pipeline_destroy(dwg_pipeline* p) {
    if (!p) return DWG_OK;
    // the pipeline's stream is the only one its buffers were used on (the
    // caller's stream joins it through events): once it is drained, every
    // block goes back to the pool at once, without waiting on other streams
    cudaStreamSynchronize(p->p.s);
    FreeScope idle(nullptr, true);
    delete p;
    return DWG_OK;
}

int dwg_pipeline_iterate(dwg_pipeline* p, int n_iters) {
    API_GUARD({
        DWG_REQUIRE(p, "pipeline_iterate: null pipeline");
        return p->p.iterate(n_iters);
    })
}

int dwg_pipeline_finalize(dwg_pipeline* p) {
    API_GUARD({
        DWG_REQUIRE(p, "pipeline_finalize: null pipeline");
        return p->p.finalize();
    })
}

int dwg_pipeline_size(dwg_pipeline* p, const char* what, long long* value) {
    API_GUARD({
        DWG_REQUIRE(p && what && value, "pipeline_size: null argument");
        Pipeline& q = p->p;
        if (!strcmp(what, "leaves"))
            *value = q.L;
        else if (!strcmp(what, "points"))
            *value = q.n;
        else if (!strcmp(what, "iterations"))
            *value = q.iter;
        else if (!strcmp(what, "grid"))  // this rank's slab (the whole grid on one GPU)
            *value = (long long)q.gres[0] * q.gres[1] * q.gnz;
        else if (!strcmp(what, "final_grid"))
            *value = (long long)q.fres[0] * q.fres[1] * q.fnz;
        else if (!strcmp(what, "grid_list_entries"))  // 0: the grid is traversed
            *value = q.glist.valid && !q.glist.too_big ? (long long)q.glist.entries : 0;
        else if (!strcmp(what, "grid_weight_slots"))
            *value = q.glist.valid && !q.glist.too_big ? q.glist.nslots : 0;
        else if (!strcmp(what, "triangles")) {
            DWG_REQUIRE(q.finalized, "pipeline_size: not finalized");
            unsigned long long T = 0;
            DWG_CHECK_CUDA(cudaMemcpyAsync(&T, q.final_ntri.ptr, sizeof(T), cudaMemcpyDeviceToHost, q.s));
            DWG_CHECK_CUDA(cudaStreamSynchronize(q.s));
            *value = (long long)T < q.final_cap ? (long long)T : q.final_cap;
        } else {
            set_error("pipeline_size: unknown item '%s'", what);
            return DWG_ERR_INVALID;
        }
        return DWG_OK;
    })
}

int dwg_pipeline_get(dwg_pipeline* p, const char* what, void* dst) {
    API_GUARD({
        DWG_REQUIRE(p && what && dst, "pipeline_get: null argument");
        Pipeline& q = p->p;
        DWG_CHECK_CUDA(cudaStreamSynchronize(q.s));
        auto cp = [&](const void* src, size_t bytes) -> int {
            DWG_CHECK_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
            return DWG_OK;
        };
        const int it = q.iter;
        if (!strcmp(what, "leaf_pos")) return cp(q.leaf_pos.ptr, sizeof(float) * 3 * q.L);
        if (!strcmp(what, "leaf_nrm")) return cp(q.leaf_nrm.ptr, sizeof(float) * 3 * q.L);
        if (!strcmp(what, "iso")) return it ? cp(q.iso_hist.ptr, sizeof(float) * it) : DWG_OK;
        if (!strcmp(what, "tri_count")) return it ? cp(q.tri_hist.ptr, sizeof(long long) * it) : DWG_OK;
        if (!strcmp(what, "zero_count")) return it ? cp(q.zero_hist.ptr, sizeof(int) * it) : DWG_OK;
        if (!strcmp(what, "terms")) return it ? cp(q.terms_hist.ptr, sizeof(unsigned long long) * it) : DWG_OK;
        if (!strcmp(what, "field")) return cp(q.field.ptr, sizeof(float) * q.gres[0] * q.gres[1] * (size_t)q.gnz);
        if (!strcmp(what, "slab")) {
            const int v[4] = {q.gz0, q.gnz, q.fz0, q.fnz};
            memcpy(dst, v, sizeof(v));
            return DWG_OK;
        }
        if (!strcmp(what, "grid_res")) {
            memcpy(dst, q.gres, sizeof(q.gres));
            return DWG_OK;
        }
        if (!strcmp(what, "grid_origin")) {
            float v[4] = {q.gorg[0], q.gorg[1], q.gorg[2], q.gh};
            memcpy(dst, v, sizeof(v));
            return DWG_OK;
        }
        DWG_REQUIRE(q.finalized, "pipeline_get: '%s' needs finalize()", what);
        if (!strcmp(what, "point_nrm")) return cp(q.point_nrm.ptr, sizeof(float) * 3 * q.n);
        if (!strcmp(what, "final_field"))
            return cp(q.final_field.ptr, sizeof(float) * q.fres[0] * q.fres[1] * (size_t)q.fnz);
        if (!strcmp(what, "final_iso")) return cp(q.final_iso.ptr, sizeof(float));
        if (!strcmp(what, "final_res")) {
            memcpy(dst, q.fres, sizeof(q.fres));
            return DWG_OK;
        }
        if (!strcmp(what, "final_origin")) {
            float v[4] = {q.forg[0], q.forg[1], q.forg[2], q.fh};
            memcpy(dst, v, sizeof(v));
            return DWG_OK;
        }
        if (!strcmp(what, "tris")) {
            unsigned long long T = 0;
            DWG_CHECK_CUDA(cudaMemcpy(&T, q.final_ntri.ptr, sizeof(T), cudaMemcpyDeviceToHost));
            long long t = (long long)T < q.final_cap ? (long long)T : q.final_cap;
            return t ? cp(q.tris.ptr, sizeof(float) * 9 * (size_t)t) : DWG_OK;
        }
        set_error("pipeline_get: unknown item '%s'", what);
        return DWG_ERR_INVALID;
    })
}

int dwg_pipeline_device_ptr(dwg_pipeline* p, const char* what, void** ptr) {
    DWG_REQUIRE(p && what && ptr, "pipeline_device_ptr: null argument");
    Pipeline& q = p->p;
    if (!strcmp(what, "leaf_pos")) *ptr = q.leaf_pos.ptr;
    else if (!strcmp(what, "leaf_nrm")) *ptr = q.leaf_nrm.ptr;
    else if (!strcmp(what, "point_nrm")) *ptr = q.point_nrm.ptr;
    else if (!strcmp(what, "tris")) *ptr = q.tris.ptr;
    else if (!strcmp(what, "field")) *ptr = q.field.ptr;
    else if (!strcmp(what, "final_field")) *ptr = q.final_field.ptr;
    else {
        set_error("pipeline_device_ptr: unknown item '%s'", what);
        return DWG_ERR_INVALID;
    }
    return DWG_OK;
}

int dwg_batch_create(const float* const* points_dev, const int* counts, int num_clouds, const dwg_params* params,
                     void* stream, dwg_batch** out) {
    API_GUARD({
        DWG_REQUIRE(out && points_dev && counts && params && num_clouds >= 1, "batch_create: bad arguments");
        *out = nullptr;
        dwg_batch* o = new dwg_batch();
        int st = o->b.setup(points_dev, counts, num_clouds, params, S(stream));
        if (st != DWG_OK) {
            delete o;
            return st;
        }
        *out = o;
        return DWG_OK;
    })
}

int dwg_batch_destroy(dwg_batch* b) {
    delete b;
    return DWG_OK;
}

int dwg_batch_iterate(dwg_batch* b, int n_iters) {
    API_GUARD({
        DWG_REQUIRE(b, "batch_iterate: null batch");
        return b->b.iterate(n_iters);
    })
}

int dwg_batch_finalize(dwg_batch* b) {
    API_GUARD({
        DWG_REQUIRE(b, "batch_finalize: null batch");
        return b->b.finalize();
    })
}

int dwg_batch_cloud(dwg_batch* b, int index, dwg_pipeline** cloud) {
    API_GUARD({
        DWG_REQUIRE(b && cloud, "batch_cloud: null argument");
        DWG_REQUIRE(index >= 0 && index < (int)b->b.clouds.size(), "batch_cloud: index %d out of range", index);
        *cloud = b->b.clouds[index].get();
        return DWG_OK;
    })
}

int dwg_autotune(const float* points_dev, int n, const dwg_params* params, float tol, int samples, int warm_iters,
                 void* stream, dwg_tune_result* out) {
    API_GUARD({
        DWG_REQUIRE(points_dev && params && out && n >= 2, "autotune: bad arguments");
        return autotune(points_dev, n, *params, tol, samples, warm_iters, S(stream), out);
    })
}

long long dwg_mlp_param_count(void) { return mlp_param_count(); }

int dwg_mlp_create(unsigned long long seed, void* stream, dwg_mlp** out) {
    API_GUARD({
        DWG_REQUIRE(out, "mlp_create: out is null");
        *out = nullptr;
        dwg_mlp* o = new dwg_mlp();
        int st = mlp_init(o->m, seed, S(stream));
        if (st != DWG_OK) {
            delete o;
            return st;
        }
        *out = o;
        return DWG_OK;
    })
}

int dwg_mlp_destroy(dwg_mlp* m) {
    delete m;
    return DWG_OK;
}

int dwg_mlp_set_params(dwg_mlp* m, const float* params_host, long long count) {
    API_GUARD({
        DWG_REQUIRE(m && params_host, "mlp_set_params: null argument");
        DWG_REQUIRE(count == mlp_param_count(), "mlp_set_params: count %lld != %lld", count, mlp_param_count());
        return mlp_set_flat(m->m, params_host, 0);
    })
}

int dwg_mlp_get_params(dwg_mlp* m, float* params_host, long long count) {
    API_GUARD({
        DWG_REQUIRE(m && params_host, "mlp_get_params: null argument");
        DWG_REQUIRE(count == mlp_param_count(), "mlp_get_params: count %lld != %lld", count, mlp_param_count());
        return mlp_get_flat(m->m, params_host, 0);
    })
}

static const char kMlpMagic[8] = {'D', 'W', 'G', 'M', 'L', 'P', '0', '1'};

int dwg_mlp_load(dwg_mlp* m, const char* path) {
    API_GUARD({
        DWG_REQUIRE(m && path, "mlp_load: null argument");
        FILE* f = fopen(path, "rb");
        DWG_REQUIRE(f, "mlp_load: cannot open %s", path);
        char magic[8];
        long long count = 0;
        const long long want = mlp_param_count();
        std::vector<float> buf((size_t)want);
        bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, kMlpMagic, 8) == 0 &&
                  fread(&count, sizeof(count), 1, f) == 1 && count == want &&
                  fread(buf.data(), sizeof(float), (size_t)want, f) == (size_t)want;
        fclose(f);
        DWG_REQUIRE(ok, "mlp_load: %s is not a parameter file of %lld floats", path, want);
        for (float v : buf) DWG_REQUIRE(std::isfinite(v), "mlp_load: %s holds a non-finite parameter", path);
        return mlp_set_flat(m->m, buf.data(), 0);
    })
}

int dwg_mlp_save(dwg_mlp* m, const char* path) {
    API_GUARD({
        DWG_REQUIRE(m && path, "mlp_save: null argument");
        const long long count = mlp_param_count();
        std::vector<float> buf((size_t)count);
        DWG_TRY(mlp_get_flat(m->m, buf.data(), 0));
        FILE* f = fopen(path, "wb");
        DWG_REQUIRE(f, "mlp_save: cannot create %s", path);
        bool ok = fwrite(kMlpMagic, 1, 8, f) == 8 && fwrite(&count, sizeof(count), 1, f) == 1 &&
                  fwrite(buf.data(), sizeof(float), (size_t)count, f) == (size_t)count;
        ok = (fclose(f) == 0) && ok;
        DWG_REQUIRE(ok, "mlp_save: write to %s failed", path);
        return DWG_OK;
    })
}

int dwg_mlp_features(const float* points_dev, int n, float* features_dev, void* stream) {
    API_GUARD({
        DWG_REQUIRE(points_dev && features_dev && n >= 2, "mlp_features: bad arguments (n=%d)", n);
        KnnIndex ix;
        DWG_TRY(knn_build(ix, points_dev, n, S(stream)));
        return mlp_features(ix, points_dev, n, features_dev, S(stream));
    })
}

int dwg_mlp_forward(dwg_mlp* m, const float* features_dev, long long n, float* out_dev, void* stream) {
    API_GUARD({
        DWG_REQUIRE(m && features_dev && out_dev && n >= 0, "mlp_forward: bad arguments");
        DWG_TRY(mlp_forward(m->m, features_dev, n, out_dev, S(stream)));
        DWG_CHECK_CUDA(cudaStreamSynchronize(S(stream)));
        return DWG_OK;
    })
}

int dwg_mlp_gradients(dwg_mlp* m, const float* features_dev, const float* targets_dev, long long n,
                      float* loss_host, float* grads_host, long long count, void* stream) {
    API_GUARD({
        DWG_REQUIRE(m && features_dev && targets_dev && grads_host && n >= 1, "mlp_gradients: bad arguments");
        DWG_REQUIRE(count == mlp_param_count(), "mlp_gradients: count %lld != %lld", count, mlp_param_count());
        DWG_TRY(mlp_backward(m->m, features_dev, targets_dev, n, loss_host, S(stream)));
        return mlp_get_grads_flat(m->m, grads_host, S(stream));
    })
}

int dwg_mlp_train_step(dwg_mlp* m, const float* features_dev, const float* targets_dev, long long n, float lr,
                       float* loss_host, void* stream) {
    API_GUARD({
        DWG_REQUIRE(m && features_dev && targets_dev && n >= 1, "mlp_train_step: bad arguments");
        DWG_REQUIRE(lr > 0.f && std::isfinite(lr), "mlp_train_step: learning rate must be positive");
        DWG_TRY(mlp_backward(m->m, features_dev, targets_dev, n, loss_host, S(stream)));
        DWG_TRY(mlp_adam(m->m, lr, 0.9f, 0.999f, 1e-8f, S(stream)));
        DWG_CHECK_CUDA(cudaStreamSynchronize(S(stream)));
        return DWG_OK;
    })
}

int dwg_mlp_init_normals(dwg_mlp* m, const float* points_dev, int n, float* normals_dev, void* stream) {
    API_GUARD({
        DWG_REQUIRE(m && points_dev && normals_dev && n >= 2, "mlp_init_normals: bad arguments (n=%d)", n);
        KnnIndex ix;
        DWG_TRY(knn_build(ix, points_dev, n, S(stream)));
        return mlp_init_normals(m->m, ix, points_dev, n, normals_dev, S(stream));
    })
}

int dwg_pipeline_create_learned(const float* points_dev, int n, const dwg_params* params, dwg_mlp* init,
                                void* stream, dwg_pipeline** out) {
    API_GUARD({
        DWG_REQUIRE(out && params && init, "pipeline_create_learned: null argument");
        DWG_REQUIRE(params->in_normal == 4, "pipeline_create_learned: params->in_normal must be 4");
        *out = nullptr;
        dwg_pipeline* o = new dwg_pipeline();
        o->p.init_mlp = &init->m;
        int st = o->p.setup(points_dev, nullptr, n, *params, S(stream));
        o->p.init_mlp = nullptr;
        if (st != DWG_OK) {
            delete o;
            return st;
        }
        *out = o;
        return DWG_OK;
    })
}

int dwg_reconstruct_host(const float* points_host, const float* normals_host, int n, const dwg_params* params,
                         float* point_normals_host, float* tris_host, long long tri_capacity, long long* num_tris,
                         void* stream) {
    API_GUARD({
        DWG_REQUIRE(points_host && params && n >= 2, "reconstruct_host: bad arguments");
        cudaStream_t st = S(stream);
        DevBuf<float> P, N;
        DWG_TRY(P.reserve((size_t)n * 3));
        DWG_CHECK_CUDA(cudaMemcpyAsync(P.ptr, points_host, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st));
        if (normals_host) {
            DWG_TRY(N.reserve((size_t)n * 3));
            DWG_CHECK_CUDA(cudaMemcpyAsync(N.ptr, normals_host, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st));
        }
        dwg_pipeline* p = nullptr;
        DWG_TRY(dwg_pipeline_create(P.ptr, normals_host ? N.ptr : nullptr, n, params, stream, &p));
        int rc = dwg_pipeline_iterate(p, params->total_iter);
        if (rc == DWG_OK) rc = dwg_pipeline_finalize(p);
        long long T = 0;
        if (rc == DWG_OK) rc = dwg_pipeline_size(p, "triangles", &T);
        if (rc == DWG_OK && point_normals_host && !params->use_leaves_generate)
            rc = dwg_pipeline_get(p, "point_nrm", point_normals_host);
        if (rc == DWG_OK && num_tris) *num_tris = T;
        if (rc == DWG_OK && tris_host && T > 0) {
            long long c = T < tri_capacity ? T : tri_capacity;
            if (c > 0) {
                cudaError_t e = cudaMemcpy(tris_host, p->p.tris.ptr, sizeof(float) * 9 * (size_t)c,
                                           cudaMemcpyDeviceToHost);
                if (e != cudaSuccess) {
                    set_error("reconstruct_host: copy failed: %s", cudaGetErrorString(e));
                    rc = DWG_ERR_CUDA;
                }
            }
            if (rc == DWG_OK && T > tri_capacity) {
                set_error("reconstruct_host: %lld triangles exceed capacity %lld", T, tri_capacity);
                rc = DWG_ERR_OVERFLOW;
            }
        }
        dwg_pipeline_destroy(p);
        return rc;
    })
}

// the file readers and writers are in io.cu

}  // extern "C"
