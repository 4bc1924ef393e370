// knn.cu -- exact kNN over a uniform cell grid.
//
// The reference builds a left-balanced kd-tree with log2(N) thrust sorts and
// walks it per query with a 30-entry stack (src/KNN_GWN.cu:42-66,490-715,
// include/cudaKDTree/cukd/traverse-cct.h:25-101).  Point clouds here are
// surfaces, so a uniform grid sized for ~3 points per occupied cell is built
// with one counting sort (histogram, scan, scatter), and each query visits
// Chebyshev shells of cells around its own cell until the k-th candidate is
// closer than anything outside the visited block.  Candidates are ranked by
// the cukd key (float bits of dist^2) << 32 | index
// (include/cudaKDTree/cukd/knn.h:279-282), with dist^2 = (dx*dx + dy*dy) + dz*dz
// in round-to-nearest single precision, and kept sorted in registers.
#include <cub/cub.cuh>

#include <climits>

#include "knn.cuh"
#include "octree.cuh"

namespace dwg {

struct KnnGrid {
    int G0, G1, G2;
    float lo0, lo1, lo2, h, inv_h;
};

__device__ __forceinline__ int cell_coord(float p, float lo, float inv_h, int G) {
    int c = (int)floorf(__fmul_rn(__fsub_rn(p, lo), inv_h));
    return c < 0 ? 0 : (c >= G ? G - 1 : c);
}

__global__ void k_knn_hist(const float* __restrict__ P, int n, KnnGrid g, int* __restrict__ counts,
                           int* __restrict__ cell_of) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int cx = cell_coord(P[(size_t)i * 3], g.lo0, g.inv_h, g.G0);
    int cy = cell_coord(P[(size_t)i * 3 + 1], g.lo1, g.inv_h, g.G1);
    int cz = cell_coord(P[(size_t)i * 3 + 2], g.lo2, g.inv_h, g.G2);
    int c = cx + g.G0 * (cy + g.G1 * cz);
    cell_of[i] = c;
    atomicAdd(&counts[c], 1);
}

__global__ void k_knn_scatter(const float* __restrict__ P, int n, const int* __restrict__ cell_of,
                              int* __restrict__ fill, float4* __restrict__ pts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int slot = atomicAdd(&fill[cell_of[i]], 1);
    pts[slot] = make_float4(P[(size_t)i * 3], P[(size_t)i * 3 + 1], P[(size_t)i * 3 + 2], __int_as_float(i));
}

int knn_build(KnnIndex& ix, const float* P, int n, cudaStream_t s) {
    DWG_REQUIRE(P != nullptr && n >= 1, "knn: need at least one point (n=%d)", n);
    ix.n = n;
    DWG_TRY(ix.bbox.reserve(6));
    DWG_TRY(bbox_device(P, n, ix.bbox.ptr, s));
    float bb[6];
    DWG_CHECK_CUDA(cudaMemcpyAsync(bb, ix.bbox.ptr, sizeof(bb), cudaMemcpyDeviceToHost, s));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    float ext[3], emax = 0.f;
    for (int d = 0; d < 3; ++d) {
        ext[d] = bb[3 + d] - bb[d];
        emax = fmaxf(emax, ext[d]);
    }
    if (!(emax > 0.f)) emax = 1.f;
    // ~3 points per occupied cell for a surface sample
    double gm = ceil(sqrt((double)n / 14.0));
    if (gm < 1) gm = 1;
    if (gm > 1024) gm = 1024;
    float h = (float)(emax / gm) * 1.0001f;
    for (;;) {
        long long tot = 1;
        for (int d = 0; d < 3; ++d) {
            int G = (int)ceil(ext[d] / h);
            if (G < 1) G = 1;
            ix.G[d] = G;
            tot *= G;
        }
        if (tot <= (1ll << 27)) break;
        h *= 1.25f;
    }
    ix.h = h;
    ix.inv_h = 1.0f / h;
    {
        int gm = max(ix.G[0], max(ix.G[1], ix.G[2]));
        int sh = 0;
        while ((gm >> sh) > 32) ++sh;
        ix.morton_shift = sh;
    }
    for (int d = 0; d < 3; ++d) ix.lo[d] = bb[d];
    long long ncell = (long long)ix.G[0] * ix.G[1] * ix.G[2];
    KnnGrid g{ix.G[0], ix.G[1], ix.G[2], ix.lo[0], ix.lo[1], ix.lo[2], ix.h, ix.inv_h};
    DevBuf<int> counts, cell_of;
    DWG_TRY(counts.reserve(ncell + 1));
    DWG_TRY(cell_of.reserve(n));
    DWG_TRY(ix.cell_start.reserve(ncell + 1));
    DWG_TRY(ix.cell_fill.reserve(ncell + 1));
    DWG_TRY(ix.pts.reserve(n));
    DWG_CHECK_CUDA(cudaMemsetAsync(counts.ptr, 0, sizeof(int) * (ncell + 1), s));
    k_knn_hist<<<div_up(n, 256), 256, 0, s>>>(P, n, g, counts.ptr, cell_of.ptr);
    DWG_CHECK_LAUNCH();
    size_t bytes = 0;
    int* cin = counts.ptr;
    int* cout = ix.cell_start.ptr;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cin, cout, (int)(ncell + 1), s));
    DWG_TRY(ix.scratch.reserve(bytes + 256));
    bytes = ix.scratch.n;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(ix.scratch.ptr, bytes, cin, cout, (int)(ncell + 1), s));
    DWG_CHECK_CUDA(cudaMemcpyAsync(ix.cell_fill.ptr, ix.cell_start.ptr, sizeof(int) * (ncell + 1),
                                   cudaMemcpyDeviceToDevice, s));
    k_knn_scatter<<<div_up(n, 256), 256, 0, s>>>(P, n, cell_of.ptr, ix.cell_fill.ptr, ix.pts.ptr);
    DWG_CHECK_LAUNCH();
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    return DWG_OK;
}

struct KnnArgs {
    KnnGrid g;
    const float4* __restrict__ pts;
    const int* __restrict__ cell_start;
    const float* __restrict__ q;
    const int* __restrict__ q_index;
    const float* __restrict__ q_source;
    long long nq;
    const unsigned long long* nq_dev;
    const int* nq_dev_i32;
    const unsigned char* __restrict__ exclude;
    const int* gate_count;
    int gate_min;
    int k;
    int* __restrict__ out;
    const int* __restrict__ order;  // query processing order (spatially bucketed)
    int* __restrict__ q_key;
    int* __restrict__ q_hist;
    int morton_shift;
};

__device__ __forceinline__ long long knn_count(const KnnArgs& a) {
    long long nq = a.nq;
    if (a.nq_dev) {
        unsigned long long d = *a.nq_dev;
        if ((long long)d < nq) nq = (long long)d;
    }
    if (a.nq_dev_i32) {
        long long d = *a.nq_dev_i32;
        if (d < nq) nq = d;
    }
    return nq;
}

__device__ __forceinline__ void knn_load_query(const KnnArgs& a, long long qi, float& qx, float& qy, float& qz) {
    if (a.q_index) {
        long long src = a.q_index[qi];
        qx = a.q_source[src * 3];
        qy = a.q_source[src * 3 + 1];
        qz = a.q_source[src * 3 + 2];
    } else {
        qx = a.q[qi * 3];
        qy = a.q[qi * 3 + 1];
        qz = a.q[qi * 3 + 2];
    }
}

__device__ __forceinline__ unsigned spread5(unsigned v) {
    v &= 31u;
    v = (v | (v << 8)) & 0x0300Fu;
    v = (v | (v << 4)) & 0x030C3u;
    v = (v | (v << 2)) & 0x09249u;
    return v;
}

// bucket the queries by the Morton code of their coarse cell (32^3 buckets)
__global__ void k_knn_qkey(KnnArgs a) {
    if (a.gate_count && *a.gate_count <= a.gate_min) return;
    const long long nq = knn_count(a);
    for (long long qi = blockIdx.x * (long long)blockDim.x + threadIdx.x; qi < nq;
         qi += (long long)gridDim.x * blockDim.x) {
        float qx, qy, qz;
        knn_load_query(a, qi, qx, qy, qz);
        unsigned cx = cell_coord(qx, a.g.lo0, a.g.inv_h, a.g.G0) >> a.morton_shift;
        unsigned cy = cell_coord(qy, a.g.lo1, a.g.inv_h, a.g.G1) >> a.morton_shift;
        unsigned cz = cell_coord(qz, a.g.lo2, a.g.inv_h, a.g.G2) >> a.morton_shift;
        int key = (int)(spread5(cx) | (spread5(cy) << 1) | (spread5(cz) << 2));
        a.q_key[qi] = key;
        atomicAdd(&a.q_hist[key], 1);
    }
}

__global__ void k_knn_qscatter(KnnArgs a, int* __restrict__ fill, int* __restrict__ order) {
    if (a.gate_count && *a.gate_count <= a.gate_min) return;
    const long long nq = knn_count(a);
    for (long long qi = blockIdx.x * (long long)blockDim.x + threadIdx.x; qi < nq;
         qi += (long long)gridDim.x * blockDim.x)
        order[atomicAdd(&fill[a.q_key[qi]], 1)] = (int)qi;
}


// top-k state of one lane: an unsorted set of KMAX keys and its maximum
template <int KMAX>
struct TopK {
    unsigned long long e[KMAX];
    unsigned long long mx;  // the k-th key (max of the set) or NONE
    int mpos;
    __device__ __forceinline__ void init(int k) {
#pragma unroll
        for (int q = 0; q < KMAX; ++q) e[q] = q < k ? ~0ull : 0ull;  // unused slots never become the max
        mx = ~0ull;
        mpos = 0;
    }
    // replace the maximum by v (v < mx) and find the new maximum
    __device__ __forceinline__ void replace_max(unsigned long long v) {
#pragma unroll
        for (int q = 0; q < KMAX; ++q)
            if (q == mpos) e[q] = v;
        mx = e[0];
        mpos = 0;
#pragma unroll
        for (int q = 1; q < KMAX; ++q)
            if (e[q] > mx) {
                mx = e[q];
                mpos = q;
            }
    }
    // ascending order: a register network for small sets, an insertion sort
    // in local memory otherwise (once per query)
    __device__ __forceinline__ void sort() {
        if (KMAX <= 16) {
#pragma unroll
            for (int pass = 0; pass < KMAX; ++pass) {
#pragma unroll
                for (int q = pass & 1; q + 1 < KMAX; q += 2) {
                    const unsigned long long a = e[q], b = e[q + 1];
                    e[q] = a < b ? a : b;
                    e[q + 1] = a < b ? b : a;
                }
            }
        } else {
            unsigned long long t[KMAX];
#pragma unroll
            for (int q = 0; q < KMAX; ++q) t[q] = e[q];
#pragma unroll 1
            for (int q = 1; q < KMAX; ++q) {
                const unsigned long long v = t[q];
                int p = q - 1;
                while (p >= 0 && t[p] > v) {
                    t[p + 1] = t[p];
                    --p;
                }
                t[p + 1] = v;
            }
#pragma unroll
            for (int q = 0; q < KMAX; ++q) e[q] = t[q];
        }
    }
};

// One thread per query; queries are processed in the order of their coarse
// Morton bucket so that neighbouring threads search neighbouring cells.  A
// query visits Chebyshev shells of cells around its own cell; a cell is
// skipped when its box is farther than the current k-th candidate; the k best
// keys are an unsorted register set whose maximum is kept in a register
// (replace-the-maximum on insertion, one sort at the end).  The search stops
// when the k-th key is closer than the boundary of the visited block.
template <int KMAX>
__global__ void __launch_bounds__(128) k_knn_thread(KnnArgs a) {
    if (a.gate_count && *a.gate_count <= a.gate_min) return;
    const long long nq = knn_count(a);
    const unsigned long long NONE = ~0ull;
    const int k = a.k;
    const float h = a.g.h;
    const float eps = 1e-4f * h + 1e-6f;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < nq;
         j += (long long)gridDim.x * blockDim.x) {
        const long long qi = a.order ? a.order[j] : j;
        float qx, qy, qz;
        knn_load_query(a, qi, qx, qy, qz);
        const int cx = cell_coord(qx, a.g.lo0, a.g.inv_h, a.g.G0);
        const int cy = cell_coord(qy, a.g.lo1, a.g.inv_h, a.g.G1);
        const int cz = cell_coord(qz, a.g.lo2, a.g.inv_h, a.g.G2);
        TopK<KMAX> top;
        top.init(k);
        for (int r = 0;; ++r) {
            const float kd2 = top.mx == NONE ? INFINITY : __uint_as_float((unsigned)(top.mx >> 32)) * 1.00001f;
            for (int dz = -r; dz <= r; ++dz) {
                const int z = cz + dz;
                if (z < 0 || z >= a.g.G2) continue;
                const float z0 = a.g.lo2 + (float)z * h - eps, z1 = z0 + h + 2.f * eps;
                const float ddz = fmaxf(0.f, fmaxf(z0 - qz, qz - z1));
                for (int dy = -r; dy <= r; ++dy) {
                    const int y = cy + dy;
                    if (y < 0 || y >= a.g.G1) continue;
                    const float y0 = a.g.lo1 + (float)y * h - eps, y1 = y0 + h + 2.f * eps;
                    const float ddy = fmaxf(0.f, fmaxf(y0 - qy, qy - y1));
                    const float dyz = ddy * ddy + ddz * ddz;
                    if (dyz > kd2) continue;
                    const bool face = (dz == -r || dz == r || dy == -r || dy == r);
                    const int step = face ? 1 : (r > 0 ? 2 * r : 1);
                    for (int dx = -r; dx <= r; dx += step) {
                        const int x = cx + dx;
                        if (x < 0 || x >= a.g.G0) continue;
                        const float x0 = a.g.lo0 + (float)x * h - eps, x1 = x0 + h + 2.f * eps;
                        const float ddx = fmaxf(0.f, fmaxf(x0 - qx, qx - x1));
                        if (ddx * ddx + dyz > kd2) continue;
                        const int c = x + a.g.G0 * (y + a.g.G1 * z);
                        const int e = a.cell_start[c + 1];
                        for (int t = a.cell_start[c]; t < e; ++t) {
                            const float4 pp = a.pts[t];
                            const int id = __float_as_int(pp.w);
                            if (a.exclude && a.exclude[id]) continue;
                            const float d2 =
                                sq3_rn(__fsub_rn(pp.x, qx), __fsub_rn(pp.y, qy), __fsub_rn(pp.z, qz));
                            const unsigned long long v = ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned)id;
                            if (v < top.mx) top.replace_max(v);
                        }
                    }
                }
            }
            if (cx - r <= 0 && cy - r <= 0 && cz - r <= 0 && cx + r >= a.g.G0 - 1 && cy + r >= a.g.G1 - 1 &&
                cz + r >= a.g.G2 - 1)
                break;
            if (top.mx != NONE) {
                float bd = INFINITY;
                if (cx - r > 0) bd = fminf(bd, qx - (a.g.lo0 + (float)(cx - r) * h));
                if (cx + r < a.g.G0 - 1) bd = fminf(bd, (a.g.lo0 + (float)(cx + r + 1) * h) - qx);
                if (cy - r > 0) bd = fminf(bd, qy - (a.g.lo1 + (float)(cy - r) * h));
                if (cy + r < a.g.G1 - 1) bd = fminf(bd, (a.g.lo1 + (float)(cy + r + 1) * h) - qy);
                if (cz - r > 0) bd = fminf(bd, qz - (a.g.lo2 + (float)(cz - r) * h));
                if (cz + r < a.g.G2 - 1) bd = fminf(bd, (a.g.lo2 + (float)(cz + r + 1) * h) - qz);
                bd -= eps;
                if (bd > 0.f && __uint_as_float((unsigned)(top.mx >> 32)) < bd * bd * 0.9999f) break;
            }
        }
        top.sort();
        // slots >= k hold 0 (below every key) and sort first; results start at KMAX - k
#pragma unroll
        for (int t = 0; t < KMAX; ++t) {
            const int o = t - (KMAX - k);
            if (o >= 0) a.out[qi * k + o] = top.e[t] == NONE ? -1 : (int)(unsigned)(top.e[t] & 0xffffffffu);
        }
    }
}

template <int KMAX>
static int knn_launch(const KnnArgs& a, long long nq, cudaStream_t s) {
    static int bps = 0;
    if (!bps) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_knn_thread<KMAX>, 128, 0);
        if (bps <= 0) bps = 1;
    }
    long long blocks = (nq + 127) / 128;
    long long cap = (long long)num_sms() * bps;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    k_knn_thread<KMAX><<<(unsigned)blocks, 128, 0, s>>>(a);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

constexpr int kKnnBuckets = 1 << 15;

int knn_query(const KnnIndex& ix, const KnnQuery& q, int k, int* out, cudaStream_t s) {
    DWG_REQUIRE(k >= 1 && k <= 64, "knn: k must be in [1, 64] (got %d)", k);
    DWG_REQUIRE(out != nullptr, "knn: output is null");
    DWG_REQUIRE(q.q || (q.q_index && q.q_source), "knn: no queries");
    if (q.nq <= 0) return DWG_OK;
    KnnArgs a;
    a.g = KnnGrid{ix.G[0], ix.G[1], ix.G[2], ix.lo[0], ix.lo[1], ix.lo[2], ix.h, ix.inv_h};
    a.pts = ix.pts.ptr;
    a.cell_start = ix.cell_start.ptr;
    a.q = q.q;
    a.q_index = q.q_index;
    a.q_source = q.q_source;
    a.nq = q.nq;
    a.nq_dev = q.nq_dev;
    a.nq_dev_i32 = q.nq_dev_i32;
    a.exclude = q.exclude;
    a.gate_count = q.gate_count;
    a.gate_min = q.gate_min;
    a.k = k;
    a.out = out;
    a.morton_shift = ix.morton_shift;
    // bucket the queries spatially (counting sort on device counts, no host sync)
    DWG_TRY(ix.q_key.reserve(q.nq));
    DWG_TRY(ix.q_order.reserve(q.nq));
    DWG_TRY(ix.q_hist.reserve(kKnnBuckets));
    DWG_TRY(ix.q_fill.reserve(kKnnBuckets));
    a.q_key = ix.q_key.ptr;
    a.q_hist = ix.q_hist.ptr;
    a.order = nullptr;
    DWG_CHECK_CUDA(cudaMemsetAsync(ix.q_hist.ptr, 0, sizeof(int) * kKnnBuckets, s));
    long long blocks = (q.nq + 255) / 256;
    long long cap = (long long)num_sms() * 8;
    if (blocks > cap) blocks = cap;
    k_knn_qkey<<<(unsigned)blocks, 256, 0, s>>>(a);
    DWG_CHECK_LAUNCH();
    size_t bytes = 0;
    int* hin = ix.q_hist.ptr;
    int* hout = ix.q_fill.ptr;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, hin, hout, kKnnBuckets, s));
    DWG_TRY(ix.q_scratch.reserve(bytes + 256));
    bytes = ix.q_scratch.n;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(ix.q_scratch.ptr, bytes, hin, hout, kKnnBuckets, s));
    k_knn_qscatter<<<(unsigned)blocks, 256, 0, s>>>(a, ix.q_fill.ptr, ix.q_order.ptr);
    DWG_CHECK_LAUNCH();
    a.order = ix.q_order.ptr;
    if (k <= 16) return knn_launch<16>(a, q.nq, s);
    if (k <= 32) return knn_launch<32>(a, q.nq, s);
    return knn_launch<64>(a, q.nq, s);
}

}  // namespace dwg
