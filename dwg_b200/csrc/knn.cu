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
};

template <int KMAX>
__global__ void __launch_bounds__(128) k_knn_query(KnnArgs a) {
    if (a.gate_count && *a.gate_count <= a.gate_min) return;
    long long nq = a.nq;
    if (a.nq_dev) {
        unsigned long long d = *a.nq_dev;
        if ((long long)d < nq) nq = (long long)d;
    }
    if (a.nq_dev_i32) {
        long long d = *a.nq_dev_i32;
        if (d < nq) nq = d;
    }
    const unsigned long long NONE = ~0ull;
    for (long long qi = blockIdx.x * (long long)blockDim.x + threadIdx.x; qi < nq;
         qi += (long long)gridDim.x * blockDim.x) {
        float qx, qy, qz;
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
        unsigned long long best[KMAX];
#pragma unroll
        for (int j = 0; j < KMAX; ++j) best[j] = NONE;
        const int cx = cell_coord(qx, a.g.lo0, a.g.inv_h, a.g.G0);
        const int cy = cell_coord(qy, a.g.lo1, a.g.inv_h, a.g.G1);
        const int cz = cell_coord(qz, a.g.lo2, a.g.inv_h, a.g.G2);
        const int k = a.k;
        for (int r = 0;; ++r) {
            for (int dz = -r; dz <= r; ++dz) {
                const int z = cz + dz;
                if (z < 0 || z >= a.g.G2) continue;
                for (int dy = -r; dy <= r; ++dy) {
                    const int y = cy + dy;
                    if (y < 0 || y >= a.g.G1) continue;
                    const bool face = (dz == -r || dz == r || dy == -r || dy == r);
                    const int step = face ? 1 : (r > 0 ? 2 * r : 1);
                    for (int dx = -r; dx <= r; dx += step) {
                        const int x = cx + dx;
                        if (x < 0 || x >= a.g.G0) continue;
                        const int c = x + a.g.G0 * (y + a.g.G1 * z);
                        const int e = a.cell_start[c + 1];
                        for (int j = a.cell_start[c]; j < e; ++j) {
                            const float4 p = a.pts[j];
                            const int id = __float_as_int(p.w);
                            if (a.exclude && a.exclude[id]) continue;
                            const float d2 = sq3_rn(__fsub_rn(p.x, qx), __fsub_rn(p.y, qy), __fsub_rn(p.z, qz));
                            unsigned long long v =
                                ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned)id;
                            bool ins = false;
#pragma unroll
                            for (int t = 0; t < KMAX; ++t)
                                if (t == k - 1) ins = v < best[t];
                            if (!ins) continue;
#pragma unroll
                            for (int t = 0; t < KMAX; ++t) {
                                if (t < k) {
                                    unsigned long long lo = best[t] < v ? best[t] : v;
                                    unsigned long long hi = best[t] < v ? v : best[t];
                                    best[t] = lo;
                                    v = hi;
                                }
                            }
                        }
                    }
                }
            }
            // stop once the block [c-r, c+r] covers the grid, or the k-th
            // candidate is closer than the block's boundary
            if (cx - r <= 0 && cy - r <= 0 && cz - r <= 0 && cx + r >= a.g.G0 - 1 && cy + r >= a.g.G1 - 1 &&
                cz + r >= a.g.G2 - 1)
                break;
            unsigned long long kth = NONE;
#pragma unroll
            for (int t = 0; t < KMAX; ++t)
                if (t == k - 1) kth = best[t];
            if (kth != NONE) {
                float bd = INFINITY;
                const float qv[3] = {qx, qy, qz};
                const int cc[3] = {cx, cy, cz};
                const int GG[3] = {a.g.G0, a.g.G1, a.g.G2};
                const float ll[3] = {a.g.lo0, a.g.lo1, a.g.lo2};
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    if (cc[d] - r > 0) bd = fminf(bd, qv[d] - (ll[d] + (float)(cc[d] - r) * a.g.h));
                    if (cc[d] + r < GG[d] - 1) bd = fminf(bd, (ll[d] + (float)(cc[d] + r + 1) * a.g.h) - qv[d]);
                }
                bd -= 1e-4f * a.g.h + 1e-6f;
                if (bd > 0.f) {
                    const float kd2 = __uint_as_float((unsigned)(kth >> 32));
                    if (kd2 < bd * bd * 0.9999f) break;
                }
            }
        }
#pragma unroll
        for (int t = 0; t < KMAX; ++t)
            if (t < k) a.out[qi * k + t] = best[t] == NONE ? -1 : (int)(unsigned)(best[t] & 0xffffffffu);
    }
}

template <int KMAX>
static int knn_launch(const KnnArgs& a, long long nq, cudaStream_t s) {
    long long blocks = (nq + 127) / 128;
    long long cap = (long long)num_sms() * 16;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    k_knn_query<KMAX><<<(unsigned)blocks, 128, 0, s>>>(a);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

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
    if (k <= 16) return knn_launch<16>(a, q.nq, s);
    if (k <= 32) return knn_launch<32>(a, q.nq, s);
    return knn_launch<64>(a, q.nq, s);
}

}  // namespace dwg
