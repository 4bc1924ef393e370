// octree.cu -- GPU build of the octreeDWG topology and its FP64 moments.
//
// The reference builds the octree recursively on the CPU
// (deps/libigl/include/igl/octree.cpp:171-335), precomputes the moments on the
// CPU (deps/libigl/include/igl/fast_winding_number.cpp:9-120) and flattens the
// result into pointer-chasing AoS nodes (src/TurboLibiGWN.cu:132-231).  Here:
//   1. every point gets its octant path as a key, computed in FP64 with the
//      same centre recursion and `>=` tests as octreeDWG;
//   2. one stable radix sort groups points by key (the sorted order is the
//      depth-first order of the leaves);
//   3. a node exists for every run of equal key prefixes at depth d whose
//      parent run holds more than one point; runs are found per level from
//      the longest common prefix of neighbouring keys;
//   4. nodes are numbered in depth-first pre-order, so each subtree is a
//      contiguous node range and a contiguous point range.
#include <cub/cub.cuh>

#include <vector>

#include "octree.cuh"

namespace dwg {

// ------------------------------------------------------------ bounding box --
__global__ void k_bbox_partial(const float* __restrict__ P, long long n, float* __restrict__ part) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        for (int d = 0; d < 3; d++) {
            float v = P[i * 3 + d];
            mn[d] = fminf(mn[d], v);
            mx[d] = fmaxf(mx[d], v);
        }
    }
    typedef cub::BlockReduce<float, 256> BR;
    __shared__ typename BR::TempStorage tmp;
    for (int d = 0; d < 3; d++) {
        float a = BR(tmp).Reduce(mn[d], cub::Min());
        __syncthreads();
        float b = BR(tmp).Reduce(mx[d], cub::Max());
        __syncthreads();
        if (threadIdx.x == 0) {
            part[blockIdx.x * 6 + d] = a;
            part[blockIdx.x * 6 + 3 + d] = b;
        }
    }
}

__global__ void k_bbox_final(const float* __restrict__ part, int nb, float* __restrict__ out) {
    typedef cub::BlockReduce<float, 256> BR;
    __shared__ typename BR::TempStorage tmp;
    for (int d = 0; d < 6; d++) {
        float v = (d < 3) ? INFINITY : -INFINITY;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            float x = part[b * 6 + d];
            v = (d < 3) ? fminf(v, x) : fmaxf(v, x);
        }
        float r = (d < 3) ? BR(tmp).Reduce(v, cub::Min()) : BR(tmp).Reduce(v, cub::Max());
        __syncthreads();
        if (threadIdx.x == 0) out[d] = r;
    }
}

int bbox_device(const float* points_dev, long long n, float* out_dev, cudaStream_t s) {
    static thread_local DevBuf<float> part;
    const int nb = 256;
    DWG_TRY(part.reserve(nb * 6));
    k_bbox_partial<<<nb, 256, 0, s>>>(points_dev, n, part.ptr);
    k_bbox_final<<<1, 256, 0, s>>>(part.ptr, nb, out_dev);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

// root cube: AABB centre, width = largest extent, in FP64 (octree.cpp:306-316)
__global__ void k_nonfinite(const float* __restrict__ x, long long m, unsigned int* __restrict__ flag) {
    unsigned int bad = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
        bad |= isfinite(x[i]) ? 0u : 1u;
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

int require_finite(const float* x, long long m, const char* what, cudaStream_t s) {
    if (m <= 0) return DWG_OK;
    DevBuf<unsigned int> flag;
    DWG_TRY(flag.reserve(1));
    DWG_CHECK_CUDA(cudaMemsetAsync(flag.ptr, 0, sizeof(unsigned int), s));
    long long blocks = (m + 255) / 256;
    if (blocks > (long long)num_sms() * 8) blocks = (long long)num_sms() * 8;
    k_nonfinite<<<(unsigned)blocks, 256, 0, s>>>(x, m, flag.ptr);
    DWG_CHECK_LAUNCH();
    unsigned int h = 0;
    DWG_CHECK_CUDA(cudaMemcpyAsync(&h, flag.ptr, sizeof(h), cudaMemcpyDeviceToHost, s));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    DWG_REQUIRE(h == 0, "%s: non-finite coordinate (NaN or infinity) in the input", what);
    return DWG_OK;
}

__global__ void k_root(const float* __restrict__ bb, double* __restrict__ root) {
    double w = 0;
    for (int d = 0; d < 3; d++) {
        double lo = bb[d], hi = bb[3 + d];
        root[d] = (lo + hi) / 2.0;
        if (hi - lo > w) w = hi - lo;
    }
    root[3] = w;
}

// ----------------------------------------------------------------- keys --
// octant path: bit0 x >= cx, bit1 y >= cy, bit2 z >= cz (octree.cpp:200-221);
// child centre = parent +/- (child width)/2 (octree.cpp:224-249,267-276)
__global__ void k_keys(const float* __restrict__ P, int n, const double* __restrict__ root, int D,
                       unsigned long long* __restrict__ keys, int* __restrict__ idx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double px = P[(size_t)i * 3], py = P[(size_t)i * 3 + 1], pz = P[(size_t)i * 3 + 2];
    double cx = root[0], cy = root[1], cz = root[2], w = root[3];
    unsigned long long key = 0;
    for (int d = 0; d < D; d++) {
        double h = w / 2.0;
        double hh = h / 2.0;
        int o = (px >= cx ? 1 : 0) | (py >= cy ? 2 : 0) | (pz >= cz ? 4 : 0);
        key = (key << 3) | (unsigned long long)o;
        cx = cx + ((o & 1) ? hh : -hh);
        cy = cy + ((o & 2) ? hh : -hh);
        cz = cz + ((o & 4) ? hh : -hh);
        w = h;
    }
    keys[i] = key;
    idx[i] = i;
}

// longest common prefix (in octal digits) with the previous key; -1 at both ends
__global__ void k_lcp(const unsigned long long* __restrict__ keys, int n, int D,
                      signed char* __restrict__ lcp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    int l = -1;
    if (i > 0 && i < n) {
        unsigned long long x = keys[i] ^ keys[i - 1];
        if (x == 0)
            l = D;
        else {
            int b = 63 - __clzll((long long)x);
            l = D - 1 - b / 3;
        }
    }
    lcp[i] = (signed char)l;
}

// a point is alone in its depth-d run iff d > max(lcp_i, lcp_{i+1}); it starts
// the nodes at depths lcp_i+1 .. leafdepth_i
__global__ void k_node_starts(const signed char* __restrict__ lcp, int n, int D,
                              int* __restrict__ nstart) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) {
        nstart[i] = 0;
        return;
    }
    int a = lcp[i], b = lcp[i + 1];
    int ld = min(D, max(a, b) + 1);
    nstart[i] = max(0, ld - a);
}

__global__ void k_level_flags(const signed char* __restrict__ lcp, int n, int d, int* __restrict__ f) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) f[i] = lcp[i] < d ? 1 : 0;
}

__global__ void k_level_starts(const signed char* __restrict__ lcp, const int* __restrict__ rank, int n,
                               int d, int* __restrict__ starts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int f = lcp[i] < d ? 1 : 0;
    if (f) starts[rank[i]] = i;
    if (i == n - 1) starts[rank[i] + f] = n;
}

__global__ void k_level_nodes(const signed char* __restrict__ lcp, const int* __restrict__ rank,
                              const int* __restrict__ starts, const int* __restrict__ node_base, int n,
                              int d, int D, int4* __restrict__ info) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int a = lcp[i];
    if (a >= d) return;
    int ld = min(D, max(a, (int)lcp[i + 1]) + 1);
    if (d > ld) return;
    int node = node_base[i] + (d - a - 1);
    int cnt = starts[rank[i] + 1] - i;
    int skip = node_base[i + cnt];
    int leaf = (cnt == 1 || d == D) ? kLeafFlag : 0;
    info[node] = make_int4(i, cnt, skip, d | leaf);
}

__global__ void k_gather(const float* __restrict__ P, const float* __restrict__ A,
                         const int* __restrict__ perm, int n, float4* __restrict__ pa,
                         float4* __restrict__ nr, int* __restrict__ inv) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int i = perm[j];
    pa[j] = make_float4(P[(size_t)i * 3], P[(size_t)i * 3 + 1], P[(size_t)i * 3 + 2], A ? A[i] : 1.0f);
    nr[j] = make_float4(0.f, 0.f, 0.f, 0.f);
    inv[i] = j;
}

__global__ void k_set_point_data(const float* __restrict__ N, const float* __restrict__ A,
                                 const float* __restrict__ R, const int* __restrict__ perm, int n,
                                 float4* __restrict__ pa, float4* __restrict__ nr) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int i = perm[j];
    if (A) pa[j].w = A[i];
    float4 v = nr[j];
    if (N) {
        v.x = N[(size_t)i * 3];
        v.y = N[(size_t)i * 3 + 1];
        v.z = N[(size_t)i * 3 + 2];
    }
    if (R) v.w = R[i];
    nr[j] = v;
}

__global__ void k_set_sorted_normals(const float* __restrict__ N, int n, float4* __restrict__ nr) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    float4 v = nr[j];
    v.x = N[(size_t)j * 3];
    v.y = N[(size_t)j * 3 + 1];
    v.z = N[(size_t)j * 3 + 2];
    nr[j] = v;
}

// ------------------------------------------------------------- moments --
// one warp per node; lanes stride the node's contiguous point range and the
// partial sums meet in a fixed shuffle tree (deterministic)
__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// nodes with more points than this are summed by a whole block
// (k_centres_big): a warp alone on the root would walk every point twice
// while the rest of the GPU idles
constexpr int kBigNode = 4096;
constexpr int kBigThreads = 512;

__global__ void k_centres(const int4* __restrict__ info, const float4* __restrict__ pa, int M,
                          double* __restrict__ cm_d, double* __restrict__ r_d, const int* __restrict__ lvl_of,
                          float4* __restrict__ node_a, float* __restrict__ node_r) {
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = warp; v < M; v += nwarps) {
        int4 iv = info[v];
        if (iv.y > kBigNode) continue;
        double sa = 0, sx = 0, sy = 0, sz = 0;
        for (int j = iv.x + lane; j < iv.x + iv.y; j += 32) {
            float4 p = pa[j];
            double a = p.w;
            sa += a;
            sx += a * (double)p.x;
            sy += a * (double)p.y;
            sz += a * (double)p.z;
        }
        sa = warp_sum_d(sa);
        sx = warp_sum_d(sx);
        sy = warp_sum_d(sy);
        sz = warp_sum_d(sz);
        sa = __shfl_sync(0xffffffffu, sa, 0);
        sx = __shfl_sync(0xffffffffu, sx, 0);
        sy = __shfl_sync(0xffffffffu, sy, 0);
        sz = __shfl_sync(0xffffffffu, sz, 0);
        double cx = sa > 0 ? sx / sa : 0.0, cy = sa > 0 ? sy / sa : 0.0, cz = sa > 0 ? sz / sa : 0.0;
        double rm = 0;
        for (int j = iv.x + lane; j < iv.x + iv.y; j += 32) {
            float4 p = pa[j];
            double dx = (double)p.x - cx, dy = (double)p.y - cy, dz = (double)p.z - cz;
            rm = fmax(rm, sqrt(dx * dx + dy * dy + dz * dz));
        }
        rm = warp_max_d(rm);
        if (lane == 0) {
            cm_d[v * 3] = cx;
            cm_d[v * 3 + 1] = cy;
            cm_d[v * 3 + 2] = cz;
            r_d[v] = rm;
            const int p = lvl_of[v];
            // leaves keep their point count in .w (they have no open test)
            node_a[p] = make_float4((float)cx, (float)cy, (float)cz,
                                    (iv.w & kLeafFlag) ? __int_as_float(iv.y) : 0.f);
            node_r[p] = (float)rm;
        }
    }
}

// the nodes above kBigNode points, a block each: thread-strided partial
// sums, then a fixed tree in shared memory (deterministic), the centre, and
// the radius as the maximum over the points (exact whatever the order)
__global__ void __launch_bounds__(kBigThreads) k_centres_big(const int4* __restrict__ info,
                                                            const float4* __restrict__ pa, int M,
                                                            double* __restrict__ cm_d, double* __restrict__ r_d,
                                                            const int* __restrict__ lvl_of,
                                                            float4* __restrict__ node_a, float* __restrict__ node_r) {
    __shared__ double red[4][kBigThreads];
    const int tid = threadIdx.x;
    for (long long v = blockIdx.x; v < M; v += gridDim.x) {
        const int4 iv = info[v];
        if (iv.y <= kBigNode) continue;  // the same node for the whole block
        double sa = 0, sx = 0, sy = 0, sz = 0;
        for (int j = iv.x + tid; j < iv.x + iv.y; j += kBigThreads) {
            const float4 p = pa[j];
            const double a = p.w;
            sa += a;
            sx += a * (double)p.x;
            sy += a * (double)p.y;
            sz += a * (double)p.z;
        }
        red[0][tid] = sa;
        red[1][tid] = sx;
        red[2][tid] = sy;
        red[3][tid] = sz;
        __syncthreads();
        for (int h = kBigThreads / 2; h > 0; h >>= 1) {
            if (tid < h)
                for (int q = 0; q < 4; ++q) red[q][tid] += red[q][tid + h];
            __syncthreads();
        }
        sa = red[0][0];
        const double cx = sa > 0 ? red[1][0] / sa : 0.0, cy = sa > 0 ? red[2][0] / sa : 0.0,
                     cz = sa > 0 ? red[3][0] / sa : 0.0;
        __syncthreads();  // every thread has read the sums before the radii reuse the buffer
        double rm = 0;
        for (int j = iv.x + tid; j < iv.x + iv.y; j += kBigThreads) {
            const float4 p = pa[j];
            const double dx = (double)p.x - cx, dy = (double)p.y - cy, dz = (double)p.z - cz;
            rm = fmax(rm, sqrt(dx * dx + dy * dy + dz * dz));
        }
        red[0][tid] = rm;
        __syncthreads();
        for (int h = kBigThreads / 2; h > 0; h >>= 1) {
            if (tid < h) red[0][tid] = fmax(red[0][tid], red[0][tid + h]);
            __syncthreads();
        }
        if (tid == 0) {
            rm = red[0][0];
            cm_d[v * 3] = cx;
            cm_d[v * 3 + 1] = cy;
            cm_d[v * 3 + 2] = cz;
            r_d[v] = rm;
            const int p = lvl_of[v];
            node_a[p] = make_float4((float)cx, (float)cy, (float)cz,
                                    (iv.w & kLeafFlag) ? __int_as_float(iv.y) : 0.f);
            node_r[p] = (float)rm;
        }
        __syncthreads();  // the buffer is free for the next node
    }
}

// sum A n per node, bottom-up one depth level at a time: a leaf sums its
// points, an internal node its children (in octant order) -- every node's sum
// has a fixed order, so the result is the same from run to run
__global__ void k_ec_level(const int* __restrict__ nodes, int p0, int count, const int4* __restrict__ info,
                           const float4* __restrict__ pa, const float4* __restrict__ nr,
                           const int* __restrict__ meta, double* __restrict__ ec_d,
                           float4* __restrict__ node_b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int p = p0 + i;
    const int v = nodes[p];
    const int4 iv = info[v];
    double ex = 0, ey = 0, ez = 0;
    if (iv.w & kLeafFlag) {
        for (int j = iv.x; j < iv.x + iv.y; ++j) {
            const double a = pa[j].w;
            const float4 q = nr[j];
            ex += a * (double)q.x;
            ey += a * (double)q.y;
            ez += a * (double)q.z;
        }
    } else {
        for (int c = v + 1; c < iv.z; c = info[c].z) {
            ex += ec_d[(size_t)c * 3];
            ey += ec_d[(size_t)c * 3 + 1];
            ez += ec_d[(size_t)c * 3 + 2];
        }
    }
    ec_d[(size_t)v * 3] = ex;
    ec_d[(size_t)v * 3 + 1] = ey;
    ec_d[(size_t)v * 3 + 2] = ez;
    node_b[p] = make_float4((float)ex, (float)ey, (float)ez, __int_as_float(meta[p]));
}

// expansion coefficients about the node's centre c, bottom-up one depth
// level at a time.  A leaf sums its points (a = p - c):
//   m1[u + 3v] = sum A a_u n_v,   m2[9i + u + 3v] = sum 0.5 a_i A a_u n_v;
// an internal node shifts its children's sums to its own centre
// (d = c_child - c):
//   m1 += m1c[u + 3v] + d_u e_v,
//   m2 += m2c[9i + u + 3v] + 0.5 (d_i m1c[u + 3v] + d_u m1c[i + 3v]) + 0.5 d_i d_u e_v
// with e = sum A n of the child.  Every sum has a fixed order.
__global__ void k_ho_level(const int* __restrict__ nodes, int p0, int count, const int4* __restrict__ info,
                           const float4* __restrict__ pa, const float4* __restrict__ nr,
                           const double* __restrict__ cm_d, const double* __restrict__ ec_d, int order,
                           double* __restrict__ ho_d, float4* __restrict__ node_h) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int p = p0 + i;
    const int v = nodes[p];
    const int4 iv = info[v];
    const double c0 = cm_d[(size_t)v * 3], c1 = cm_d[(size_t)v * 3 + 1], c2 = cm_d[(size_t)v * 3 + 2];
    double m[36];
#pragma unroll
    for (int t = 0; t < 36; ++t) m[t] = 0.0;
    if (iv.w & kLeafFlag) {
        for (int j = iv.x; j < iv.x + iv.y; ++j) {
            const float4 q = pa[j];
            const float4 nn = nr[j];
            const double A = q.w;
            const double a[3] = {(double)q.x - c0, (double)q.y - c1, (double)q.z - c2};
            const double an[3] = {A * (double)nn.x, A * (double)nn.y, A * (double)nn.z};
#pragma unroll
            for (int vv = 0; vv < 3; ++vv)
#pragma unroll
                for (int u = 0; u < 3; ++u) {
                    const double t1 = a[u] * an[vv];
                    m[u + 3 * vv] += t1;
                    if (order >= 2) {
#pragma unroll
                        for (int k = 0; k < 3; ++k) m[9 + 9 * k + u + 3 * vv] += 0.5 * a[k] * t1;
                    }
                }
        }
    } else {
        for (int ch = v + 1; ch < iv.z; ch = info[ch].z) {
            const double d[3] = {cm_d[(size_t)ch * 3] - c0, cm_d[(size_t)ch * 3 + 1] - c1,
                                 cm_d[(size_t)ch * 3 + 2] - c2};
            const double e[3] = {ec_d[(size_t)ch * 3], ec_d[(size_t)ch * 3 + 1], ec_d[(size_t)ch * 3 + 2]};
            const double* hc = ho_d + (size_t)ch * 36;
            double m1c[9];
#pragma unroll
            for (int t = 0; t < 9; ++t) m1c[t] = hc[t];
#pragma unroll
            for (int vv = 0; vv < 3; ++vv)
#pragma unroll
                for (int u = 0; u < 3; ++u) {
                    m[u + 3 * vv] += m1c[u + 3 * vv] + d[u] * e[vv];
                    if (order >= 2) {
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                            m[9 + 9 * k + u + 3 * vv] += hc[9 + 9 * k + u + 3 * vv] +
                                                         0.5 * (d[k] * m1c[u + 3 * vv] + d[u] * m1c[k + 3 * vv]) +
                                                         0.5 * d[k] * d[u] * e[vv];
                    }
                }
        }
    }
    double* ho = ho_d + (size_t)v * 36;
#pragma unroll
    for (int t = 0; t < 36; ++t) ho[t] = m[t];
    // traversal record, contracted for evaluation (32 floats, 8 float4):
    //   [0..8] m1, [9] trace m1, [10..12] g_k = sum_u m2[k,u,u] + sum_i m2[i,i,k]
    //   + sum_i m2[i,k,i], [13..30] s(i<=u, v) = m2[i,u,v] + m2[u,i,v] (i != u)
    //   for v = 0..2 and (i,u) = 00 01 02 11 12 22
    float r[32];
#pragma unroll
    for (int t = 0; t < 9; ++t) r[t] = (float)m[t];
    r[9] = (float)(m[0] + m[4] + m[8]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double g = 0;
#pragma unroll
        for (int u = 0; u < 3; ++u)
            g += m[9 + 9 * k + u + 3 * u] + m[9 + 9 * u + u + 3 * k] + m[9 + 9 * u + k + 3 * u];
        r[10 + k] = (float)g;
    }
    {
        int o = 13;
#pragma unroll
        for (int vv = 0; vv < 3; ++vv)
#pragma unroll
            for (int i2 = 0; i2 < 3; ++i2)
#pragma unroll
                for (int u = i2; u < 3; ++u)
                    r[o++] = (float)(i2 == u ? m[9 + 9 * i2 + u + 3 * vv]
                                             : m[9 + 9 * i2 + u + 3 * vv] + m[9 + 9 * u + i2 + 3 * vv]);
    }
    r[31] = 0.f;
    float4* h = node_h + (size_t)p * 8;
#pragma unroll
    for (int t = 0; t < 8; ++t) h[t] = make_float4(r[4 * t], r[4 * t + 1], r[4 * t + 2], r[4 * t + 3]);
}

// level-order position of every node and the traversal meta word
__global__ void k_lvl_of(const int* __restrict__ level_nodes, int M, int* __restrict__ lvl_of) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < M) lvl_of[level_nodes[p]] = p;
}

__global__ void k_node_meta(const int4* __restrict__ info, const int* __restrict__ level_nodes,
                            const int* __restrict__ lvl_of, int M, int* __restrict__ meta) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= M) return;
    const int v = level_nodes[p];
    const int4 iv = info[v];
    unsigned m;
    if (iv.w & kLeafFlag) {
        m = kMetaLeafBit | (iv.y == 1 ? (unsigned)kMetaSingle : 0u) | ((unsigned)iv.x & kMetaIndex);
    } else {
        int nch = 0;
        for (int c = v + 1; c < iv.z && nch < 9; c = info[c].z) ++nch;
        m = ((unsigned)lvl_of[v + 1] & kMetaIndex) | ((unsigned)(nch - 1) << 28);
    }
    meta[p] = (int)m;
}

__global__ void k_depth_key(const int4* __restrict__ info, int M, unsigned* __restrict__ key, int* __restrict__ id) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= M) return;
    key[v] = (unsigned)(info[v].w & 0xff);
    id[v] = v;
}

// Open threshold of a node for opening ratio beta.  With t = beta*R rounded,
// the far test of the reference, sqrt_rn(d2) > t, holds for an up-set of
// floats d2 (sqrt_rn is monotone), so one float T decides it exactly:
// far <=> d2 > T, T the largest float d2 that is not far.  Estimate: the
// boundary is B = (t + ulp(t)/2)^2 (exact in FP64); d2 == B (when B is a
// float) rounds half to even, i.e. is far exactly when t's last mantissa bit
// is 1.  The estimate is then confirmed with the test itself.
__device__ __forceinline__ bool open_far(float d2, float t) { return __fsqrt_rn(d2) > t; }

__global__ void k_node_thr(const float* __restrict__ node_r, const int* __restrict__ meta, int M, float beta,
                           float4* __restrict__ node_a, unsigned int* __restrict__ err) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= M) return;
    if ((unsigned)meta[v] & kMetaLeafBit) return;
    const float t = __fmul_rn(beta, node_r[v]);
    float thr;
    if (t == 0.f) {
        thr = 0.0f;  // every d2 > 0 is far
    } else {
        const double hulp = ((double)nextafterf(t, INFINITY) - (double)t) * 0.5;
        const double b = ((double)t + hulp) * ((double)t + hulp);
        thr = __double2float_rd(b);
        if ((double)thr == b && (__float_as_uint(t) & 1u)) thr = nextafterf(thr, 0.f);
        // confirm: thr is not far and the next float is (a few steps at most)
        for (int it = 0; it < 4 && open_far(thr, t); ++it) thr = nextafterf(thr, 0.f);
        for (int it = 0; it < 4 && !open_far(nextafterf(thr, INFINITY), t); ++it) thr = nextafterf(thr, INFINITY);
        if (open_far(thr, t) || !open_far(nextafterf(thr, INFINITY), t)) atomicOr(err, 8u);
    }
    float4 a = node_a[v];
    a.w = thr;
    node_a[v] = a;
}


// ---------------------------------------------------------- leaf centres --
__global__ void k_leaf_flags(const int4* __restrict__ info, int M, int min_count, int* __restrict__ f) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= M) return;
    int4 iv = info[v];
    f[v] = ((iv.w & kLeafFlag) && iv.y > min_count) ? 1 : 0;
}

// cell centre of a node, by the same FP64 recursion as the keys
__global__ void k_leaf_centres(const int4* __restrict__ info, const int* __restrict__ f,
                               const int* __restrict__ rank, int M,
                               const unsigned long long* __restrict__ keys,
                               const double* __restrict__ root, int D, float* __restrict__ out,
                               int* __restrict__ out_node) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= M || !f[v]) return;
    int4 iv = info[v];
    int depth = iv.w & 0xff;
    unsigned long long key = keys[iv.x];
    double cx = root[0], cy = root[1], cz = root[2], w = root[3];
    for (int d = 0; d < depth; d++) {
        int o = (int)((key >> (3 * (D - 1 - d))) & 7ull);
        double h = w / 2.0;
        double hh = h / 2.0;
        cx = cx + ((o & 1) ? hh : -hh);
        cy = cy + ((o & 2) ? hh : -hh);
        cz = cz + ((o & 4) ? hh : -hh);
        w = h;
    }
    int r = rank[v];
    out[(size_t)r * 3] = (float)cx;
    out[(size_t)r * 3 + 1] = (float)cy;
    out[(size_t)r * 3 + 2] = (float)cz;
    out_node[r] = v;
}

// ------------------------------------------------------------- host side --
template <typename F>
static int cub_call(DevBuf<unsigned char>& scratch, F&& f) {
    size_t bytes = 0;
    cudaError_t e = f((void*)nullptr, bytes);
    if (e != cudaSuccess) {
        set_error("cub size query failed: %s", cudaGetErrorString(e));
        return DWG_ERR_CUDA;
    }
    DWG_TRY(scratch.reserve(bytes + 256));
    size_t have = scratch.n;
    e = f((void*)scratch.ptr, have);
    if (e != cudaSuccess) {
        set_error("cub call failed: %s", cudaGetErrorString(e));
        return DWG_ERR_CUDA;
    }
    return DWG_OK;
}

int octree_build(Octree& t, const float* P, int n, int D, const float* A, cudaStream_t s) {
    DWG_REQUIRE(n >= 1, "octree: need at least one point (n=%d)", n);
    DWG_REQUIRE(D >= 1 && D <= kMaxDepth, "octree: max_depth must be in [1, %d] (got %d)", kMaxDepth, D);
    DWG_REQUIRE(P != nullptr, "octree: null points");
    DWG_TRY(require_finite(P, 3ll * n, "octree", s));
    t.n = n;
    t.max_depth = D;
    DevBuf<float> bb;
    DWG_TRY(bb.reserve(6));
    DWG_TRY(bbox_device(P, n, bb.ptr, s));
    DWG_TRY(t.root_dev.reserve(4));
    k_root<<<1, 1, 0, s>>>(bb.ptr, t.root_dev.ptr);
    DevBuf<unsigned long long> keys_in;
    DevBuf<int> idx_in;
    DWG_TRY(keys_in.reserve(n));
    DWG_TRY(idx_in.reserve(n));
    DWG_TRY(t.keys.reserve(n));
    DWG_TRY(t.perm.reserve(n));
    DWG_TRY(t.inv_perm.reserve(n));
    k_keys<<<div_up(n, 256), 256, 0, s>>>(P, n, t.root_dev.ptr, D, keys_in.ptr, idx_in.ptr);
    DWG_CHECK_LAUNCH();
    unsigned long long* kin = keys_in.ptr;
    unsigned long long* kout = t.keys.ptr;
    int* vin = idx_in.ptr;
    int* vout = t.perm.ptr;
    DWG_TRY(cub_call(t.scratch, [&](void* tmp, size_t& bytes) {
        return cub::DeviceRadixSort::SortPairs(tmp, bytes, kin, kout, vin, vout, n, 0, 3 * D, s);
    }));
    DevBuf<signed char> lcp;
    DevBuf<int> nstart, node_base;
    DWG_TRY(lcp.reserve(n + 1));
    DWG_TRY(nstart.reserve(n + 1));
    DWG_TRY(node_base.reserve(n + 1));
    k_lcp<<<div_up(n + 1, 256), 256, 0, s>>>(t.keys.ptr, n, D, lcp.ptr);
    k_node_starts<<<div_up(n + 1, 256), 256, 0, s>>>(lcp.ptr, n, D, nstart.ptr);
    DWG_CHECK_LAUNCH();
    int* ns = nstart.ptr;
    int* nb = node_base.ptr;
    DWG_TRY(cub_call(t.scratch, [&](void* tmp, size_t& bytes) {
        return cub::DeviceScan::ExclusiveSum(tmp, bytes, ns, nb, n + 1, s);
    }));
    int M = 0;
    DWG_CHECK_CUDA(cudaMemcpyAsync(&M, node_base.ptr + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    DWG_CHECK_CUDA(cudaMemcpyAsync(t.root, t.root_dev.ptr, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    t.M = M;
    DWG_TRY(t.info.reserve(M));
    DevBuf<int> flags, rank, starts;
    DWG_TRY(flags.reserve(n));
    DWG_TRY(rank.reserve(n));
    DWG_TRY(starts.reserve(n + 1));
    for (int d = 0; d <= D; d++) {
        k_level_flags<<<div_up(n, 256), 256, 0, s>>>(lcp.ptr, n, d, flags.ptr);
        int* fp = flags.ptr;
        int* rp = rank.ptr;
        DWG_TRY(cub_call(t.scratch, [&](void* tmp, size_t& bytes) {
            return cub::DeviceScan::ExclusiveSum(tmp, bytes, fp, rp, n, s);
        }));
        k_level_starts<<<div_up(n, 256), 256, 0, s>>>(lcp.ptr, rank.ptr, n, d, starts.ptr);
        k_level_nodes<<<div_up(n, 256), 256, 0, s>>>(lcp.ptr, rank.ptr, starts.ptr, node_base.ptr, n, d, D,
                                                      t.info.ptr);
        DWG_CHECK_LAUNCH();
    }
    {
        // level order: stable radix sort of the nodes by depth
        DevBuf<unsigned> dkey, dkey2;
        DevBuf<int> ids;
        DWG_TRY(dkey.reserve(M));
        DWG_TRY(dkey2.reserve(M));
        DWG_TRY(ids.reserve(M));
        DWG_TRY(t.level_nodes.reserve(M));
        DWG_TRY(t.lvl_of.reserve(M));
        DWG_TRY(t.node_meta.reserve(M));
        k_depth_key<<<div_up(M, 256), 256, 0, s>>>(t.info.ptr, M, dkey.ptr, ids.ptr);
        DWG_CHECK_LAUNCH();
        unsigned* k0 = dkey.ptr;
        unsigned* k1 = dkey2.ptr;
        int* v0 = ids.ptr;
        int* v1 = t.level_nodes.ptr;
        DWG_TRY(cub_call(t.scratch, [&](void* tmp, size_t& bytes) {
            return cub::DeviceRadixSort::SortPairs(tmp, bytes, k0, k1, v0, v1, M, 0, 5, s);
        }));
        std::vector<unsigned> h(M);
        DWG_CHECK_CUDA(cudaMemcpyAsync(h.data(), dkey2.ptr, sizeof(unsigned) * M, cudaMemcpyDeviceToHost, s));
        DWG_CHECK_CUDA(cudaStreamSynchronize(s));
        for (int d = 0; d <= kMaxDepth + 1; ++d) t.level_off[d] = M;
        for (int p = M - 1; p >= 0; --p) t.level_off[h[p]] = p;
        t.level_off[0] = 0;
        for (int d = kMaxDepth; d >= 0; --d)
            if (t.level_off[d] > t.level_off[d + 1]) t.level_off[d] = t.level_off[d + 1];
        k_lvl_of<<<div_up(M, 256), 256, 0, s>>>(t.level_nodes.ptr, M, t.lvl_of.ptr);
        k_node_meta<<<div_up(M, 256), 256, 0, s>>>(t.info.ptr, t.level_nodes.ptr, t.lvl_of.ptr, M, t.node_meta.ptr);
        DWG_CHECK_LAUNCH();
        DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    }
    DWG_TRY(t.pa.reserve(n));
    DWG_TRY(t.nr.reserve(n));
    k_gather<<<div_up(n, 256), 256, 0, s>>>(P, A, t.perm.ptr, n, t.pa.ptr, t.nr.ptr, t.inv_perm.ptr);
    DWG_CHECK_LAUNCH();
    DWG_TRY(t.node_a.reserve(M));
    DWG_TRY(t.node_b.reserve(M));
    DWG_TRY(t.node_r.reserve(M));
    DWG_TRY(t.cm_d.reserve((size_t)M * 3));
    DWG_TRY(t.r_d.reserve(M));
    DWG_TRY(t.ec_d.reserve((size_t)M * 3));
    DWG_TRY(t.work.reserve(2));
    DWG_CHECK_CUDA(cudaMemsetAsync(t.work.ptr, 0, 2 * sizeof(unsigned int), s));
    DWG_CHECK_CUDA(cudaMemsetAsync(t.node_b.ptr, 0, sizeof(float4) * M, s));
    DWG_CHECK_CUDA(cudaMemsetAsync(t.ec_d.ptr, 0, sizeof(double) * 3 * M, s));
    DWG_TRY(octree_update_centres(t, s));
    DWG_TRY(octree_update_normals(t, s));  // fills the node meta words
    return DWG_OK;
}

int octree_set_point_data(Octree& t, const float* N, const float* A, const float* R, cudaStream_t s) {
    if (!N && !A && !R) return DWG_OK;
    k_set_point_data<<<div_up(t.n, 256), 256, 0, s>>>(N, A, R, t.perm.ptr, t.n, t.pa.ptr, t.nr.ptr);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

int octree_set_sorted_normals(Octree& t, const float* N, cudaStream_t s) {
    k_set_sorted_normals<<<div_up(t.n, 256), 256, 0, s>>>(N, t.n, t.nr.ptr);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

static unsigned moment_blocks(int M) {
    long long warps = M;
    long long blocks = (warps * 32 + 255) / 256;
    long long cap = (long long)num_sms() * 16;
    return (unsigned)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

int octree_update_centres(Octree& t, cudaStream_t s) {
    k_centres<<<moment_blocks(t.M), 256, 0, s>>>(t.info.ptr, t.pa.ptr, t.M, t.cm_d.ptr, t.r_d.ptr, t.lvl_of.ptr,
                                                  t.node_a.ptr, t.node_r.ptr);
    DWG_CHECK_LAUNCH();
    if (t.n > kBigNode) {
        k_centres_big<<<num_sms() * 2, kBigThreads, 0, s>>>(t.info.ptr, t.pa.ptr, t.M, t.cm_d.ptr, t.r_d.ptr,
                                                            t.lvl_of.ptr, t.node_a.ptr, t.node_r.ptr);
        DWG_CHECK_LAUNCH();
    }
    t.thr_beta = -1.f;
    return DWG_OK;
}

int octree_set_beta(Octree& t, float beta, cudaStream_t s) {
    if (t.thr_beta == beta) return DWG_OK;
    k_node_thr<<<div_up(t.M, 256), 256, 0, s>>>(t.node_r.ptr, t.node_meta.ptr, t.M, beta, t.node_a.ptr,
                                                 t.work.ptr + 1);
    DWG_CHECK_LAUNCH();
    t.thr_beta = beta;
    return DWG_OK;
}

int octree_update_normals(Octree& t, cudaStream_t s) {
    for (int d = t.max_depth; d >= 0; --d) {
        int cnt = t.level_off[d + 1] - t.level_off[d];
        if (cnt <= 0) continue;
        k_ec_level<<<div_up(cnt, 128), 128, 0, s>>>(t.level_nodes.ptr, t.level_off[d], cnt, t.info.ptr, t.pa.ptr,
                                                     t.nr.ptr, t.node_meta.ptr, t.ec_d.ptr, t.node_b.ptr);
    }
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

int octree_update_expansion(Octree& t, int order, cudaStream_t s) {
    DWG_REQUIRE(order >= 1 && order <= 2, "octree: expansion order must be 1 or 2 (got %d)", order);
    DWG_TRY(t.ho_d.reserve((size_t)t.M * 36));
    DWG_TRY(t.node_h.reserve((size_t)t.M * 8));
    for (int d = t.max_depth; d >= 0; --d) {
        int cnt = t.level_off[d + 1] - t.level_off[d];
        if (cnt <= 0) continue;
        k_ho_level<<<div_up(cnt, 64), 64, 0, s>>>(t.level_nodes.ptr, t.level_off[d], cnt, t.info.ptr, t.pa.ptr,
                                                   t.nr.ptr, t.cm_d.ptr, t.ec_d.ptr, order, t.ho_d.ptr,
                                                   t.node_h.ptr);
    }
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

int octree_leaf_centres(Octree& t, int min_count, DevBuf<float>& out_xyz, DevBuf<int>& out_node,
                        int* num_leaves, cudaStream_t s) {
    DevBuf<int> f, rank;
    DWG_TRY(f.reserve(t.M));
    DWG_TRY(rank.reserve(t.M));
    k_leaf_flags<<<div_up(t.M, 256), 256, 0, s>>>(t.info.ptr, t.M, min_count, f.ptr);
    int* fp = f.ptr;
    int* rp = rank.ptr;
    int M = t.M;
    DWG_TRY(cub_call(t.scratch, [&](void* tmp, size_t& bytes) {
        return cub::DeviceScan::ExclusiveSum(tmp, bytes, fp, rp, M, s);
    }));
    int last_rank = 0, last_flag = 0;
    DWG_CHECK_CUDA(cudaMemcpyAsync(&last_rank, rank.ptr + M - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    DWG_CHECK_CUDA(cudaMemcpyAsync(&last_flag, f.ptr + M - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    int L = last_rank + last_flag;
    *num_leaves = L;
    DWG_TRY(out_xyz.reserve((size_t)(L ? L : 1) * 3));
    DWG_TRY(out_node.reserve(L ? L : 1));
    k_leaf_centres<<<div_up(M, 256), 256, 0, s>>>(t.info.ptr, f.ptr, rank.ptr, M, t.keys.ptr, t.root_dev.ptr,
                                                  t.max_depth, out_xyz.ptr, out_node.ptr);
    DWG_CHECK_LAUNCH();
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    return DWG_OK;
}

}  // namespace dwg
