// normals.cu -- normal initialisation, diffusion and repair.
//
// Single-precision expressions that decide the next iteration's normals use
// round-to-nearest intrinsics in a fixed order, so that the oracle reproduces
// them bit for bit.  The triangle->point scatter is summed in 2^-40 fixed
// point with 64-bit integer atomics: the result does not depend on the order
// in which the atomics land (the reference adds FP32 atomics,
// src/TurboDWG.cu:199-201, whose sum depends on scheduling).
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "normals.cuh"
#include "octree.cuh"

namespace dwg {

constexpr double kFix = 1099511627776.0;  // 2^40

// GaussMapInitNormals, src/TurboNormalInit.cu:3-27
__global__ void k_gauss_map(const float* __restrict__ P, int n, const float* __restrict__ bb,
                            float* __restrict__ N) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float c[3], v[3];
    for (int d = 0; d < 3; ++d) {
        c[d] = __fdiv_rn(__fadd_rn(bb[d], bb[3 + d]), 2.0f);
        v[d] = __fsub_rn(P[(size_t)i * 3 + d], c[d]);
    }
    float sc = inv_len_eps(__fsqrt_rn(sq3_rn(v[0], v[1], v[2])));
    for (int d = 0; d < 3; ++d) N[(size_t)i * 3 + d] = __fmul_rn(v[d], sc);
}

int gauss_map(const float* P, int n, float* N, cudaStream_t s) {
    DWG_REQUIRE(P && N && n >= 1, "gauss_map: bad arguments");
    DevBuf<float> bb;
    DWG_TRY(bb.reserve(6));
    DWG_TRY(bbox_device(P, n, bb.ptr, s));
    k_gauss_map<<<div_up(n, 256), 256, 0, s>>>(P, n, bb.ptr, N);
    DWG_CHECK_LAUNCH();
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));  // bb is released on return
    return DWG_OK;
}

// UpdateNormals (src/TurboDWG.cu:179-204), fixed point
__global__ void k_scatter(const int* __restrict__ knn, const float* __restrict__ tn, long long T,
                          const unsigned long long* __restrict__ Tdev, int k, int L,
                          unsigned long long* __restrict__ acc) {
    long long nt = T;
    if (Tdev && (long long)*Tdev < nt) nt = (long long)*Tdev;
    long long total = nt * k;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long t = e / k;
        int i = knn[e];
        if (i < 0 || i >= L) continue;
        for (int d = 0; d < 3; ++d) {
            long long f = __double2ll_rn((double)tn[t * 3 + d] * kFix);
            atomicAdd(&acc[(size_t)i * 3 + d], (unsigned long long)f);
        }
    }
}

// NormalizeNormals (src/TurboDWG.cu:238-266); also clears the accumulator
__global__ void k_finalize(long long* __restrict__ acc, int L, float* __restrict__ N,
                           unsigned char* __restrict__ is_zero, int* __restrict__ zero_count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool zero = false;
    if (i < L) {
        float t[3];
        for (int d = 0; d < 3; ++d) {
            t[d] = __double2float_rn(__ll2double_rn(acc[(size_t)i * 3 + d]) * (1.0 / kFix));
            acc[(size_t)i * 3 + d] = 0;
        }
        float len = __fsqrt_rn(sq3_rn(t[0], t[1], t[2]));
        zero = (double)len < 1e-10;
        if (!zero) {
            float sc = inv_len_eps(len);
            for (int d = 0; d < 3; ++d) N[(size_t)i * 3 + d] = __fmul_rn(t[d], sc);
        }
        if (is_zero) is_zero[i] = zero ? 1 : 0;
    }
    unsigned m = __ballot_sync(0xffffffffu, zero);
    if ((threadIdx.x & 31) == 0 && m && zero_count) atomicAdd(zero_count, __popc(m));
}

int diffuse_scatter(const int* knn, const float* tn, long long T, const unsigned long long* Tdev, int k, int L,
                    long long* acc, cudaStream_t s) {
    DWG_REQUIRE(knn && tn && acc && L >= 1 && k >= 1, "diffuse_normals: bad arguments");
    if (T > 0) {
        long long blocks = (T * k + 255) / 256;
        long long cap = (long long)num_sms() * 16;
        if (blocks > cap) blocks = cap;
        k_scatter<<<(unsigned)blocks, 256, 0, s>>>(knn, tn, T, Tdev, k, L, (unsigned long long*)acc);
        DWG_CHECK_LAUNCH();
    }
    return DWG_OK;
}

int diffuse_finish(int L, float* N, long long* acc, unsigned char* is_zero, int* zero_count, cudaStream_t s) {
    DWG_REQUIRE(N && acc && L >= 1, "diffuse_normals: bad arguments");
    if (zero_count) DWG_CHECK_CUDA(cudaMemsetAsync(zero_count, 0, sizeof(int), s));
    k_finalize<<<div_up(L, 256), 256, 0, s>>>(acc, L, N, is_zero, zero_count);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

int diffuse_normals(const int* knn, const float* tn, long long T, const unsigned long long* Tdev, int k, int L,
                    float* N, long long* acc, unsigned char* is_zero, int* zero_count, cudaStream_t s) {
    DWG_TRY(diffuse_scatter(knn, tn, T, Tdev, k, L, acc, s));
    return diffuse_finish(L, N, acc, is_zero, zero_count, s);
}

// The seed of each flagged point: points do not move between calls, so any k
// distinct unflagged points bound its k-th nearest unflagged distance from
// above, and its k neighbours of the last call that queried it usually still
// qualify (and are usually its k nearest again).  The key is the largest of
// their squared distances, computed as the searches compute them and rounded
// up, over every index: the k nearest keys all lie below it.  Points whose
// recorded neighbours are incomplete, repeated or flagged get none (~0).
__global__ void k_seed_keys(const int* __restrict__ list, const int* __restrict__ count, int gate_min,
                            const int* __restrict__ prev, int k, int L, const unsigned char* __restrict__ is_zero,
                            const float* __restrict__ P, unsigned long long* __restrict__ seed) {
    const int z = *count;
    if (z <= gate_min) return;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < z; j += gridDim.x * blockDim.x) {
        const int i = list[j];
        const float qx = P[(size_t)i * 3], qy = P[(size_t)i * 3 + 1], qz = P[(size_t)i * 3 + 2];
        int ids[kKnnBoundK];
        bool ok = true;
        float mx = 0.f;
        for (int t = 0; t < k && ok; ++t) {
            const int c = prev[(size_t)i * k + t];
            ok = c >= 0 && c < L && !is_zero[c];
            for (int u = 0; u < t && ok; ++u) ok = ids[u] != c;
            if (!ok) break;
            ids[t] = c;
            const float d2 = sq3_rn(__fsub_rn(P[(size_t)c * 3], qx), __fsub_rn(P[(size_t)c * 3 + 1], qy),
                                    __fsub_rn(P[(size_t)c * 3 + 2], qz));
            mx = fmaxf(mx, d2);
        }
        seed[j] = ok ? ((unsigned long long)__float_as_uint(mx * 1.00002f) << 32) | 0xffffffffull : ~0ull;
    }
}

// SimpleUpdateNonzeroNormals (src/TurboDWG.cu:322-359); the neighbours are
// also recorded per point for the next call's seeds
__global__ void k_zero_apply(const int* __restrict__ list, const int* __restrict__ count, int gate_min,
                             const int* __restrict__ nb, int k, float* __restrict__ N, int* __restrict__ prev) {
    const int z = *count;
    if (z <= gate_min) return;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < z; j += gridDim.x * blockDim.x) {
        if (prev)
            for (int t = 0; t < k; ++t) prev[(size_t)list[j] * k + t] = nb[(size_t)j * k + t];
        float sx = 0.f, sy = 0.f, sz = 0.f;
        for (int t = 0; t < k; ++t) {
            int c = nb[(size_t)j * k + t];
            if (c < 0) continue;
            sx = __fadd_rn(sx, N[(size_t)c * 3]);
            sy = __fadd_rn(sy, N[(size_t)c * 3 + 1]);
            sz = __fadd_rn(sz, N[(size_t)c * 3 + 2]);
        }
        float sc = inv_len_eps(__fsqrt_rn(sq3_rn(sx, sy, sz)));
        int i = list[j];
        N[(size_t)i * 3] = __fmul_rn(sx, sc);
        N[(size_t)i * 3 + 1] = __fmul_rn(sy, sc);
        N[(size_t)i * 3 + 2] = __fmul_rn(sz, sc);
    }
}

int zero_repair(const KnnIndex& ix, const float* pos, int L, float* N, const unsigned char* is_zero, int k,
                int min_zero, ZeroRepairWs& ws, cudaStream_t s) {
    DWG_REQUIRE(pos && N && is_zero && L >= 1 && k >= 1 && k <= 64, "zero_repair: bad arguments");
    DWG_TRY(ws.list.reserve(L));
    DWG_TRY(ws.count.reserve(1));
    DWG_TRY(ws.nb.reserve((size_t)L * k));
    thrust::counting_iterator<int> it(0);
    size_t bytes = 0;
    int* lp = ws.list.ptr;
    int* cp = ws.count.ptr;
    DWG_CHECK_CUDA(cub::DeviceSelect::Flagged(nullptr, bytes, it, is_zero, lp, cp, L, s));
    DWG_TRY(ws.scratch.reserve(bytes + 256));
    bytes = ws.scratch.n;
    DWG_CHECK_CUDA(cub::DeviceSelect::Flagged(ws.scratch.ptr, bytes, it, is_zero, lp, cp, L, s));
    // the neighbours are the k nearest among the unflagged points, in key
    // order: the query runs on the index of those points alone
    DWG_TRY(knn_build_subset(ix, is_zero, ws.sub, s));
    KnnQuery q;
    q.q_index = ws.list.ptr;
    q.q_source = pos;
    q.nq = L;
    q.nq_dev_i32 = ws.count.ptr;
    q.gate_count = ws.count.ptr;
    q.gate_min = min_zero;
    long long blocks = (long long)num_sms() * 4;
    // seeds from the neighbours recorded by earlier calls (k <= 16: the
    // cell-grouped search); the record starts empty
    int* prev = nullptr;
    if (k <= kKnnBoundK) {
        if (!ws.prev.ptr || ws.prev.n < (size_t)L * k || ws.prev_k != k) {
            DWG_TRY(ws.prev.reserve((size_t)L * k));
            DWG_CHECK_CUDA(cudaMemsetAsync(ws.prev.ptr, 0xff, sizeof(int) * (size_t)L * k, s));
            ws.prev_k = k;
        }
        DWG_TRY(ws.seed.reserve(L));
        k_seed_keys<<<(unsigned)blocks, 256, 0, s>>>(ws.list.ptr, ws.count.ptr, min_zero, ws.prev.ptr, k, L, is_zero,
                                                     pos, ws.seed.ptr);
        DWG_CHECK_LAUNCH();
        q.seed = ws.seed.ptr;
        prev = ws.prev.ptr;
    }
    DWG_TRY(knn_query(ws.sub, q, k, ws.nb.ptr, s));
    k_zero_apply<<<(unsigned)blocks, 256, 0, s>>>(ws.list.ptr, ws.count.ptr, min_zero, ws.nb.ptr, k, N, prev);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

__global__ void k_iota(int* __restrict__ v, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

__global__ void k_area_div(float* __restrict__ areas, const int* __restrict__ idx, int k) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) areas[idx[i]] /= 1000.0f;
}

int outlier_filter(float* areas, int n, float thr, cudaStream_t s) {
    DWG_REQUIRE(areas && n >= 1, "outlier_filter: bad arguments");
    if (!(thr > 0.f)) return DWG_OK;
    const int k = (int)ceilf((float)n * thr);
    if (k <= 0) return DWG_OK;
    DevBuf<float> keys_out;
    DevBuf<int> ids, ids_out;
    DevBuf<unsigned char> tmp;
    DWG_TRY(keys_out.reserve(n));
    DWG_TRY(ids.reserve(n));
    DWG_TRY(ids_out.reserve(n));
    k_iota<<<div_up(n, 256), 256, 0, s>>>(ids.ptr, n);
    DWG_CHECK_LAUNCH();
    size_t bytes = 0;
    DWG_CHECK_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, areas, keys_out.ptr, ids.ptr, ids_out.ptr, n,
                                                             0, 32, s));
    DWG_TRY(tmp.reserve(bytes + 256));
    bytes = tmp.n;
    DWG_CHECK_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.ptr, bytes, areas, keys_out.ptr, ids.ptr, ids_out.ptr,
                                                             n, 0, 32, s));
    const int kk = k < n ? k : n;
    k_area_div<<<div_up(kk, 256), 256, 0, s>>>(areas, ids_out.ptr, kk);
    DWG_CHECK_LAUNCH();
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));  // the sort buffers are released on return
    return DWG_OK;
}

// LoadNormals (src/TurboDWG.cu:206-236)
__global__ void k_load_normals(const int* __restrict__ knn, int k, long long nq, const float* __restrict__ LN,
                               float* __restrict__ out) {
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= nq) return;
    float s[3] = {0.f, 0.f, 0.f};
    for (int t = 0; t < k; ++t) {
        int c = knn[q * k + t];
        if (c < 0) continue;
        for (int d = 0; d < 3; ++d) s[d] = __fadd_rn(s[d], LN[(size_t)c * 3 + d]);
    }
    for (int d = 0; d < 3; ++d) s[d] = __fdiv_rn(s[d], (float)k);
    float sc = inv_len_eps(__fsqrt_rn(sq3_rn(s[0], s[1], s[2])));
    for (int d = 0; d < 3; ++d) out[q * 3 + d] = __fmul_rn(s[d], sc);
}

int load_normals(const int* knn, int k, long long nq, const float* LN, float* out, cudaStream_t s) {
    DWG_REQUIRE(knn && LN && out && k >= 1, "load_normals: bad arguments");
    if (nq <= 0) return DWG_OK;
    k_load_normals<<<div_up(nq, 256), 256, 0, s>>>(knn, k, nq, LN, out);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

// SimpleUpdateRadii (src/TurboDWG.cu:361-391), offset initialised per neighbour
__global__ void k_radii(const float* __restrict__ P, int n, const int* __restrict__ knn, int k,
                        float* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float acc = 0.f;
    for (int t = 0; t < k; ++t) {
        int c = knn[(size_t)i * k + t];
        if (c < 0) continue;
        float dx = __fsub_rn(P[(size_t)i * 3], P[(size_t)c * 3]);
        float dy = __fsub_rn(P[(size_t)i * 3 + 1], P[(size_t)c * 3 + 1]);
        float dz = __fsub_rn(P[(size_t)i * 3 + 2], P[(size_t)c * 3 + 2]);
        acc = __fadd_rn(acc, sq3_rn(dx, dy, dz));
    }
    acc = __fdiv_rn(acc, (float)k);
    float r = __fsqrt_rn(acc);
    r = (r < 0.0015f) ? 0.0015f : r;
    r = (r > 0.015f) ? 0.015f : r;
    out[i] = r;
}

int radii(const float* P, int n, const int* knn, int k, float* out, cudaStream_t s) {
    DWG_REQUIRE(P && knn && out && n >= 1 && k >= 1, "radii: bad arguments");
    k_radii<<<div_up(n, 256), 256, 0, s>>>(P, n, knn, k, out);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

constexpr int kMeanBlocks = 256;

__global__ void k_mean_partial(const float* __restrict__ x, long long n, double* __restrict__ part) {
    long long chunk = (n + kMeanBlocks - 1) / kMeanBlocks;
    long long b0 = blockIdx.x * chunk, b1 = b0 + chunk < n ? b0 + chunk : n;
    double acc = 0;
    for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) acc += (double)x[i];
    typedef cub::BlockReduce<double, 256> BR;
    __shared__ typename BR::TempStorage tmp;
    double t = BR(tmp).Sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_mean_final(const double* __restrict__ part, long long n, float* __restrict__ out,
                             const int* __restrict__ half, float* __restrict__ hist, const int* __restrict__ iter) {
    typedef cub::BlockReduce<double, kMeanBlocks> BR;
    __shared__ typename BR::TempStorage tmp;
    double t = BR(tmp).Sum(part[threadIdx.x]);
    if (threadIdx.x == 0) {
        float m = (float)(t / (double)n);
        if (half && *half) m = m * 0.5f;
        *out = m;
        if (hist && iter) hist[*iter] = m;
    }
}

int mean_to_iso(const float* x, long long n, float* mean_dev, const int* half_dev, float* iso_hist,
                const int* iter_dev, DevBuf<double>& partial, cudaStream_t s) {
    DWG_REQUIRE(x && mean_dev && n >= 1, "mean: bad arguments");
    DWG_TRY(partial.reserve(kMeanBlocks));
    k_mean_partial<<<kMeanBlocks, 256, 0, s>>>(x, n, partial.ptr);
    k_mean_final<<<1, kMeanBlocks, 0, s>>>(partial.ptr, n, mean_dev, half_dev, iso_hist, iter_dev);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

}  // namespace dwg
