// mlp.cu -- learned normal initialiser: covariance features and a small MLP
// trained and evaluated with this file's own kernels.
//
// Features (12 per point, from its 16 nearest points, self included):
// eigenvalues of the neighbourhood covariance divided by their sum (3), the
// eigenvectors of the smallest and of the largest eigenvalue, each turned to
// point away from the centre of the cloud's bounding box (3 + 3), and the
// offset from the point to the centroid of a wider neighbourhood (the 64
// nearest of every 4th point, ~256 points) divided by that neighbourhood's
// RMS spread (3): over 16 points the offset that tells convex from concave
// is buried in the sampling noise.  The network maps them to a 3-vector
// that is normalised into an initial normal.
//
// GEMMs run on the tensor cores with mma.sync m16n8k16 (BF16 inputs, FP32
// accumulation); activations are rounded to BF16 where they feed a GEMM and
// kept in FP32 elsewhere.  Training is mean cosine loss with Adam.
#include <cmath>
#include <random>
#include <vector>

#include "mlp.cuh"
#include "octree.cuh"

namespace dwg {

// ---------------------------------------------------------------- features --
// eigen-decomposition of a symmetric 3x3 matrix: eigenvalues by the closed
// trigonometric form of the characteristic cubic (O. K. Smith, CACM 1961),
// eigenvectors as the largest cross product of two rows of (A - lambda I)
__device__ void eig_vec(const double a[6], double lam, double out[3], const double fallback[3]) {
    // a = (xx, yy, zz, xy, xz, yz)
    const double r0[3] = {a[0] - lam, a[3], a[4]};
    const double r1[3] = {a[3], a[1] - lam, a[5]};
    const double r2[3] = {a[4], a[5], a[2] - lam};
    double c[3][3] = {{r0[1] * r1[2] - r0[2] * r1[1], r0[2] * r1[0] - r0[0] * r1[2], r0[0] * r1[1] - r0[1] * r1[0]},
                      {r0[1] * r2[2] - r0[2] * r2[1], r0[2] * r2[0] - r0[0] * r2[2], r0[0] * r2[1] - r0[1] * r2[0]},
                      {r1[1] * r2[2] - r1[2] * r2[1], r1[2] * r2[0] - r1[0] * r2[2], r1[0] * r2[1] - r1[1] * r2[0]}};
    int best = 0;
    double bn = -1;
    for (int i = 0; i < 3; ++i) {
        double nn = c[i][0] * c[i][0] + c[i][1] * c[i][1] + c[i][2] * c[i][2];
        if (nn > bn) {
            bn = nn;
            best = i;
        }
    }
    if (bn < 1e-60) {
        for (int d = 0; d < 3; ++d) out[d] = fallback[d];
        return;
    }
    const double inv = 1.0 / sqrt(bn);
    for (int d = 0; d < 3; ++d) out[d] = c[best][d] * inv;
}

__global__ void k_features(const float* __restrict__ P, int n, const int* __restrict__ nb, int k,
                           const float* __restrict__ S, const int* __restrict__ nbw, int kw,
                           const float* __restrict__ bb, float* __restrict__ F) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double px = P[(size_t)i * 3], py = P[(size_t)i * 3 + 1], pz = P[(size_t)i * 3 + 2];
    double cx = 0, cy = 0, cz = 0;
    int cnt = 0;
    for (int j = 0; j < k; ++j) {
        const int q = nb[(size_t)i * k + j];
        if (q < 0) continue;
        cx += P[(size_t)q * 3];
        cy += P[(size_t)q * 3 + 1];
        cz += P[(size_t)q * 3 + 2];
        ++cnt;
    }
    cnt = cnt > 0 ? cnt : 1;
    cx /= cnt;
    cy /= cnt;
    cz /= cnt;
    double a[6] = {0, 0, 0, 0, 0, 0};
    for (int j = 0; j < k; ++j) {
        const int q = nb[(size_t)i * k + j];
        if (q < 0) continue;
        const double dx = P[(size_t)q * 3] - cx, dy = P[(size_t)q * 3 + 1] - cy, dz = P[(size_t)q * 3 + 2] - cz;
        a[0] += dx * dx;
        a[1] += dy * dy;
        a[2] += dz * dz;
        a[3] += dx * dy;
        a[4] += dx * dz;
        a[5] += dy * dz;
    }
    for (int t = 0; t < 6; ++t) a[t] /= cnt;
    // eigenvalues
    const double m = (a[0] + a[1] + a[2]) / 3.0;
    const double k0 = a[0] - m, k1 = a[1] - m, k2 = a[2] - m;
    const double p2 = (k0 * k0 + k1 * k1 + k2 * k2 + 2.0 * (a[3] * a[3] + a[4] * a[4] + a[5] * a[5])) / 6.0;
    double l1, l2, l3;
    if (p2 < 1e-60) {
        l1 = l2 = l3 = m;
    } else {
        const double pp = sqrt(p2);
        const double det = k0 * (k1 * k2 - a[5] * a[5]) - a[3] * (a[3] * k2 - a[5] * a[4]) + a[4] * (a[3] * a[5] - k1 * a[4]);
        double r = det / (2.0 * pp * pp * pp);
        r = r < -1.0 ? -1.0 : (r > 1.0 ? 1.0 : r);
        const double phi = acos(r) / 3.0;
        l1 = m + 2.0 * pp * cos(phi);
        l3 = m + 2.0 * pp * cos(phi + 2.0943951023931957);
        l2 = 3.0 * m - l1 - l3;
    }
    // direction from the bounding-box centre (orients the eigenvectors)
    const double gx = px - 0.5 * ((double)bb[0] + bb[3]), gy = py - 0.5 * ((double)bb[1] + bb[4]),
                 gz = pz - 0.5 * ((double)bb[2] + bb[5]);
    double gn = sqrt(gx * gx + gy * gy + gz * gz);
    const double g[3] = {gn > 0 ? gx / gn : 0.0, gn > 0 ? gy / gn : 0.0, gn > 0 ? gz / gn : 1.0};
    const double ex[3] = {1, 0, 0};
    double v3[3], v1[3];
    eig_vec(a, l3, v3, g);
    eig_vec(a, l1, v1, ex);
    if (v3[0] * g[0] + v3[1] * g[1] + v3[2] * g[2] < 0)
        for (int d = 0; d < 3; ++d) v3[d] = -v3[d];
    if (v1[0] * g[0] + v1[1] * g[1] + v1[2] * g[2] < 0)
        for (int d = 0; d < 3; ++d) v1[d] = -v1[d];
    const double sum = fmax(l1 + l2 + l3, 1e-30);
    float* f = F + (size_t)i * kMlpIn;
    f[0] = (float)(fmax(l1, 0.0) / sum);
    f[1] = (float)(fmax(l2, 0.0) / sum);
    f[2] = (float)(fmax(l3, 0.0) / sum);
    for (int d = 0; d < 3; ++d) f[3 + d] = (float)v3[d];
    for (int d = 0; d < 3; ++d) f[6 + d] = (float)v1[d];
    // centroid offset over the wide neighbourhood (kw nearest points of the
    // subsample S), over its RMS spread
    double wx = 0, wy = 0, wz = 0;
    int wc = 0;
    for (int j = 0; j < kw; ++j) {
        const int q = nbw[(size_t)i * kw + j];
        if (q < 0) continue;
        wx += S[(size_t)q * 3];
        wy += S[(size_t)q * 3 + 1];
        wz += S[(size_t)q * 3 + 2];
        ++wc;
    }
    wc = wc > 0 ? wc : 1;
    wx /= wc;
    wy /= wc;
    wz /= wc;
    double ws = 0;
    for (int j = 0; j < kw; ++j) {
        const int q = nbw[(size_t)i * kw + j];
        if (q < 0) continue;
        const double dx = S[(size_t)q * 3] - wx, dy = S[(size_t)q * 3 + 1] - wy, dz = S[(size_t)q * 3 + 2] - wz;
        ws += dx * dx + dy * dy + dz * dz;
    }
    const double wsc = 1.0 / sqrt(fmax(ws / wc, 1e-30));
    f[9] = (float)((wx - px) * wsc);
    f[10] = (float)((wy - py) * wsc);
    f[11] = (float)((wz - pz) * wsc);
}

__global__ void k_subsample(const float* __restrict__ P, int n, int stride, float* __restrict__ S) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = (n + stride - 1) / stride;
    if (j >= m) return;
    for (int d = 0; d < 3; ++d) S[(size_t)j * 3 + d] = P[(size_t)j * stride * 3 + d];
}

int mlp_features(const KnnIndex& ix, const float* P, int n, float* F, cudaStream_t s) {
    DWG_REQUIRE(P && F && n >= 1, "mlp_features: bad arguments");
    DWG_REQUIRE(ix.n >= 1, "mlp_features: empty index");
    const int k = ix.n < kMlpFeatureK ? ix.n : kMlpFeatureK;
    DevBuf<int> nb, nbw;
    DWG_TRY(nb.reserve((size_t)n * k));
    KnnQuery q;
    q.q = P;
    q.nq = n;
    DWG_TRY(knn_query(ix, q, k, nb.ptr, s));
    // wide neighbourhood: the kMlpWideK nearest of every kMlpWideStride-th point
    const int m = (n + kMlpWideStride - 1) / kMlpWideStride;
    DevBuf<float> S;
    DWG_TRY(S.reserve((size_t)m * 3));
    k_subsample<<<div_up(m, 256), 256, 0, s>>>(P, n, kMlpWideStride, S.ptr);
    DWG_CHECK_LAUNCH();
    KnnIndex iw;
    DWG_TRY(knn_build(iw, S.ptr, m, s));
    const int kw = m < kMlpWideK ? m : kMlpWideK;
    DWG_TRY(nbw.reserve((size_t)n * kw));
    DWG_TRY(knn_query(iw, q, kw, nbw.ptr, s));
    k_features<<<div_up(n, 128), 128, 0, s>>>(P, n, nb.ptr, k, S.ptr, nbw.ptr, kw, ix.bbox.ptr, F);
    DWG_CHECK_LAUNCH();
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    return DWG_OK;
}

// ------------------------------------------------------------------- GEMM --
__device__ __forceinline__ unsigned pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (unsigned)__bfloat16_as_ushort(lo) | ((unsigned)__bfloat16_as_ushort(hi) << 16);
}

// C[M x N] (FP32, ldc) (+)= op(A)[M x K] op(B)[K x N], BF16 operands.
// op(A)(r, c) = TA ? A[c * lda + r] : A[r * lda + c]
// op(B)(k, c) = TB ? B[c * ldb + k] : B[k * ldb + c]
// One warp computes a 16 x 32 tile with mma.sync.m16n8k16 (fragment layout of
// the PTX ISA: lane = 4 g + t holds rows g, g+8 and columns 2t, 2t+1, +8).
template <bool TA, bool TB>
__global__ void __launch_bounds__(128) k_gemm(const __nv_bfloat16* __restrict__ A, int lda,
                                              const __nv_bfloat16* __restrict__ B, int ldb, float* __restrict__ C,
                                              int ldc, int M, int N, int K, int accumulate, int k_chunk) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = (blockIdx.x * 4 + warp) * 16;
    const int n0 = blockIdx.y * 32;
    if (m0 >= M) return;
    // split K: slice z covers [kb, ke) and writes its own M x N partial
    const int kb = blockIdx.z * k_chunk;
    const int ke = kb + k_chunk < K ? kb + k_chunk : K;
    C += (size_t)blockIdx.z * M * ldc;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    auto ldA = [&](int r, int c) -> __nv_bfloat16 {
        if (r >= M || c >= ke) return zero;
        return TA ? A[(size_t)c * lda + r] : A[(size_t)r * lda + c];
    };
    auto ldB = [&](int k, int c) -> __nv_bfloat16 {
        if (k >= ke || c >= N) return zero;
        return TB ? B[(size_t)c * ldb + k] : B[(size_t)k * ldb + c];
    };
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
    for (int k0 = kb; k0 < ke; k0 += 16) {
        const int r0 = m0 + g, r1 = m0 + g + 8, c0 = k0 + 2 * t, c1 = k0 + 2 * t + 8;
        const unsigned a0 = pack_bf16(ldA(r0, c0), ldA(r0, c0 + 1));
        const unsigned a1 = pack_bf16(ldA(r1, c0), ldA(r1, c0 + 1));
        const unsigned a2 = pack_bf16(ldA(r0, c1), ldA(r0, c1 + 1));
        const unsigned a3 = pack_bf16(ldA(r1, c1), ldA(r1, c1 + 1));
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int col = n0 + 8 * j + g;
            const unsigned b0 = pack_bf16(ldB(c0, col), ldB(c0 + 1, col));
            const unsigned b1 = pack_bf16(ldB(c1, col), ldB(c1 + 1, col));
            asm volatile(
                "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                "{%0,%1,%2,%3};\n"
                : "+f"(acc[j][0]), "+f"(acc[j][1]), "+f"(acc[j][2]), "+f"(acc[j][3])
                : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int col = n0 + 8 * j + 2 * t;
        const int rows[2] = {m0 + g, m0 + g + 8};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = rows[h];
            if (r >= M) continue;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int cc = col + e;
                if (cc >= N) continue;
                float* dst = C + (size_t)r * ldc + cc;
                const float v = acc[j][2 * h + e];
                *dst = accumulate ? *dst + v : v;
            }
        }
    }
}

// sums the partial products of the K slices in slice order (deterministic)
__global__ void k_sum_slices(const float* __restrict__ part, int slices, long long mn, float* __restrict__ C) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= mn) return;
    float acc = 0.f;
    for (int z = 0; z < slices; ++z) acc += part[(size_t)z * mn + i];
    C[i] = acc;
}

template <bool TA, bool TB>
static int gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, float* C, int ldc, int M, int N, int K,
                bool accumulate, cudaStream_t s, DevBuf<float>* split_ws = nullptr) {
    // a long K over a small output (weight gradients: K = batch) is split into
    // slices of 1024 so that the whole GPU works on it
    int slices = 1, chunk = K;
    if (split_ws && !accumulate && ldc == N && (long long)div_up(M, 64) * div_up(N, 32) < 148 && K > 2048) {
        chunk = 1024;
        slices = (int)div_up(K, chunk);
        DWG_TRY(split_ws->reserve((size_t)slices * M * N));
    }
    dim3 grid(div_up(M, 64), div_up(N, 32), slices);
    float* dst = slices > 1 ? split_ws->ptr : C;
    k_gemm<TA, TB><<<grid, 128, 0, s>>>(A, lda, B, ldb, dst, ldc, M, N, K, accumulate ? 1 : 0, chunk);
    DWG_CHECK_LAUNCH();
    if (slices > 1) {
        const long long mn = (long long)M * N;
        k_sum_slices<<<div_up(mn, 256), 256, 0, s>>>(split_ws->ptr, slices, mn, C);
        DWG_CHECK_LAUNCH();
    }
    return DWG_OK;
}

// ------------------------------------------------------------ elementwise --
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.7071067811865476f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.7071067811865476f)) + x * 0.3989422804014327f * expf(-0.5f * x * x);
}

__global__ void k_pack_x(const float* __restrict__ F, long long n, __nv_bfloat16* __restrict__ X) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n * kMlpInPad) return;
    const long long r = i / kMlpInPad;
    const int c = (int)(i % kMlpInPad);
    X[i] = __float2bfloat16_rn(c < kMlpIn ? F[r * kMlpIn + c] : 0.f);
}

// z += b; h = bf16(gelu(z)) (hidden layers) -- z keeps the FP32 pre-activation
__global__ void k_bias_act(float* __restrict__ z, const float* __restrict__ b, __nv_bfloat16* __restrict__ h,
                           long long rows, int cols, int act) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    const float v = z[i] + b[i % cols];
    z[i] = v;
    if (act) h[i] = __float2bfloat16_rn(gelu(v));
}

// cosine loss of the first 3 outputs; dY (BF16, 8 columns) and the loss sum
__global__ void k_cos_loss(const float* __restrict__ y, const float* __restrict__ tgt, long long rows,
                           __nv_bfloat16* __restrict__ dy, float* __restrict__ loss) {
    long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    float l = 0.f;
    if (r < rows) {
        const float* yr = y + r * kMlpOutPad;
        const float* tr = tgt + r * 3;
        const float nn = sqrtf(yr[0] * yr[0] + yr[1] * yr[1] + yr[2] * yr[2]) + 1e-12f;
        const float yh[3] = {yr[0] / nn, yr[1] / nn, yr[2] / nn};
        const float c = yh[0] * tr[0] + yh[1] * tr[1] + yh[2] * tr[2];
        l = (1.0f - c) / (float)rows;
        for (int d = 0; d < kMlpOutPad; ++d) {
            float g = 0.f;
            if (d < 3) g = -(tr[d] - c * yh[d]) / nn / (float)rows;
            dy[r * kMlpOutPad + d] = __float2bfloat16_rn(g);
        }
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l);
}

// dZ = dH * gelu'(z): FP32 kept for the bias gradient, BF16 for the GEMMs
__global__ void k_gelu_back(const float* __restrict__ dh, const float* __restrict__ z, long long n,
                            float* __restrict__ dz, __nv_bfloat16* __restrict__ dzb) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = dh[i] * gelu_grad(z[i]);
    dz[i] = v;
    dzb[i] = __float2bfloat16_rn(v);
}

// column sums (bias gradients), one block per column, fixed order
__global__ void k_colsum_f32(const float* __restrict__ x, long long rows, int cols, float* __restrict__ out) {
    const int c = blockIdx.x;
    float acc = 0.f;
    for (long long r = threadIdx.x; r < rows; r += blockDim.x) acc += x[r * cols + c];
    __shared__ float sh[256];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = sh[0];
}

__global__ void k_colsum_bf16(const __nv_bfloat16* __restrict__ x, long long rows, int cols, float* __restrict__ out) {
    const int c = blockIdx.x;
    float acc = 0.f;
    for (long long r = threadIdx.x; r < rows; r += blockDim.x) acc += __bfloat162float(x[r * cols + c]);
    __shared__ float sh[256];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = sh[0];
}

__global__ void k_to_bf16(const float* __restrict__ x, long long n, __nv_bfloat16* __restrict__ y) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, long long n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_take3(const float* __restrict__ y, long long rows, float* __restrict__ out) {
    long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= rows) return;
    for (int d = 0; d < 3; ++d) out[r * 3 + d] = y[r * kMlpOutPad + d];
}

// --------------------------------------------------------------- host side --
static int ensure_cap(Mlp& m, long long B) {
    if (B <= m.cap) return DWG_OK;
    DWG_TRY(m.x.reserve((size_t)B * kMlpInPad));
    for (int l = 0; l < kMlpLayers; ++l) {
        DWG_TRY(m.z[l].reserve((size_t)B * m.dout[l]));
        DWG_TRY(m.h[l].reserve((size_t)B * m.dout[l]));
    }
    DWG_TRY(m.dz.reserve((size_t)B * kMlpHidden));
    DWG_TRY(m.dzb.reserve((size_t)B * kMlpHidden));
    DWG_TRY(m.dhb.reserve((size_t)B * kMlpHidden));
    m.cap = B;
    return DWG_OK;
}

static int refresh_bf16(Mlp& m, cudaStream_t s) {
    for (int l = 0; l < kMlpLayers; ++l) {
        const long long nw = (long long)m.din[l] * m.dout[l];
        k_to_bf16<<<div_up(nw, 256), 256, 0, s>>>(m.w[l].ptr, nw, m.wb[l].ptr);
    }
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

int mlp_init(Mlp& m, unsigned long long seed, cudaStream_t s) {
    std::mt19937_64 gen(seed);
    const int real_in[kMlpLayers] = {kMlpIn, kMlpHidden, kMlpHidden, kMlpHidden};
    const int real_out[kMlpLayers] = {kMlpHidden, kMlpHidden, kMlpHidden, kMlpOut};
    for (int l = 0; l < kMlpLayers; ++l) {
        const int din = m.din[l], dout = m.dout[l];
        std::vector<float> w((size_t)din * dout, 0.f), b(dout, 0.f);
        const float lim = std::sqrt(6.0f / (float)real_in[l]);
        std::uniform_real_distribution<float> U(-lim, lim);
        for (int i = 0; i < real_in[l]; ++i)
            for (int o = 0; o < real_out[l]; ++o) w[(size_t)i * dout + o] = U(gen) * (l == kMlpLayers - 1 ? 0.3f : 1.f);
        DWG_TRY(m.w[l].reserve(w.size()));
        DWG_TRY(m.b[l].reserve(b.size()));
        DWG_TRY(m.wb[l].reserve(w.size()));
        DWG_TRY(m.gw[l].reserve(w.size()));
        DWG_TRY(m.gb[l].reserve(b.size()));
        for (auto* buf : {&m.mw[l], &m.vw[l]}) {
            DWG_TRY(buf->reserve(w.size()));
            DWG_CHECK_CUDA(cudaMemsetAsync(buf->ptr, 0, sizeof(float) * w.size(), s));
        }
        for (auto* buf : {&m.mb[l], &m.vb[l]}) {
            DWG_TRY(buf->reserve(b.size()));
            DWG_CHECK_CUDA(cudaMemsetAsync(buf->ptr, 0, sizeof(float) * b.size(), s));
        }
        DWG_CHECK_CUDA(cudaMemcpyAsync(m.w[l].ptr, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice, s));
        DWG_CHECK_CUDA(cudaMemcpyAsync(m.b[l].ptr, b.data(), sizeof(float) * b.size(), cudaMemcpyHostToDevice, s));
    }
    DWG_TRY(m.loss.reserve(1));
    m.step = 0;
    DWG_TRY(refresh_bf16(m, s));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    return DWG_OK;
}

long long mlp_param_count() {
    const Mlp m;
    long long c = 0;
    for (int l = 0; l < kMlpLayers; ++l) c += (long long)m.din[l] * m.dout[l] + m.dout[l];
    return c;
}

int mlp_set_flat(Mlp& m, const float* params_host, cudaStream_t s) {
    DWG_REQUIRE(params_host, "mlp_set_flat: null parameters");
    const float* src = params_host;
    for (int l = 0; l < kMlpLayers; ++l) {
        const size_t nw = (size_t)m.din[l] * m.dout[l];
        DWG_CHECK_CUDA(cudaMemcpyAsync(m.w[l].ptr, src, sizeof(float) * nw, cudaMemcpyHostToDevice, s));
        src += nw;
        DWG_CHECK_CUDA(cudaMemcpyAsync(m.b[l].ptr, src, sizeof(float) * m.dout[l], cudaMemcpyHostToDevice, s));
        src += m.dout[l];
    }
    DWG_TRY(refresh_bf16(m, s));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    return DWG_OK;
}

static int copy_flat(const DevBuf<float>* w, const DevBuf<float>* b, const Mlp& m, float* dst, cudaStream_t s) {
    DWG_REQUIRE(dst, "mlp: null output");
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    for (int l = 0; l < kMlpLayers; ++l) {
        const size_t nw = (size_t)m.din[l] * m.dout[l];
        DWG_CHECK_CUDA(cudaMemcpy(dst, w[l].ptr, sizeof(float) * nw, cudaMemcpyDeviceToHost));
        dst += nw;
        DWG_CHECK_CUDA(cudaMemcpy(dst, b[l].ptr, sizeof(float) * m.dout[l], cudaMemcpyDeviceToHost));
        dst += m.dout[l];
    }
    return DWG_OK;
}

int mlp_get_flat(Mlp& m, float* params_host, cudaStream_t s) { return copy_flat(m.w, m.b, m, params_host, s); }
int mlp_get_grads_flat(Mlp& m, float* grads_host, cudaStream_t s) { return copy_flat(m.gw, m.gb, m, grads_host, s); }

// forward of rows [0, B) of the packed input m.x; leaves z[3] = outputs
static int forward_packed(Mlp& m, long long B, cudaStream_t s) {
    const __nv_bfloat16* in = m.x.ptr;
    int ld = kMlpInPad;
    for (int l = 0; l < kMlpLayers; ++l) {
        DWG_TRY(gemm<false, false>(in, ld, m.wb[l].ptr, m.dout[l], m.z[l].ptr, m.dout[l], (int)B, m.dout[l], m.din[l],
                                   false, s));
        const long long nz = B * m.dout[l];
        k_bias_act<<<div_up(nz, 256), 256, 0, s>>>(m.z[l].ptr, m.b[l].ptr, m.h[l].ptr, B, m.dout[l],
                                                   l < kMlpLayers - 1 ? 1 : 0);
        DWG_CHECK_LAUNCH();
        in = m.h[l].ptr;
        ld = m.dout[l];
    }
    return DWG_OK;
}

int mlp_forward(Mlp& m, const float* F, long long n, float* out, cudaStream_t s) {
    DWG_REQUIRE(F && out && n >= 0, "mlp_forward: bad arguments");
    const long long chunk = 1 << 16;
    DWG_TRY(ensure_cap(m, n < chunk ? (n > 0 ? n : 1) : chunk));
    for (long long r0 = 0; r0 < n; r0 += chunk) {
        const long long B = n - r0 < chunk ? n - r0 : chunk;
        k_pack_x<<<div_up(B * kMlpInPad, 256), 256, 0, s>>>(F + r0 * kMlpIn, B, m.x.ptr);
        DWG_CHECK_LAUNCH();
        DWG_TRY(forward_packed(m, B, s));
        k_take3<<<div_up(B, 256), 256, 0, s>>>(m.z[kMlpLayers - 1].ptr, B, out + r0 * 3);
        DWG_CHECK_LAUNCH();
    }
    return DWG_OK;
}

int mlp_backward(Mlp& m, const float* F, const float* T, long long B, float* loss_host, cudaStream_t s) {
    DWG_REQUIRE(F && T && B >= 1 && B < (1ll << 31), "mlp_backward: bad arguments");
    DWG_TRY(ensure_cap(m, B));
    k_pack_x<<<div_up(B * kMlpInPad, 256), 256, 0, s>>>(F, B, m.x.ptr);
    DWG_CHECK_LAUNCH();
    DWG_TRY(forward_packed(m, B, s));
    DWG_CHECK_CUDA(cudaMemsetAsync(m.loss.ptr, 0, sizeof(float), s));
    // dY in BF16 (8 columns), reusing dzb
    k_cos_loss<<<div_up(B, 256), 256, 0, s>>>(m.z[kMlpLayers - 1].ptr, T, B, m.dzb.ptr, m.loss.ptr);
    DWG_CHECK_LAUNCH();
    const __nv_bfloat16* dzb = m.dzb.ptr;  // dZ of the current layer, BF16
    for (int l = kMlpLayers - 1; l >= 0; --l) {
        const int din = m.din[l], dout = m.dout[l];
        const __nv_bfloat16* hin = l > 0 ? m.h[l - 1].ptr : m.x.ptr;
        // bias gradient
        if (l == kMlpLayers - 1)
            k_colsum_bf16<<<dout, 256, 0, s>>>(dzb, B, dout, m.gb[l].ptr);
        else
            k_colsum_f32<<<dout, 256, 0, s>>>(m.dz.ptr, B, dout, m.gb[l].ptr);
        DWG_CHECK_LAUNCH();
        // dW = H_in^T dZ
        DWG_TRY(gemm<true, false>(hin, din, dzb, dout, m.gw[l].ptr, dout, din, dout, (int)B, false, s, &m.split));
        if (l == 0) break;
        // dH_in = dZ W^T (FP32 into dz scratch), then dZ_in = dH_in * gelu'(z_in)
        float* dh = m.dz.ptr;
        DWG_TRY(gemm<false, true>(dzb, dout, m.wb[l].ptr, dout, dh, din, (int)B, din, dout, false, s));
        // the BF16 dZ of the layer below must not overwrite the one being read:
        // alternate between the two BF16 scratch buffers
        __nv_bfloat16* next = (dzb == m.dzb.ptr) ? m.dhb.ptr : m.dzb.ptr;
        k_gelu_back<<<div_up(B * din, 256), 256, 0, s>>>(dh, m.z[l - 1].ptr, B * din, m.dz.ptr, next);
        DWG_CHECK_LAUNCH();
        dzb = next;
    }
    if (loss_host) {
        DWG_CHECK_CUDA(cudaMemcpyAsync(loss_host, m.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost, s));
        DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    }
    return DWG_OK;
}

int mlp_adam(Mlp& m, float lr, float b1, float b2, float eps, cudaStream_t s) {
    m.step += 1;
    const float c1 = 1.f - std::pow(b1, (float)m.step), c2 = 1.f - std::pow(b2, (float)m.step);
    for (int l = 0; l < kMlpLayers; ++l) {
        const long long nw = (long long)m.din[l] * m.dout[l];
        k_adam<<<div_up(nw, 256), 256, 0, s>>>(m.w[l].ptr, m.mw[l].ptr, m.vw[l].ptr, m.gw[l].ptr, nw, lr, b1, b2, eps,
                                               c1, c2);
        k_adam<<<div_up(m.dout[l], 256), 256, 0, s>>>(m.b[l].ptr, m.mb[l].ptr, m.vb[l].ptr, m.gb[l].ptr, m.dout[l], lr,
                                                      b1, b2, eps, c1, c2);
    }
    DWG_CHECK_LAUNCH();
    return refresh_bf16(m, s);
}

__global__ void k_unit_or_gauss(const float* __restrict__ y, const float* __restrict__ P, int n,
                                const float* __restrict__ bb, float* __restrict__ N) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float a = y[(size_t)i * 3], b = y[(size_t)i * 3 + 1], c = y[(size_t)i * 3 + 2];
    const float len = sqrtf(a * a + b * b + c * c);
    if (len > 1e-12f && isfinite(len)) {
        N[(size_t)i * 3] = a / len;
        N[(size_t)i * 3 + 1] = b / len;
        N[(size_t)i * 3 + 2] = c / len;
        return;
    }
    // Gauss map (src/TurboNormalInit.cu:3-44)
    float v[3];
    for (int d = 0; d < 3; ++d) v[d] = __fsub_rn(P[(size_t)i * 3 + d], __fdiv_rn(__fadd_rn(bb[d], bb[3 + d]), 2.0f));
    const float sc = inv_len_eps(__fsqrt_rn(sq3_rn(v[0], v[1], v[2])));
    for (int d = 0; d < 3; ++d) N[(size_t)i * 3 + d] = __fmul_rn(v[d], sc);
}

int mlp_init_normals(Mlp& m, const KnnIndex& ix, const float* P, int n, float* N, cudaStream_t s) {
    DWG_REQUIRE(P && N && n >= 1, "mlp_init_normals: bad arguments");
    DevBuf<float> F, y;
    DWG_TRY(F.reserve((size_t)n * kMlpIn));
    DWG_TRY(y.reserve((size_t)n * 3));
    DWG_TRY(mlp_features(ix, P, n, F.ptr, s));
    DWG_TRY(mlp_forward(m, F.ptr, n, y.ptr, s));
    k_unit_or_gauss<<<div_up(n, 256), 256, 0, s>>>(y.ptr, P, n, ix.bbox.ptr, N);
    DWG_CHECK_LAUNCH();
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));  // F and y are released on return
    return DWG_OK;
}

}  // namespace dwg
