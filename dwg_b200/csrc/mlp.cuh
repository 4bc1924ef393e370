// mlp.cuh -- the learned normal initialiser: per-point features and a small
// MLP (12 -> 128 -> 128 -> 128 -> 3, GELU) with BF16 weights and activations
// feeding tensor-core GEMMs that accumulate in FP32.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "knn.cuh"

namespace dwg {

constexpr int kMlpIn = 12;    // features
constexpr int kMlpInPad = 16; // padded to the MMA k step
constexpr int kMlpHidden = 128;
constexpr int kMlpOut = 3;
constexpr int kMlpOutPad = 8;  // padded to the MMA n step
constexpr int kMlpLayers = 4;
constexpr int kMlpFeatureK = 16;  // neighbours of the covariance features
constexpr int kMlpWideK = 64;     // neighbours of the centroid offset ...
constexpr int kMlpWideStride = 4; // ... among every 4th point

struct Mlp {
    // layer l maps dims[l] -> dims[l+1] (padded): W_l is [din x dout] row-major
    int din[kMlpLayers] = {kMlpInPad, kMlpHidden, kMlpHidden, kMlpHidden};
    int dout[kMlpLayers] = {kMlpHidden, kMlpHidden, kMlpHidden, kMlpOutPad};
    DevBuf<float> w[kMlpLayers], b[kMlpLayers];             // FP32 master
    DevBuf<__nv_bfloat16> wb[kMlpLayers];                   // BF16 copy for the GEMMs
    DevBuf<float> mw[kMlpLayers], vw[kMlpLayers], mb[kMlpLayers], vb[kMlpLayers];  // Adam
    DevBuf<float> gw[kMlpLayers], gb[kMlpLayers];           // gradients
    long long step = 0;
    // activations of the last forward (batch capacity)
    long long cap = 0;
    DevBuf<__nv_bfloat16> x;                                // [B x 16]
    DevBuf<float> z[kMlpLayers];                            // pre-activations
    DevBuf<__nv_bfloat16> h[kMlpLayers];                    // post-activations (h[3] unused)
    DevBuf<float> dz;                                       // [B x 128] scratch
    DevBuf<__nv_bfloat16> dzb, dhb;
    DevBuf<float> loss;
    DevBuf<float> split;  // partial products of split-K weight-gradient GEMMs
};

// Flat parameter layout (host and files): for l = 0..3, W_l [din x dout]
// row-major then b_l [dout], padded sizes; padding entries are zero.
long long mlp_param_count();

int mlp_init(Mlp& m, unsigned long long seed, cudaStream_t s);
int mlp_set_flat(Mlp& m, const float* params_host, cudaStream_t s);
int mlp_get_flat(Mlp& m, float* params_host, cudaStream_t s);
int mlp_get_grads_flat(Mlp& m, float* grads_host, cudaStream_t s);
// features [n x 12] of points (xyz, n) from their k=16 nearest neighbours in
// `ix` (built on the same points); the eigenvectors are oriented away from the
// centre of the index's bounding box
int mlp_features(const KnnIndex& ix, const float* points, int n, float* features, cudaStream_t s);
// raw network outputs [n x 3]
int mlp_forward(Mlp& m, const float* features, long long n, float* out, cudaStream_t s);
// loss = mean(1 - <y/|y|, t>); fills the gradients; loss_host may be null
int mlp_backward(Mlp& m, const float* features, const float* targets, long long n, float* loss_host,
                 cudaStream_t s);
int mlp_adam(Mlp& m, float lr, float beta1, float beta2, float eps, cudaStream_t s);
// initial normals of points indexed by `ix`: features, forward, normalise;
// an output of length below 1e-12 or not finite falls back to the Gauss map
// about the centre of the index's bounding box
int mlp_init_normals(Mlp& m, const KnnIndex& ix, const float* points, int n, float* normals, cudaStream_t s);

}  // namespace dwg
