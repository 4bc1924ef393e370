// tune.cu -- autotuner for the grid sums: Barnes-Hut opening ratio and brick
// shape.
//
// For one cloud: build the pipeline, run a few DWG iterations so that the
// normals are realistic, then
//   1. draw `samples` grid samples (seeded) and sum them exactly (every node
//      opened; correctly rounded terms, FP64 accumulation);
//   2. for each candidate opening ratio, the RMS and max error of the
//      Barnes-Hut sums at those samples against the exact ones;
//   3. among the ratios within `tol` (tol <= 0: within the error of the
//      reference's beta = 2.3), time a full grid evaluation and keep the
//      fastest; then time the four brick shapes at that ratio.
// The reference setting (beta 2.3, 4x4x2 bricks) is timed beside it.
#include <algorithm>
#include <random>
#include <vector>

#include "pipeline.cuh"
#include "tune.cuh"

namespace dwg {

static const float kBetas[] = {1.5f, 1.8f, 2.0f, 2.3f, 2.6f, 3.0f, 3.5f, 4.5f};

__global__ void k_sample_grid(const long long* __restrict__ idx, int m, int rx, int ry, float ox, float oy, float oz,
                              float h, float* __restrict__ q) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const long long v = idx[i];
    const long long x = v % rx, y = (v / rx) % ry, z = v / ((long long)rx * ry);
    q[(size_t)i * 3] = __fadd_rn(ox, __fmul_rn((float)x, h));
    q[(size_t)i * 3 + 1] = __fadd_rn(oy, __fmul_rn((float)y, h));
    q[(size_t)i * 3 + 2] = __fadd_rn(oz, __fmul_rn((float)z, h));
}

static int time_grid(Pipeline& p, const dwg_gwn_params& gp, float* ms, cudaStream_t s) {
    GwnQuery qg;
    for (int d = 0; d < 3; ++d) {
        qg.res[d] = p.gres[d];
        qg.origin[d] = p.gorg[d];
    }
    qg.spacing = p.gh;
    cudaEvent_t e0, e1;
    DWG_CHECK_CUDA(cudaEventCreate(&e0));
    DWG_CHECK_CUDA(cudaEventCreate(&e1));
    std::vector<float> t;
    int st = DWG_OK;
    for (int r = 0; r < 4 && st == DWG_OK; ++r) {  // first one warms up
        cudaEventRecord(e0, s);
        st = gwn_eval(p.t2, qg, gp, p.field.ptr, nullptr, nullptr, s, p.cur_sigma.ptr);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = DWG_ERR_CUDA;
        float x = 0.f;
        cudaEventElapsedTime(&x, e0, e1);
        if (r > 0) t.push_back(x);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != DWG_OK) return st;
    std::sort(t.begin(), t.end());
    *ms = t[t.size() / 2];
    return DWG_OK;
}

int autotune(const float* points_dev, int n, const dwg_params& prm, float tol, int samples, int warm_iters,
             cudaStream_t stream, dwg_tune_result* out) {
    DWG_REQUIRE(out && samples >= 32, "autotune: bad arguments");
    Pipeline p;
    DWG_TRY(p.setup(points_dev, nullptr, n, prm, stream));
    DWG_TRY(p.iterate(warm_iters > 0 ? warm_iters : 1));
    cudaStream_t s = p.s;
    DWG_TRY(p.join_in());
    const long long ng = (long long)p.gres[0] * p.gres[1] * p.gres[2];
    const int m = (int)std::min<long long>(samples, ng);
    // seeded sample of grid indices
    std::vector<long long> idx((size_t)m);
    std::mt19937_64 gen(12345);
    std::uniform_int_distribution<long long> U(0, ng - 1);
    for (auto& v : idx) v = U(gen);
    DevBuf<long long> idx_d;
    DevBuf<float> q, w_exact, w;
    DWG_TRY(idx_d.reserve(m));
    DWG_TRY(q.reserve((size_t)m * 3));
    DWG_TRY(w_exact.reserve(m));
    DWG_TRY(w.reserve(m));
    DWG_CHECK_CUDA(cudaMemcpyAsync(idx_d.ptr, idx.data(), sizeof(long long) * m, cudaMemcpyHostToDevice, s));
    k_sample_grid<<<div_up(m, 256), 256, 0, s>>>(idx_d.ptr, m, p.gres[0], p.gres[1], p.gorg[0], p.gorg[1],
                                                 p.gorg[2], p.gh, q.ptr);
    DWG_CHECK_LAUNCH();
    GwnQuery qs;
    qs.q = q.ptr;
    qs.nq = m;
    dwg_gwn_params gp = p.gwn_params();
    // exact sums: every node opened (a threshold no distance exceeds)
    dwg_gwn_params ge = gp;
    ge.beta = 1e18f;
    ge.precision = 2;
    DWG_TRY(gwn_eval(p.t2, qs, ge, w_exact.ptr, nullptr, nullptr, s, p.cur_sigma.ptr));
    std::vector<float> we((size_t)m), wb((size_t)m);
    DWG_CHECK_CUDA(cudaMemcpyAsync(we.data(), w_exact.ptr, sizeof(float) * m, cudaMemcpyDeviceToHost, s));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    // error of each opening ratio against the exact sums
    double fsq = 0;
    for (int i = 0; i < m; ++i) fsq += (double)we[i] * we[i];
    constexpr int nb = sizeof(kBetas) / sizeof(kBetas[0]);
    float rms_of[nb], max_of[nb];
    float ref_rms = 0.f;
    for (int bi = 0; bi < nb; ++bi) {
        dwg_gwn_params gb = gp;
        gb.beta = kBetas[bi];
        DWG_TRY(gwn_eval(p.t2, qs, gb, w.ptr, nullptr, nullptr, s, p.cur_sigma.ptr));
        DWG_CHECK_CUDA(cudaMemcpyAsync(wb.data(), w.ptr, sizeof(float) * m, cudaMemcpyDeviceToHost, s));
        DWG_CHECK_CUDA(cudaStreamSynchronize(s));
        double se = 0, mx = 0;
        for (int i = 0; i < m; ++i) {
            const double e = (double)wb[i] - (double)we[i];
            se += e * e;
            mx = std::max(mx, std::fabs(e));
        }
        rms_of[bi] = (float)std::sqrt(se / m);
        max_of[bi] = (float)mx;
        if (kBetas[bi] == 2.3f) ref_rms = rms_of[bi];
    }
    // tol <= 0: no less accurate than the reference's beta = 2.3
    const float limit = tol > 0.f ? tol : ref_rms * 1.000001f;
    float best_beta = -1.f, best_ms = 0.f, best_rms = 0.f, best_max = 0.f;
    for (int bi = 0; bi < nb; ++bi) {
        if (rms_of[bi] > limit) continue;
        dwg_gwn_params gb = gp;
        gb.beta = kBetas[bi];
        float ms = 0.f;
        DWG_TRY(time_grid(p, gb, &ms, s));
        if (best_beta < 0.f || ms < best_ms) {
            best_beta = kBetas[bi];
            best_ms = ms;
            best_rms = rms_of[bi];
            best_max = max_of[bi];
        }
    }
    out->ref_rms_err = ref_rms;
    out->field_rms = (float)std::sqrt(fsq / m);
    DWG_REQUIRE(best_beta > 0.f, "autotune: no opening ratio reaches RMS error %g", limit);
    // brick shape at that ratio
    int best_tile = 0;
    float tile_ms = 0.f;
    for (int tile = 0; tile < 4; ++tile) {
        dwg_gwn_params gt = gp;
        gt.beta = best_beta;
        gt.tile = tile;
        float ms = 0.f;
        DWG_TRY(time_grid(p, gt, &ms, s));
        if (tile == 0 || ms < tile_ms) {
            tile_ms = ms;
            best_tile = tile;
        }
    }
    best_ms = tile_ms;
    // the reference setting
    dwg_gwn_params gr = gp;
    gr.beta = 2.3f;
    gr.tile = 0;
    float ref_ms = 0.f;
    DWG_TRY(time_grid(p, gr, &ref_ms, s));
    out->beta = best_beta;
    out->tile = best_tile;
    out->rms_err = best_rms;
    out->max_err = best_max;
    out->grid_ms = best_ms;
    out->ref_ms = ref_ms;
    return p.join_out();
}

}  // namespace dwg
