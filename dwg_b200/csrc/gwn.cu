// gwn.cu -- Barnes-Hut generalised-winding-number sums, one warp per 32 queries.
//
// The reference (src/TurboLibiGWN.cu:328-836) runs one thread per query over
// pointer-chasing AoS nodes with a stackless DFS.  Here a warp walks the
// octree for 32 spatially coherent queries at once (a 4x4x2 brick of grid
// samples, or 32 consecutive Morton-ordered points).  Every stack entry
// carries the mask of lanes that opened the node, so each lane still takes
// exactly the reference's per-query decisions -- a child is a dipole term
// when |CM - q| > beta R, otherwise it is opened, and leaves are summed point
// by point -- while node and point loads are warp-broadcast.  Sums are FP32
// with an optional compensated (two-sum) accumulator per lane.
#include "gwn.cuh"

namespace dwg {

constexpr int kGwnWarps = 8;
constexpr int kGwnStack = 8 * (kMaxDepth + 1) + 8;
constexpr float kFourPi = 12.566370614359172f;

// MUFU approximations without the subnormal fix-up paths
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2_ftz(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_ftz(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// One term of the sum for offset (dx,dy,dz) = p - q and d = A (p - q).n.
// Screened (src/TurboLibiGWN.cu:530-584): rho = max(|p-q|, s),
// v = (sigma rho + 1) d / (e^{sigma rho} 4 pi rho^3 + 1e-7) with the sign of d,
// skipped when |p-q| <= 1e-10.  Plain (:351-360): v = d / (4 pi |p-q|^3 + 1e-8).
// PREC < 2 uses the MUFU approximations (sigma_l2e = sigma log2 e);
// PREC 2 uses correctly rounded sqrt / division and expf.
template <bool SCREENED, int PREC>
__device__ __forceinline__ bool gwn_term(float dx, float dy, float dz, float d, float s, float sigma,
                                         float sigma_l2e, float& v) {
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    if (SCREENED) {
        if (!(r2 > 1e-20f)) return false;  // |p - q| <= 1e-10
        const float r = (PREC >= 2) ? sqrtf(r2) : r2 * rsqrt_ftz(r2);
        const float rho = fmaxf(r, s);
        const float e = (PREC >= 2) ? expf(sigma * rho) : ex2_ftz(rho * sigma_l2e);
        const float r3 = rho * rho * rho;
        const float den = fmaf(e, kFourPi * r3, 1e-7f);
        const float num = fmaf(sigma, rho, 1.0f) * d;
        const float res = (PREC >= 2) ? __fdiv_rn(num, den) : num * rcp_ftz(den);
        v = copysignf(fabsf(res), d);
        return true;
    } else {
        if (r2 == 0.0f) {
            v = 0.0f;
            return true;
        }
        const float r = (PREC >= 2) ? sqrtf(r2) : r2 * rsqrt_ftz(r2);
        const float den = fmaf(kFourPi * r, r2, 1e-8f);
        v = (PREC >= 2) ? __fdiv_rn(d, den) : d * rcp_ftz(den);
        return true;
    }
}

template <int PREC>
__device__ __forceinline__ void acc_add(float& s, float& c, float v) {
    if (PREC == 0) {
        s += v;
    } else {
        // Knuth two-sum: s + v = t + err exactly
        float t = __fadd_rn(s, v);
        float bp = __fsub_rn(t, s);
        float err = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(v, bp));
        s = t;
        c = __fadd_rn(c, err);
    }
}

struct GwnArgs {
    const int4* __restrict__ info;
    const float4* __restrict__ node_a;
    const float4* __restrict__ node_b;
    const float* __restrict__ node_r;
    const float4* __restrict__ pa;
    const float4* __restrict__ nr;
    float beta, sigma, screen;
    const float* sigma_dev;
    int use_radii;
    const float* __restrict__ q;
    long long nq;
    int rx, ry, rz;
    float ox, oy, oz, h;
    int bx, by;  // bricks per row / column
    long long ngroups;
    float* __restrict__ out;
    unsigned long long* terms_total;
    int* per_query_terms;
    unsigned int* work;  // [0] counter, [1] error flags (sticky)
    int num_nodes, num_points;
};

template <bool GRID, bool SCREENED, int PREC>
__global__ void __launch_bounds__(kGwnWarps * 32, 4) k_gwn(GwnArgs a) {
    __shared__ int2 stack[kGwnWarps][kGwnStack];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const float sigma = a.sigma_dev ? *a.sigma_dev : a.sigma;
    const float sigma_l2e = sigma * 1.4426950408889634f;
    unsigned long long my_terms = 0;
    for (;;) {
        unsigned g = 0;
        if (lane == 0) g = atomicAdd(&a.work[0], 1u);
        g = __shfl_sync(FULL, g, 0);
        if ((long long)g >= a.ngroups) break;
        bool valid;
        float qx = 0.f, qy = 0.f, qz = 0.f;
        long long qi;
        if (GRID) {
            int bxi = (int)(g % (unsigned)a.bx);
            unsigned t = g / (unsigned)a.bx;
            int byi = (int)(t % (unsigned)a.by);
            int bzi = (int)(t / (unsigned)a.by);
            int x = bxi * 4 + (lane & 3), y = byi * 4 + ((lane >> 2) & 3), z = bzi * 2 + (lane >> 4);
            valid = x < a.rx && y < a.ry && z < a.rz;
            qi = (long long)x + (long long)a.rx * ((long long)y + (long long)a.ry * z);
            qx = __fadd_rn(a.ox, __fmul_rn((float)x, a.h));
            qy = __fadd_rn(a.oy, __fmul_rn((float)y, a.h));
            qz = __fadd_rn(a.oz, __fmul_rn((float)z, a.h));
        } else {
            qi = (long long)g * 32 + lane;
            valid = qi < a.nq;
            if (valid) {
                qx = a.q[qi * 3];
                qy = a.q[qi * 3 + 1];
                qz = a.q[qi * 3 + 2];
            }
        }
        const unsigned vm = __ballot_sync(FULL, valid);
        float s = 0.f, c = 0.f;
        int nterm = 0;

        auto leaf_points = [&](int start, int cnt) {
            for (int j = start; j < start + cnt; ++j) {
                float4 p = a.pa[j];
                float4 nn = a.nr[j];
                float dx = p.x - qx, dy = p.y - qy, dz = p.z - qz;
                float d = p.w * fmaf(dx, nn.x, fmaf(dy, nn.y, dz * nn.z));
                float sc = a.use_radii ? nn.w : a.screen;
                float v;
                if (gwn_term<SCREENED, PREC>(dx, dy, dz, d, sc, sigma, sigma_l2e, v)) {
                    acc_add<PREC>(s, c, v);
                    ++nterm;
                }
            }
        };

        // one child record (level order): a single-point leaf is one term, a
        // larger leaf is summed point by point, an internal node is a dipole
        // term when far for this lane and is opened (pushed with the lanes
        // that need it) otherwise
        auto child = [&](int cidx, const float4& na, const float4& nb, bool act, int& sp) {
            const unsigned meta = (unsigned)__float_as_int(nb.w);
            if (meta & kMetaLeafBit) {
                if ((meta & kMetaSingle) && !a.use_radii) {
                    if (act) {
                        const float dx = na.x - qx, dy = na.y - qy, dz = na.z - qz;
                        const float d = fmaf(dx, nb.x, fmaf(dy, nb.y, dz * nb.z));
                        float v;
                        if (gwn_term<SCREENED, PREC>(dx, dy, dz, d, a.screen, sigma, sigma_l2e, v)) {
                            acc_add<PREC>(s, c, v);
                            ++nterm;
                        }
                    }
                } else {
                    const int st = (int)(meta & kMetaIndex), cnt = __float_as_int(na.w);
                    if (cnt < 0 || st + cnt > a.num_points) {
                        if (lane == 0) atomicOr(&a.work[1], 4u);
                    } else if (act) {
                        leaf_points(st, cnt);
                    }
                }
                return;
            }
            bool near = false;
            if (act) {
                // opening test sqrt_rn(d2) > beta*R, d2 in round-to-nearest
                // single precision (src/TurboLibiGWN.cu:636-644), as a
                // comparison of d2 with the node's exact threshold
                const float dx = __fsub_rn(na.x, qx), dy = __fsub_rn(na.y, qy), dz = __fsub_rn(na.z, qz);
                const float d2 = sq3_rn(dx, dy, dz);
                const float thr = fabsf(na.w);
                bool far = d2 > thr;
                if (!far && d2 == thr && signbit(na.w)) far = __fsqrt_rn(d2) > __fmul_rn(a.beta, a.node_r[cidx]);
                if (far) {
                    const float d = fmaf(dx, nb.x, fmaf(dy, nb.y, dz * nb.z));
                    float v;
                    if (gwn_term<SCREENED, PREC>(dx, dy, dz, d, a.screen, sigma, sigma_l2e, v)) {
                        acc_add<PREC>(s, c, v);
                        ++nterm;
                    }
                } else {
                    near = true;
                }
            }
            const unsigned nm = __ballot_sync(FULL, near);
            if (nm) {
                if (sp < kGwnStack) {
                    if (lane == 0) stack[w][sp] = make_int2(cidx, (int)nm);
                    ++sp;
                } else if (lane == 0) {
                    atomicOr(&a.work[1], 1u);
                }
            }
        };

        int sp = 0;
        {
            const float4 ra = a.node_a[0], rb = a.node_b[0];
            const unsigned rm = (unsigned)__float_as_int(rb.w);
            if (rm & kMetaLeafBit) {
                child(0, ra, rb, valid, sp);  // a leaf root is summed; nothing is pushed
            } else {
                if (lane == 0) stack[w][0] = make_int2(0, (int)vm);
                sp = 1;
            }
        }
        while (sp > 0) {
            __syncwarp();
            const int2 e = stack[w][--sp];
            __syncwarp();
            if (e.x < 0 || e.x >= a.num_nodes) {
                if (lane == 0) atomicOr(&a.work[1], 2u);
                continue;
            }
            const bool act = (((unsigned)e.y) >> lane) & 1u;
            const unsigned pm = (unsigned)__float_as_int(a.node_b[e.x].w);
            const int first = (int)(pm & kMetaIndex);
            const int nch = (int)((pm >> 28) & 7u) + 1;
            // structural guard: children come after the parent, inside the table
            if ((pm & kMetaLeafBit) || first <= e.x || first + nch > a.num_nodes) {
                if (lane == 0) atomicOr(&a.work[1], 2u);
                continue;
            }
            float4 na = a.node_a[first], nb = a.node_b[first];
            for (int j = 0; j < nch; ++j) {
                float4 na2, nb2;
                if (j + 1 < nch) {  // load the next sibling while this one is evaluated
                    na2 = a.node_a[first + j + 1];
                    nb2 = a.node_b[first + j + 1];
                }
                child(first + j, na, nb, act, sp);
                na = na2;
                nb = nb2;
            }
        }
        if (valid) {
            a.out[qi] = (PREC == 0) ? s : __fadd_rn(s, c);
            if (a.per_query_terms) a.per_query_terms[qi] = nterm;
        }
        my_terms += (unsigned long long)nterm;
    }
    if (a.terms_total) {
        for (int o = 16; o > 0; o >>= 1) my_terms += __shfl_down_sync(FULL, my_terms, o);
        if (lane == 0 && my_terms) atomicAdd(a.terms_total, my_terms);
    }
}

template <bool GRID, bool SCREENED, int PREC>
static int launch(const GwnArgs& a, cudaStream_t s) {
    static int blocks_per_sm = 0;
    if (!blocks_per_sm) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_gwn<GRID, SCREENED, PREC>,
                                                      kGwnWarps * 32, 0);
        if (blocks_per_sm <= 0) blocks_per_sm = 1;
    }
    long long want = (a.ngroups + kGwnWarps - 1) / kGwnWarps;
    long long grid = (long long)num_sms() * blocks_per_sm;
    if (want < grid) grid = want > 0 ? want : 1;
    k_gwn<GRID, SCREENED, PREC><<<(unsigned)grid, kGwnWarps * 32, 0, s>>>(a);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

template <bool GRID>
static int dispatch(const GwnArgs& a, const dwg_gwn_params& p, cudaStream_t s) {
    const int prec = p.precision < 0 ? 0 : (p.precision > 2 ? 2 : p.precision);
    if (p.screened) {
        if (prec == 0) return launch<GRID, true, 0>(a, s);
        if (prec == 1) return launch<GRID, true, 1>(a, s);
        return launch<GRID, true, 2>(a, s);
    }
    if (prec == 0) return launch<GRID, false, 0>(a, s);
    if (prec == 1) return launch<GRID, false, 1>(a, s);
    return launch<GRID, false, 2>(a, s);
}

int gwn_eval(const Octree& t, const GwnQuery& q, const dwg_gwn_params& p, float* out,
             unsigned long long* terms_total, int* per_query_terms, cudaStream_t s,
             const float* sigma_dev) {
    DWG_REQUIRE(t.M > 0, "gwn: octree is empty");
    DWG_REQUIRE(out != nullptr, "gwn: output is null");
    GwnArgs a;
    a.info = t.info.ptr;
    DWG_TRY(octree_set_beta(const_cast<Octree&>(t), p.beta, s));
    a.node_a = t.node_a.ptr;
    a.node_b = t.node_b.ptr;
    a.node_r = t.node_r.ptr;
    a.pa = t.pa.ptr;
    a.nr = t.nr.ptr;
    a.beta = p.beta;
    a.sigma = p.sigma;
    a.sigma_dev = sigma_dev;
    a.screen = p.screen;
    a.use_radii = p.use_radii;
    a.out = out;
    a.terms_total = terms_total;
    a.per_query_terms = per_query_terms;
    DWG_TRY(t.work.reserve(2));
    a.work = t.work.ptr;
    a.num_nodes = t.M;
    a.num_points = t.n;
    // the counter restarts with every launch; the error word is sticky
    DWG_CHECK_CUDA(cudaMemsetAsync(t.work.ptr, 0, sizeof(unsigned int), s));
    if (q.q) {
        a.q = q.q;
        a.nq = q.nq;
        a.rx = a.ry = a.rz = 0;
        a.ox = a.oy = a.oz = a.h = 0.f;
        a.bx = a.by = 1;
        a.ngroups = (q.nq + 31) / 32;
        if (a.ngroups == 0) return DWG_OK;
        return dispatch<false>(a, p, s);
    }
    DWG_REQUIRE(q.res[0] > 0 && q.res[1] > 0 && q.res[2] > 0, "gwn: bad grid resolution");
    a.q = nullptr;
    a.nq = (long long)q.res[0] * q.res[1] * q.res[2];
    a.rx = q.res[0];
    a.ry = q.res[1];
    a.rz = q.res[2];
    a.ox = q.origin[0];
    a.oy = q.origin[1];
    a.oz = q.origin[2];
    a.h = q.spacing;
    a.bx = (q.res[0] + 3) / 4;
    a.by = (q.res[1] + 3) / 4;
    a.ngroups = (long long)a.bx * a.by * ((q.res[2] + 1) / 2);
    DWG_REQUIRE(a.ngroups < (1ll << 32), "gwn: grid too large");
    return dispatch<true>(a, p, s);
}

}  // namespace dwg
