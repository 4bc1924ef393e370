// gwn.cu -- Barnes-Hut generalised-winding-number sums, one warp per 32 queries.
//
// The reference (src/TurboLibiGWN.cu:328-836) runs one thread per query over
// pointer-chasing AoS nodes with a stackless DFS.  Here a warp walks the
// octree for 32 spatially coherent queries at once (a 4x4x2 brick of grid
// samples, or 32 consecutive Morton-ordered points).  Every stack entry
// carries the mask of lanes that opened the node, so each lane still takes
// exactly the reference's per-query decisions -- a child is a dipole term
// when |CM - q| > beta R, otherwise it is opened, and leaves are summed point
// by point -- while node and point loads are warp-broadcast.  Terms are
// FP32; each query's sum is FP32 (precision 0), FP64 (precision 1 and 2) or
// compensated FP32 (precision 3, Neumaier).
#include "gwn.cuh"

#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

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
// PREC != 2 uses the MUFU approximations (sigma_l2e = sigma log2 e);
// PREC 2 uses correctly rounded sqrt / division and expf.
template <bool SCREENED, int PREC>
__device__ __forceinline__ bool gwn_term_r2(float r2, float d, float s, float sigma, float sigma_l2e, float& v) {
    if (SCREENED) {
        if (!(r2 > 1e-20f)) return false;  // |p - q| <= 1e-10
        const float r = (PREC == 2) ? sqrtf(r2) : r2 * rsqrt_ftz(r2);
        const float rho = fmaxf(r, s);
        const float e = (PREC == 2) ? expf(sigma * rho) : ex2_ftz(rho * sigma_l2e);
        const float r3 = rho * rho * rho;
        const float den = fmaf(e, kFourPi * r3, 1e-7f);
        // the reference forces the sign of d onto the term
        // (src/TurboLibiGWN.cu:550-584); den > 0, so |sigma rho + 1| d does
        // that (an operand modifier, no extra instruction)
        const float num = fabsf(fmaf(sigma, rho, 1.0f)) * d;
        v = (PREC == 2) ? __fdiv_rn(num, den) : num * rcp_ftz(den);
        return true;
    } else {
        if (r2 == 0.0f) {
            v = 0.0f;
            return true;
        }
        const float r = (PREC == 2) ? sqrtf(r2) : r2 * rsqrt_ftz(r2);
        const float den = fmaf(kFourPi * r, r2, 1e-8f);
        v = (PREC == 2) ? __fdiv_rn(d, den) : d * rcp_ftz(den);
        return true;
    }
}

template <bool SCREENED, int PREC>
__device__ __forceinline__ bool gwn_term(float dx, float dy, float dz, float d, float s, float sigma,
                                         float sigma_l2e, float& v) {
    return gwn_term_r2<SCREENED, PREC>(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), d, s, sigma, sigma_l2e, v);
}

// A sum of FP32 terms kept in FP32 with Neumaier's compensation (the
// improved Kahan-Babuska summation, Neumaier 1974): s is the rounded running
// sum and c collects the rounding error of every addition, taken exactly
// from the larger and the smaller operand; the sum is s + c, rounded once.
// Its error is about that of summing in twice the precision, independent of
// the number of terms up to ~1/eps of them.
struct CompSum {
    float s, c;
    CompSum() = default;
    __device__ CompSum(float v) : s(v), c(0.f) {}
    __device__ __forceinline__ void add(float v) {
        const float t = __fadd_rn(s, v);
        const bool sbig = fabsf(s) >= fabsf(v);
        const float big = sbig ? s : v, small = sbig ? v : s;
        c = __fadd_rn(c, __fadd_rn(__fsub_rn(big, t), small));
        s = t;
    }
    __device__ __forceinline__ CompSum& operator+=(const CompSum& o) {
        add(o.s);
        c = __fadd_rn(c, o.c);
        return *this;
    }
    __device__ __forceinline__ explicit operator float() const { return __fadd_rn(s, c); }
};

// per-query accumulator: FP32 (PREC 0); FP64 (PREC 1 and 2: each FP32 term
// converted exactly and added in double, one conversion and one add per
// term); compensated FP32 (PREC 3)
template <int PREC>
struct AccType {
    using T = double;
};
template <>
struct AccType<0> {
    using T = float;
};
template <>
struct AccType<3> {
    using T = CompSum;
};

// brick shapes of 32 grid samples (x, y, z extents) a warp evaluates together
template <int SHAPE>
struct Brick;
template <>
struct Brick<0> {
    static constexpr int X = 4, Y = 4, Z = 2;
};
template <>
struct Brick<1> {
    static constexpr int X = 8, Y = 4, Z = 1;
};
template <>
struct Brick<2> {
    static constexpr int X = 2, Y = 4, Z = 4;
};
template <>
struct Brick<3> {
    static constexpr int X = 8, Y = 2, Z = 2;
};

__host__ __device__ inline void brick_extent(int shape, int& x, int& y, int& z) {
    x = shape == 1 || shape == 3 ? 8 : (shape == 2 ? 2 : 4);
    y = shape == 3 ? 2 : 4;
    z = shape == 1 ? 1 : (shape == 0 ? 2 : (shape == 2 ? 4 : 2));
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
    int zoff;  // global z index of local sample 0 (grid slabs)
    float ox, oy, oz, h;
    int bx, by;  // bricks per row / column
    long long ngroups;
    float* __restrict__ out;
    unsigned long long* terms_total;
    int* per_query_terms;
    unsigned int* work;  // [0] counter, [1] error flags (sticky)
    int num_nodes, num_points;
    const float4* __restrict__ node_h;  // expansion records, 8 float4 each (plain sums, order >= 1)
    // interaction lists (grids): per-group entry counts (counting pass), the
    // groups' first entries (ngroups + 1) and the entries
    unsigned int* list_count;
    const unsigned long long* __restrict__ list_off;
    int4* list;
    // cached screening weights of the list's node entries (grids, NQ = 2):
    // slot c holds, per entry and lane, the weights of the lane's two
    // samples; wsel picks the launch's mode and slot on the device
    float2* wbuf;
    unsigned long long wstride;  // float2 per slot = entries * 32
    GwnWeightState* wsel;
};

// The screening weight of a far-node term with the MUFU approximations:
// g = |sigma rho + 1| / (e^{sigma rho} 4 pi rho^3 + 1e-7), 0 where no term is
// taken; the term is g d.  g depends on the geometry and sigma only, so the
// interaction-list replay can keep it across iterations with the same sigma
// and still produce the same bits.
__device__ __forceinline__ float screen_weight_masked(bool take, float r2, float s, float sigma, float sigma_l2e,
                                                      bool& ok) {
    ok = take && r2 > 1e-20f;  // |p - q| <= 1e-10 is skipped
    const float r2s = ok ? r2 : 1.0f;
    const float rho = fmaxf(r2s * rsqrt_ftz(r2s), s);
    const float den = fmaf(ex2_ftz(rho * sigma_l2e), kFourPi * (rho * rho * rho), 1e-7f);
    // the reference forces the sign of d onto the term
    // (src/TurboLibiGWN.cu:550-584); den > 0 and |sigma rho + 1| > 0 do that
    const float g = fabsf(fmaf(sigma, rho, 1.0f)) * rcp_ftz(den);
    return ok ? g : 0.f;
}

template <bool SCREENED, int PREC>
__device__ __forceinline__ float gwn_term_masked(bool take, float r2, float d, float s, float sigma,
                                                 float sigma_l2e, bool& counted) {
    float v = 0.f;
    counted = false;
    if (SCREENED && PREC != 2) {
        v = __fmul_rn(screen_weight_masked(take, r2, s, sigma, sigma_l2e, counted), d);
    } else if (SCREENED) {
        const bool ok = take && r2 > 1e-20f;  // |p - q| <= 1e-10 is skipped
        const float r2s = ok ? r2 : 1.0f;
        const float rho = fmaxf(sqrtf(r2s), s);
        const float den = fmaf(expf(sigma * rho), kFourPi * (rho * rho * rho), 1e-7f);
        // the reference forces the sign of d onto the term
        // (src/TurboLibiGWN.cu:550-584); den > 0, so |sigma rho + 1| d does
        // that (an operand modifier, no extra instruction)
        const float t = __fdiv_rn(fabsf(fmaf(sigma, rho, 1.0f)) * d, den);
        v = ok ? t : 0.f;
        counted = ok;
    } else {
        const bool zero = r2 == 0.0f;  // a zero distance is a term of value 0
        const float r2s = (take && !zero) ? r2 : 1.0f;
        const float r = (PREC == 2) ? sqrtf(r2s) : r2s * rsqrt_ftz(r2s);
        const float den = fmaf(kFourPi * r, r2s, 1e-8f);
        const float t = (PREC == 2) ? __fdiv_rn(d, den) : d * rcp_ftz(den);
        v = (take && !zero) ? t : 0.f;
        counted = take;
    }
    return v;
}

// Higher-order far field of the plain sum (igl::fast_winding_number
// expansion_eval, deps/libigl/include/igl/fast_winding_number.cpp:187-241):
// with loc = CM - q, r = |loc| and the node's coefficients m1 (9), m2 (27),
//   order 1: sum_uv (delta_uv / (4 pi r^3) - 3 loc_u loc_v / (4 pi r^5)) m1[u + 3v]
//          = tr(m1) / (4 pi r^3) - 3 loc^T m1 loc / (4 pi r^5)
//   order 2: + sum_i sum_uv (15 loc_i loc_u loc_v / (4 pi r^7)
//              - 3 (loc_i delta_uv + loc_v delta_ui + loc_u delta_vi) / (4 pi r^5)) m2[9i + u + 3v]
//          = 15 sum_v loc_v sum_{i<=u} loc_i loc_u s(i,u,v) / (4 pi r^7) - 3 loc.g / (4 pi r^5)
// on the node record's contraction (m1, tr m1, g, s; see octree.cuh); the
// order-0 dipole is the usual term.
template <int ORDER, int PREC>
__device__ __forceinline__ float fwn_correction(float lx, float ly, float lz, float r2, const float4* __restrict__ H) {
    const float r = (PREC == 2) ? sqrtf(r2) : r2 * rsqrt_ftz(r2);
    const float p3 = kFourPi * r * r * r;
    const float p5 = p3 * r * r;
    const float d = (PREC == 2) ? __fdiv_rn(1.0f, p3) : rcp_ftz(p3);
    const float c5 = (PREC == 2) ? __fdiv_rn(-3.0f, p5) : -3.0f * rcp_ftz(p5);
    float h[32];
#pragma unroll
    for (int t = 0; t < (ORDER >= 2 ? 8 : 3); ++t) {
        const float4 c = H[t];
        h[4 * t] = c.x;
        h[4 * t + 1] = c.y;
        h[4 * t + 2] = c.z;
        h[4 * t + 3] = c.w;
    }
    // loc^T m1 loc
    const float mx = fmaf(h[0], lx, fmaf(h[3], ly, h[6] * lz));
    const float my = fmaf(h[1], lx, fmaf(h[4], ly, h[7] * lz));
    const float mz = fmaf(h[2], lx, fmaf(h[5], ly, h[8] * lz));
    const float q1 = fmaf(lx, mx, fmaf(ly, my, lz * mz));
    float w = fmaf(d, h[9], c5 * q1);
    if (ORDER >= 2) {
        const float p7 = p5 * r * r;
        const float i15 = (PREC == 2) ? __fdiv_rn(15.0f, p7) : 15.0f * rcp_ftz(p7);
        const float l00 = lx * lx, l01 = lx * ly, l02 = lx * lz, l11 = ly * ly, l12 = ly * lz, l22 = lz * lz;
        float cub = 0.f;
        const float lv[3] = {lx, ly, lz};
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const float* sv = h + 13 + 6 * v;
            const float t = fmaf(l00, sv[0], fmaf(l01, sv[1], fmaf(l02, sv[2], fmaf(l11, sv[3], fmaf(l12, sv[4], l22 * sv[5])))));
            cub = fmaf(lv[v], t, cub);
        }
        const float lg = fmaf(lx, h[10], fmaf(ly, h[11], lz * h[12]));
        w = fmaf(i15, cub, fmaf(c5, lg, w));
    }
    return w;
}

// Queries per lane: grids take NQ_GRID samples per lane (the brick of SHAPE
// stacked NQ_GRID times in z), point queries one (consecutive points spread
// over more of the tree than grid bricks, which costs more than it shares).
#ifndef DWG_NQ_GRID
#define DWG_NQ_GRID 2
#endif
constexpr int kNqGrid = DWG_NQ_GRID;

// The sums of group g: 32 x NQ queries, NQ per lane.  The warp walks the
// octree once for all of them: each stack entry carries, per query slot, the
// mask of the lanes whose query opened the node, so every query takes exactly
// the reference's per-query decisions -- a child is a dipole term when
// |CM - q| > beta R, otherwise it is opened, and leaves are summed point by
// point -- while the traversal (stack pops, record loads, the loop over
// children) is shared.  Terms are evaluated branch-free and masked, so that a
// lane's queries never split the warp; each query's terms keep their
// depth-first order (its value does not depend on NQ or the brick shape).
// Returns the lane's term count.
// the grid samples of group g for this lane: the brick of SHAPE stacked NQ
// times in z
template <int SHAPE, int NQ>
__device__ __forceinline__ void grid_queries(const GwnArgs& a, unsigned long long g, int lane, bool* valid,
                                             long long* qi, float* qx, float* qy, float* qz) {
    using B = Brick<SHAPE>;
    const long long bxi = (long long)(g % (unsigned long long)a.bx);
    const unsigned long long t = g / (unsigned long long)a.bx;
    const long long byi = (long long)(t % (unsigned long long)a.by);
    const long long bzi = (long long)(t / (unsigned long long)a.by);
    const long long x = bxi * B::X + (lane % B::X), y = byi * B::Y + ((lane / B::X) % B::Y);
    const long long z0 = bzi * (NQ * B::Z) + lane / (B::X * B::Y);
    const bool xy_ok = x < a.rx && y < a.ry;
    const float fx = __fadd_rn(a.ox, __fmul_rn((float)x, a.h));
    const float fy = __fadd_rn(a.oy, __fmul_rn((float)y, a.h));
#pragma unroll
    for (int u = 0; u < NQ; ++u) {
        const long long z = z0 + u * B::Z;
        valid[u] = xy_ok && z < a.rz;
        qi[u] = x + (long long)a.rx * (y + (long long)a.ry * z);
        qx[u] = fx;
        qy[u] = fy;
        qz[u] = __fadd_rn(a.oz, __fmul_rn((float)(z + a.zoff), a.h));
    }
}

// the samples of group g: a grid brick, or 32 * NQ consecutive points
template <bool GRID, int SHAPE, int NQ>
__device__ __forceinline__ void group_queries(const GwnArgs& a, unsigned long long g, int lane, bool* valid,
                                              long long* qi, float* qx, float* qy, float* qz) {
    if (GRID) {
        grid_queries<SHAPE, NQ>(a, g, lane, valid, qi, qx, qy, qz);
    } else {
#pragma unroll
        for (int u = 0; u < NQ; ++u) {
            qi[u] = (long long)g * (32 * NQ) + u * 32 + lane;
            valid[u] = qi[u] < a.nq;
            qx[u] = qy[u] = qz[u] = 0.f;
            if (valid[u]) {
                qx[u] = a.q[qi[u] * 3];
                qy[u] = a.q[qi[u] * 3 + 1];
                qz[u] = a.q[qi[u] * 3 + 2];
            }
        }
    }
}

// kept screening weights of one lane and list entry: one per sample slot
template <int NQ>
struct WeightOf {
    using T = float2;
    __device__ static T pack(const float* g) { return make_float2(g[0], g[1]); }
    __device__ static void unpack(const T& w, float* g) {
        g[0] = w.x;
        g[1] = w.y;
    }
};
template <>
struct WeightOf<1> {
    using T = float;
    __device__ static T pack(const float* g) { return g[0]; }
    __device__ static void unpack(const T& w, float* g) { g[0] = w; }
};

// the points of a leaf, one term each, for one query
template <bool SCREENED, int PREC, typename Acc>
__device__ __forceinline__ void leaf_terms(const GwnArgs& a, int start, int cnt, float qx, float qy, float qz,
                                           float sigma, float sigma_l2e, Acc& sum, int& nt) {
    for (int j = start; j < start + cnt; ++j) {
        const float4 p = a.pa[j];
        const float4 nn = a.nr[j];
        const float dx = p.x - qx, dy = p.y - qy, dz = p.z - qz;
        const float d = p.w * fmaf(dx, nn.x, fmaf(dy, nn.y, dz * nn.z));
        const float sc = a.use_radii ? nn.w : a.screen;
        float v;
        if (gwn_term<SCREENED, PREC>(dx, dy, dz, d, sc, sigma, sigma_l2e, v)) {
            sum += (Acc)v;
            ++nt;
        }
    }
}

// (A n) . (p - q) of a node for one sample
__device__ __forceinline__ float node_dot(const float4& nb, float dx, float dy, float dz) {
    return fmaf(dz, nb.z, fmaf(dy, nb.y, dx * nb.x));
}

// one far-node term, masked to the lanes that take it (shared by the
// traversal and the replay of its interaction list, so both give the same bits)
// (returns the screening weight g of the term for PREC != 2, 0 otherwise)
template <bool SCREENED, int PREC, typename Acc>
__device__ __forceinline__ float node_term(const GwnArgs& a, const float4& na, const float4& nb, float dx, float dy,
                                           float dz, float d2, bool take, float sigma, float sigma_l2e, Acc& sum,
                                           int& nt) {
    // x and y parts first: the samples of a lane share x and y
    const float dd = node_dot(nb, dx, dy, dz);
    bool k;
    float v, g = 0.f;
    if (SCREENED && PREC != 2) {
        g = screen_weight_masked(take, d2, a.screen, sigma, sigma_l2e, k);
        v = __fmul_rn(g, dd);  // never contracted into the sum: a kept g gives the same bits
    } else {
        v = gwn_term_masked<SCREENED, PREC>(take, d2, dd, a.screen, sigma, sigma_l2e, k);
    }
    sum += (Acc)v;  // v is 0 where no term is taken
    nt += (int)k;
    return g;
}

// MODE 0 sums; MODE 1 counts the group's interaction-list entries (visits
// where some lane takes a term, and multi-point leaves); MODE 2 writes them:
// (record, term masks per query slot) in visit order.  Modes 1 and 2 do the
// traversal only.
template <bool GRID, bool SCREENED, int PREC, int SHAPE, int NQ, int ORDER, int MODE = 0>
__device__ __forceinline__ int gwn_group(const GwnArgs& a, unsigned long long g, int lane,
                                         int* __restrict__ stk_node, unsigned* __restrict__ stk_mask,
                                         unsigned* __restrict__ stk_meta, float4* __restrict__ crec, float sigma,
                                         float sigma_l2e) {
    const unsigned FULL = 0xffffffffu;
    bool valid[NQ];
    long long qi[NQ];
    float qx[NQ], qy[NQ], qz[NQ];
    group_queries<GRID, SHAPE, NQ>(a, g, lane, valid, qi, qx, qy, qz);
    using Acc = typename AccType<PREC>::T;
    Acc sum[NQ];
    int nt[NQ];
#pragma unroll
    for (int u = 0; u < NQ; ++u) {
        sum[u] = 0;
        nt[u] = 0;
    }

    static_assert(MODE == 0 || (NQ <= 3 && ORDER == 0), "interaction lists: order 0, at most 3 slots");
    unsigned rec = 0;  // list entries of this group (warp-uniform)
    int4* const out_list = (MODE == 2) ? a.list + a.list_off[g] : nullptr;
    auto leaf_points = [&](int start, int cnt, int u) {
        leaf_terms<SCREENED, PREC>(a, start, cnt, qx[u], qy[u], qz[u], sigma, sigma_l2e, sum[u], nt[u]);
    };
    auto record = [&](int word, const unsigned* m) {
        if (MODE == 2 && lane == 0)
            out_list[rec] = make_int4(word, (int)m[0], NQ > 1 ? (int)m[1] : 0, NQ > 2 ? (int)m[2] : 0);
        ++rec;
    };

    // one child record (level order).  A single-point leaf is always a term;
    // an internal node is a dipole term when far for the query (sqrt_rn(d2)
    // > beta R in round-to-nearest single precision, src/TurboLibiGWN.cu:
    // 636-644, as one comparison of d2 with the node's exact threshold) and is
    // opened (pushed with the queries that need it) otherwise; both use the
    // same d2.  Larger leaves (every leaf when radii apply) are summed point
    // by point.
    auto child = [&](int cidx, const float4& na, const float4& nb, const bool* act, int& sp) {
        const unsigned meta = (unsigned)__float_as_int(nb.w);
        const bool leaf = (meta & kMetaLeafBit) != 0;
        if (leaf && (!(meta & kMetaSingle) || a.use_radii)) {
            const int st = (int)(meta & kMetaIndex), cnt = __float_as_int(na.w);
            if (cnt < 0 || st + cnt > a.num_points) {
                if (lane == 0) atomicOr(&a.work[1], 4u);
            } else if (MODE == 0) {
#pragma unroll
                for (int u = 0; u < NQ; ++u)
                    if (act[u]) leaf_points(st, cnt, u);
            } else {
                unsigned m[NQ];
#pragma unroll
                for (int u = 0; u < NQ; ++u) m[u] = __ballot_sync(FULL, act[u]);
                record(cidx | (int)0x80000000, m);
            }
            return;
        }
        float dx[NQ], dy[NQ], dz[NQ], d2[NQ];
        bool far[NQ], take[NQ];
        bool any = false;
#pragma unroll
        for (int u = 0; u < NQ; ++u) {
            dx[u] = __fsub_rn(na.x, qx[u]);
            dy[u] = __fsub_rn(na.y, qy[u]);
            dz[u] = __fsub_rn(na.z, qz[u]);
            d2[u] = sq3_rn(dx[u], dy[u], dz[u]);
            far[u] = leaf || d2[u] > na.w;
            take[u] = act[u] && far[u];
            any = any || take[u];
        }
        if (MODE != 0) {
            unsigned m[NQ];
            unsigned anym = 0;
#pragma unroll
            for (int u = 0; u < NQ; ++u) {
                m[u] = __ballot_sync(FULL, take[u]);
                anym |= m[u];
            }
            if (anym) record(cidx, m);
        } else if (__any_sync(FULL, any)) {
#pragma unroll
            for (int u = 0; u < NQ; ++u) {
                if (ORDER == 0) {
                    node_term<SCREENED, PREC>(a, na, nb, dx[u], dy[u], dz[u], d2[u], take[u], sigma, sigma_l2e, sum[u],
                                              nt[u]);
                } else {
                    // x and y parts first: the samples of a lane share x and y
                    const float dd = fmaf(dz[u], nb.z, fmaf(dy[u], nb.y, dx[u] * nb.x));
                    bool k;
                    float v = gwn_term_masked<SCREENED, PREC>(take[u], d2[u], dd, a.screen, sigma, sigma_l2e, k);
                    if (!SCREENED && !leaf) {
                        // far internal node: add the expansion terms (leaves are exact)
                        const float c = fwn_correction<ORDER, PREC>(dx[u], dy[u], dz[u], take[u] ? d2[u] : 1.0f,
                                                                    a.node_h + (size_t)cidx * 8);
                        v += take[u] ? c : 0.f;
                    }
                    sum[u] += (Acc)v;  // v is 0 where no term is taken
                    nt[u] += (int)k;
                }
            }
        }
        unsigned nm[NQ];
        unsigned anym = 0;
#pragma unroll
        for (int u = 0; u < NQ; ++u) {
            nm[u] = __ballot_sync(FULL, act[u] && !far[u]);
            anym |= nm[u];
        }
        if (anym) {
            if (sp < kGwnStack) {
                if (lane == 0) {
                    stk_node[sp] = cidx;
                    stk_meta[sp] = meta;  // its children's place: no load when it is popped
#pragma unroll
                    for (int u = 0; u < NQ; ++u) stk_mask[sp * NQ + u] = nm[u];
                }
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
            unsigned m[NQ];
#pragma unroll
            for (int u = 0; u < NQ; ++u) m[u] = __ballot_sync(FULL, valid[u]);
            if (lane == 0) {
                stk_node[0] = 0;
                stk_meta[0] = rm;
#pragma unroll
                for (int u = 0; u < NQ; ++u) stk_mask[u] = m[u];
            }
            sp = 1;
        }
    }
    while (sp > 0) {
        __syncwarp();
        --sp;
        const int node = stk_node[sp];
        const unsigned pm = stk_meta[sp];
        bool act[NQ];
#pragma unroll
        for (int u = 0; u < NQ; ++u) act[u] = (stk_mask[sp * NQ + u] >> lane) & 1u;
        __syncwarp();
        if (node < 0 || node >= a.num_nodes) {
            if (lane == 0) atomicOr(&a.work[1], 2u);
            continue;
        }
        const int first = (int)(pm & kMetaIndex);
        const int nch = (int)((pm >> 28) & 7u) + 1;
        // structural guard: children come after the parent, inside the table
        if ((pm & kMetaLeafBit) || first <= node || first + nch > a.num_nodes) {
            if (lane == 0) atomicOr(&a.work[1], 2u);
            continue;
        }
        // the (at most 8, contiguous) children's records at once, a lane
        // each, into shared memory; the loop top's __syncwarp ordered the
        // previous node's reads of them before these writes
        if (lane < nch) {
            crec[lane] = a.node_a[first + lane];
            crec[8 + lane] = a.node_b[first + lane];
        }
        __syncwarp();
        for (int j = 0; j < nch; ++j) {
            const float4 na = crec[j], nb = crec[8 + j];
            child(first + j, na, nb, act, sp);
        }
    }
    if (MODE == 1) {
        if (lane == 0) a.list_count[g] = rec;
        return 0;
    }
    if (MODE == 2) return 0;
    int total = 0;
#pragma unroll
    for (int u = 0; u < NQ; ++u) {
        if (valid[u]) {
            a.out[qi[u]] = (float)sum[u];
            if (a.per_query_terms) a.per_query_terms[qi[u]] = nt[u];
        }
        total += nt[u];
    }
    return total;
}

template <bool GRID>
__host__ __device__ constexpr int nq_of() {
    return GRID ? kNqGrid : 1;
}

template <bool GRID, bool SCREENED, int PREC, int SHAPE, int ORDER, int MODE = 0>
__global__ void __launch_bounds__(kGwnWarps * 32, (GRID && kNqGrid >= 4) ? 2 : 3) k_gwn(GwnArgs a) {
    constexpr int NQ = nq_of<GRID>();
    __shared__ int stk_node[kGwnWarps][kGwnStack];
    __shared__ unsigned stk_mask[kGwnWarps][kGwnStack * NQ];
    __shared__ unsigned stk_meta[kGwnWarps][kGwnStack];
    __shared__ float4 crec[kGwnWarps][16];
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
        my_terms += (unsigned long long)gwn_group<GRID, SCREENED, PREC, SHAPE, NQ, ORDER, MODE>(
            a, g, lane, stk_node[w], stk_mask[w], stk_meta[w], crec[w], sigma, sigma_l2e);
    }
    if (a.terms_total) {
        for (int o = 16; o > 0; o >>= 1) my_terms += __shfl_down_sync(FULL, my_terms, o);
        if (lane == 0 && my_terms) atomicAdd(a.terms_total, my_terms);
    }
}

// Replay of the recorded interaction lists of a grid: every group walks its
// entries in visit order and evaluates exactly the terms (and multi-point
// leaves) the traversal evaluated, with the same arithmetic, so the sums are
// bit-identical; the traversal itself (stack, opening tests, votes) is gone.
// With weight slots (a.wsel), mode 1 also writes the screening weight of
// every node entry and sample; in mode 2 the launch returns at once and
// k_gwn_wread reads them back.
template <bool GRID, bool SCREENED, int PREC, int SHAPE>
__global__ void __launch_bounds__(kGwnWarps * 32, 3) k_gwn_replay(GwnArgs a) {
    constexpr int NQ = nq_of<GRID>();
    using WT = WeightOf<NQ>;
    using W = typename WT::T;
    using Acc = typename AccType<PREC>::T;
    __shared__ float4 rrec[kGwnWarps][64];  // per warp: the batch's node records (a, then b)
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    float4* const ra = rrec[threadIdx.x >> 5];
    float4* const rb = ra + 32;
    const float sigma = a.sigma_dev ? *a.sigma_dev : a.sigma;
    const float sigma_l2e = sigma * 1.4426950408889634f;
    int wmode = 0;
    W* wp = nullptr;
    if (SCREENED && PREC != 2 && a.wsel) {
        wmode = a.wsel->mode;
        if (wmode == 2) return;  // k_gwn_wread reads the kept weights
        wp = reinterpret_cast<W*>(a.wbuf) + (size_t)a.wsel->slot * a.wstride;
    }
    unsigned long long my_terms = 0, my_node_terms = 0;
    for (;;) {
        unsigned g = 0;
        if (lane == 0) g = atomicAdd(&a.work[0], 1u);
        g = __shfl_sync(FULL, g, 0);
        if ((long long)g >= a.ngroups) break;
        bool valid[NQ];
        long long qi[NQ];
        float qx[NQ], qy[NQ], qz[NQ];
        group_queries<GRID, SHAPE, NQ>(a, g, lane, valid, qi, qx, qy, qz);
        Acc sum[NQ];
        int nt[NQ], ntn = 0;
#pragma unroll
        for (int u = 0; u < NQ; ++u) {
            sum[u] = 0;
            nt[u] = 0;
        }
        const unsigned long long e0 = a.list_off[g], e1 = a.list_off[g + 1];
        // the group's entries arrive 32 at a time in one coalesced load and
        // are handed out by shuffles; their node records are loaded at the
        // same time, a lane each, into shared memory (no dependent global
        // load per entry)
        for (unsigned long long base = e0; base < e1; base += 32) {
            const int4 mine = base + lane < e1 ? a.list[base + lane] : make_int4(0, 0, 0, 0);
            const int cnt = e1 - base < 32 ? (int)(e1 - base) : 32;
            if (base + lane < e1 && mine.x >= 0) {
                ra[lane] = a.node_a[mine.x];
                rb[lane] = a.node_b[mine.x];
            }
            __syncwarp();
            for (int j = 0; j < cnt; ++j) {
                const int ex = __shfl_sync(FULL, mine.x, j);
                const unsigned m[3] = {(unsigned)__shfl_sync(FULL, mine.y, j), (unsigned)__shfl_sync(FULL, mine.z, j),
                                       (unsigned)__shfl_sync(FULL, mine.w, j)};
                if (ex < 0) {  // a multi-point leaf: its points for the lanes that reached it
                    const int cidx = ex & 0x7fffffff;
                    const unsigned meta = (unsigned)__float_as_int(a.node_b[cidx].w);
                    const int st = (int)(meta & kMetaIndex), pc = __float_as_int(a.node_a[cidx].w);
#pragma unroll
                    for (int u = 0; u < NQ; ++u)
                        if ((m[u] >> lane) & 1u)
                            leaf_terms<SCREENED, PREC>(a, st, pc, qx[u], qy[u], qz[u], sigma, sigma_l2e, sum[u],
                                                       nt[u]);
                } else {
                    const float4 na = ra[j], nb = rb[j];
                    float gw[NQ];
#pragma unroll
                    for (int u = 0; u < NQ; ++u) {
                        const float dx = __fsub_rn(na.x, qx[u]);
                        const float dy = __fsub_rn(na.y, qy[u]);
                        const float dz = __fsub_rn(na.z, qz[u]);
                        const int before = nt[u];
                        gw[u] = node_term<SCREENED, PREC>(a, na, nb, dx, dy, dz, sq3_rn(dx, dy, dz),
                                                          ((m[u] >> lane) & 1u) != 0, sigma, sigma_l2e, sum[u],
                                                          nt[u]);
                        ntn += nt[u] - before;
                    }
                    if (wmode == 1) __stcs(wp + (base + j) * 32 + lane, WT::pack(gw));
                }
            }
            __syncwarp();  // the records are read before the next batch's overwrite them
        }
#pragma unroll
        for (int u = 0; u < NQ; ++u) {
            if (valid[u]) a.out[qi[u]] = (float)sum[u];
            my_terms += (unsigned long long)nt[u];
        }
        my_node_terms += (unsigned long long)ntn;
    }
    if (a.terms_total) {
        for (int o = 16; o > 0; o >>= 1) my_terms += __shfl_down_sync(FULL, my_terms, o);
        if (lane == 0 && my_terms) atomicAdd(a.terms_total, my_terms);
    }
    if (wmode == 1) {
        for (int o = 16; o > 0; o >>= 1) my_node_terms += __shfl_down_sync(FULL, my_node_terms, o);
        if (lane == 0 && my_node_terms) atomicAdd(&a.wsel->node_terms[a.wsel->slot], my_node_terms);
    }
}

// Replay that reads the kept screening weights of this sigma (mode 2; other
// modes return at once): per node entry one dot product and one product per
// sample, g (A n).(p - q), with the replay's roundings, so the sums keep
// their bits.  The kernel is bound by the weights' HBM stream (256 bytes per
// entry for grid cells, 128 for points), so each warp streams its group's
// entries and weights through a ring of kWreadRing chunks of kWreadChunk
// entries in shared memory, two chunks in flight while it sums the third:
// one lane hands each chunk to the bulk-copy (TMA) engine as two 1-D copies
// (the chunk's weights and its entries are contiguous in global memory) that
// complete on the ring slot's mbarrier.  Grid cells (two samples per lane,
// 8-byte weights): two 256-thread blocks per SM, 106 KB of ring and node
// records each; points (one sample, 4-byte weights): three blocks of 58 KB,
// so that more warps cover the node records' round trips.  The node terms a
// slot stands for were counted when it was written.
constexpr int kWreadChunk = 16;
template <bool GRID>
__host__ __device__ constexpr int wread_blocks() {
    return GRID ? 2 : 3;
}

// the points of a multi-point leaf for one sample, out of line (rare in the
// read path; its registers stay off the loop).  The running sum goes in and
// comes back, so the points add to it in order, as in leaf_terms.
template <typename Acc>
struct LeafSum {
    Acc sum;
    int nt;
};
template <bool SCREENED, int PREC, typename Acc>
__device__ __noinline__ LeafSum<Acc> leaf_points_ool(const float4* __restrict__ pa, const float4* __restrict__ nr,
                                                     int use_radii, float screen, int start, int cnt, float qx,
                                                     float qy, float qz, float sigma, float sigma_l2e, Acc sum) {
    LeafSum<Acc> r{sum, 0};
    for (int j = start; j < start + cnt; ++j) {
        const float4 p = pa[j];
        const float4 nn = nr[j];
        const float dx = p.x - qx, dy = p.y - qy, dz = p.z - qz;
        const float d = p.w * fmaf(dx, nn.x, fmaf(dy, nn.y, dz * nn.z));
        const float sc = use_radii ? nn.w : screen;
        float v;
        if (gwn_term<SCREENED, PREC>(dx, dy, dz, d, sc, sigma, sigma_l2e, v)) {
            r.sum += (Acc)v;
            ++r.nt;
        }
    }
    return r;
}
constexpr int kWreadRing = 3;
// per warp: the ring's weights (3 slots x C entries x 32 lanes x WSIZE
// bytes), its entries (16 bytes each), then the node records of the chunk
// being summed (two float4 per entry); every part a multiple of 16 bytes
template <int WSIZE>
__host__ __device__ constexpr int wread_warp_bytes() {
    return kWreadRing * kWreadChunk * (32 * WSIZE + 16) + 2 * kWreadChunk * 16;
}
template <bool GRID>
__host__ __device__ constexpr int wread_smem() {
    return kGwnWarps * wread_warp_bytes<(int)sizeof(typename WeightOf<nq_of<GRID>()>::T)>();
}

// 1-D bulk copies global -> shared (the TMA engine), completed on an
// mbarrier: the barrier's phase completes when its one arrival (with the
// expected byte count) and all the copies' bytes have landed.
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// bounded: gives up (false) after about a second of suspended waits
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    for (int it = 0; it < (1 << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// chunk c of entries [e0, e1) into a ring slot: its weights (32 per entry)
// and its entries, two bulk copies issued by lane 0 onto the slot's barrier.
// Returns whether the chunk exists (was issued).  Sizes are multiples of 16
// bytes and both sources 16-byte aligned (256-byte aligned buffers, whole
// entries of 16 bytes and of 32 weights).  The warp's reads of the slot's
// previous chunk are complete (the caller's __syncwarp); the proxy fence
// orders them before the copy's writes.
template <typename W>
__device__ __forceinline__ bool wread_issue(const W* __restrict__ wp, const int4* __restrict__ list,
                                            unsigned long long e0, unsigned long long e1, unsigned long long c,
                                            W* ws, int4* ls, unsigned long long* bar, int lane) {
    const unsigned long long first = e0 + c * kWreadChunk;
    if (first >= e1) return false;
    if (lane == 0) {
        const unsigned cnt =
            (unsigned)(e1 - first < (unsigned long long)kWreadChunk ? e1 - first : kWreadChunk);
        const unsigned wb = cnt * 32u * (unsigned)sizeof(W), lb = cnt * 16u;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(bar, wb + lb);
        bulk_copy_g2s(ws, wp + first * 32, wb, bar);
        bulk_copy_g2s(ls, list + first, lb, bar);
    }
    return true;
}

template <bool GRID, bool SCREENED, int PREC, int SHAPE>
__global__ void __launch_bounds__(kGwnWarps * 32, wread_blocks<GRID>()) k_gwn_wread(GwnArgs a) {
    constexpr int NQ = nq_of<GRID>();
    constexpr int C = kWreadChunk;
    using WT = WeightOf<NQ>;
    using W = typename WT::T;
    constexpr int WS = (int)sizeof(W);
    constexpr int WB = wread_warp_bytes<WS>();
    static_assert(WS % 4 == 0 && (32 * WS) % 16 == 0, "weight rows of whole 16-byte units");
    using Acc = typename AccType<PREC>::T;
    extern __shared__ __align__(16) unsigned char wread_smem[];
    __shared__ __align__(8) unsigned long long wbar[kGwnWarps][kWreadRing];
    const unsigned FULL = 0xffffffffu;
    GwnWeightState* const wst = a.wsel;
    if (wst->mode != 2) return;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    W* const wring = reinterpret_cast<W*>(wread_smem + warp * WB);
    int4* const lring = reinterpret_cast<int4*>(wread_smem + warp * WB + kWreadRing * C * 32 * WS);
    float4* const rec = reinterpret_cast<float4*>(wread_smem + warp * WB + kWreadRing * C * (32 * WS + 16));
    unsigned long long* const bar = wbar[warp];
    if (lane == 0) {
        for (int r = 0; r < kWreadRing; ++r) mbar_init(bar + r);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    unsigned parity = 0;  // bit r: the phase of ring slot r to wait for next
    unsigned pend = 0;    // bit r: slot r has a chunk in flight
    bool wait_ok = true;  // warp-uniform
    const W* const wp = reinterpret_cast<const W*>(a.wbuf) + (size_t)wst->slot * a.wstride;
    if (a.terms_total && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(a.terms_total, wst->node_terms[wst->slot]);
    const float sigma = a.sigma_dev ? *a.sigma_dev : a.sigma;
    const float sigma_l2e = sigma * 1.4426950408889634f;
    unsigned long long my_terms = 0;
    for (;;) {
        unsigned g = 0;
        if (lane == 0) g = atomicAdd(&wst->work, 1u);
        g = __shfl_sync(FULL, g, 0);
        if ((long long)g >= a.ngroups) break;
        bool valid[NQ];
        long long qi[NQ];
        float qx[NQ], qy[NQ], qz[NQ];
        group_queries<GRID, SHAPE, NQ>(a, g, lane, valid, qi, qx, qy, qz);
        Acc sum[NQ];
        int nt[NQ];
#pragma unroll
        for (int u = 0; u < NQ; ++u) {
            sum[u] = 0;
            nt[u] = 0;
        }
        const unsigned long long e0 = a.list_off[g], e1 = a.list_off[g + 1];
        const unsigned long long nchunk = (e1 - e0 + C - 1) / C;
        __syncwarp();  // the ring's last readers (previous group) are done
        // a group's chunk c sits in ring slot c % kWreadRing (every issued
        // chunk is waited for before its group ends, so no copy spans groups)
#pragma unroll
        for (int c = 0; c < kWreadRing - 1; ++c)
            if (wread_issue(wp, a.list, e0, e1, c, wring + c * C * 32, lring + c * C, bar + c, lane))
                pend |= 1u << c;
        for (unsigned long long c = 0; c < nchunk; ++c) {
            const int r = (int)(c % kWreadRing);
            // chunk c has landed (c + 1 may be in flight): every lane waits
            // (each needs the copy's bytes visible); after a wait that gave
            // up, the slot's contents are unknown: the warp reads none of
            // them (its entries index node records)
            wait_ok = __all_sync(FULL, mbar_wait(bar + r, (parity >> r) & 1u));
            if (!wait_ok) break;
            parity ^= 1u << r;
            pend &= ~(1u << r);
            const W* wc = wring + r * C * 32;
            const int4* lc = lring + r * C;
            const unsigned long long first = e0 + c * C;
            const int cnt = e1 - first < (unsigned long long)C ? (int)(e1 - first) : C;
            // the chunk's node records (for a multi-point leaf, its node's)
            // are loaded at once, a lane each, into shared memory: one round
            // trip per chunk rather than one per entry.  A full chunk of node
            // entries (the common case) is then summed unrolled.
            if (lane < cnt) {
                const int x = lc[lane].x & 0x7fffffff;
                rec[lane] = a.node_a[x];
                rec[C + lane] = a.node_b[x];
            }
            const bool full = cnt == C && __ballot_sync(FULL, lc[lane & (C - 1)].x < 0) == 0;
            __syncwarp();  // the warp's previous readers passed the chunk-end __syncwarp
            if (full) {
#pragma unroll
                for (int k = 0; k < C; ++k) {
                    const float4 na = rec[k], nb = rec[C + k];
                    float wu[NQ];
                    WT::unpack(wc[k * 32 + lane], wu);
#pragma unroll
                    for (int u = 0; u < NQ; ++u) {
                        const float dd = node_dot(nb, __fsub_rn(na.x, qx[u]), __fsub_rn(na.y, qy[u]),
                                                  __fsub_rn(na.z, qz[u]));
                        sum[u] += (Acc)__fmul_rn(wu[u], dd);
                    }
                }
            }
            for (int k = full ? C : 0; k < cnt; ++k) {
                const int4 e = lc[k];
                const float4 na = rec[k], nb = rec[C + k];
                if (e.x < 0) {  // a multi-point leaf: its points for the lanes that reached it
                    const unsigned meta = (unsigned)__float_as_int(nb.w);
                    const int st = (int)(meta & kMetaIndex), pc = __float_as_int(na.w);
#pragma unroll
                    for (int u = 0; u < NQ; ++u) {
                        if (((unsigned)(u == 0 ? e.y : (u == 1 ? e.z : e.w)) >> lane) & 1u) {
                            const LeafSum<Acc> r = leaf_points_ool<SCREENED, PREC, Acc>(
                                a.pa, a.nr, a.use_radii, a.screen, st, pc, qx[u], qy[u], qz[u], sigma, sigma_l2e,
                                sum[u]);
                            sum[u] = r.sum;
                            nt[u] += r.nt;
                        }
                    }
                } else {
                    float wu[NQ];
                    WT::unpack(wc[k * 32 + lane], wu);
#pragma unroll
                    for (int u = 0; u < NQ; ++u) {
                        const float dd = node_dot(nb, __fsub_rn(na.x, qx[u]), __fsub_rn(na.y, qy[u]),
                                                  __fsub_rn(na.z, qz[u]));
                        sum[u] += (Acc)__fmul_rn(wu[u], dd);
                    }
                }
            }
            __syncwarp();  // ring slot (c + 2) % 3 = (c - 1) % 3 was read in the previous pass
            const unsigned long long nx = c + kWreadRing - 1;
            const int rn = (int)(nx % kWreadRing);
            if (wread_issue(wp, a.list, e0, e1, nx, wring + rn * C * 32, lring + rn * C, bar + rn, lane))
                pend |= 1u << rn;
        }
#pragma unroll
        for (int u = 0; u < NQ; ++u) {
            if (valid[u]) a.out[qi[u]] = (float)sum[u];
            my_terms += (unsigned long long)nt[u];
        }
        if (!wait_ok) break;
    }
    // every issued chunk was waited for, so no copy outlives the block,
    // unless a wait gave up (a copy that never landed): that is reported,
    // and the chunks still in flight get one more bounded wait each
    if (!wait_ok) {
        if (lane == 0) atomicOr(&a.work[1], 16u);
        for (int r = 0; r < kWreadRing; ++r)
            if ((pend >> r) & 1u) (void)mbar_wait(bar + r, (parity >> r) & 1u);
    }
    if (a.terms_total) {
        for (int o = 16; o > 0; o >>= 1) my_terms += __shfl_down_sync(FULL, my_terms, o);
        if (lane == 0 && my_terms) atomicAdd(a.terms_total, my_terms);
    }
}

// Chooses the weight slot of the next replay launch on the device: a launch
// that wrote a slot has completed when this runs (same stream), so its slot
// becomes valid; then a valid slot with this (sigma, screen) is read, else
// the first free slot is written, else the terms are evaluated as usual.
__global__ void k_weight_select(GwnWeightState* __restrict__ w, const float* __restrict__ sigma_dev, float sigma,
                                float screen) {
    if (w->mode == 1) w->valid[w->slot] = 1;
    const float sg = sigma_dev ? *sigma_dev : sigma;
    w->mode = 0;
    w->slot = 0;
    w->work = 0;
    for (int c = 0; c < w->nslots; ++c)
        if (w->valid[c] && w->sigma[c] == sg && w->screen[c] == screen) {
            w->mode = 2;
            w->slot = c;
            return;
        }
    for (int c = 0; c < w->nslots; ++c)
        if (!w->valid[c] && (w->pref[c] == 0.f || w->pref[c] == sg)) {
            w->mode = 1;
            w->slot = c;
            w->sigma[c] = sg;
            w->screen[c] = screen;
            w->node_terms[c] = 0;
            return;
        }
}

struct SlotPrefs {
    float s[kGwnWeightSlots];
};
// the sigmas that L's slots are kept for: L.pref when it holds fewer slots
// than it wants, else none (every sigma of the schedule has a slot)
static SlotPrefs slot_prefs(const GwnList& L, int nslots) {
    SlotPrefs p{};
    if (nslots < L.wslots)
        for (int c = 0; c < nslots && c < kGwnWeightSlots; ++c) p.s[c] = L.pref[c];
    return p;
}

__global__ void k_weight_reset(GwnWeightState* __restrict__ w, int nslots, SlotPrefs pref) {
    w->mode = 0;
    w->slot = 0;
    w->nslots = nslots;
    w->work = 0;
    for (int c = 0; c < kGwnWeightSlots; ++c) {
        w->valid[c] = 0;
        w->sigma[c] = 0.f;
        w->screen[c] = 0.f;
        w->pref[c] = pref.s[c];
        w->node_terms[c] = 0;
    }
}

int gwn_list_drop_weights(GwnList& L, cudaStream_t s) {
    if (!L.valid || L.nslots <= 0) return DWG_OK;
    k_weight_reset<<<1, 1, 0, s>>>(L.wstate.ptr, L.nslots, slot_prefs(L, L.nslots));
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

void gwn_list_release(GwnList& L) {
    L.count.release();
    L.off.release();
    L.ent.release();
    L.scratch.release();
    L.w.release();
    L.wstate.release();
    L.nslots = 0;
    L.entries = 0;
    L.ngroups = 0;
    L.valid = false;
    L.too_big = false;
}

int gwn_list_add_weights(GwnList& L, int nslots, cudaStream_t s) {
    // the weight state exists when the recording could keep weights (screened
    // terms with the MUFU approximations)
    DWG_REQUIRE(L.valid && !L.too_big && L.wstate.ptr && L.nslots == 0 && L.entries > 0,
                "gwn lists: no recorded list without weights to add them to");
    DWG_REQUIRE(nslots >= 1 && nslots <= L.wslots && nslots <= kGwnWeightSlots, "gwn lists: bad slot count %d",
                nslots);
    const size_t wb = L.grid ? sizeof(WeightOf<nq_of<true>()>::T) : sizeof(WeightOf<nq_of<false>()>::T);
    const size_t per = (size_t)L.entries * 32 * wb;
    DWG_TRY(L.w.reserve(((size_t)nslots * per + sizeof(float2) - 1) / sizeof(float2)));
    L.nslots = nslots;
    k_weight_reset<<<1, 1, 0, s>>>(L.wstate.ptr, nslots, slot_prefs(L, nslots));
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

// Grid sums of many clouds in one persistent launch: the groups of all
// clouds form one work list (prefix[c] = first group of cloud c), taken in
// order by the warps of the grid, so that small clouds do not idle the GPU.
template <bool SCREENED, int PREC, int SHAPE>
__global__ void __launch_bounds__(kGwnWarps * 32, kNqGrid >= 4 ? 2 : 3)
    k_gwn_batch(const GwnArgs* __restrict__ table, const unsigned long long* __restrict__ prefix, int nclouds,
                unsigned long long* __restrict__ work) {
    __shared__ int stk_node[kGwnWarps][kGwnStack];
    __shared__ unsigned stk_mask[kGwnWarps][kGwnStack * kNqGrid];
    __shared__ unsigned stk_meta[kGwnWarps][kGwnStack];
    __shared__ float4 crec[kGwnWarps][16];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const unsigned long long total = prefix[nclouds];
    for (;;) {
        unsigned long long g = 0;
        if (lane == 0) g = atomicAdd(work, 1ull);
        g = __shfl_sync(FULL, g, 0);
        if (g >= total) break;
        int lo = 0, hi = nclouds - 1;  // last cloud with prefix <= g
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= g) lo = mid;
            else hi = mid - 1;
        }
        const GwnArgs& a = table[lo];
        const float sigma = a.sigma_dev ? *a.sigma_dev : a.sigma;
        int nt = gwn_group<true, SCREENED, PREC, SHAPE, kNqGrid, 0>(a, g - prefix[lo], lane, stk_node[w], stk_mask[w],
                                                                stk_meta[w], crec[w], sigma,
                                                                sigma * 1.4426950408889634f);
        if (a.terms_total) {
            for (int o = 16; o > 0; o >>= 1) nt += __shfl_down_sync(FULL, nt, o);
            if (lane == 0 && nt) atomicAdd(a.terms_total, (unsigned long long)nt);
        }
    }
}

template <typename K>
static int blocks_for(K kernel) {
    int bps = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, kGwnWarps * 32, 0);
    return bps > 0 ? bps : 1;
}

template <bool GRID, bool SCREENED, int PREC, int SHAPE, int ORDER>
static int launch(const GwnArgs& a, cudaStream_t s) {
    static int blocks_per_sm = 0;
    if (!blocks_per_sm) blocks_per_sm = blocks_for(k_gwn<GRID, SCREENED, PREC, SHAPE, ORDER>);
    long long want = (a.ngroups + kGwnWarps - 1) / kGwnWarps;
    long long grid = (long long)num_sms() * blocks_per_sm;
    if (want < grid) grid = want > 0 ? want : 1;
    k_gwn<GRID, SCREENED, PREC, SHAPE, ORDER><<<(unsigned)grid, kGwnWarps * 32, 0, s>>>(a);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

template <bool GRID, bool SCREENED, int PREC, int ORDER>
static int launch_shape(const GwnArgs& a, int shape, cudaStream_t s) {
    if (!GRID) return launch<GRID, SCREENED, PREC, 0, ORDER>(a, s);
    switch (shape) {
        case 1: return launch<GRID, SCREENED, PREC, 1, ORDER>(a, s);
        case 2: return launch<GRID, SCREENED, PREC, 2, ORDER>(a, s);
        case 3: return launch<GRID, SCREENED, PREC, 3, ORDER>(a, s);
        default: return launch<GRID, SCREENED, PREC, 0, ORDER>(a, s);
    }
}

template <bool GRID, int PREC>
static int launch_plain(const GwnArgs& a, const dwg_gwn_params& p, cudaStream_t s) {
    if (p.order == 1) return launch_shape<GRID, false, PREC, 1>(a, p.tile, s);
    if (p.order == 2) return launch_shape<GRID, false, PREC, 2>(a, p.tile, s);
    return launch_shape<GRID, false, PREC, 0>(a, p.tile, s);
}

template <bool GRID>
static int dispatch(const GwnArgs& a, const dwg_gwn_params& p, cudaStream_t s) {
    const int prec = p.precision < 0 ? 0 : (p.precision > 3 ? 3 : p.precision);
    if (p.screened) {
        if (prec == 0) return launch_shape<GRID, true, 0, 0>(a, p.tile, s);
        if (prec == 1) return launch_shape<GRID, true, 1, 0>(a, p.tile, s);
        if (prec == 3) return launch_shape<GRID, true, 3, 0>(a, p.tile, s);
        return launch_shape<GRID, true, 2, 0>(a, p.tile, s);
    }
    if (prec == 0) return launch_plain<GRID, 0>(a, p, s);
    if (prec == 1) return launch_plain<GRID, 1>(a, p, s);
    if (prec == 3) return launch_plain<GRID, 3>(a, p, s);
    return launch_plain<GRID, 2>(a, p, s);
}

// the kernel arguments of a sum (everything but the launch); *empty is set
// for an empty point query set
static int make_args(const Octree& t, const GwnQuery& q, const dwg_gwn_params& p, float* out,
                     unsigned long long* terms_total, int* per_query_terms, cudaStream_t s, const float* sigma_dev,
                     GwnArgs& a, bool* empty) {
    *empty = false;
    DWG_REQUIRE(t.M > 0, "gwn: octree is empty");
    DWG_REQUIRE(out != nullptr, "gwn: output is null");
    DWG_REQUIRE(p.order >= 0 && p.order <= 2, "gwn: expansion order must be 0, 1 or 2 (got %d)", p.order);
    DWG_REQUIRE(p.order == 0 || !p.screened, "gwn: expansion orders above 0 apply to the plain sum only");
    a.info = t.info.ptr;
    DWG_TRY(octree_set_beta(const_cast<Octree&>(t), p.beta, s));
    a.node_h = nullptr;
    a.list_count = nullptr;
    a.list_off = nullptr;
    a.list = nullptr;
    a.wbuf = nullptr;
    a.wstride = 0;
    a.wsel = nullptr;
    if (p.order > 0) {
        DWG_TRY(octree_update_expansion(const_cast<Octree&>(t), p.order, s));
        a.node_h = t.node_h.ptr;
    }
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
        a.zoff = 0;
        a.ox = a.oy = a.oz = a.h = 0.f;
        a.bx = a.by = 1;
        a.ngroups = (q.nq + 31) / 32;  // one point per lane
        *empty = a.ngroups == 0;
        return DWG_OK;
    }
    DWG_REQUIRE(q.res[0] > 0 && q.res[1] > 0 && q.res[2] > 0, "gwn: bad grid resolution");
    a.q = nullptr;
    a.nq = (long long)q.res[0] * q.res[1] * q.res[2];
    a.rx = q.res[0];
    a.ry = q.res[1];
    a.rz = q.res[2];
    a.zoff = q.zoff;
    a.ox = q.origin[0];
    a.oy = q.origin[1];
    a.oz = q.origin[2];
    a.h = q.spacing;
    DWG_REQUIRE(p.tile >= 0 && p.tile <= 3, "gwn: tile must be in [0, 3]");
    int ex, ey, ez;
    brick_extent(p.tile, ex, ey, ez);
    a.bx = (q.res[0] + ex - 1) / ex;
    a.by = (q.res[1] + ey - 1) / ey;
    a.ngroups = (long long)a.bx * a.by * ((q.res[2] + kNqGrid * ez - 1) / (kNqGrid * ez));  // bricks stacked in z
    DWG_REQUIRE(a.ngroups < (1ll << 32), "gwn: grid too large");
    return DWG_OK;
}

int gwn_eval(const Octree& t, const GwnQuery& q, const dwg_gwn_params& p, float* out,
             unsigned long long* terms_total, int* per_query_terms, cudaStream_t s,
             const float* sigma_dev) {
    GwnArgs a;
    bool empty = false;
    DWG_TRY(make_args(t, q, p, out, terms_total, per_query_terms, s, sigma_dev, a, &empty));
    if (empty) return DWG_OK;
    return q.q ? dispatch<false>(a, p, s) : dispatch<true>(a, p, s);
}

// ------------------------------------------------------ interaction lists --
GwnList::~GwnList() = default;

__global__ void k_list_total(const unsigned int* __restrict__ count, unsigned long long* __restrict__ off,
                             long long n) {
    off[n] = off[n - 1] + count[n - 1];
}

template <bool GRID, bool SCREENED, int PREC, int SHAPE>
static int listed_shape(GwnArgs& a, GwnList& L, const Octree& t, cudaStream_t s, size_t max_bytes, bool* fallback) {
    constexpr int NQ = nq_of<GRID>();
    using W = typename WeightOf<NQ>::T;
    static int bps = 0;
    if (!bps) bps = blocks_for(k_gwn_replay<GRID, SCREENED, PREC, SHAPE>);
    const long long grid_all = (long long)num_sms() * bps;
    const unsigned grid = (unsigned)(a.ngroups < grid_all * kGwnWarps ? (a.ngroups + kGwnWarps - 1) / kGwnWarps
                                                                      : grid_all);
    *fallback = false;
    if (!L.valid) {
        // count the entries of every group, place them, record them
        DWG_TRY(L.count.reserve(a.ngroups));
        DWG_TRY(L.off.reserve(a.ngroups + 1));
        GwnArgs c = a;
        c.list_count = L.count.ptr;
        c.out = nullptr;
        c.terms_total = nullptr;
        DWG_CHECK_CUDA(cudaMemsetAsync(t.work.ptr, 0, sizeof(unsigned int), s));
        k_gwn<GRID, SCREENED, PREC, SHAPE, 0, 1><<<grid, kGwnWarps * 32, 0, s>>>(c);
        DWG_CHECK_LAUNCH();
        size_t bytes = 0;
        DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, L.count.ptr, L.off.ptr, (int)a.ngroups, s));
        DWG_TRY(L.scratch.reserve(bytes + 256));
        bytes = L.scratch.n;
        DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(L.scratch.ptr, bytes, L.count.ptr, L.off.ptr, (int)a.ngroups, s));
        k_list_total<<<1, 1, 0, s>>>(L.count.ptr, L.off.ptr, a.ngroups);
        DWG_CHECK_LAUNCH();
        unsigned long long total = 0;
        DWG_CHECK_CUDA(cudaMemcpyAsync(&total, L.off.ptr + a.ngroups, sizeof(total), cudaMemcpyDeviceToHost, s));
        DWG_CHECK_CUDA(cudaStreamSynchronize(s));
        if (!max_bytes) max_bytes = device_free_bytes() / 4;  // no budget given: a quarter of the free memory
        // too large to keep, or no room for it: traverse every time
        if (total * sizeof(int4) > max_bytes || L.ent.reserve(total ? total : 1) != DWG_OK) {
            L.too_big = true;
            L.count.release();
            L.off.release();
            L.ent.release();
            *fallback = true;
            return DWG_OK;
        }
        c.list_off = L.off.ptr;
        c.list = L.ent.ptr;
        DWG_CHECK_CUDA(cudaMemsetAsync(t.work.ptr, 0, sizeof(unsigned int), s));
        k_gwn<GRID, SCREENED, PREC, SHAPE, 0, 2><<<grid, kGwnWarps * 32, 0, s>>>(c);
        DWG_CHECK_LAUNCH();
        L.entries = total;
        L.valid = true;
        // weight slots: 8 bytes per entry and lane each, together at most a
        // third of the free memory and 64 GB
        L.nslots = 0;
        if (SCREENED && PREC != 2 && L.wslots > 0 && total > 0) {
            const size_t fr = device_free_bytes();
            const unsigned long long per = total * 32ull * sizeof(W);
            unsigned long long cap = std::min<unsigned long long>(fr / 3, 64ull << 30);
            if (L.wmax) {  // a budget shared with the entries just kept
                const unsigned long long lb = total * (unsigned long long)sizeof(int4);
                cap = std::min<unsigned long long>(cap, L.wmax > lb ? L.wmax - lb : 0);
            }
            int n = (int)std::min<unsigned long long>((unsigned long long)std::min(L.wslots, kGwnWeightSlots),
                                                      cap / per);
            if (n > 0 && L.w.reserve(((size_t)n * per + sizeof(float2) - 1) / sizeof(float2)) != DWG_OK) n = 0;
            L.nslots = n;
            DWG_TRY(L.wstate.reserve(1));
            k_weight_reset<<<1, 1, 0, s>>>(L.wstate.ptr, n, slot_prefs(L, n));
            DWG_CHECK_LAUNCH();
        }
    }
    a.list_off = L.off.ptr;
    a.list = L.ent.ptr;
    if (L.nslots > 0) {
        a.wbuf = L.w.ptr;
        a.wstride = L.entries * 32ull;
        a.wsel = L.wstate.ptr;
        k_weight_select<<<1, 1, 0, s>>>(L.wstate.ptr, a.sigma_dev, a.sigma, a.screen);
        DWG_CHECK_LAUNCH();
    }
    DWG_CHECK_CUDA(cudaMemsetAsync(t.work.ptr, 0, sizeof(unsigned int), s));
    k_gwn_replay<GRID, SCREENED, PREC, SHAPE><<<grid, kGwnWarps * 32, 0, s>>>(a);
    DWG_CHECK_LAUNCH();
    if (L.nslots > 0) {
        // the ring's shared memory is opted into per device
        static int bpw_dev[64] = {0};
        int dev = 0;
        DWG_CHECK_CUDA(cudaGetDevice(&dev));
        DWG_REQUIRE(dev >= 0 && dev < 64, "gwn: device %d out of range", dev);
        int& bpw = bpw_dev[dev];
        if (!bpw) {
            DWG_CHECK_CUDA(cudaFuncSetAttribute(k_gwn_wread<GRID, SCREENED, PREC, SHAPE>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, wread_smem<GRID>()));
            DWG_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpw, k_gwn_wread<GRID, SCREENED, PREC, SHAPE>,
                                                                         kGwnWarps * 32, wread_smem<GRID>()));
            if (bpw < 1) bpw = 1;
        }
        const long long all = (long long)num_sms() * bpw;
        const unsigned gw = (unsigned)(a.ngroups < all * kGwnWarps ? (a.ngroups + kGwnWarps - 1) / kGwnWarps : all);
        k_gwn_wread<GRID, SCREENED, PREC, SHAPE><<<gw, kGwnWarps * 32, wread_smem<GRID>(), s>>>(a);
        DWG_CHECK_LAUNCH();
    }
    return DWG_OK;
}

template <bool GRID, int PREC>
static int listed_prec(GwnArgs& a, GwnList& L, const Octree& t, int tile, cudaStream_t s, size_t max_bytes,
                       bool* fallback) {
    if (!GRID) return listed_shape<GRID, true, PREC, 0>(a, L, t, s, max_bytes, fallback);
    switch (tile) {
        case 1: return listed_shape<GRID, true, PREC, 1>(a, L, t, s, max_bytes, fallback);
        case 2: return listed_shape<GRID, true, PREC, 2>(a, L, t, s, max_bytes, fallback);
        case 3: return listed_shape<GRID, true, PREC, 3>(a, L, t, s, max_bytes, fallback);
        default: return listed_shape<GRID, true, PREC, 0>(a, L, t, s, max_bytes, fallback);
    }
}

template <bool GRID>
static int listed_dispatch(GwnArgs& a, GwnList& L, const Octree& t, const dwg_gwn_params& p, cudaStream_t s,
                           size_t max_bytes) {
    const int prec = p.precision < 0 ? 0 : (p.precision > 3 ? 3 : p.precision);
    bool fallback = false;
    if (prec == 0) DWG_TRY(listed_prec<GRID, 0>(a, L, t, p.tile, s, max_bytes, &fallback));
    else if (prec == 1) DWG_TRY(listed_prec<GRID, 1>(a, L, t, p.tile, s, max_bytes, &fallback));
    else if (prec == 3) DWG_TRY(listed_prec<GRID, 3>(a, L, t, p.tile, s, max_bytes, &fallback));
    else DWG_TRY(listed_prec<GRID, 2>(a, L, t, p.tile, s, max_bytes, &fallback));
    if (fallback) {
        DWG_CHECK_CUDA(cudaMemsetAsync(t.work.ptr, 0, sizeof(unsigned int), s));
        return dispatch<GRID>(a, p, s);
    }
    return DWG_OK;
}

int gwn_eval_listed(const Octree& t, const GwnQuery& q, const dwg_gwn_params& p, GwnList& L, float* out,
                    unsigned long long* terms_total, cudaStream_t s, const float* sigma_dev, size_t max_bytes,
                    int wslots) {
    DWG_REQUIRE(p.screened && p.order == 0, "gwn lists: screened sums only");
    GwnArgs a;
    bool empty = false;
    DWG_TRY(make_args(t, q, p, out, terms_total, nullptr, s, sigma_dev, a, &empty));
    if (empty) return DWG_OK;
    const bool grid = !q.q;
    const bool same = L.ngroups == a.ngroups && L.grid == grid && L.qptr == q.q && L.nq == a.nq &&
                      L.tile == (grid ? p.tile : 0) && L.res[0] == q.res[0] && L.res[1] == q.res[1] &&
                      L.res[2] == q.res[2] && L.zoff == q.zoff && L.origin[0] == q.origin[0] &&
                      L.origin[1] == q.origin[1] && L.origin[2] == q.origin[2] && L.spacing == q.spacing &&
                      L.beta == p.beta && L.use_radii == p.use_radii && L.wslots == wslots;
    if (!same) {  // other samples or other decisions: record again
        L.valid = false;
        L.too_big = false;
    }
    if (L.too_big) return grid ? dispatch<true>(a, p, s) : dispatch<false>(a, p, s);
    L.ngroups = a.ngroups;
    L.grid = grid;
    L.qptr = q.q;
    L.nq = a.nq;
    L.tile = grid ? p.tile : 0;
    for (int d = 0; d < 3; ++d) {
        L.res[d] = q.res[d];
        L.origin[d] = q.origin[d];
    }
    L.zoff = q.zoff;
    L.spacing = q.spacing;
    L.beta = p.beta;
    L.use_radii = p.use_radii;
    L.wslots = wslots;
    return grid ? listed_dispatch<true>(a, L, t, p, s, max_bytes) : listed_dispatch<false>(a, L, t, p, s, max_bytes);
}

// ------------------------------------------------------------- batches --
static void fill_args(GwnArgs& a, const Octree& t, const GwnBatchItem& it, const dwg_gwn_params& p) {
    a.info = t.info.ptr;
    a.node_a = t.node_a.ptr;
    a.node_b = t.node_b.ptr;
    a.node_r = t.node_r.ptr;
    a.pa = t.pa.ptr;
    a.nr = t.nr.ptr;
    a.beta = p.beta;
    a.sigma = p.sigma;
    a.sigma_dev = it.sigma_dev;
    a.screen = p.screen;
    a.use_radii = p.use_radii;
    a.q = nullptr;
    a.rx = it.res[0];
    a.ry = it.res[1];
    a.rz = it.res[2];
    a.zoff = 0;
    a.nq = (long long)a.rx * a.ry * a.rz;
    a.ox = it.origin[0];
    a.oy = it.origin[1];
    a.oz = it.origin[2];
    a.h = it.spacing;
    int ex, ey, ez;
    brick_extent(p.tile, ex, ey, ez);
    a.bx = (a.rx + ex - 1) / ex;
    a.by = (a.ry + ey - 1) / ey;
    a.ngroups = (long long)a.bx * a.by * ((a.rz + kNqGrid * ez - 1) / (kNqGrid * ez));
    a.out = it.out;
    a.terms_total = it.terms_total;
    a.per_query_terms = nullptr;
    a.work = t.work.ptr;  // error word at [1]
    a.node_h = nullptr;
    a.list_count = nullptr;
    a.list_off = nullptr;
    a.list = nullptr;
    a.wbuf = nullptr;
    a.wstride = 0;
    a.wsel = nullptr;
    a.num_nodes = t.M;
    a.num_points = t.n;
}

struct GwnBatchImpl {
    DevBuf<GwnArgs> table;
    DevBuf<unsigned long long> prefix, work;
    int n = 0;
    dwg_gwn_params p{};
};

GwnBatch::~GwnBatch() { delete impl; }

int gwn_batch_prepare(GwnBatch& b, const GwnBatchItem* items, int n, const dwg_gwn_params& p, cudaStream_t s) {
    DWG_REQUIRE(items && n >= 1, "gwn batch: no clouds");
    DWG_REQUIRE(p.screened, "gwn batch: screened sums only");
    DWG_REQUIRE(p.tile >= 0 && p.tile <= 3, "gwn batch: tile must be in [0, 3]");
    if (!b.impl) b.impl = new GwnBatchImpl();
    GwnBatchImpl& B = *b.impl;
    std::vector<GwnArgs> host((size_t)n);
    std::vector<unsigned long long> pre((size_t)n + 1, 0);
    for (int i = 0; i < n; ++i) {
        DWG_REQUIRE(items[i].tree && items[i].tree->M > 0 && items[i].out, "gwn batch: cloud %d is incomplete", i);
        DWG_REQUIRE(items[i].res[0] > 0 && items[i].res[1] > 0 && items[i].res[2] > 0,
                    "gwn batch: cloud %d has a bad grid", i);
        DWG_TRY(octree_set_beta(*items[i].tree, items[i].beta > 0.f ? items[i].beta : p.beta, s));
        fill_args(host[i], *items[i].tree, items[i], p);
        pre[i + 1] = pre[i] + (unsigned long long)host[i].ngroups;
    }
    DWG_TRY(B.table.reserve(n));
    DWG_TRY(B.prefix.reserve(n + 1));
    DWG_TRY(B.work.reserve(1));
    DWG_CHECK_CUDA(cudaMemcpyAsync(B.table.ptr, host.data(), sizeof(GwnArgs) * n, cudaMemcpyHostToDevice, s));
    DWG_CHECK_CUDA(cudaMemcpyAsync(B.prefix.ptr, pre.data(), sizeof(unsigned long long) * (n + 1),
                                   cudaMemcpyHostToDevice, s));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));  // host vectors go out of scope
    B.n = n;
    B.p = p;
    b.groups = pre[n];
    return DWG_OK;
}

template <bool SCREENED, int PREC, int SHAPE>
static int launch_batch(GwnBatchImpl& B, unsigned long long groups, cudaStream_t s) {
    static int bps = 0;
    if (!bps) bps = blocks_for(k_gwn_batch<SCREENED, PREC, SHAPE>);
    long long want = (long long)((groups + kGwnWarps - 1) / kGwnWarps);
    long long grid = (long long)num_sms() * bps;
    if (want < grid) grid = want > 0 ? want : 1;
    k_gwn_batch<SCREENED, PREC, SHAPE><<<(unsigned)grid, kGwnWarps * 32, 0, s>>>(B.table.ptr, B.prefix.ptr, B.n,
                                                                                 B.work.ptr);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

template <int PREC>
static int launch_batch_shape(GwnBatchImpl& B, unsigned long long groups, cudaStream_t s) {
    switch (B.p.tile) {
        case 1: return launch_batch<true, PREC, 1>(B, groups, s);
        case 2: return launch_batch<true, PREC, 2>(B, groups, s);
        case 3: return launch_batch<true, PREC, 3>(B, groups, s);
        default: return launch_batch<true, PREC, 0>(B, groups, s);
    }
}

int gwn_batch_launch(GwnBatch& b, cudaStream_t s) {
    DWG_REQUIRE(b.impl && b.impl->n > 0, "gwn batch: not prepared");
    GwnBatchImpl& B = *b.impl;
    DWG_CHECK_CUDA(cudaMemsetAsync(B.work.ptr, 0, sizeof(unsigned long long), s));
    const int prec = B.p.precision < 0 ? 0 : (B.p.precision > 3 ? 3 : B.p.precision);
    if (prec == 0) return launch_batch_shape<0>(B, b.groups, s);
    if (prec == 1) return launch_batch_shape<1>(B, b.groups, s);
    if (prec == 3) return launch_batch_shape<3>(B, b.groups, s);
    return launch_batch_shape<2>(B, b.groups, s);
}

}  // namespace dwg
