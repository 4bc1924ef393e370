// gwn_eval.cu -- values and gradients of the winding-number sums, one thread
// per query, with the Barnes-Hut decisions of the warp kernels (gwn.cu).
//
// The DWG loop needs values only, and gwn.cu sums those with one warp per 32
// coherent queries.  This file serves the two other uses of the same sums:
//
//  * the analytic gradient grad_q w (the reference has none): for a term
//    v = G(rho) dot with dot = ne.(p - q) (ne = A n of a point, sum A n of a
//    far node),
//        screened  G = |sigma rho + 1| / (e^{sigma rho} 4 pi rho^3 + 1e-7),
//                  rho = max(|p - q|, s),
//                  grad v = -G ne + dot G'(rho) grad rho,
//                  grad rho = -(p - q) / r for r > s, 0 where s takes over;
//        plain     G = 1 / (4 pi r^3 + 1e-8),
//                  grad v = -ne G + dot 12 pi r G^2 (p - q);
//    the far field is the order-0 dipole, whose gradient this is;
//  * FP64 sums: terms and sums in double from the FP64 moments (cm_d, ec_d)
//    and the points' float data, the yardstick a caller checks the FP32 sums
//    against on the GPU (the CPU oracle does the same on the host).
//
// Decisions: a child record is far when sq3_rn(CM_f - q) > its open
// threshold (exactly the warp kernels' test, so the same terms are taken);
// leaves are always summed point by point.  The traversal walks the level-
// order records with a per-level (first child, count, next) stack.
#include "gwn.cuh"

namespace dwg {

constexpr double kFourPiD = 12.566370614359172953850573533118;

struct ThreadArgs {
    const float4* __restrict__ node_a;
    const float4* __restrict__ node_b;
    const int* __restrict__ level_nodes;
    const double* __restrict__ cm_d;
    const double* __restrict__ ec_d;
    const float4* __restrict__ pa;
    const float4* __restrict__ nr;
    float sigma, screen;
    int use_radii;
    const float* __restrict__ q;
    long long nq;
    int rx, ry, rz, zoff;
    float ox, oy, oz, h;
    int num_nodes, num_points;
    void* out_w;
    void* out_g;
    unsigned int* err;
};

// One term and its gradient, terms in T (float: IEEE sqrt and division and
// CUDA's expf; or double), accumulated in double.
template <typename T, bool SCREENED, bool GRAD>
__device__ __forceinline__ void add_term(T dx, T dy, T dz, T nx, T ny, T nz, T s, T sigma, double& w, double* g) {
    const T r2 = dx * dx + dy * dy + dz * dz;
    const T dot = dx * nx + dy * ny + dz * nz;
    if (SCREENED) {
        if (!(r2 > (T)1e-20)) return;  // |p - q| <= 1e-10 is skipped
        const T r = sqrt(r2);
        const T rho = r > s ? r : s;
        const T e = exp(sigma * rho);
        const T r3 = rho * rho * rho;
        const T den = e * ((T)kFourPiD * r3) + (T)1e-7;
        const T up = fabs(sigma * rho + (T)1);
        const T G = up / den;
        w += (double)(G * dot);
        if (GRAD) {
            const T dden = e * (sigma * (T)kFourPiD * r3 + (T)(3.0 * kFourPiD) * rho * rho);
            const T Gp = (sigma * den - up * dden) / (den * den);
            const T k = r > s ? -dot * Gp / r : (T)0;
            g[0] += (double)(k * dx - G * nx);
            g[1] += (double)(k * dy - G * ny);
            g[2] += (double)(k * dz - G * nz);
        }
    } else {
        if (r2 == (T)0) return;  // a zero distance is a term of value 0
        const T r = sqrt(r2);
        const T den = (T)kFourPiD * r * r2 + (T)1e-8;
        w += (double)(dot / den);
        if (GRAD) {
            const T k = dot * (T)(3.0 * kFourPiD) * r / (den * den);
            g[0] += (double)(k * dx - nx / den);
            g[1] += (double)(k * dy - ny / den);
            g[2] += (double)(k * dz - nz / den);
        }
    }
}

template <typename T, bool SCREENED, bool GRAD>
__device__ __forceinline__ void leaf_points_thread(const ThreadArgs& a, int st, int cnt, float qx, float qy, float qz,
                                                   double& w, double* g) {
    const T sig = (T)a.sigma;
    for (int j = st; j < st + cnt; ++j) {
        const float4 p = a.pa[j];
        const float4 n = a.nr[j];
        const T s = (T)(a.use_radii ? n.w : a.screen);
        add_term<T, SCREENED, GRAD>((T)p.x - (T)qx, (T)p.y - (T)qy, (T)p.z - (T)qz, (T)p.w * (T)n.x,
                                    (T)p.w * (T)n.y, (T)p.w * (T)n.z, s, sig, w, g);
    }
}

template <typename T, bool SCREENED, bool GRAD>
__global__ void __launch_bounds__(128) k_gwn_thread(ThreadArgs a) {
    using TO = T;  // output type
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.nq; i += stride) {
        float qx, qy, qz;
        if (a.q) {
            qx = a.q[i * 3];
            qy = a.q[i * 3 + 1];
            qz = a.q[i * 3 + 2];
        } else {  // the grid sample of the warp kernels: origin + index * spacing, rounded per operation
            const long long x = i % a.rx, t = i / a.rx;
            const long long y = t % a.ry, z = t / a.ry;
            qx = __fadd_rn(a.ox, __fmul_rn((float)x, a.h));
            qy = __fadd_rn(a.oy, __fmul_rn((float)y, a.h));
            qz = __fadd_rn(a.oz, __fmul_rn((float)(z + a.zoff), a.h));
        }
        double w = 0, g[3] = {0, 0, 0};
        int first[kMaxDepth + 2], count[kMaxDepth + 2], next[kMaxDepth + 2];
        int lev = 0;
        {
            const unsigned rm = (unsigned)__float_as_int(a.node_b[0].w);
            if (rm & kMetaLeafBit) {
                const int st = (int)(rm & kMetaIndex), cnt = __float_as_int(a.node_a[0].w);
                if (cnt >= 0 && st + cnt <= a.num_points)
                    leaf_points_thread<T, SCREENED, GRAD>(a, st, cnt, qx, qy, qz, w, g);
                else
                    atomicOr(a.err, 4u);
            } else {
                first[0] = (int)(rm & kMetaIndex);
                count[0] = (int)((rm >> 28) & 7u) + 1;
                next[0] = 0;
                lev = 1;
            }
        }
        while (lev > 0) {
            const int L = lev - 1;
            if (next[L] == count[L]) {
                --lev;
                continue;
            }
            const int c = first[L] + next[L]++;
            if (c < 0 || c >= a.num_nodes) {
                atomicOr(a.err, 2u);
                --lev;
                continue;
            }
            const float4 na = a.node_a[c], nb = a.node_b[c];
            const unsigned meta = (unsigned)__float_as_int(nb.w);
            if (meta & kMetaLeafBit) {
                const int st = (int)(meta & kMetaIndex), cnt = __float_as_int(na.w);
                if (cnt < 0 || st + cnt > a.num_points) {
                    atomicOr(a.err, 4u);
                    continue;
                }
                leaf_points_thread<T, SCREENED, GRAD>(a, st, cnt, qx, qy, qz, w, g);
                continue;
            }
            const float dxf = __fsub_rn(na.x, qx), dyf = __fsub_rn(na.y, qy), dzf = __fsub_rn(na.z, qz);
            if (sq3_rn(dxf, dyf, dzf) > na.w) {  // far: the node's dipole term
                if (sizeof(T) == 8) {
                    const int v = a.level_nodes[c];
                    const double* cm = a.cm_d + (size_t)v * 3;
                    const double* ec = a.ec_d + (size_t)v * 3;
                    add_term<T, SCREENED, GRAD>((T)(cm[0] - (double)qx), (T)(cm[1] - (double)qy),
                                                (T)(cm[2] - (double)qz), (T)ec[0], (T)ec[1], (T)ec[2],
                                                (T)a.screen, (T)a.sigma, w, g);
                } else {
                    add_term<T, SCREENED, GRAD>((T)dxf, (T)dyf, (T)dzf, (T)nb.x, (T)nb.y, (T)nb.z, (T)a.screen,
                                                (T)a.sigma, w, g);
                }
                continue;
            }
            // opened: its children become the next level
            const int fc = (int)(meta & kMetaIndex), nch = (int)((meta >> 28) & 7u) + 1;
            if (fc <= c || fc + nch > a.num_nodes || lev >= kMaxDepth + 2) {
                atomicOr(a.err, 2u);
                continue;
            }
            first[lev] = fc;
            count[lev] = nch;
            next[lev] = 0;
            ++lev;
        }
        if (a.out_w) static_cast<TO*>(a.out_w)[i] = (TO)w;
        if (GRAD && a.out_g) {
            TO* og = static_cast<TO*>(a.out_g) + i * 3;
            og[0] = (TO)g[0];
            og[1] = (TO)g[1];
            og[2] = (TO)g[2];
        }
    }
}

template <typename T, bool SCREENED, bool GRAD>
static int launch_thread(const ThreadArgs& a, cudaStream_t s) {
    const long long blocks = std::min<long long>((a.nq + 127) / 128, (long long)num_sms() * 16);
    k_gwn_thread<T, SCREENED, GRAD><<<(unsigned)(blocks > 0 ? blocks : 1), 128, 0, s>>>(a);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

int gwn_eval_thread(const Octree& t, const GwnQuery& q, const dwg_gwn_params& p, bool fp64, void* out_w,
                    void* out_g, cudaStream_t s) {
    DWG_REQUIRE(t.M > 0, "gwn: octree is empty");
    DWG_REQUIRE(out_w || out_g, "gwn: no output");
    DWG_REQUIRE(p.order == 0, "gwn: gradients and FP64 sums take the order-0 far field");
    DWG_REQUIRE(p.beta >= 0.f, "gwn: beta must be >= 0");
    DWG_TRY(octree_set_beta(const_cast<Octree&>(t), p.beta, s));
    DWG_TRY(t.work.reserve(2));
    ThreadArgs a;
    a.node_a = t.node_a.ptr;
    a.node_b = t.node_b.ptr;
    a.level_nodes = t.level_nodes.ptr;
    a.cm_d = t.cm_d.ptr;
    a.ec_d = t.ec_d.ptr;
    a.pa = t.pa.ptr;
    a.nr = t.nr.ptr;
    a.sigma = p.sigma;
    a.screen = p.screen;
    a.use_radii = p.use_radii;
    a.num_nodes = t.M;
    a.num_points = t.n;
    a.out_w = out_w;
    a.out_g = out_g;
    a.err = t.work.ptr + 1;
    if (q.q) {
        a.q = q.q;
        a.nq = q.nq;
        a.rx = a.ry = a.rz = a.zoff = 0;
        a.ox = a.oy = a.oz = a.h = 0.f;
    } else {
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
    }
    if (a.nq == 0) return DWG_OK;
    const bool grad = out_g != nullptr;
    if (fp64) {
        if (p.screened) return grad ? launch_thread<double, true, true>(a, s) : launch_thread<double, true, false>(a, s);
        return grad ? launch_thread<double, false, true>(a, s) : launch_thread<double, false, false>(a, s);
    }
    if (p.screened) return grad ? launch_thread<float, true, true>(a, s) : launch_thread<float, true, false>(a, s);
    return grad ? launch_thread<float, false, true>(a, s) : launch_thread<float, false, false>(a, s);
}

}  // namespace dwg
