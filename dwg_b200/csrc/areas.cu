// areas.cu -- PCA normals and point areas (the reference's --com_As 1 mode).
//
// The reference computes both on the host with third-party code: PCL's
// NormalEstimation (k = 10, viewpoint at the bounding-box centre,
// include/DWGProcess.h:152-200) and libigl's CGAL-based point_areas
// (deps/libigl/include/igl/copyleft/cgal/point_areas.cpp:39-210).  Here each
// point is one thread.  The covariance and its cyclic Jacobi eigen
// decomposition use only +, -, *, / and sqrt in FP64, each rounded once
// (this file is compiled without contraction into fused multiply-adds), in
// a fixed order, so the results do not depend on the thread or the device.
//
// The area of point i needs the 2-D Delaunay triangles around it among its
// kept neighbours; a triangle (i, b, c) is Delaunay when no other neighbour
// lies strictly inside its circumcircle.  Leaves are octree cell centres, a
// lattice, so cocircular neighbours are common: the decisions are made
// exactly (orientation in 64-bit integers, the in-circle determinant by a
// floating-point filter with an exact 128-bit fallback) on coordinates
// rounded to 2^-24 of the neighbourhood's extent, and each cocircular
// polygon is triangulated as the fan from point i.
#include <cmath>

#include "areas.cuh"

namespace dwg {

constexpr int kAreaMaxK = 32;

// cyclic Jacobi rotations on a symmetric 3x3 matrix (each rotation zeroes
// its pivot); w ascending, V[:, i] the unit eigenvector of w[i]
__device__ void jacobi3(const double A_in[3][3], double w[3], double V[3][3]) {
    double a[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            a[i][j] = A_in[i][j];
            V[i][j] = i == j ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 32; sweep++) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        const double dg = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off <= 1e-36 * dg) break;
#pragma unroll
        for (int p = 0; p < 2; p++)
#pragma unroll
            for (int q = p + 1; q < 3; q++) {
                if (a[p][q] == 0.0) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
#pragma unroll
                for (int k = 0; k < 3; k++) {  // columns p, q
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
#pragma unroll
                for (int k = 0; k < 3; k++) {  // rows p, q
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                a[p][q] = 0.0;
                a[q][p] = 0.0;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    // ascending eigenvalues, ties in index order
    int ord[3] = {0, 1, 2};
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = i + 1; j < 3; j++)
            if (a[ord[j]][ord[j]] < a[ord[i]][ord[i]]) {
                const int t = ord[i];
                ord[i] = ord[j];
                ord[j] = t;
            }
    double Vs[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        w[i] = a[ord[i]][ord[i]];
#pragma unroll
        for (int k = 0; k < 3; k++) Vs[k][i] = V[k][ord[i]];
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) V[i][k] = Vs[i][k];
}

// mean and covariance (divided by m) of the rows of nb with a non-negative id
__device__ int covariance_row(const float* __restrict__ P, const int* __restrict__ row, int k, double c[3],
                              double C[3][3]) {
    c[0] = c[1] = c[2] = 0;
    int m = 0;
    for (int j = 0; j < k; j++) {
        const int q = row[j];
        if (q < 0) continue;
        for (int d = 0; d < 3; d++) c[d] += (double)P[(size_t)q * 3 + d];
        ++m;
    }
    if (m == 0) return 0;
    for (int d = 0; d < 3; d++) c[d] /= m;
    for (int r = 0; r < 3; r++)
        for (int q = 0; q < 3; q++) C[r][q] = 0.0;
    for (int j = 0; j < k; j++) {
        const int q = row[j];
        if (q < 0) continue;
        double e[3];
        for (int d = 0; d < 3; d++) e[d] = (double)P[(size_t)q * 3 + d] - c[d];
        for (int r = 0; r < 3; r++)
            for (int qq = 0; qq < 3; qq++) C[r][qq] += e[r] * e[qq];
    }
    for (int r = 0; r < 3; r++)
        for (int q = 0; q < 3; q++) C[r][q] /= m;
    return m;
}

__global__ void k_pca_normals(const float* __restrict__ P, int n, const int* __restrict__ nb, int k,
                              const float* __restrict__ view, float* __restrict__ N) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double nv[3] = {0, 0, 1};
    double c[3], C[3][3];
    if (covariance_row(P, nb + (size_t)i * k, k, c, C) >= 3) {
        double w[3], V[3][3];
        jacobi3(C, w, V);
        for (int d = 0; d < 3; d++) nv[d] = V[d][0];
    }
    // flipNormalTowardsViewpoint: (view - p) . n >= 0
    double dp = 0;
    for (int d = 0; d < 3; d++) dp += ((double)view[d] - (double)P[(size_t)i * 3 + d]) * nv[d];
    const double sg = dp < 0 ? -1.0 : 1.0;
    for (int d = 0; d < 3; d++) N[(size_t)i * 3 + d] = (float)(sg * nv[d]);
}

// exact orientation of integer points (|coordinates| <= 2^24): > 0 counter-clockwise
__device__ __forceinline__ long long orient_q(long long ax, long long ay, long long bx, long long by, long long cx,
                                              long long cy) {
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}

// sign of the in-circle determinant of d against the circle through a, b, c
// (> 0: d inside when a, b, c are counter-clockwise).  With |coordinates| <=
// 2^24 every difference, lift and 2x2 minor is exact in FP64; only the three
// products and two sums round, so |error| < 4u * sum|products| (u = 2^-53)
// and a larger determinant has the sign of the exact one.  Otherwise the
// determinant is evaluated exactly in 128-bit integers.
__device__ int incircle_q(long long ax, long long ay, long long bx, long long by, long long cx, long long cy,
                          long long dx, long long dy) {
    const double adx = (double)(ax - dx), ady = (double)(ay - dy), bdx = (double)(bx - dx),
                 bdy = (double)(by - dy), cdx = (double)(cx - dx), cdy = (double)(cy - dy);
    const double t1 = (adx * adx + ady * ady) * (bdx * cdy - cdx * bdy);
    const double t2 = (bdx * bdx + bdy * bdy) * (adx * cdy - cdx * ady);
    const double t3 = (cdx * cdx + cdy * cdy) * (adx * bdy - bdx * ady);
    const double det = (t1 - t2) + t3;
    const double bound = ((fabs(t1) + fabs(t2)) + fabs(t3)) * 0x1p-51;
    if (det > bound) return 1;
    if (det < -bound) return -1;
    const __int128 Adx = ax - dx, Ady = ay - dy, Bdx = bx - dx, Bdy = by - dy, Cdx = cx - dx, Cdy = cy - dy;
    const __int128 e = (Adx * Adx + Ady * Ady) * (Bdx * Cdy - Cdx * Bdy) -
                       (Bdx * Bdx + Bdy * Bdy) * (Adx * Cdy - Cdx * Ady) +
                       (Cdx * Cdx + Cdy * Cdy) * (Adx * Bdy - Bdx * Ady);
    return e > 0 ? 1 : (e < 0 ? -1 : 0);
}

__global__ void k_point_areas(const float* __restrict__ P, int n, const int* __restrict__ nb, int k,
                              const float* __restrict__ N, float* __restrict__ A) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int* row = nb + (size_t)i * k;
    const int q0 = row[0];
    if (q0 < 0) {
        A[i] = 0.f;
        return;
    }
    // the neighbours whose normal agrees with the first one's (self),
    // point_areas.cpp:97-106
    int ids[kAreaMaxK];
    int m = 0;
    const double n0x = N[(size_t)q0 * 3], n0y = N[(size_t)q0 * 3 + 1], n0z = N[(size_t)q0 * 3 + 2];
    for (int j = 0; j < k; ++j) {
        const int q = row[j];
        if (q < 0) continue;
        double d = 0;
        d += n0x * (double)N[(size_t)q * 3];
        d += n0y * (double)N[(size_t)q * 3 + 1];
        d += n0z * (double)N[(size_t)q * 3 + 2];
        if (d > 0) ids[m++] = q;
    }
    if (m <= 2) {
        A[i] = 0.f;
        return;
    }
    // PCA plane (point_areas.cpp:114-133): scores on the two largest
    // principal directions
    double c[3], C[3][3], w[3], V[3][3];
    covariance_row(P, ids, m, c, C);
    jacobi3(C, w, V);
    double u[kAreaMaxK], v[kAreaMaxK];
    double mx = 0;
    for (int j = 0; j < m; j++) {
        double e[3];
        for (int d = 0; d < 3; d++) e[d] = (double)P[(size_t)ids[j] * 3 + d] - c[d];
        u[j] = e[0] * V[0][2] + e[1] * V[1][2] + e[2] * V[2][2];
        v[j] = e[0] * V[0][1] + e[1] * V[1][1] + e[2] * V[2][1];
        if (fabs(u[j]) > mx) mx = fabs(u[j]);
        if (fabs(v[j]) > mx) mx = fabs(v[j]);
    }
    if (!(mx > 0) || !isfinite(mx)) {
        A[i] = 0.f;
        return;
    }
    // coordinates rounded to 2^-24 of the extent; coincident points after
    // rounding are one vertex (the first)
    const double scale = ldexp(1.0, 23 - ilogb(mx));
    int qx[kAreaMaxK], qy[kAreaMaxK], keep[kAreaMaxK];
    int mk = 0;
    for (int j = 0; j < m; j++) {
        const int x = (int)__double2ll_rn(u[j] * scale), y = (int)__double2ll_rn(v[j] * scale);
        bool dup = false;
        for (int t = 0; t < mk && !dup; t++) dup = qx[t] == x && qy[t] == y;
        if (dup) continue;
        qx[mk] = x;
        qy[mk] = y;
        keep[mk++] = j;
    }
    double acc = 0;
    for (int b = 1; b < mk; ++b) {
        for (int cc = b + 1; cc < mk; ++cc) {
            const long long orient = orient_q(qx[0], qy[0], qx[b], qy[b], qx[cc], qy[cc]);
            if (orient == 0) continue;  // collinear: no face
            // Delaunay: no point strictly inside the circumcircle; points on
            // it form a cocircular polygon, triangulated as the fan from the
            // point itself (b, c adjacent: no cocircular point beyond b-c)
            bool ok = true;
            for (int t = 1; t < mk && ok; ++t) {
                if (t == b || t == cc) continue;
                int sg = incircle_q(qx[0], qy[0], qx[b], qy[b], qx[cc], qy[cc], qx[t], qy[t]);
                if (orient < 0) sg = -sg;
                if (sg > 0) ok = false;
                if (sg == 0) {
                    const long long side = orient_q(qx[b], qy[b], qx[cc], qy[cc], qx[t], qy[t]);
                    if ((side > 0) != (orient > 0) && side != 0) ok = false;
                }
            }
            if (!ok) continue;
            // triangle XYZ with X the point itself (point_areas.cpp:160-193)
            const int jb = keep[b], jc = keep[cc];
            const double ax = u[0], ay = v[0], bx = u[jb], by = v[jb], cx = u[jc], cy = v[jc];
            const double x = sqrt((bx - cx) * (bx - cx) + (by - cy) * (by - cy));
            const double y = sqrt((ax - cx) * (ax - cx) + (ay - cy) * (ay - cy));
            const double z = sqrt((bx - ax) * (bx - ax) + (by - ay) * (by - ay));
            const double cosX = (z * z + y * y - x * x) / (2 * y * z);
            const double cosY = (z * z + x * x - y * y) / (2 * x * z);
            const double cosZ = (x * x + y * y - z * z) / (2 * y * x);
            double b0 = x * cosX, b1 = y * cosY, b2 = z * cosZ;
            const double bs = b0 + b1 + b2;
            b0 /= bs;
            b1 /= bs;
            b2 /= bs;
            const double full = 0.25 * sqrt((x + (y + z)) * (z - (x - y)) * (z + (x - y)) * (x + (y - z)));
            if (cosX < 0) {
                acc += 0.5 * full;
            } else if (cosY < 0 || cosZ < 0) {
                acc += 0.25 * full;
            } else {
                acc += (b1 * full + b2 * full) / 2;
            }
        }
    }
    A[i] = isfinite(acc) ? (float)acc : 0.f;
}

// splitmix64 (S. Vigna) of an index: the seeded random stream of the leaf normals
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__global__ void k_random_normals(float* __restrict__ N, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double scale = (1.0 / 9007199254740992.0) * 6.283185307179586;
    const double u = (double)(mix64((unsigned long long)i * 2) >> 11) * scale;
    const double v = (double)(mix64((unsigned long long)i * 2 + 1) >> 11) * scale;
    N[(size_t)i * 3] = (float)(sin(u) * cos(v));
    N[(size_t)i * 3 + 1] = (float)(sin(u) * sin(v));
    N[(size_t)i * 3 + 2] = (float)cos(u);
}

// centre of a bounding box (min xyz, max xyz): (upper + lower) / 2 in float
__global__ void k_box_centre(const float* __restrict__ box, float* __restrict__ out) {
    if (threadIdx.x < 3) out[threadIdx.x] = __fmul_rn(__fadd_rn(box[threadIdx.x], box[3 + threadIdx.x]), 0.5f);
}

int pca_normals(const float* P, int n, const int* nb, int k, const float* view_dev, float* N, cudaStream_t s) {
    DWG_REQUIRE(P && nb && view_dev && N && n >= 1 && k >= 1, "pca_normals: bad arguments");
    k_pca_normals<<<div_up(n, 128), 128, 0, s>>>(P, n, nb, k, view_dev, N);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

int point_areas(const float* P, int n, const int* nb, int k, const float* N, float* A, cudaStream_t s) {
    DWG_REQUIRE(P && nb && N && A && n >= 1 && k >= 1 && k <= kAreaMaxK, "point_areas: bad arguments (k=%d)", k);
    k_point_areas<<<div_up(n, 64), 64, 0, s>>>(P, n, nb, k, N, A);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

int random_normals(float* N, int n, cudaStream_t s) {
    DWG_REQUIRE(N && n >= 0, "random_normals: bad arguments");
    if (n == 0) return DWG_OK;
    k_random_normals<<<div_up(n, 256), 256, 0, s>>>(N, n);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

int box_centre(const float* P, int n, float* box6_dev, float* view_dev, cudaStream_t s) {
    DWG_TRY(bbox_device(P, n, box6_dev, s));
    k_box_centre<<<1, 32, 0, s>>>(box6_dev, view_dev);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

}  // namespace dwg
