/*
 * dwg_oracle.c -- CPU restatement of the DWG reconstruction hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  See
 * dwg_oracle.h for the contract.  Build: oracle/Makefile (gcc, -ffp-contract=off
 * so that single-precision expressions round exactly like the CUDA code's
 * explicit __f*_rn intrinsics).
 */
#include "dwg_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PI_D 3.14159265358979323846

static void* xmalloc(size_t n) {
    void* p = malloc(n ? n : 1);
    if (!p) abort();
    return p;
}
static void* xcalloc(size_t n, size_t s) {
    void* p = calloc(n ? n : 1, s ? s : 1);
    if (!p) abort();
    return p;
}

/* ------------------------------------------------------------------------ */
/* octree: igl::octreeDWG, deps/libigl/include/igl/octree.cpp:171-335         */
/* ------------------------------------------------------------------------ */
struct dwgo_octree {
    int n_nodes, cap, max_depth, n_points;
    int* children;   /* cap*8 */
    double* centers; /* cap*3 */
    double* widths;
    int* depth;
    int** lists;
    int* lcount;
    long long* list_off; /* flattened after build */
    int* flat;
};

static void oct_grow(dwgo_octree* t, int need) {
    if (need <= t->cap) return;
    int nc = t->cap ? t->cap : 64;
    while (nc < need) nc *= 2;
    t->children = realloc(t->children, (size_t)nc * 8 * sizeof(int));
    t->centers = realloc(t->centers, (size_t)nc * 3 * sizeof(double));
    t->widths = realloc(t->widths, (size_t)nc * sizeof(double));
    t->depth = realloc(t->depth, (size_t)nc * sizeof(int));
    t->lists = realloc(t->lists, (size_t)nc * sizeof(int*));
    t->lcount = realloc(t->lcount, (size_t)nc * sizeof(int));
    if (!t->children || !t->centers || !t->widths || !t->depth || !t->lists || !t->lcount) abort();
    t->cap = nc;
}

/* octant numbering: bit0 x >= cx, bit1 y >= cy, bit2 z >= cz (octree.cpp:200-221) */
static int oct_octant(const double* p, const double* c) {
    int i = 0;
    if (p[0] >= c[0]) i += 1;
    if (p[1] >= c[1]) i += 2;
    if (p[2] >= c[2]) i += 4;
    return i;
}

/* child centre: parent +/- h per axis, x positive for odd, y for {2,3,6,7},
 * z for >3 (octree.cpp:224-249) */
static void oct_translate(const double* pc, double h, int ci, double* out) {
    out[0] = pc[0] + ((ci % 2) ? h : -h);
    out[1] = pc[1] + ((ci == 2 || ci == 3 || ci == 6 || ci == 7) ? h : -h);
    out[2] = pc[2] + ((ci > 3) ? h : -h);
}

static void oct_helper(dwgo_octree* t, const double* P, int index, int depth) {
    /* split rule: more than one point and depth below the cap (octree.cpp:264) */
    if (t->lcount[index] > 1 && depth < t->max_depth) {
        int m = t->n_nodes;
        oct_grow(t, m + 8);
        double h = t->widths[index] / 2.0;
        double cc[3] = {t->centers[index * 3], t->centers[index * 3 + 1], t->centers[index * 3 + 2]};
        for (int i = 0; i < 8; i++) {
            t->children[index * 8 + i] = m + i;
            for (int j = 0; j < 8; j++) t->children[(m + i) * 8 + j] = -1;
            oct_translate(cc, h / 2.0, i, &t->centers[(m + i) * 3]);
            t->widths[m + i] = h;
            t->depth[m + i] = depth + 1;
            t->lists[m + i] = NULL;
            t->lcount[m + i] = 0;
        }
        /* distribute in list order (stable) */
        int cnt[8] = {0};
        int* oc = xmalloc((size_t)t->lcount[index] * sizeof(int));
        for (int j = 0; j < t->lcount[index]; j++) {
            int pi = t->lists[index][j];
            oc[j] = oct_octant(&P[(size_t)pi * 3], cc);
            cnt[oc[j]]++;
        }
        for (int i = 0; i < 8; i++) t->lists[m + i] = xmalloc((size_t)(cnt[i] ? cnt[i] : 1) * sizeof(int));
        for (int j = 0; j < t->lcount[index]; j++) {
            int c = m + oc[j];
            t->lists[c][t->lcount[c]++] = t->lists[index][j];
        }
        free(oc);
        t->n_nodes = m + 8;
        for (int i = 0; i < 8; i++) oct_helper(t, P, m + i, depth + 1);
    }
}

dwgo_octree* dwgo_octree_build(const double* P, int n, int max_depth) {
    dwgo_octree* t = xcalloc(1, sizeof(dwgo_octree));
    t->max_depth = max_depth;
    t->n_points = n;
    oct_grow(t, 1);
    t->n_nodes = 1;
    for (int j = 0; j < 8; j++) t->children[j] = -1;
    t->lists[0] = xmalloc((size_t)(n ? n : 1) * sizeof(int));
    for (int i = 0; i < n; i++) t->lists[0][i] = i;
    t->lcount[0] = n;
    /* root: AABB centre, width = largest extent (octree.cpp:306-316) */
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) {
            double v = P[(size_t)i * 3 + d];
            if (v < mn[d]) mn[d] = v;
            if (v > mx[d]) mx[d] = v;
        }
    double w = 0;
    for (int d = 0; d < 3; d++) {
        t->centers[d] = (mn[d] + mx[d]) / 2.0;
        if (mx[d] - mn[d] > w) w = mx[d] - mn[d];
    }
    t->widths[0] = w;
    t->depth[0] = 0;
    oct_helper(t, P, 0, 0);
    /* flatten lists */
    t->list_off = xmalloc((size_t)(t->n_nodes + 1) * sizeof(long long));
    long long tot = 0;
    for (int i = 0; i < t->n_nodes; i++) {
        t->list_off[i] = tot;
        tot += t->lcount[i];
    }
    t->list_off[t->n_nodes] = tot;
    t->flat = xmalloc((size_t)(tot ? tot : 1) * sizeof(int));
    for (int i = 0; i < t->n_nodes; i++) {
        if (t->lcount[i]) memcpy(t->flat + t->list_off[i], t->lists[i], (size_t)t->lcount[i] * sizeof(int));
        free(t->lists[i]);
    }
    free(t->lists);
    t->lists = NULL;
    return t;
}

void dwgo_octree_free(dwgo_octree* t) {
    if (!t) return;
    free(t->children);
    free(t->centers);
    free(t->widths);
    free(t->depth);
    free(t->lcount);
    free(t->list_off);
    free(t->flat);
    free(t);
}

int dwgo_octree_num_nodes(const dwgo_octree* t) { return t->n_nodes; }

void dwgo_octree_export(const dwgo_octree* t, int* children, double* centers,
                        double* widths, int* counts, int* depth) {
    for (int i = 0; i < t->n_nodes; i++) {
        if (children) memcpy(children + (size_t)i * 8, t->children + (size_t)i * 8, 8 * sizeof(int));
        if (centers) memcpy(centers + (size_t)i * 3, t->centers + (size_t)i * 3, 3 * sizeof(double));
        if (widths) widths[i] = t->widths[i];
        if (counts) counts[i] = t->lcount[i];
        if (depth) depth[i] = t->depth[i];
    }
}

void dwgo_octree_lists(const dwgo_octree* t, long long* list_off, int* lists) {
    memcpy(list_off, t->list_off, (size_t)(t->n_nodes + 1) * sizeof(long long));
    memcpy(lists, t->flat, (size_t)t->list_off[t->n_nodes] * sizeof(int));
}

static void dfs_emit(const dwgo_octree* t, int node, int* perm, int* start, int* k) {
    if (start) start[node] = *k;
    if (t->lcount[node] == 0) return;
    if (t->children[(size_t)node * 8] == -1) {
        for (long long j = t->list_off[node]; j < t->list_off[node + 1]; j++) {
            if (perm) perm[*k] = t->flat[j];
            (*k)++;
        }
        return;
    }
    for (int c = 0; c < 8; c++) dfs_emit(t, t->children[(size_t)node * 8 + c], perm, start, k);
}

void dwgo_octree_dfs_order(const dwgo_octree* t, int* perm) {
    int k = 0;
    dfs_emit(t, 0, perm, NULL, &k);
}

void dwgo_octree_dfs_starts(const dwgo_octree* t, int* start) {
    int k = 0;
    dfs_emit(t, 0, NULL, start, &k);
}

/* ------------------------------------------------------------------------ */
/* moments: fast_winding_number.cpp:9-120, expansion order 0                 */
/* ------------------------------------------------------------------------ */
void dwgo_moments(const dwgo_octree* t, const float* P, const float* N,
                  const float* A, double* CM, double* R, double* EC) {
    for (int nd = 0; nd < t->n_nodes; nd++) {
        double at = 0, cm[3] = {0, 0, 0}, ec[3] = {0, 0, 0};
        for (long long j = t->list_off[nd]; j < t->list_off[nd + 1]; j++) {
            int i = t->flat[j];
            double a = A[i];
            at += a;
            for (int d = 0; d < 3; d++) {
                cm[d] += a * (double)P[(size_t)i * 3 + d];
                ec[d] += a * (double)N[(size_t)i * 3 + d];
            }
        }
        /* empty nodes are never visited by the traversal; 0/0 becomes 0 here */
        for (int d = 0; d < 3; d++) cm[d] = (at > 0) ? cm[d] / at : 0.0;
        double rmax = 0;
        for (long long j = t->list_off[nd]; j < t->list_off[nd + 1]; j++) {
            int i = t->flat[j];
            double dx = (double)P[(size_t)i * 3] - cm[0], dy = (double)P[(size_t)i * 3 + 1] - cm[1],
                   dz = (double)P[(size_t)i * 3 + 2] - cm[2];
            double r = sqrt(dx * dx + dy * dy + dz * dz);
            if (r > rmax) rmax = r;
        }
        if (CM)
            for (int d = 0; d < 3; d++) CM[(size_t)nd * 3 + d] = cm[d];
        if (EC)
            for (int d = 0; d < 3; d++) EC[(size_t)nd * 3 + d] = ec[d];
        if (R) R[nd] = rmax;
    }
}

/* ------------------------------------------------------------------------ */
/* GWN kernels: src/TurboLibiGWN.cu:328-511 (plain), :513-812 (screened)      */
/* ------------------------------------------------------------------------ */
/* screened term, evaluated in FP64.  rho = max(r, s); the value carries the
 * sign of d = A (p-q).n (the reference's sign-fix branches, :550-584). */
static inline int term_screened(double dx, double dy, double dz, double dot_an,
                                double s, double sigma, double* out) {
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (!(r > 1e-10)) return 0;
    double rho = (s > r) ? s : r;
    double up = (rho * sigma + 1.0) * dot_an;
    double down = exp(rho * sigma) * (4.0 * PI_D * rho * rho * rho) + 1e-7;
    double res = fabs(up / down);
    *out = (dot_an > 0.0) ? res : -res;
    return 1;
}

static inline double term_plain(double dx, double dy, double dz, double dot_an) {
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    return dot_an / (4.0 * PI_D * r * r * r + 1e-8);
}

/* Gradients with respect to the query q of the two terms above (the
 * reference has none; they are the analytic derivatives).  With
 * (dx,dy,dz) = p - q, ne the term's weighted normal (A n, or sum A n of a
 * node) and dot = ne.(p - q):
 *   screened  v = G(rho) dot, G = (sigma rho + 1) / (e^{sigma rho} 4 pi rho^3 + 1e-7),
 *             grad v = -G ne + dot G'(rho) grad rho, grad rho = -(p - q)/r when
 *             r > s and 0 when the screen radius s takes over;
 *   plain     v = dot / (4 pi r^3 + 1e-8),
 *             grad v = -ne / den + dot 12 pi r (p - q) / den^2.
 * Terms the value skips (r <= 1e-10 screened, r == 0 plain) add nothing. */
static inline void grad_screened(double dx, double dy, double dz, const double ne[3], double s, double sigma,
                                 double g[3]) {
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (!(r > 1e-10)) return;
    const double rho = (s > r) ? s : r;
    const double e = exp(rho * sigma);
    const double den = e * (4.0 * PI_D * rho * rho * rho) + 1e-7;
    const double up = rho * sigma + 1.0;
    const double G = up / den;
    const double dot = dx * ne[0] + dy * ne[1] + dz * ne[2];
    const double dden = e * (sigma * 4.0 * PI_D * rho * rho * rho + 12.0 * PI_D * rho * rho);
    const double Gp = (sigma * den - up * dden) / (den * den);
    const double k = (s > r) ? 0.0 : -dot * Gp / r; /* dot G' grad rho = k (p - q) */
    g[0] += -G * ne[0] + k * dx;
    g[1] += -G * ne[1] + k * dy;
    g[2] += -G * ne[2] + k * dz;
}

static inline void grad_plain(double dx, double dy, double dz, const double ne[3], double g[3]) {
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (r == 0.0) return;
    const double den = 4.0 * PI_D * r * r * r + 1e-8;
    const double dot = dx * ne[0] + dy * ne[1] + dz * ne[2];
    const double k = dot * 12.0 * PI_D * r / (den * den);
    g[0] += -ne[0] / den + k * dx;
    g[1] += -ne[1] / den + k * dy;
    g[2] += -ne[2] / den + k * dz;
}

/* higher-order far-field terms of igl::fast_winding_number's expansion_eval
 * (deps/libigl/include/igl/fast_winding_number.cpp:187-241), loc = CM - q:
 * order 1 adds sum_uv SecondDerivative(u,v) m1[u + 3v] with
 * SecondDerivative = loc loc^T (-3 / (4 pi r^5)) + I / (4 pi r^3); order 2 adds
 * sum_i sum_uv ThirdDerivative_i(u,v) m2[9i + u + 3v] with
 * ThirdDerivative_i = 15 loc_i loc loc^T / (4 pi r^7)
 *                     - 3 / (4 pi r^5) (loc_i I + e_i loc^T + loc e_i^T) */
static double expansion_terms(double lx, double ly, double lz, const double* h, int order) {
    const double loc[3] = {lx, ly, lz};
    const double r = sqrt(lx * lx + ly * ly + lz * lz);
    const double p3 = 4.0 * PI_D * r * r * r;
    const double p5 = p3 * r * r;
    const double d = 1.0 / p3;
    double w = 0;
    for (int v = 0; v < 3; v++)
        for (int u = 0; u < 3; u++) {
            double sd = loc[u] * loc[v] * (-3.0 / p5);
            if (u == v) sd += d;
            w += sd * h[u + 3 * v];
        }
    if (order >= 2) {
        const double p7 = p5 * r * r;
        for (int i = 0; i < 3; i++)
            for (int v = 0; v < 3; v++)
                for (int u = 0; u < 3; u++) {
                    double rcd = 0;
                    if (u == v) rcd += loc[i];
                    if (u == i) rcd += loc[v];
                    if (v == i) rcd += loc[u];
                    const double td = 15.0 * loc[i] * (loc[u] * (loc[v] / p7)) + (-3.0 / p5) * rcd;
                    w += td * h[9 + 9 * i + u + 3 * v];
                }
    }
    return w;
}

typedef struct {
    const dwgo_octree* t;
    const float *P, *N, *A, *radii;
    const double *CM, *EC;
    const double* HO; /* expansion coefficients, 36 per node (order >= 1) */
    int order;
    float* CMf; /* float copies used for the opening decision */
    float* Rf;
    const float* Q;
    long long nq;
    float beta, sigma, screen;
    int screened, use_radii;
    double* out;
    double* gout; /* nq x 3 gradients, or NULL */
    long long* terms;
    long long next;
    pthread_mutex_t mu;
} bh_ctx;

static inline void add_points(const bh_ctx* c, int node, double qx, double qy, double qz,
                              double* acc, double* g, long long* nt) {
    const dwgo_octree* t = c->t;
    for (long long j = t->list_off[node]; j < t->list_off[node + 1]; j++) {
        int i = t->flat[j];
        double dx = (double)c->P[(size_t)i * 3] - qx, dy = (double)c->P[(size_t)i * 3 + 1] - qy,
               dz = (double)c->P[(size_t)i * 3 + 2] - qz;
        double dot = (double)c->A[i] *
                     (dx * c->N[(size_t)i * 3] + dy * c->N[(size_t)i * 3 + 1] + dz * c->N[(size_t)i * 3 + 2]);
        double ne[3] = {0, 0, 0};
        if (g)
            for (int d = 0; d < 3; d++) ne[d] = (double)c->A[i] * (double)c->N[(size_t)i * 3 + d];
        if (c->screened) {
            double s = c->use_radii ? (double)c->radii[i] : (double)c->screen, v;
            if (term_screened(dx, dy, dz, dot, s, c->sigma, &v)) {
                *acc += v;
                (*nt)++;
                if (g) grad_screened(dx, dy, dz, ne, s, c->sigma, g);
            }
        } else {
            *acc += term_plain(dx, dy, dz, dot);
            (*nt)++;
            if (g) grad_plain(dx, dy, dz, ne, g);
        }
    }
}

/* opening decision in single precision, same operation order as the CUDA
 * kernel: dist = sqrt((dx*dx + dy*dy) + dz*dz) > beta * R (TurboLibiGWN.cu:632-644) */
static inline int is_far(const bh_ctx* c, int node, float qx, float qy, float qz) {
    float dx = c->CMf[(size_t)node * 3] - qx;
    float dy = c->CMf[(size_t)node * 3 + 1] - qy;
    float dz = c->CMf[(size_t)node * 3 + 2] - qz;
    float xx = dx * dx, yy = dy * dy, zz = dz * dz;
    float d2 = xx + yy;
    d2 = d2 + zz;
    float dist = sqrtf(d2);
    float lim = c->beta * c->Rf[node];
    return dist > lim;
}

static void bh_visit(const bh_ctx* c, int node, float qxf, float qyf, float qzf, double* acc, double* g,
                     long long* nt) {
    const dwgo_octree* t = c->t;
    double qx = qxf, qy = qyf, qz = qzf;
    if (t->children[(size_t)node * 8] == -1) {
        add_points(c, node, qx, qy, qz, acc, g, nt);
        return;
    }
    for (int k = 0; k < 8; k++) {
        int ch = t->children[(size_t)node * 8 + k];
        if (t->lcount[ch] <= 0) continue;
        if (is_far(c, ch, qxf, qyf, qzf)) {
            if (t->children[(size_t)ch * 8] == -1) {
                add_points(c, ch, qx, qy, qz, acc, g, nt);
            } else {
                double dx = c->CM[(size_t)ch * 3] - qx, dy = c->CM[(size_t)ch * 3 + 1] - qy,
                       dz = c->CM[(size_t)ch * 3 + 2] - qz;
                const double* ne = c->EC + (size_t)ch * 3;
                double dot = dx * ne[0] + dy * ne[1] + dz * ne[2];
                if (c->screened) {
                    double v;
                    if (term_screened(dx, dy, dz, dot, (double)c->screen, c->sigma, &v)) {
                        *acc += v;
                        (*nt)++;
                        if (g) grad_screened(dx, dy, dz, ne, (double)c->screen, c->sigma, g);
                    }
                } else {
                    *acc += term_plain(dx, dy, dz, dot) +
                            (c->order > 0 ? expansion_terms(dx, dy, dz, c->HO + (size_t)ch * 36, c->order) : 0.0);
                    (*nt)++;
                    if (g) grad_plain(dx, dy, dz, ne, g);
                }
            }
        } else {
            bh_visit(c, ch, qxf, qyf, qzf, acc, g, nt);
        }
    }
}

static void* bh_worker(void* arg) {
    bh_ctx* c = (bh_ctx*)arg;
    const long long chunk = 256;
    for (;;) {
        pthread_mutex_lock(&c->mu);
        long long s = c->next;
        c->next += chunk;
        pthread_mutex_unlock(&c->mu);
        if (s >= c->nq) break;
        long long e = s + chunk < c->nq ? s + chunk : c->nq;
        for (long long q = s; q < e; q++) {
            double acc = 0, g[3] = {0, 0, 0};
            long long nt = 0;
            if (c->t->lcount[0] > 0)
                bh_visit(c, 0, c->Q[q * 3], c->Q[q * 3 + 1], c->Q[q * 3 + 2], &acc, c->gout ? g : NULL, &nt);
            c->out[q] = acc;
            if (c->gout)
                for (int d = 0; d < 3; d++) c->gout[q * 3 + d] = g[d];
            if (c->terms) c->terms[q] = nt;
        }
    }
    return NULL;
}

static void run_threads(void* (*fn)(void*), void* ctx, int nthreads) {
    if (nthreads <= 1) {
        fn(ctx);
        return;
    }
    pthread_t* th = xmalloc((size_t)nthreads * sizeof(pthread_t));
    for (int i = 0; i < nthreads; i++) pthread_create(&th[i], NULL, fn, ctx);
    for (int i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
    free(th);
}

static void gwn_bh_impl(const dwgo_octree* t, const float* P, const float* N,
                        const float* A, const float* radii, const double* CM,
                        const double* R, const double* EC, const double* HO, int order,
                        const float* Q, long long nq, float beta, float sigma, int screened,
                        int use_radii, float screen, int nthreads, double* out, double* gout,
                        long long* terms) {
    bh_ctx c;
    memset(&c, 0, sizeof(c));
    c.gout = gout;
    c.HO = HO;
    c.order = order;
    c.t = t;
    c.P = P;
    c.N = N;
    c.A = A;
    c.radii = radii;
    c.CM = CM;
    c.EC = EC;
    c.CMf = xmalloc((size_t)t->n_nodes * 3 * sizeof(float));
    c.Rf = xmalloc((size_t)t->n_nodes * sizeof(float));
    for (long long i = 0; i < (long long)t->n_nodes * 3; i++) c.CMf[i] = (float)CM[i];
    for (int i = 0; i < t->n_nodes; i++) c.Rf[i] = (float)R[i];
    c.Q = Q;
    c.nq = nq;
    c.beta = beta;
    c.sigma = sigma;
    c.screen = screen;
    c.screened = screened;
    c.use_radii = use_radii;
    c.out = out;
    c.terms = terms;
    pthread_mutex_init(&c.mu, NULL);
    run_threads(bh_worker, &c, nthreads);
    pthread_mutex_destroy(&c.mu);
    free(c.CMf);
    free(c.Rf);
}

void dwgo_gwn_bh(const dwgo_octree* t, const float* P, const float* N,
                 const float* A, const float* radii, const double* CM,
                 const double* R, const double* EC, const float* Q, long long nq,
                 float beta, float sigma, int screened, int use_radii,
                 float screen, int nthreads, double* out, long long* terms) {
    gwn_bh_impl(t, P, N, A, radii, CM, R, EC, NULL, 0, Q, nq, beta, sigma, screened, use_radii, screen,
                nthreads, out, NULL, terms);
}

void dwgo_gwn_bh_grad(const dwgo_octree* t, const float* P, const float* N,
                      const float* A, const float* radii, const double* CM,
                      const double* R, const double* EC, const float* Q, long long nq,
                      float beta, float sigma, int screened, int use_radii,
                      float screen, int nthreads, double* out, double* grad_out) {
    gwn_bh_impl(t, P, N, A, radii, CM, R, EC, NULL, 0, Q, nq, beta, sigma, screened, use_radii, screen,
                nthreads, out, grad_out, NULL);
}

void dwgo_fwn(const dwgo_octree* t, const float* P, const float* N, const float* A,
              const double* CM, const double* R, const double* EC, const double* HO, int order,
              const float* Q, long long nq, float beta, int nthreads, double* out, long long* terms) {
    gwn_bh_impl(t, P, N, A, NULL, CM, R, EC, HO, order, Q, nq, beta, 0.f, 0, 0, 0.f, nthreads, out, NULL, terms);
}

void dwgo_expansion(const dwgo_octree* t, const float* P, const float* N, const float* A,
                    const double* CM, double* HO) {
    for (int nd = 0; nd < t->n_nodes; nd++) {
        double* h = HO + (size_t)nd * 36;
        memset(h, 0, sizeof(double) * 36);
        for (long long j = t->list_off[nd]; j < t->list_off[nd + 1]; j++) {
            const int i = t->flat[j];
            double a[3], an[3];
            for (int d = 0; d < 3; d++) {
                a[d] = (double)P[(size_t)i * 3 + d] - CM[(size_t)nd * 3 + d];
                an[d] = (double)A[i] * (double)N[(size_t)i * 3 + d];
            }
            /* TempCoeffs = A point^T N (col-major), then 0.5 point(k) TempCoeffs
             * (fast_winding_number.cpp:89-104) */
            for (int v = 0; v < 3; v++)
                for (int u = 0; u < 3; u++) {
                    const double tc = (double)A[i] * a[u] * (double)N[(size_t)i * 3 + v];
                    h[u + 3 * v] += tc;
                    for (int k = 0; k < 3; k++) h[9 + 9 * k + u + 3 * v] += 0.5 * a[k] * tc;
                }
            (void)an;
        }
    }
}

typedef struct {
    const float *P, *N, *A, *radii, *Q;
    int n;
    long long nq;
    float sigma, screen;
    int screened, use_radii;
    double* out;
    long long next;
    pthread_mutex_t mu;
} ex_ctx;

static void* ex_worker(void* arg) {
    ex_ctx* c = (ex_ctx*)arg;
    for (;;) {
        pthread_mutex_lock(&c->mu);
        long long s = c->next;
        c->next += 64;
        pthread_mutex_unlock(&c->mu);
        if (s >= c->nq) break;
        long long e = s + 64 < c->nq ? s + 64 : c->nq;
        for (long long q = s; q < e; q++) {
            double qx = c->Q[q * 3], qy = c->Q[q * 3 + 1], qz = c->Q[q * 3 + 2], acc = 0;
            for (int i = 0; i < c->n; i++) {
                double dx = (double)c->P[(size_t)i * 3] - qx, dy = (double)c->P[(size_t)i * 3 + 1] - qy,
                       dz = (double)c->P[(size_t)i * 3 + 2] - qz;
                double dot = (double)c->A[i] * (dx * c->N[(size_t)i * 3] + dy * c->N[(size_t)i * 3 + 1] +
                                                dz * c->N[(size_t)i * 3 + 2]);
                if (c->screened) {
                    double s = c->use_radii ? (double)c->radii[i] : (double)c->screen, v;
                    if (term_screened(dx, dy, dz, dot, s, c->sigma, &v)) acc += v;
                } else {
                    acc += term_plain(dx, dy, dz, dot);
                }
            }
            c->out[q] = acc;
        }
    }
    return NULL;
}

void dwgo_gwn_exact(const float* P, const float* N, const float* A,
                    const float* radii, int n, const float* Q, long long nq,
                    float sigma, int screened, int use_radii, float screen,
                    int nthreads, double* out) {
    ex_ctx c;
    memset(&c, 0, sizeof(c));
    c.P = P;
    c.N = N;
    c.A = A;
    c.radii = radii;
    c.Q = Q;
    c.n = n;
    c.nq = nq;
    c.sigma = sigma;
    c.screen = screen;
    c.screened = screened;
    c.use_radii = use_radii;
    c.out = out;
    pthread_mutex_init(&c.mu, NULL);
    run_threads(ex_worker, &c, nthreads);
    pthread_mutex_destroy(&c.mu);
}

/* ------------------------------------------------------------------------ */
/* voxel grid: deps/libigl/include/igl/voxel_grid.cpp:11-87, grid.cpp:11-45  */
/* Sample positions are closed-form: origin + index * spacing (single        */
/* precision), instead of the materialised Eigen matrix of the reference.    */
/* ------------------------------------------------------------------------ */
void dwgo_voxel_grid(const float* P, int n, float offset, int s, int res[3],
                     float origin[3], float* spacing) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) {
            float v = P[(size_t)i * 3 + d];
            if (v < mn[d]) mn[d] = v;
            if (v > mx[d]) mx[d] = v;
        }
    float diag[3];
    for (int d = 0; d < 3; d++) {
        mn[d] = mn[d] - offset;
        mx[d] = mx[d] + offset;
        diag[d] = mx[d] - mn[d];
    }
    int si = 0;
    for (int d = 1; d < 3; d++)
        if (diag[d] > diag[si]) si = d;
    float s_len = diag[si];
    float sf = (float)(s - 2);
    for (int d = 0; d < 3; d++) {
        if (d == si)
            res[d] = s - 2;
        else {
            float v = sf * diag[d];
            v = v / s_len;
            res[d] = (int)ceilf(v);
        }
        res[d] += 2;
    }
    float Aa[3];
    for (int d = 0; d < 3; d++) {
        float ps = 1.0f / ((float)res[d] - 1.0f);
        float den = 1.0f - 2.0f * ps;
        Aa[d] = diag[d] / den;
    }
    int ai = 0;
    for (int d = 1; d < 3; d++)
        if (Aa[d] > Aa[ai]) ai = d;
    float h = Aa[ai] / ((float)res[ai] - 1.0f);
    for (int d = 0; d < 3; d++) {
        float c = (mn[d] + mx[d]) / 2.0f;
        float half = 0.5f * ((float)res[d] - 1.0f);
        float ext = half * h;
        origin[d] = c - ext;
    }
    *spacing = h;
}

void dwgo_grid_points(const int res[3], const float origin[3], float spacing, float* out) {
    long long k = 0;
    for (int z = 0; z < res[2]; z++)
        for (int y = 0; y < res[1]; y++)
            for (int x = 0; x < res[0]; x++, k++) {
                float fx = (float)x * spacing, fy = (float)y * spacing, fz = (float)z * spacing;
                out[k * 3] = origin[0] + fx;
                out[k * 3 + 1] = origin[1] + fy;
                out[k * 3 + 2] = origin[2] + fz;
            }
}

/* ------------------------------------------------------------------------ */
/* marching cubes tables                                                     */
/* Corner c sits at (x + (b0 != b1), y + b1, z + !b2) (src/TurboMC.cu:408-413)*/
/* edge e joins (e & 7, e<4 ? (e+1)&3 : e<8 ? 4+((e-3)&3) : e-4) (:433-434). */
/* Edge masks follow from the corners.  The triangles of each case are the   */
/* reference's (src/TurboMC.cu:57-314), handed in by dwgo_mc_set_triangles   */
/* from the fixture tests/golden/mc_reference_loops.json (the front end does */
/* this when it loads the library).  dwgo_mc_polygons gives the polygons the */
/* cube geometry implies, fanned from their lowest edge, for the tests that  */
/* check the triangles against them: on every face, crossing edges pair up;  */
/* an ambiguous face cuts off the corners above the iso value; loops are     */
/* oriented so that, seen from outside the cube with the face corners        */
/* counter-clockwise, each face segment runs from the crossing entered from  */
/* a corner below the iso value.                                             */
/* ------------------------------------------------------------------------ */
static signed char mc_ref_tris[256 * 16];
static int mc_ref_tris_set = 0;

void dwgo_mc_set_triangles(const signed char* tri_table) {
    memcpy(mc_ref_tris, tri_table, sizeof(mc_ref_tris));
    mc_ref_tris_set = 1;
}
static const int MC_CORNER[8][3] = {{0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1},
                                    {0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}};
static int mc_edge_a(int e) { return e & 7; }
static int mc_edge_b(int e) { return e < 4 ? ((e + 1) & 3) : (e < 8 ? 4 + ((e - 3) & 3) : e - 4); }
static int mc_edge_of(int a, int b) {
    for (int e = 0; e < 12; e++)
        if ((mc_edge_a(e) == a && mc_edge_b(e) == b) || (mc_edge_a(e) == b && mc_edge_b(e) == a)) return e;
    return -1;
}

void dwgo_mc_polygons(int* edge_table, signed char* tri_table) {
    /* faces: the 4 corners of each face in counter-clockwise order seen from
     * outside */
    int faces[6][4];
    int nf = 0;
    for (int axis = 0; axis < 3; axis++)
        for (int val = 0; val < 2; val++) {
            int cs[4], k = 0;
            for (int c = 0; c < 8; c++)
                if (MC_CORNER[c][axis] == val) cs[k++] = c;
            int o[4] = {cs[0], -1, -1, -1};
            for (int i = 1; i < 4; i++)
                for (int j = 0; j < 4; j++) {
                    int c = cs[j], used = 0, dist = 0;
                    for (int u = 0; u < i; u++)
                        if (o[u] == c) used = 1;
                    for (int d = 0; d < 3; d++) dist += abs(MC_CORNER[c][d] - MC_CORNER[o[i - 1]][d]);
                    if (!used && dist == 1) {
                        o[i] = c;
                        break;
                    }
                }
            /* orientation: (v0 x v1) . outward normal > 0 */
            double cen[3] = {0, 0, 0};
            for (int i = 0; i < 4; i++)
                for (int d = 0; d < 3; d++) cen[d] += MC_CORNER[o[i]][d] / 4.0;
            double v0[3], v1[3], cr[3];
            for (int d = 0; d < 3; d++) {
                v0[d] = MC_CORNER[o[0]][d] - cen[d];
                v1[d] = MC_CORNER[o[1]][d] - cen[d];
            }
            cr[0] = v0[1] * v1[2] - v0[2] * v1[1];
            cr[1] = v0[2] * v1[0] - v0[0] * v1[2];
            cr[2] = v0[0] * v1[1] - v0[1] * v1[0];
            double outn = val ? 1.0 : -1.0;
            if (cr[axis] * outn < 0) {
                int tmp = o[1];
                o[1] = o[3];
                o[3] = tmp;
            }
            for (int i = 0; i < 4; i++) faces[nf][i] = o[i];
            nf++;
        }
    for (int ci = 0; ci < 256; ci++) {
        int inside[8];
        for (int c = 0; c < 8; c++) inside[c] = (ci >> c) & 1;
        int et = 0;
        for (int e = 0; e < 12; e++)
            if (inside[mc_edge_a(e)] != inside[mc_edge_b(e)]) et |= 1 << e;
        if (edge_table) edge_table[ci] = et;
        int nxt[12];
        for (int e = 0; e < 12; e++) nxt[e] = -1;
        for (int f = 0; f < 6; f++) {
            int ce[4], cin[4], n = 0;
            for (int k = 0; k < 4; k++) {
                int a = faces[f][k], b = faces[f][(k + 1) & 3];
                if (inside[a] != inside[b]) {
                    ce[n] = mc_edge_of(a, b);
                    cin[n] = inside[a];
                    n++;
                }
            }
            int pa[2][2], np = 0;
            if (n == 2) {
                pa[0][0] = 0;
                pa[0][1] = 1;
                np = 1;
            } else if (n == 4) {
                if (inside[faces[f][0]]) { /* cut off the two corners above iso */
                    pa[0][0] = 3; pa[0][1] = 0;
                    pa[1][0] = 1; pa[1][1] = 2;
                } else {
                    pa[0][0] = 0; pa[0][1] = 1;
                    pa[1][0] = 2; pa[1][1] = 3;
                }
                np = 2;
            }
            for (int s = 0; s < np; s++) {
                int x = pa[s][0], y = pa[s][1];
                if (cin[x] == 0)
                    nxt[ce[x]] = ce[y];
                else
                    nxt[ce[y]] = ce[x];
            }
        }
        signed char* row = tri_table ? tri_table + ci * 16 : NULL;
        int w = 0;
        int seen[12] = {0};
        for (int e = 0; e < 12; e++) {
            if (nxt[e] < 0 || seen[e]) continue;
            int loop[12], ln = 0, c = e;
            do {
                loop[ln++] = c;
                seen[c] = 1;
                c = nxt[c];
            } while (c != e && ln < 12);
            /* e is the lowest edge of the loop (edges scanned in order) */
            for (int k = 1; k + 1 < ln; k++) {
                if (row) {
                    row[w] = (signed char)loop[0];
                    row[w + 1] = (signed char)loop[k];
                    row[w + 2] = (signed char)loop[k + 1];
                }
                w += 3;
            }
        }
        if (row)
            for (; w < 16; w++) row[w] = -1;
    }
}

void dwgo_mc_tables(int* edge_table, signed char* tri_table) {
    if (!mc_ref_tris_set) {
        fprintf(stderr, "dwg oracle: marching-cubes triangles not set (dwgo_mc_set_triangles)\n");
        abort();
    }
    dwgo_mc_polygons(edge_table, NULL);
    if (tri_table) memcpy(tri_table, mc_ref_tris, sizeof(mc_ref_tris));
}

long long dwgo_marching_cubes(const float* field, const int res[3],
                              const float origin[3], float spacing, float iso,
                              float* tris, float* centroids, float* normals,
                              long long cap, unsigned char* cases) {
    static int et[256];
    static signed char tt[256 * 16];
    static int init = 0;
    if (!init) {
        dwgo_mc_tables(et, tt);
        init = 1;
    }
    long long nx = res[0], ny = res[1], nz = res[2], T = 0;
    for (long long z = 0; z + 1 < nz; z++)
        for (long long y = 0; y + 1 < ny; y++)
            for (long long x = 0; x + 1 < nx; x++) {
                float v[8], p[8][3];
                int ci = 0;
                for (int c = 0; c < 8; c++) {
                    long long gx = x + MC_CORNER[c][0], gy = y + MC_CORNER[c][1], gz = z + MC_CORNER[c][2];
                    v[c] = field[gx + nx * (gy + ny * gz)];
                    float fx = (float)gx * spacing, fy = (float)gy * spacing, fz = (float)gz * spacing;
                    p[c][0] = origin[0] + fx;
                    p[c][1] = origin[1] + fy;
                    p[c][2] = origin[2] + fz;
                    if (v[c] > iso) ci |= 1 << c;
                }
                if (cases) cases[x + (nx - 1) * (y + (ny - 1) * z)] = (unsigned char)ci;
                if (!et[ci]) continue;
                float vl[12][3];
                for (int e = 0; e < 12; e++) {
                    if (!(et[ci] & (1 << e))) continue;
                    int a = mc_edge_a(e), b = mc_edge_b(e);
                    /* vertex_interp, src/TurboMC.cu:373-381 */
                    float num = v[a] - iso;
                    float dv = v[b] - v[a];
                    float den = (float)((double)dv + 1e-10);
                    float ell = num / den;
                    for (int d = 0; d < 3; d++) {
                        float dp = p[b][d] - p[a][d];
                        float m = ell * dp;
                        vl[e][d] = p[a][d] - m;
                    }
                }
                for (int k = 0; k < 16 && tt[ci * 16 + k] >= 0; k += 3, T++) {
                    if (T >= cap) continue;
                    const float* P0 = vl[(int)tt[ci * 16 + k]];
                    const float* P1 = vl[(int)tt[ci * 16 + k + 1]];
                    const float* P2 = vl[(int)tt[ci * 16 + k + 2]];
                    if (tris)
                        for (int d = 0; d < 3; d++) {
                            tris[T * 9 + d] = P0[d];
                            tris[T * 9 + 3 + d] = P1[d];
                            tris[T * 9 + 6 + d] = P2[d];
                        }
                    if (centroids)
                        for (int d = 0; d < 3; d++) {
                            float s = P0[d] + P1[d];
                            s = s + P2[d];
                            centroids[T * 3 + d] = s / 3.0f;
                        }
                    if (normals) {
                        float u[3], w[3];
                        for (int d = 0; d < 3; d++) {
                            u[d] = P1[d] - P0[d];
                            w[d] = P2[d] - P0[d];
                        }
                        float a0 = u[1] * w[2], b0 = u[2] * w[1];
                        float a1 = u[2] * w[0], b1 = u[0] * w[2];
                        float a2 = u[0] * w[1], b2 = u[1] * w[0];
                        float cx = a0 - b0, cy = a1 - b1, cz = a2 - b2;
                        float xx = cx * cx, yy = cy * cy, zz = cz * cz;
                        float l2 = xx + yy;
                        l2 = l2 + zz;
                        float len = sqrtf(l2);
                        float den = (float)((double)len + 1e-8);
                        float sc = -(1.0f / den);
                        normals[T * 3] = cx * sc;
                        normals[T * 3 + 1] = cy * sc;
                        normals[T * 3 + 2] = cz * sc;
                    }
                }
            }
    return T;
}

/* ------------------------------------------------------------------------ */
/* kNN: brute force with the cukd candidate key (dist2 bits << 32 | id),     */
/* include/cudaKDTree/cukd/knn.h:279-282,404-414                            */
/* ------------------------------------------------------------------------ */
static inline uint64_t knn_key(float d2, int id) {
    uint32_t b;
    memcpy(&b, &d2, 4);
    return ((uint64_t)b << 32) | (uint32_t)id;
}
static inline float sqdist_f(const float* a, const float* b) {
    float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    float xx = dx * dx, yy = dy * dy, zz = dz * dz;
    float d2 = xx + yy;
    d2 = d2 + zz;
    return d2;
}

typedef struct {
    const float *P, *Q;
    int n, k;
    long long nq;
    int* out;
    long long next;
    pthread_mutex_t mu;
} knn_ctx;

static void* knn_worker(void* arg) {
    knn_ctx* c = (knn_ctx*)arg;
    uint64_t* best = xmalloc((size_t)c->k * sizeof(uint64_t));
    for (;;) {
        pthread_mutex_lock(&c->mu);
        long long s = c->next;
        c->next += 64;
        pthread_mutex_unlock(&c->mu);
        if (s >= c->nq) break;
        long long e = s + 64 < c->nq ? s + 64 : c->nq;
        for (long long q = s; q < e; q++) {
            for (int j = 0; j < c->k; j++) best[j] = UINT64_MAX;
            for (int i = 0; i < c->n; i++) {
                uint64_t key = knn_key(sqdist_f(&c->P[(size_t)i * 3], &c->Q[q * 3]), i);
                if (key >= best[c->k - 1]) continue;
                int j = c->k - 1;
                while (j > 0 && best[j - 1] > key) {
                    best[j] = best[j - 1];
                    j--;
                }
                best[j] = key;
            }
            for (int j = 0; j < c->k; j++)
                c->out[q * c->k + j] = best[j] == UINT64_MAX ? -1 : (int)(uint32_t)best[j];
        }
    }
    free(best);
    return NULL;
}

void dwgo_knn(const float* P, int n, const float* Q, long long nq, int k,
              int nthreads, int* out) {
    knn_ctx c;
    memset(&c, 0, sizeof(c));
    c.P = P;
    c.Q = Q;
    c.n = n;
    c.k = k;
    c.nq = nq;
    c.out = out;
    pthread_mutex_init(&c.mu, NULL);
    run_threads(knn_worker, &c, nthreads);
    pthread_mutex_destroy(&c.mu);
}

/* ------------------------------------------------------------------------ */
/* normals                                                                    */
/* ------------------------------------------------------------------------ */
#define FIX_SCALE 1099511627776.0 /* 2^40 */

/* UpdateNormals + NormalizeNormals (src/TurboDWG.cu:179-204,238-266).  The
 * scatter is accumulated in 2^-40 fixed point (int64), which makes it
 * independent of summation order; the reference adds FP32 atomics in an
 * unspecified order. */
int dwgo_diffuse_normals(const int* knn, const float* tri_normals,
                         long long T, int k, int L, float* normals,
                         unsigned char* is_zero) {
    int64_t* acc = xcalloc((size_t)L * 3, sizeof(int64_t));
    for (long long t = 0; t < T; t++) {
        int64_t f[3];
        for (int d = 0; d < 3; d++) f[d] = llrint((double)tri_normals[t * 3 + d] * FIX_SCALE);
        for (int j = 0; j < k; j++) {
            int i = knn[t * k + j];
            if (i < 0 || i >= L) continue;
            for (int d = 0; d < 3; d++) acc[(size_t)i * 3 + d] += f[d];
        }
    }
    int zc = 0;
    for (int i = 0; i < L; i++) {
        float tv[3];
        for (int d = 0; d < 3; d++) tv[d] = (float)((double)acc[(size_t)i * 3 + d] * (1.0 / FIX_SCALE));
        float xx = tv[0] * tv[0], yy = tv[1] * tv[1], zz = tv[2] * tv[2];
        float l2 = xx + yy;
        l2 = l2 + zz;
        float len = sqrtf(l2);
        if ((double)len < 1e-10) {
            zc++;
            if (is_zero) is_zero[i] = 1;
        } else {
            if (is_zero) is_zero[i] = 0;
            float sc = 1.0f / (float)((double)len + 1e-8);
            for (int d = 0; d < 3; d++) normals[(size_t)i * 3 + d] = tv[d] * sc;
        }
    }
    free(acc);
    return zc;
}

/* LoadZeroData + kNN on the non-zero subset + SimpleUpdateNonzeroNormals
 * (src/TurboDWG.cu:145-177,322-359,585-644); subsets keep index order. */
void dwgo_zero_repair(const float* Lpos, int L, float* normals,
                      const unsigned char* is_zero, int k, int nthreads) {
    int nz = 0, nn = 0;
    for (int i = 0; i < L; i++) {
        if (is_zero[i]) nz++;
        else nn++;
    }
    if (nz == 0 || nn == 0) return;
    int kk = k < nn ? k : nn;
    float* zp = xmalloc((size_t)nz * 3 * sizeof(float));
    float* np = xmalloc((size_t)nn * 3 * sizeof(float));
    float* nnrm = xmalloc((size_t)nn * 3 * sizeof(float));
    int* zi = xmalloc((size_t)nz * sizeof(int));
    int a = 0, b = 0;
    for (int i = 0; i < L; i++) {
        if (is_zero[i]) {
            memcpy(&zp[(size_t)a * 3], &Lpos[(size_t)i * 3], 12);
            zi[a++] = i;
        } else {
            memcpy(&np[(size_t)b * 3], &Lpos[(size_t)i * 3], 12);
            memcpy(&nnrm[(size_t)b * 3], &normals[(size_t)i * 3], 12);
            b++;
        }
    }
    int* nb = xmalloc((size_t)nz * kk * sizeof(int));
    dwgo_knn(np, nn, zp, nz, kk, nthreads, nb);
    for (int z = 0; z < nz; z++) {
        float s[3] = {0, 0, 0};
        for (int j = 0; j < kk; j++) {
            int c = nb[(size_t)z * kk + j];
            for (int d = 0; d < 3; d++) s[d] = s[d] + nnrm[(size_t)c * 3 + d];
        }
        float xx = s[0] * s[0], yy = s[1] * s[1], zz = s[2] * s[2];
        float l2 = xx + yy;
        l2 = l2 + zz;
        float sc = 1.0f / (float)((double)sqrtf(l2) + 1e-8);
        for (int d = 0; d < 3; d++) normals[(size_t)zi[z] * 3 + d] = s[d] * sc;
    }
    free(zp);
    free(np);
    free(nnrm);
    free(zi);
    free(nb);
}

/* GaussMapInitNormals (src/TurboNormalInit.cu:3-44): centre = middle of the
 * points' bounding box. */
void dwgo_gauss_map(const float* P, int n, float* normals) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) {
            float v = P[(size_t)i * 3 + d];
            if (v < mn[d]) mn[d] = v;
            if (v > mx[d]) mx[d] = v;
        }
    float c[3];
    for (int d = 0; d < 3; d++) {
        float s = mn[d] + mx[d];
        c[d] = s / 2.0f;
    }
    for (int i = 0; i < n; i++) {
        float v[3];
        for (int d = 0; d < 3; d++) v[d] = P[(size_t)i * 3 + d] - c[d];
        float xx = v[0] * v[0], yy = v[1] * v[1], zz = v[2] * v[2];
        float l2 = xx + yy;
        l2 = l2 + zz;
        float sc = 1.0f / (float)((double)sqrtf(l2) + 1e-8);
        for (int d = 0; d < 3; d++) normals[(size_t)i * 3 + d] = v[d] * sc;
    }
}

/* LoadNormals (src/TurboDWG.cu:206-236) */
void dwgo_load_normals(const int* knn, int k, long long nq,
                       const float* leaf_normals, float* out) {
    for (long long q = 0; q < nq; q++) {
        float s[3] = {0, 0, 0};
        for (int j = 0; j < k; j++) {
            int c = knn[q * k + j];
            for (int d = 0; d < 3; d++) s[d] = s[d] + leaf_normals[(size_t)c * 3 + d];
        }
        for (int d = 0; d < 3; d++) s[d] = s[d] / (float)k;
        float xx = s[0] * s[0], yy = s[1] * s[1], zz = s[2] * s[2];
        float l2 = xx + yy;
        l2 = l2 + zz;
        float sc = 1.0f / (float)((double)sqrtf(l2) + 1e-8);
        for (int d = 0; d < 3; d++) out[q * 3 + d] = s[d] * sc;
    }
}

/* SimpleUpdateRadii (src/TurboDWG.cu:361-391) with the per-neighbour offset
 * initialised (the reference leaves it uninitialised at :375-379):
 * r = clamp(sqrt(mean_j |p_i - p_j|^2), 0.0015, 0.015), self included. */
void dwgo_radii(const float* P, int n, const int* knn, int k, float* radii) {
    for (int i = 0; i < n; i++) {
        float acc = 0.0f;
        for (int j = 0; j < k; j++) {
            int c = knn[(size_t)i * k + j];
            acc = acc + sqdist_f(&P[(size_t)i * 3], &P[(size_t)c * 3]);
        }
        acc = acc / (float)k;
        float r = sqrtf(acc);
        r = (r < 0.0015f) ? 0.0015f : r;
        r = (r > 0.015f) ? 0.015f : r;
        radii[i] = r;
    }
}

/* ---- --com_As 1: PCA normals, point areas, seeded random leaf normals ---- */

/* eigen decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations
 * (each rotation zeroes its pivot exactly); w ascending, V[:, i] the unit
 * eigenvector of w[i].  Only +, -, *, / and sqrt, each rounded once, in a
 * fixed order: the GPU evaluates the same sequence and gets the same bits. */
static void jacobi3(const double A_in[3][3], double w[3], double V[3][3]) {
    double a[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            a[i][j] = A_in[i][j];
            V[i][j] = i == j ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 32; sweep++) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        const double dg = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off <= 1e-36 * dg) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                if (a[p][q] == 0.0) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; k++) { /* columns p, q */
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; k++) { /* rows p, q */
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                a[p][q] = 0.0;
                a[q][p] = 0.0;
                for (int k = 0; k < 3; k++) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    /* ascending eigenvalues, ties in index order */
    int ord[3] = {0, 1, 2};
    for (int i = 0; i < 3; i++)
        for (int j = i + 1; j < 3; j++)
            if (a[ord[j]][ord[j]] < a[ord[i]][ord[i]]) {
                const int t = ord[i];
                ord[i] = ord[j];
                ord[j] = t;
            }
    double Vs[3][3];
    for (int i = 0; i < 3; i++) {
        w[i] = a[ord[i]][ord[i]];
        for (int k = 0; k < 3; k++) Vs[k][i] = V[k][ord[i]];
    }
    memcpy(V, Vs, sizeof(Vs));
}

/* mean c and covariance C (divided by m) of the points ids[0..m) */
static void covariance(const float* P, const int* ids, int m, double c[3], double C[3][3]) {
    c[0] = c[1] = c[2] = 0;
    for (int j = 0; j < m; j++)
        for (int d = 0; d < 3; d++) c[d] += (double)P[(size_t)ids[j] * 3 + d];
    for (int d = 0; d < 3; d++) c[d] /= m;
    memset(C, 0, sizeof(double) * 9);
    for (int j = 0; j < m; j++) {
        double e[3];
        for (int d = 0; d < 3; d++) e[d] = (double)P[(size_t)ids[j] * 3 + d] - c[d];
        for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++) C[r][q] += e[r] * e[q];
    }
    for (int r = 0; r < 3; r++)
        for (int q = 0; q < 3; q++) C[r][q] /= m;
}

void dwgo_pca_normals(const float* P, int n, const int* knn, int k, const float view[3], float* normals) {
    int* ids = xmalloc((size_t)k * sizeof(int));
    for (int i = 0; i < n; i++) {
        int m = 0;
        for (int j = 0; j < k; j++)
            if (knn[(size_t)i * k + j] >= 0) ids[m++] = knn[(size_t)i * k + j];
        double nv[3] = {0, 0, 1};
        if (m >= 3) {
            double c[3], C[3][3], w[3], V[3][3];
            covariance(P, ids, m, c, C);
            jacobi3(C, w, V);
            for (int d = 0; d < 3; d++) nv[d] = V[d][0];
        }
        /* flipNormalTowardsViewpoint: (view - p) . n >= 0 */
        double dp = 0;
        for (int d = 0; d < 3; d++) dp += ((double)view[d] - (double)P[(size_t)i * 3 + d]) * nv[d];
        const double sg = dp < 0 ? -1.0 : 1.0;
        for (int d = 0; d < 3; d++) normals[(size_t)i * 3 + d] = (float)(sg * nv[d]);
    }
    free(ids);
}

/* exact orientation of integer points (|coordinates| < 2^24): > 0 counter-clockwise */
static long long orient_q(long long ax, long long ay, long long bx, long long by, long long cx, long long cy) {
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}

/* exact in-circle determinant sign of d against the circle through a, b, c
 * (> 0: d inside when a, b, c are counter-clockwise), 128-bit integers */
static int incircle_q(long long ax, long long ay, long long bx, long long by, long long cx, long long cy,
                      long long dx, long long dy) {
    const __int128 adx = ax - dx, ady = ay - dy, bdx = bx - dx, bdy = by - dy, cdx = cx - dx, cdy = cy - dy;
    const __int128 det = (adx * adx + ady * ady) * (bdx * cdy - cdx * bdy) -
                         (bdx * bdx + bdy * bdy) * (adx * cdy - cdx * ady) +
                         (cdx * cdx + cdy * cdy) * (adx * bdy - bdx * ady);
    return det > 0 ? 1 : (det < 0 ? -1 : 0);
}

void dwgo_point_areas(const float* P, int n, const int* knn, int k, const float* normals, float* areas) {
    int* ids = xmalloc((size_t)k * sizeof(int));
    double* u = xmalloc((size_t)k * sizeof(double));
    double* v = xmalloc((size_t)k * sizeof(double));
    long long* qx = xmalloc((size_t)k * sizeof(long long));
    long long* qy = xmalloc((size_t)k * sizeof(long long));
    int* keep = xmalloc((size_t)k * sizeof(int));
    for (int i = 0; i < n; i++) {
        const int q0 = knn[(size_t)i * k];
        areas[i] = 0.f;
        if (q0 < 0) continue;
        /* neighbours whose normal agrees with the first one's (point_areas.cpp:97-106) */
        int m = 0;
        for (int j = 0; j < k; j++) {
            const int q = knn[(size_t)i * k + j];
            if (q < 0) continue;
            double d = 0;
            for (int t = 0; t < 3; t++) d += (double)normals[(size_t)q0 * 3 + t] * (double)normals[(size_t)q * 3 + t];
            if (d > 0) ids[m++] = q;
        }
        if (m <= 2) continue;
        /* PCA plane (point_areas.cpp:114-133): scores on the two largest
         * principal directions */
        double c[3], C[3][3], w[3], V[3][3];
        covariance(P, ids, m, c, C);
        jacobi3(C, w, V);
        double mx = 0;
        for (int j = 0; j < m; j++) {
            double e[3];
            for (int d = 0; d < 3; d++) e[d] = (double)P[(size_t)ids[j] * 3 + d] - c[d];
            u[j] = e[0] * V[0][2] + e[1] * V[1][2] + e[2] * V[2][2];
            v[j] = e[0] * V[0][1] + e[1] * V[1][1] + e[2] * V[2][1];
            if (fabs(u[j]) > mx) mx = fabs(u[j]);
            if (fabs(v[j]) > mx) mx = fabs(v[j]);
        }
        if (!(mx > 0) || !isfinite(mx)) continue;
        /* the 2-D Delaunay triangulation decided exactly on coordinates
         * rounded to a grid of 2^-24 of the extent; coincident points after
         * rounding are one vertex (the first) */
        const double scale = ldexp(1.0, 23 - ilogb(mx));
        int mk = 0;
        for (int j = 0; j < m; j++) {
            const long long x = llrint(u[j] * scale), y = llrint(v[j] * scale);
            int dup = 0;
            for (int t = 0; t < mk && !dup; t++) dup = qx[t] == x && qy[t] == y;
            if (dup) continue;
            qx[mk] = x;
            qy[mk] = y;
            keep[mk++] = j;
        }
        double acc = 0;
        for (int b = 1; b < mk; b++)
            for (int cc = b + 1; cc < mk; cc++) {
                const long long orient = orient_q(qx[0], qy[0], qx[b], qy[b], qx[cc], qy[cc]);
                if (orient == 0) continue; /* collinear: no face */
                /* Delaunay: no point strictly inside the circumcircle; points
                 * on it form a cocircular polygon, triangulated as the fan
                 * from the point itself (its neighbours on the polygon are
                 * adjacent: no cocircular point beyond the chord b-c) */
                int ok = 1;
                for (int t = 1; t < mk && ok; t++) {
                    if (t == b || t == cc) continue;
                    int sg = incircle_q(qx[0], qy[0], qx[b], qy[b], qx[cc], qy[cc], qx[t], qy[t]);
                    if (orient < 0) sg = -sg;
                    if (sg > 0) ok = 0;
                    if (sg == 0) {
                        const long long side = orient_q(qx[b], qy[b], qx[cc], qy[cc], qx[t], qy[t]);
                        if ((side > 0) != (orient > 0) && side != 0) ok = 0;
                    }
                }
                if (!ok) continue;
                /* triangle XYZ with X the point itself (point_areas.cpp:160-193) */
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
                if (cosX < 0)
                    acc += 0.5 * full;
                else if (cosY < 0 || cosZ < 0)
                    acc += 0.25 * full;
                else
                    acc += (b1 * full + b2 * full) / 2;
            }
        areas[i] = isfinite(acc) ? (float)acc : 0.f;
    }
    free(ids);
    free(u);
    free(v);
    free(qx);
    free(qy);
    free(keep);
}

/* splitmix64 (S. Vigna) of an index: integer mixing, identical on the GPU */
static uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

void dwgo_random_normals(int n, float* normals) {
    for (int i = 0; i < n; i++) {
        const double u = (double)(mix64((uint64_t)i * 2) >> 11) * (1.0 / 9007199254740992.0) * 6.283185307179586;
        const double v = (double)(mix64((uint64_t)i * 2 + 1) >> 11) * (1.0 / 9007199254740992.0) * 6.283185307179586;
        normals[(size_t)i * 3] = (float)(sin(u) * cos(v));
        normals[(size_t)i * 3 + 1] = (float)(sin(u) * sin(v));
        normals[(size_t)i * 3 + 2] = (float)cos(u);
    }
}

/* ------------------------------------------------------------------------ */
/* full reconstruction                                                        */
/* ------------------------------------------------------------------------ */
struct dwgo_run {
    int L, N, iters;
    long long T;
    int fres[3], ires[3];
    float* leaf_pos;
    float* leaf_nrm;
    float* point_nrm;
    float* tris;
    float* iso;
    long long* tri_count;
    int* zero_count;
    float* final_field;
    float final_iso;
};

static float sigma_schedule(int t, float lambda) {
    /* src/TurboDWG.cu:526-533 */
    float s = lambda;
    if (t < 4) s = 20.0f;
    if (t > 0 && t % 7 == 0) s = 10.0f;
    return s;
}

static double* to_double(const float* a, long long n) {
    double* d = xmalloc((size_t)n * sizeof(double));
    for (long long i = 0; i < n; i++) d[i] = a[i];
    return d;
}

/* one GWN evaluation at points and at a grid + the mean of the point field */
static void field_pass(const dwgo_octree* tr, const float* pos, int n, const float* nrm,
                       const float* A, const float* radii, const double* CM, const double* R,
                       const dwgo_params* prm, float sigma, const int res[3], const float org[3],
                       float h, int nthreads, float* grid_field, double* mean_out) {
    double* EC = xmalloc((size_t)tr->n_nodes * 3 * sizeof(double));
    dwgo_moments(tr, pos, nrm, A, NULL, NULL, EC);
    double* wp = xmalloc((size_t)n * sizeof(double));
    dwgo_gwn_bh(tr, pos, nrm, A, radii, CM, R, EC, pos, n, prm->beta, sigma, 1, prm->use_radii,
                prm->screen, nthreads, wp, NULL);
    double sum = 0;
    for (int i = 0; i < n; i++) sum += wp[i];
    *mean_out = sum / (double)n;
    long long ng = (long long)res[0] * res[1] * res[2];
    float* gp = xmalloc((size_t)ng * 3 * sizeof(float));
    dwgo_grid_points(res, org, h, gp);
    double* wg = xmalloc((size_t)ng * sizeof(double));
    dwgo_gwn_bh(tr, pos, nrm, A, radii, CM, R, EC, gp, ng, prm->beta, sigma, 1, prm->use_radii,
                prm->screen, nthreads, wg, NULL);
    for (long long i = 0; i < ng; i++) grid_field[i] = (float)wg[i];
    free(EC);
    free(wp);
    free(gp);
    free(wg);
}

static const float* g_filter_keys;
static int cmp_desc_stable(const void* x, const void* y) {
    const int a = *(const int*)x, b = *(const int*)y;
    if (g_filter_keys[a] > g_filter_keys[b]) return -1;
    if (g_filter_keys[a] < g_filter_keys[b]) return 1;
    return a < b ? -1 : (a > b);
}

void dwgo_outlier_filter(float* A, int n, float thr) {
    if (!(thr > 0.f) || n <= 0) return;
    int k = (int)ceilf((float)n * thr);
    if (k > n) k = n;
    if (k <= 0) return;
    int* idx = xmalloc((size_t)n * sizeof(int));
    for (int i = 0; i < n; i++) idx[i] = i;
    g_filter_keys = A;
    qsort(idx, (size_t)n, sizeof(int), cmp_desc_stable);
    for (int i = 0; i < k; i++) A[idx[i]] /= 1000.0f;
    free(idx);
}

dwgo_run* dwgo_reconstruct(const float* P, int n, const float* N_in,
                           const dwgo_params* prm, int nthreads) {
    dwgo_run* run = xcalloc(1, sizeof(dwgo_run));
    run->N = n;
    /* octree on the points (include/DWGProcess.h:227) */
    double* Pd = to_double(P, (long long)n * 3);
    dwgo_octree* t1 = dwgo_octree_build(Pd, n, prm->max_depth);
    /* leaves: BFS order, cell centres of leaves with > min_num points
     * (GetOctreeLeaves, include/DWGProcess.h:383-428) */
    int M1 = t1->n_nodes;
    int* queue = xmalloc((size_t)M1 * sizeof(int));
    int* lnode = xmalloc((size_t)M1 * sizeof(int));
    int qh = 0, qt = 0, L = 0;
    queue[qt++] = 0;
    while (qh < qt) {
        int idx = queue[qh++];
        if (t1->children[(size_t)idx * 8] == -1) {
            if (t1->lcount[idx] > prm->min_num) lnode[L++] = idx;
            continue;
        }
        for (int c = 0; c < 8; c++) {
            int ch = t1->children[(size_t)idx * 8 + c];
            if (ch != -1 && t1->lcount[ch] > 0) queue[qt++] = ch;
        }
    }
    float* lpos0 = xmalloc((size_t)L * 3 * sizeof(float));
    for (int i = 0; i < L; i++)
        for (int d = 0; d < 3; d++) lpos0[(size_t)i * 3 + d] = (float)t1->centers[(size_t)lnode[i] * 3 + d];
    float* lnrm0 = xcalloc((size_t)L * 3, sizeof(float));
    /* --com_As 1: PCA normals (10 nearest, viewpoint at the box centre)
     * replace the input unless in_normal is 1 (include/DWGProcess.h:152-200) */
    float* Npca = NULL;
    if (prm->com_as && prm->in_normal != 1) {
        const int kp = n < 10 ? n : 10;
        int* nb = xmalloc((size_t)n * kp * sizeof(int));
        dwgo_knn(P, n, P, n, kp, nthreads, nb);
        float lo[3], hi[3], view[3];
        for (int d = 0; d < 3; d++) lo[d] = hi[d] = P[d];
        for (int i = 1; i < n; i++)
            for (int d = 0; d < 3; d++) {
                const float x = P[(size_t)i * 3 + d];
                if (x < lo[d]) lo[d] = x;
                if (x > hi[d]) hi[d] = x;
            }
        for (int d = 0; d < 3; d++) view[d] = (hi[d] + lo[d]) / 2.0f;
        Npca = xmalloc((size_t)n * 3 * sizeof(float));
        dwgo_pca_normals(P, n, nb, kp, view, Npca);
        free(nb);
        N_in = Npca;
    }
    if ((prm->in_normal != 3 || prm->com_as) && N_in) {
        /* SmoothNormalstoOctreeLeaves (include/DWGProcess.h:430-472), then
         * the whole-matrix normalisation of :537 */
        double* acc = xcalloc((size_t)L * 3, sizeof(double));
        double fro = 0;
        for (int i = 0; i < L; i++) {
            int nd = lnode[i];
            double W = t1->widths[nd];
            for (long long j = t1->list_off[nd]; j < t1->list_off[nd + 1]; j++) {
                int pi = t1->flat[j];
                for (int d = 0; d < 3; d++) {
                    double x = ((double)P[(size_t)pi * 3 + d] - t1->centers[(size_t)nd * 3 + d]) / W;
                    acc[(size_t)i * 3 + d] += exp(-(x * x) / 4.0) * (double)N_in[(size_t)pi * 3 + d];
                }
            }
            for (int d = 0; d < 3; d++) fro += acc[(size_t)i * 3 + d] * acc[(size_t)i * 3 + d];
        }
        fro = sqrt(fro);
        for (long long i = 0; i < (long long)L * 3; i++) lnrm0[i] = (float)(fro > 0 ? acc[i] / fro : acc[i]);
        free(acc);
    }
    /* canonical leaf order: depth-first order of the octree on the leaves */
    double* Ld = to_double(lpos0, (long long)L * 3);
    dwgo_octree* t2tmp = dwgo_octree_build(Ld, L, prm->max_depth);
    int* perm = xmalloc((size_t)(L ? L : 1) * sizeof(int));
    dwgo_octree_dfs_order(t2tmp, perm);
    dwgo_octree_free(t2tmp);
    float* lpos = xmalloc((size_t)L * 3 * sizeof(float));
    float* lnrm = xmalloc((size_t)L * 3 * sizeof(float));
    for (int i = 0; i < L; i++)
        for (int d = 0; d < 3; d++) {
            lpos[(size_t)i * 3 + d] = lpos0[(size_t)perm[i] * 3 + d];
            lnrm[(size_t)i * 3 + d] = lnrm0[(size_t)perm[i] * 3 + d];
        }
    free(lpos0);
    free(lnrm0);
    for (long long i = 0; i < (long long)L * 3; i++) Ld[i] = lpos[i];
    dwgo_octree* t2 = dwgo_octree_build(Ld, L, prm->max_depth);
    free(Ld);
    float* lA = xmalloc((size_t)L * sizeof(float));
    for (int i = 0; i < L; i++) lA[i] = prm->area;
    if (prm->com_as) {
        /* leaf areas from the 15 nearest leaves and the smoothed normals
         * (GetRadiiandAs, include/DWGProcess.h:345-378) */
        const int ka = L < 15 ? L : 15;
        int* nb = xmalloc((size_t)L * ka * sizeof(int));
        dwgo_knn(lpos, L, lpos, L, ka, nthreads, nb);
        dwgo_point_areas(lpos, L, nb, ka, lnrm, lA);
        free(nb);
    }
    float* lrad = xmalloc((size_t)L * sizeof(float));
    if (prm->use_radii) {
        int* nb = xmalloc((size_t)L * prm->kw * sizeof(int));
        dwgo_knn(lpos, L, lpos, L, prm->kw, nthreads, nb);
        dwgo_radii(lpos, L, nb, prm->kw, lrad);
        free(nb);
    } else {
        for (int i = 0; i < L; i++) lrad[i] = prm->screen;
    }
    /* iteration grid from the points (include/DWGProcess.h:672) */
    float org1[3], h1;
    dwgo_voxel_grid(P, n, prm->offset_1, prm->grid_reso, run->ires, org1, &h1);
    long long ng1 = (long long)run->ires[0] * run->ires[1] * run->ires[2];
    double* CM2 = xmalloc((size_t)t2->n_nodes * 3 * sizeof(double));
    double* R2 = xmalloc((size_t)t2->n_nodes * sizeof(double));
    dwgo_moments(t2, lpos, lnrm, lA, CM2, R2, NULL);
    /* OutlierFilter runs on the GPU copy of the areas (src/TurboDWG.cu:512):
     * the centres of mass and radii keep the areas of the host precompute,
     * the per-iteration sums of A n use the filtered ones */
    dwgo_outlier_filter(lA, L, prm->as_thres);
    if (prm->in_normal == 2 && prm->com_as) dwgo_random_normals(L, lnrm); /* include/DWGProcess.h:643-657 */
    if (prm->in_normal == 3) dwgo_gauss_map(lpos, L, lnrm);

    run->iters = prm->total_iter;
    run->iso = xcalloc((size_t)(prm->total_iter ? prm->total_iter : 1), sizeof(float));
    run->tri_count = xcalloc((size_t)(prm->total_iter ? prm->total_iter : 1), sizeof(long long));
    run->zero_count = xcalloc((size_t)(prm->total_iter ? prm->total_iter : 1), sizeof(int));
    float* gfield = xmalloc((size_t)ng1 * sizeof(float));
    long long cap = ng1 / 2 > 1000000 ? ng1 / 2 : 1000000;
    float* cent = xmalloc((size_t)cap * 3 * sizeof(float));
    float* tnrm = xmalloc((size_t)cap * 3 * sizeof(float));
    unsigned char* isz = xmalloc((size_t)(L ? L : 1));
    for (int it = 0; it < prm->total_iter; it++) {
        float sigma = sigma_schedule(it, prm->lambda);
        double mean;
        field_pass(t2, lpos, L, lnrm, lA, lrad, CM2, R2, prm, sigma, run->ires, org1, h1, nthreads,
                   gfield, &mean);
        float iso = (float)mean;
        if (it % 5 == 0 && it != 0) iso = iso * 0.5f; /* src/TurboDWG.cu:547-550 */
        run->iso[it] = iso;
        long long T = dwgo_marching_cubes(gfield, run->ires, org1, h1, iso, NULL, cent, tnrm, cap, NULL);
        if (T > cap) T = cap;
        run->tri_count[it] = T;
        int* nb = xmalloc((size_t)(T ? T : 1) * prm->knn_tri * sizeof(int));
        dwgo_knn(lpos, L, cent, T, prm->knn_tri, nthreads, nb);
        int zc = dwgo_diffuse_normals(nb, tnrm, T, prm->knn_tri, L, lnrm, isz);
        free(nb);
        run->zero_count[it] = zc;
        if (zc > prm->knn_zero) dwgo_zero_repair(lpos, L, lnrm, isz, prm->knn_zero, nthreads);
    }
    free(gfield);
    run->L = L;
    run->leaf_pos = lpos;
    run->leaf_nrm = lnrm;

    /* final meshing */
    float* pn = xmalloc((size_t)n * 3 * sizeof(float));
    float org2[3], h2;
    if (prm->use_leaves_generate == 1) {
        /* src/TurboDWG.cu:768-806 */
        dwgo_voxel_grid(lpos, L, 0.01f, prm->final_reso, run->fres, org2, &h2);
        long long ng2 = (long long)run->fres[0] * run->fres[1] * run->fres[2];
        if (prm->use_radii) {
            int* nb = xmalloc((size_t)L * prm->final_kw * sizeof(int));
            dwgo_knn(lpos, L, lpos, L, prm->final_kw, nthreads, nb);
            dwgo_radii(lpos, L, nb, prm->final_kw, lrad);
            free(nb);
        }
        run->final_field = xmalloc((size_t)ng2 * sizeof(float));
        double mean;
        field_pass(t2, lpos, L, lnrm, lA, lrad, CM2, R2, prm, prm->lambda, run->fres, org2, h2,
                   nthreads, run->final_field, &mean);
        run->final_iso = (float)mean;
        memset(pn, 0, (size_t)n * 3 * sizeof(float));
    } else {
        /* src/TurboDWG.cu:808-924 */
        dwgo_voxel_grid(P, n, prm->offset_2, prm->final_reso, run->fres, org2, &h2);
        long long ng2 = (long long)run->fres[0] * run->fres[1] * run->fres[2];
        int* nb = xmalloc((size_t)n * prm->normal_kw * sizeof(int));
        dwgo_knn(lpos, L, P, n, prm->normal_kw, nthreads, nb);
        dwgo_load_normals(nb, prm->normal_kw, n, lnrm, pn);
        free(nb);
        float* pA = xmalloc((size_t)n * sizeof(float));
        for (int i = 0; i < n; i++) pA[i] = prm->area;
        if (prm->com_as) {
            /* point areas from the 15 nearest points and the loaded normals
             * (include/DWGProcess.h:783-792); the moments below use them
             * (UpdateGWNInfo, src/TurboDWG.cu:931) */
            const int ka = n < 15 ? n : 15;
            int* nb3 = xmalloc((size_t)n * ka * sizeof(int));
            dwgo_knn(P, n, P, n, ka, nthreads, nb3);
            dwgo_point_areas(P, n, nb3, ka, pn, pA);
            free(nb3);
        }
        float* prad = xmalloc((size_t)n * sizeof(float));
        if (prm->use_radii) {
            int* nb2 = xmalloc((size_t)n * prm->final_kw * sizeof(int));
            dwgo_knn(P, n, P, n, prm->final_kw, nthreads, nb2);
            dwgo_radii(P, n, nb2, prm->final_kw, prad);
            free(nb2);
        } else {
            for (int i = 0; i < n; i++) prad[i] = prm->screen;
        }
        double* CM1 = xmalloc((size_t)t1->n_nodes * 3 * sizeof(double));
        double* R1 = xmalloc((size_t)t1->n_nodes * sizeof(double));
        dwgo_moments(t1, P, pn, pA, CM1, R1, NULL);
        dwgo_outlier_filter(pA, n, prm->as_thres); /* src/TurboDWG.cu:876, :935, as above */
        run->final_field = xmalloc((size_t)ng2 * sizeof(float));
        double mean;
        field_pass(t1, P, n, pn, pA, prad, CM1, R1, prm, prm->lambda, run->fres, org2, h2, nthreads,
                   run->final_field, &mean);
        run->final_iso = (float)mean;
        free(pA);
        free(prad);
        free(CM1);
        free(R1);
    }
    run->point_nrm = pn;
    long long ng2 = (long long)run->fres[0] * run->fres[1] * run->fres[2];
    long long cap2 = ng2 / 2 > 1000000 ? ng2 / 2 : 1000000;
    long long T = dwgo_marching_cubes(run->final_field, run->fres, org2, h2, run->final_iso, NULL, NULL,
                                      NULL, 0, NULL);
    if (T > cap2) T = cap2;
    run->tris = xmalloc((size_t)(T ? T : 1) * 9 * sizeof(float));
    dwgo_marching_cubes(run->final_field, run->fres, org2, h2, run->final_iso, run->tris, NULL, NULL, T,
                        NULL);
    run->T = T;

    free(cent);
    free(tnrm);
    free(isz);
    free(lA);
    free(lrad);
    free(CM2);
    free(R2);
    free(perm);
    free(queue);
    free(lnode);
    free(Npca);
    free(Pd);
    dwgo_octree_free(t1);
    dwgo_octree_free(t2);
    return run;
}

void dwgo_run_free(dwgo_run* r) {
    if (!r) return;
    free(r->leaf_pos);
    free(r->leaf_nrm);
    free(r->point_nrm);
    free(r->tris);
    free(r->iso);
    free(r->tri_count);
    free(r->zero_count);
    free(r->final_field);
    free(r);
}

long long dwgo_run_size(const dwgo_run* r, int what) {
    switch (what) {
        case 0: return r->L;
        case 1: return r->N;
        case 2: return r->T;
        case 3: return r->iters;
        case 4: case 5: case 6: return r->fres[what - 4];
        case 7: case 8: case 9: return r->ires[what - 7];
        default: return -1;
    }
}

int dwgo_run_get(const dwgo_run* r, const char* name, void* dst) {
    long long ng2 = (long long)r->fres[0] * r->fres[1] * r->fres[2];
    if (!strcmp(name, "leaf_pos")) memcpy(dst, r->leaf_pos, (size_t)r->L * 12);
    else if (!strcmp(name, "leaf_nrm")) memcpy(dst, r->leaf_nrm, (size_t)r->L * 12);
    else if (!strcmp(name, "point_nrm")) memcpy(dst, r->point_nrm, (size_t)r->N * 12);
    else if (!strcmp(name, "tris")) memcpy(dst, r->tris, (size_t)r->T * 36);
    else if (!strcmp(name, "iso")) memcpy(dst, r->iso, (size_t)r->iters * 4);
    else if (!strcmp(name, "tri_count")) memcpy(dst, r->tri_count, (size_t)r->iters * 8);
    else if (!strcmp(name, "zero_count")) memcpy(dst, r->zero_count, (size_t)r->iters * 4);
    else if (!strcmp(name, "final_field")) memcpy(dst, r->final_field, (size_t)ng2 * 4);
    else if (!strcmp(name, "final_iso")) memcpy(dst, &r->final_iso, 4);
    else return -1;
    return 0;
}
