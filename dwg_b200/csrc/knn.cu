// knn.cu -- exact kNN over a uniform cell grid.
//
// The reference builds a left-balanced kd-tree with log2(N) thrust sorts and
// walks it per query with a 30-entry stack (src/KNN_GWN.cu:42-66,490-715,
// include/cudaKDTree/cukd/traverse-cct.h:25-101).  Point clouds here are
// surfaces, so a uniform grid sized for ~3 points per occupied cell is built
// with one counting sort (histogram, scan, scatter), and each query visits
// Chebyshev shells of cells around its own cell until the k-th candidate is
// closer than anything outside the visited block.  Candidates are ranked by
// the cukd key (float bits of dist^2) << 32 | index
// (include/cudaKDTree/cukd/knn.h:279-282), with dist^2 = (dx*dx + dy*dy) + dz*dz
// in round-to-nearest single precision, and kept sorted in registers.
#include <cub/cub.cuh>

#include <climits>
#include <vector>

#include "knn.cuh"
#include "octree.cuh"

namespace dwg {

struct KnnGrid {
    int G0, G1, G2;
    float lo0, lo1, lo2, h, inv_h;
};

__device__ __forceinline__ int cell_coord(float p, float lo, float inv_h, int G) {
    int c = (int)floorf(__fmul_rn(__fsub_rn(p, lo), inv_h));
    return c < 0 ? 0 : (c >= G ? G - 1 : c);
}

__global__ void k_knn_hist(const float* __restrict__ P, int n, KnnGrid g, int* __restrict__ counts,
                           int* __restrict__ cell_of) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int cx = cell_coord(P[(size_t)i * 3], g.lo0, g.inv_h, g.G0);
    int cy = cell_coord(P[(size_t)i * 3 + 1], g.lo1, g.inv_h, g.G1);
    int cz = cell_coord(P[(size_t)i * 3 + 2], g.lo2, g.inv_h, g.G2);
    int c = cx + g.G0 * (cy + g.G1 * cz);
    cell_of[i] = c;
    atomicAdd(&counts[c], 1);
}

__global__ void k_knn_scatter(const float* __restrict__ P, int n, const int* __restrict__ cell_of,
                              int* __restrict__ fill, float4* __restrict__ pts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int slot = atomicAdd(&fill[cell_of[i]], 1);
    pts[slot] = make_float4(P[(size_t)i * 3], P[(size_t)i * 3 + 1], P[(size_t)i * 3 + 2], __int_as_float(i));
}

// The occupancy pyramid: node c of level l >= 1 holds the mask of its
// occupied children (bit t for the child 2 * (i, j, k) + (t & 1, t >> 1 & 1,
// t >> 2), cells at level 1), so a node is occupied iff its byte is nonzero
// and a walk skips empty children without loading them.  One launch fills
// every level of a zeroed pyramid: a thread per level-1 node ORs in its mask,
// then climbs while it is the first child to make its parent nonzero (the old
// byte of the OR), so every occupied node's bit reaches its parent once and
// no thread waits for another.
struct PyrDims {
    int levels;
    int ldim[KnnIndex::kMaxLevels][3];
    long long loff[KnnIndex::kMaxLevels];
};

// OR v into the byte at p (a 32-bit atomic on its word; the buffer is padded
// to whole words); returns the byte before
__device__ __forceinline__ unsigned atomic_or_byte(unsigned char* p, unsigned v) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    unsigned* w = reinterpret_cast<unsigned*>(a & ~(uintptr_t)3);
    const unsigned sh = (unsigned)(a & 3) * 8u;
    return (atomicOr(w, v << sh) >> sh) & 0xffu;
}

__global__ void k_pyr_fill(const int* __restrict__ cell_start, int G0, int G1, int G2, PyrDims pd,
                           unsigned char* __restrict__ occ) {
    const int D0 = pd.ldim[1][0], D1 = pd.ldim[1][1], D2 = pd.ldim[1][2];
    const long long m = (long long)D0 * D1 * D2;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < m;
         c += (long long)gridDim.x * blockDim.x) {
        int i = (int)(c % D0), j = (int)((c / D0) % D1), k = (int)(c / ((long long)D0 * D1));
        unsigned o = 0;
        for (int t = 0; t < 8; ++t) {
            const int x = 2 * i + (t & 1), y = 2 * j + ((t >> 1) & 1), z = 2 * k + (t >> 2);
            if (x >= G0 || y >= G1 || z >= G2) continue;
            const long long f = x + (long long)G0 * (y + (long long)G1 * z);
            o |= (cell_start[f + 1] > cell_start[f] ? 1u : 0u) << t;
        }
        if (!o) continue;
        atomic_or_byte(occ + pd.loff[1] + c, o);
        for (int l = 2; l <= pd.levels; ++l) {
            const int t = (i & 1) | ((j & 1) << 1) | ((k & 1) << 2);
            i >>= 1;
            j >>= 1;
            k >>= 1;
            const long long p = pd.loff[l] + i + (long long)pd.ldim[l][0] * (j + (long long)pd.ldim[l][1] * k);
            if (atomic_or_byte(occ + p, 1u << t) != 0) break;  // the parent was occupied: its ancestors know
        }
    }
}

// level dimensions and offsets of the occupancy pyramid of ix's grid
static int pyramid_dims(KnnIndex& ix) {
    ix.levels = 0;
    int d[3] = {ix.G[0], ix.G[1], ix.G[2]};
    ix.ldim[0][0] = d[0];
    ix.ldim[0][1] = d[1];
    ix.ldim[0][2] = d[2];
    long long total = 0;
    int L = 0;
    while (d[0] > 1 || d[1] > 1 || d[2] > 1) {
        DWG_REQUIRE(L + 1 < KnnIndex::kMaxLevels, "knn: grid too large for the occupancy pyramid");
        ++L;
        for (int t = 0; t < 3; ++t) {
            d[t] = (d[t] + 1) / 2;
            ix.ldim[L][t] = d[t];
        }
        ix.loff[L] = total;
        total += (long long)d[0] * d[1] * d[2];
    }
    ix.levels = L;
    // padded to whole 32-bit words (the fill ORs bytes through word atomics)
    if (L > 0) DWG_TRY(ix.occ.reserve((size_t)total + 4));
    return DWG_OK;
}

// the occupancy masks of every level from ix.cell_start (stream-ordered)
static int pyramid_fill(KnnIndex& ix, cudaStream_t s) {
    if (ix.levels < 1) return DWG_OK;
    PyrDims pd;
    pd.levels = ix.levels;
    for (int l = 0; l < KnnIndex::kMaxLevels; ++l) {
        pd.loff[l] = ix.loff[l];
        for (int d = 0; d < 3; ++d) pd.ldim[l][d] = ix.ldim[l][d];
    }
    DWG_CHECK_CUDA(cudaMemsetAsync(ix.occ.ptr, 0, ix.occ.n, s));
    const long long m = (long long)ix.ldim[1][0] * ix.ldim[1][1] * ix.ldim[1][2];
    long long blocks = div_up(m, 256);
    const long long cap = (long long)num_sms() * 8;
    if (blocks > cap) blocks = cap;
    k_pyr_fill<<<(unsigned)blocks, 256, 0, s>>>(ix.cell_start.ptr, ix.G[0], ix.G[1], ix.G[2], pd, ix.occ.ptr);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

static int build_pyramid(KnnIndex& ix, cudaStream_t s) {
    DWG_TRY(pyramid_dims(ix));
    return pyramid_fill(ix, s);
}

int knn_build(KnnIndex& ix, const float* P, int n, cudaStream_t s) {
    DWG_REQUIRE(P != nullptr && n >= 1, "knn: need at least one point (n=%d)", n);
    DWG_TRY(require_finite(P, 3ll * n, "knn", s));
    ix.n = n;
    DWG_TRY(ix.bbox.reserve(6));
    DWG_TRY(bbox_device(P, n, ix.bbox.ptr, s));
    float bb[6];
    DWG_CHECK_CUDA(cudaMemcpyAsync(bb, ix.bbox.ptr, sizeof(bb), cudaMemcpyDeviceToHost, s));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    float ext[3], emax = 0.f;
    for (int d = 0; d < 3; ++d) {
        ext[d] = bb[3 + d] - bb[d];
        emax = fmaxf(emax, ext[d]);
    }
    if (!(emax > 0.f)) emax = 1.f;
    // ~3 points per occupied cell for a surface sample
    double gm = ceil(sqrt((double)n / 14.0));
    if (gm < 1) gm = 1;
    if (gm > 1024) gm = 1024;
    float h = (float)(emax / gm) * 1.0001f;
    for (;;) {
        long long tot = 1;
        for (int d = 0; d < 3; ++d) {
            int G = (int)ceil(ext[d] / h);
            if (G < 1) G = 1;
            ix.G[d] = G;
            tot *= G;
        }
        if (tot <= (1ll << 27)) break;
        h *= 1.25f;
    }
    ix.h = h;
    ix.inv_h = 1.0f / h;
    {
        int gm = max(ix.G[0], max(ix.G[1], ix.G[2]));
        int sh = 0;
        while ((gm >> sh) > 32) ++sh;
        ix.morton_shift = sh;
    }
    for (int d = 0; d < 3; ++d) ix.lo[d] = bb[d];
    long long ncell = (long long)ix.G[0] * ix.G[1] * ix.G[2];
    KnnGrid g{ix.G[0], ix.G[1], ix.G[2], ix.lo[0], ix.lo[1], ix.lo[2], ix.h, ix.inv_h};
    DevBuf<int> counts, cell_of;
    DWG_TRY(counts.reserve(ncell + 1));
    DWG_TRY(cell_of.reserve(n));
    DWG_TRY(ix.cell_start.reserve(ncell + 1));
    DWG_TRY(ix.cell_fill.reserve(ncell + 1));
    DWG_TRY(ix.pts.reserve(n));
    DWG_CHECK_CUDA(cudaMemsetAsync(counts.ptr, 0, sizeof(int) * (ncell + 1), s));
    k_knn_hist<<<div_up(n, 256), 256, 0, s>>>(P, n, g, counts.ptr, cell_of.ptr);
    DWG_CHECK_LAUNCH();
    size_t bytes = 0;
    int* cin = counts.ptr;
    int* cout = ix.cell_start.ptr;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cin, cout, (int)(ncell + 1), s));
    DWG_TRY(ix.scratch.reserve(bytes + 256));
    bytes = ix.scratch.n;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(ix.scratch.ptr, bytes, cin, cout, (int)(ncell + 1), s));
    DWG_CHECK_CUDA(cudaMemcpyAsync(ix.cell_fill.ptr, ix.cell_start.ptr, sizeof(int) * (ncell + 1),
                                   cudaMemcpyDeviceToDevice, s));
    k_knn_scatter<<<div_up(n, 256), 256, 0, s>>>(P, n, cell_of.ptr, ix.cell_fill.ptr, ix.pts.ptr);
    DWG_CHECK_LAUNCH();
    DWG_TRY(build_pyramid(ix, s));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    return DWG_OK;
}

struct KnnArgs {
    KnnGrid g;
    const float4* __restrict__ pts;
    const int* __restrict__ cell_start;
    const float* __restrict__ q;
    const int* __restrict__ q_index;
    const float* __restrict__ q_source;
    long long nq;
    const unsigned long long* nq_dev;
    const int* nq_dev_i32;
    const unsigned char* __restrict__ exclude;
    const int* gate_count;
    int gate_min;
    int k;
    int* __restrict__ out;
    const int* __restrict__ order;  // query processing order (spatially bucketed)
    int* __restrict__ q_key;
    int* __restrict__ q_hist;
    int morton_shift;
    // per-cell bound of the 16th-neighbour distance (null: none), seeds the
    // per-thread search of queries with k <= 16
    const float* __restrict__ kb;
    // queries whose pyramid walk ran past kDeepBudget visits go on this list
    // (null: no budget) and are finished by k_knn_deep
    int* __restrict__ deep;
    float* __restrict__ deep_bound;  // per entry: a bound on the k-th squared distance (its walk's k-th key)
    int* __restrict__ deep_count;
    // per query (null: none): a key above its k-th nearest key, ~0 for none
    const unsigned long long* __restrict__ seed;
    // occupancy pyramid
    const unsigned char* __restrict__ occ;
    int levels;
    int ldim[KnnIndex::kMaxLevels][3];
    long long loff[KnnIndex::kMaxLevels];
};

// a seed key as a distance from the query that holds its k nearest: +inf
// for none
__device__ __forceinline__ float seed_radius(unsigned long long sd) {
    return sd == ~0ull ? INFINITY : sqrtf(__uint_as_float((unsigned)(sd >> 32))) * 1.00002f + 1e-7f;
}

__device__ __forceinline__ long long knn_count(const KnnArgs& a) {
    long long nq = a.nq;
    if (a.nq_dev) {
        unsigned long long d = *a.nq_dev;
        if ((long long)d < nq) nq = (long long)d;
    }
    if (a.nq_dev_i32) {
        long long d = *a.nq_dev_i32;
        if (d < nq) nq = d;
    }
    return nq;
}

__device__ __forceinline__ void knn_load_query(const KnnArgs& a, long long qi, float& qx, float& qy, float& qz) {
    if (a.q_index) {
        long long src = a.q_index[qi];
        qx = a.q_source[src * 3];
        qy = a.q_source[src * 3 + 1];
        qz = a.q_source[src * 3 + 2];
    } else {
        qx = a.q[qi * 3];
        qy = a.q[qi * 3 + 1];
        qz = a.q[qi * 3 + 2];
    }
}

__device__ __forceinline__ unsigned spread5(unsigned v) {
    v &= 31u;
    v = (v | (v << 8)) & 0x0300Fu;
    v = (v | (v << 4)) & 0x030C3u;
    v = (v | (v << 2)) & 0x09249u;
    return v;
}

// bucket the queries by the Morton code of their coarse cell (32^3 buckets)
__global__ void k_knn_qkey(KnnArgs a) {
    if (a.gate_count && *a.gate_count <= a.gate_min) return;
    const long long nq = knn_count(a);
    for (long long qi = blockIdx.x * (long long)blockDim.x + threadIdx.x; qi < nq;
         qi += (long long)gridDim.x * blockDim.x) {
        float qx, qy, qz;
        knn_load_query(a, qi, qx, qy, qz);
        unsigned cx = cell_coord(qx, a.g.lo0, a.g.inv_h, a.g.G0) >> a.morton_shift;
        unsigned cy = cell_coord(qy, a.g.lo1, a.g.inv_h, a.g.G1) >> a.morton_shift;
        unsigned cz = cell_coord(qz, a.g.lo2, a.g.inv_h, a.g.G2) >> a.morton_shift;
        int key = (int)(spread5(cx) | (spread5(cy) << 1) | (spread5(cz) << 2));
        a.q_key[qi] = key;
        atomicAdd(&a.q_hist[key], 1);
    }
}

__global__ void k_knn_qscatter(KnnArgs a, int* __restrict__ fill, int* __restrict__ order) {
    if (a.gate_count && *a.gate_count <= a.gate_min) return;
    const long long nq = knn_count(a);
    for (long long qi = blockIdx.x * (long long)blockDim.x + threadIdx.x; qi < nq;
         qi += (long long)gridDim.x * blockDim.x)
        order[atomicAdd(&fill[a.q_key[qi]], 1)] = (int)qi;
}


// top-k state of one lane: an unsorted set of KMAX keys and its maximum
// (value, slot) of the largest of v[LO, LO + N), the lowest slot among equal
// values (what a scan from LO with a strict comparison finds), by a
// tournament: depth log2 N instead of a chain of N - 1 dependent compares
template <int LO, int N, typename T, int M>
__device__ __forceinline__ void tour_max(const T (&v)[M], T& m, int& p) {
    if constexpr (N == 1) {
        m = v[LO];
        p = LO;
    } else {
        T m1, m2;
        int p1, p2;
        tour_max<LO, N / 2>(v, m1, p1);
        tour_max<LO + N / 2, N - N / 2>(v, m2, p2);
        const bool r = m2 > m1;
        m = r ? m2 : m1;
        p = r ? p2 : p1;
    }
}

// Batcher's odd-even merge sort on 16 inputs, 63 comparators in 10 layers
// (the iterative form: for p = 1, 2, 4, 8, for d = p, p/2, ..., 1, for j =
// d mod p, step 2d, for i < d, join i + j and i + j + d when both lie in the
// same block of 2p); comparator t orders slots kSortLo[t] < kSortHi[t].  On
// fewer slots the missing ones count as +infinity: a comparator that touches
// one never swaps and is left out (59 remain for 15 slots, 32 for 10; the
// odd-even transposition network took 105 and 45).
constexpr int kSortNet = 63;
constexpr unsigned char kSortLo[kSortNet] = {0, 2, 4, 6, 8, 10, 12, 14, 0, 1, 4, 5, 8, 9, 12, 13, 1, 5, 9, 13, 0, 1, 2, 3, 8, 9, 10, 11, 2, 3, 10, 11, 1, 3, 5, 9, 11, 13, 0, 1, 2, 3, 4, 5, 6, 7, 4, 5, 6, 7, 2, 3, 6, 7, 10, 11, 1, 3, 5, 7, 9, 11, 13};
constexpr unsigned char kSortHi[kSortNet] = {1, 3, 5, 7, 9, 11, 13, 15, 2, 3, 6, 7, 10, 11, 14, 15, 2, 6, 10, 14, 4, 5, 6, 7, 12, 13, 14, 15, 4, 5, 12, 13, 2, 4, 6, 10, 12, 14, 8, 9, 10, 11, 12, 13, 14, 15, 8, 9, 10, 11, 4, 5, 8, 9, 12, 13, 2, 4, 6, 8, 10, 12, 14};

template <int KMAX>
struct TopK {
    unsigned long long e[KMAX];
    unsigned long long mx;  // the k-th key (max of the set) or NONE
    int mpos;
    int fill;  // keys entered so far, up to k: the slots fill in order before any maximum search
    __device__ __forceinline__ void init(int k) {
#pragma unroll
        for (int q = 0; q < KMAX; ++q) e[q] = q < k ? ~0ull : 0ull;  // unused slots never become the max
        mx = ~0ull;
        mpos = 0;
        fill = 0;
    }
    // k slots holding the key T: only keys below T enter, and T must bound
    // the k-th key from above so that every slot is replaced
    __device__ __forceinline__ void init_bound(int k, unsigned long long T) {
#pragma unroll
        for (int q = 0; q < KMAX; ++q) e[q] = q < k ? T : 0ull;
        mx = T;
        mpos = 0;
        fill = 0;
    }
    // enter v (v < mx): the first k keys take the slots in turn (the
    // maximum stays the initial key until the last slot is taken, then it is
    // searched once), later keys replace the maximum
    __device__ __forceinline__ void push(unsigned long long v, int k) {
        if (fill < k) {
#pragma unroll
            for (int q = 0; q < KMAX; ++q)
                if (q == fill) e[q] = v;
            if (++fill == k) {
                max_slot();
            }
        } else {
            replace_max(v);
        }
    }
    template <int T>
    __device__ __forceinline__ void sort_net() {
        if constexpr (T < kSortNet) {
            constexpr int lo = kSortLo[T], hi = kSortHi[T];
            if constexpr (hi < KMAX) {
                const unsigned long long a = e[lo], b = e[hi];
                e[lo] = a < b ? a : b;
                e[hi] = a < b ? b : a;
            }
            sort_net<T + 1>();
        }
    }
    // mx and mpos: the largest key and its lowest slot
    __device__ __forceinline__ void max_slot() {
        if constexpr (KMAX <= 16) {
            tour_max<0, KMAX>(e, mx, mpos);
        } else {
            mx = e[0];
            mpos = 0;
#pragma unroll
            for (int q = 1; q < KMAX; ++q)
                if (e[q] > mx) {
                    mx = e[q];
                    mpos = q;
                }
        }
    }
    // drop e[0] of a sorted set: the keys move down one slot, NONE enters on top
    __device__ __forceinline__ void shift_down() {
#pragma unroll
        for (int q = 0; q + 1 < KMAX; ++q) e[q] = e[q + 1];
        e[KMAX - 1] = ~0ull;
    }
    // replace the maximum by v (v < mx) and find the new maximum (a warp's
    // lanes take the same steps whether or not their slots are all filled)
    __device__ __forceinline__ void replace_max(unsigned long long v) {
#pragma unroll
        for (int q = 0; q < KMAX; ++q)
            if (q == mpos) e[q] = v;
        max_slot();
    }
    // ascending order (once per query): up to 16 slots the sorting network
    // of sort_net, more slots an insertion sort in local memory
    __device__ __forceinline__ void sort() {
        if constexpr (KMAX <= 16) {
            sort_net<0>();
        } else {
            unsigned long long t[KMAX];
#pragma unroll
            for (int q = 0; q < KMAX; ++q) t[q] = e[q];
#pragma unroll 1
            for (int q = 1; q < KMAX; ++q) {
                const unsigned long long v = t[q];
                int p = q - 1;
                while (p >= 0 && t[p] > v) {
                    t[p + 1] = t[p];
                    --p;
                }
                t[p + 1] = v;
            }
#pragma unroll
            for (int q = 0; q < KMAX; ++q) e[q] = t[q];
        }
    }
};

// Exact continuation of a query's search over the occupancy pyramid, after
// the Chebyshev shells 0 and 1 around its cell (cx, cy, cz) were scanned.
// Depth-first from the 1x1x1 top level, the children of a node in the order
// of their octant's distance from the query's octant (same octant, then the
// three face neighbours, the three edge neighbours, the opposite one); a
// node is skipped when it is empty (its bit in the parent's child mask: no
// load) or its (eps-widened) box is farther than the current k-th candidate.
// The walk is stackless: a 4-bit child counter per level in one 64-bit word,
// the child masks of the nodes on the path (a byte per level in two 64-bit
// words) and the current node's coordinates.  With a deep list the walk
// gives up after kDeepBudget child visits (returns false): a query that far
// from its neighbours is finished by a warp of k_knn_deep instead of holding
// a thread (and its warp) for the length of a long walk.
constexpr int kDeepBudget = 128;
template <int KMAX>
__device__ __forceinline__ bool knn_pyramid(const KnnArgs& a, float qx, float qy, float qz, int cx, int cy, int cz,
                                            TopK<KMAX>& top) {
    const unsigned long long NONE = ~0ull;
    const float h = a.g.h;
    const float eps = 1e-4f * h + 1e-6f;
    const int top_l = a.levels;
    int lvl = top_l, ci = 0, cj = 0, ck = 0;
    unsigned long long ctr = 0;
    int visits = 0;
    // byte l of (mk1:mk0): the child mask of the path's node at level l
    unsigned long long mk0 = 0ull, mk1 = 0ull;
    {
        const unsigned long long tm = (unsigned long long)a.occ[a.loff[top_l]] << (8 * (top_l & 7));
        if (top_l < 8) mk0 = tm;
        else mk1 = tm;
    }
    for (;;) {
        const int sh = 4 * lvl;
        const int c = (int)((ctr >> sh) & 15ull);
        if (c == 8) {
            if (lvl == top_l) break;
            ctr &= ~(15ull << sh);
            ++lvl;
            ci >>= 1;
            cj >>= 1;
            ck >>= 1;
            continue;
        }
        ctr += 1ull << sh;
        if (a.deep && ++visits > kDeepBudget) return false;
        // octant of the query about the node's midpoint
        const int half = 1 << (lvl - 1);
        const float mx = a.g.lo0 + (float)((ci << lvl) + half) * h;
        const float my = a.g.lo1 + (float)((cj << lvl) + half) * h;
        const float mz = a.g.lo2 + (float)((ck << lvl) + half) * h;
        const int qo = (qx >= mx ? 1 : 0) | (qy >= my ? 2 : 0) | (qz >= mz ? 4 : 0);
        const int oc = qo ^ (int)((0x76534210u >> (4 * c)) & 7u);
        // empty or outside the grid (such children have no bit)
        if (!(((lvl < 8 ? mk0 : mk1) >> (8 * (lvl & 7) + oc)) & 1ull)) continue;
        const int nl = lvl - 1;
        const int ni = (ci << 1) | (oc & 1), nj = (cj << 1) | ((oc >> 1) & 1), nk = (ck << 1) | (oc >> 2);
        const float kd2 = top.mx == NONE ? INFINITY : __uint_as_float((unsigned)(top.mx >> 32)) * 1.00001f;
        const float x0 = a.g.lo0 + (float)(ni << nl) * h - eps, x1 = a.g.lo0 + (float)((ni + 1) << nl) * h + eps;
        const float y0 = a.g.lo1 + (float)(nj << nl) * h - eps, y1 = a.g.lo1 + (float)((nj + 1) << nl) * h + eps;
        const float z0 = a.g.lo2 + (float)(nk << nl) * h - eps, z1 = a.g.lo2 + (float)((nk + 1) << nl) * h + eps;
        const float ddx = fmaxf(0.f, fmaxf(x0 - qx, qx - x1));
        const float ddy = fmaxf(0.f, fmaxf(y0 - qy, qy - y1));
        const float ddz = fmaxf(0.f, fmaxf(z0 - qz, qz - z1));
        if (ddx * ddx + ddy * ddy + ddz * ddz > kd2) continue;
        if (nl == 0) {
            if (abs(ni - cx) <= 1 && abs(nj - cy) <= 1 && abs(nk - cz) <= 1) continue;  // scanned already
            const int cell = ni + a.g.G0 * (nj + a.g.G1 * nk);
            const int e = a.cell_start[cell + 1];
            for (int t = a.cell_start[cell]; t < e; ++t) {
                const float4 pp = a.pts[t];
                const int id = __float_as_int(pp.w);
                if (a.exclude && a.exclude[id]) continue;
                const float d2 = sq3_rn(__fsub_rn(pp.x, qx), __fsub_rn(pp.y, qy), __fsub_rn(pp.z, qz));
                const unsigned long long v = ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned)id;
                if (v < top.mx) top.push(v, a.k);
            }
            continue;
        }
        const int* D = a.ldim[nl];
        const unsigned long long cm = a.occ[a.loff[nl] + ni + (long long)D[0] * (nj + (long long)D[1] * nk)];
        const int bs = 8 * (nl & 7);
        if (nl < 8) mk0 = (mk0 & ~(0xffull << bs)) | (cm << bs);
        else mk1 = (mk1 & ~(0xffull << bs)) | (cm << bs);
        lvl = nl;
        ci = ni;
        cj = nj;
        ck = nk;
    }
    return true;
}

// One thread per query; queries are processed in the order of their coarse
// Morton bucket so that neighbouring threads search neighbouring cells.  A
// query visits Chebyshev shells of cells around its own cell; a cell is
// skipped when its box is farther than the current k-th candidate; the k best
// keys are an unsorted register set whose maximum is kept in a register
// (replace-the-maximum on insertion, one sort at the end).  The search stops
// when the k-th key is closer than the boundary of the visited block.
template <int KMAX>
__global__ void __launch_bounds__(128, KMAX <= 10 ? 4 : 1) k_knn_thread(KnnArgs a) {
    if (a.gate_count && *a.gate_count <= a.gate_min) return;
    const long long nq = knn_count(a);
    const unsigned long long NONE = ~0ull;
    const int k = a.k;
    const float h = a.g.h;
    const float eps = 1e-4f * h + 1e-6f;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < nq;
         j += (long long)gridDim.x * blockDim.x) {
        const long long qi = a.order ? a.order[j] : j;
        float qx, qy, qz;
        knn_load_query(a, qi, qx, qy, qz);
        const int cx = cell_coord(qx, a.g.lo0, a.g.inv_h, a.g.G0);
        const int cy = cell_coord(qy, a.g.lo1, a.g.inv_h, a.g.G1);
        const int cz = cell_coord(qz, a.g.lo2, a.g.inv_h, a.g.G2);
        TopK<KMAX> top;
        bool deferred = false;
        if (a.kb && k <= kKnnBoundK) {
            // start from k copies of the key of the bound kb[c] + |q - x_c|
            // on the 16th distance: everything beyond it is pruned at once
            const float ex = qx - (a.g.lo0 + ((float)cx + 0.5f) * h), ey = qy - (a.g.lo1 + ((float)cy + 0.5f) * h),
                        ez = qz - (a.g.lo2 + ((float)cz + 0.5f) * h);
            const float rq = (a.kb[cx + a.g.G0 * (cy + a.g.G1 * cz)] + sqrtf(ex * ex + ey * ey + ez * ez) * 1.00002f) *
                                 1.00002f + 1e-7f;
            top.init_bound(k, ((unsigned long long)__float_as_uint(rq * rq * 1.00002f) << 32) | 0xffffffffull);
        } else {
            top.init(k);
        }
        if (a.seed) {
            const unsigned long long sd = a.seed[qi];
            if (sd < top.mx) top.init_bound(k, sd);
        }
        for (int r = 0;; ++r) {
            const float kd2 = top.mx == NONE ? INFINITY : __uint_as_float((unsigned)(top.mx >> 32)) * 1.00001f;
            for (int dz = -r; dz <= r; ++dz) {
                const int z = cz + dz;
                if (z < 0 || z >= a.g.G2) continue;
                const float z0 = a.g.lo2 + (float)z * h - eps, z1 = z0 + h + 2.f * eps;
                const float ddz = fmaxf(0.f, fmaxf(z0 - qz, qz - z1));
                for (int dy = -r; dy <= r; ++dy) {
                    const int y = cy + dy;
                    if (y < 0 || y >= a.g.G1) continue;
                    const float y0 = a.g.lo1 + (float)y * h - eps, y1 = y0 + h + 2.f * eps;
                    const float ddy = fmaxf(0.f, fmaxf(y0 - qy, qy - y1));
                    const float dyz = ddy * ddy + ddz * ddz;
                    if (dyz > kd2) continue;
                    const bool face = (dz == -r || dz == r || dy == -r || dy == r);
                    const int step = face ? 1 : (r > 0 ? 2 * r : 1);
                    for (int dx = -r; dx <= r; dx += step) {
                        const int x = cx + dx;
                        if (x < 0 || x >= a.g.G0) continue;
                        const float x0 = a.g.lo0 + (float)x * h - eps, x1 = x0 + h + 2.f * eps;
                        const float ddx = fmaxf(0.f, fmaxf(x0 - qx, qx - x1));
                        if (ddx * ddx + dyz > kd2) continue;
                        const int c = x + a.g.G0 * (y + a.g.G1 * z);
                        const int e = a.cell_start[c + 1];
                        for (int t = a.cell_start[c]; t < e; ++t) {
                            const float4 pp = a.pts[t];
                            const int id = __float_as_int(pp.w);
                            if (a.exclude && a.exclude[id]) continue;
                            const float d2 =
                                sq3_rn(__fsub_rn(pp.x, qx), __fsub_rn(pp.y, qy), __fsub_rn(pp.z, qz));
                            const unsigned long long v = ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned)id;
                            if (v < top.mx) top.push(v, k);
                        }
                    }
                }
            }
            if (cx - r <= 0 && cy - r <= 0 && cz - r <= 0 && cx + r >= a.g.G0 - 1 && cy + r >= a.g.G1 - 1 &&
                cz + r >= a.g.G2 - 1)
                break;
            if (top.mx != NONE) {
                float bd = INFINITY;
                if (cx - r > 0) bd = fminf(bd, qx - (a.g.lo0 + (float)(cx - r) * h));
                if (cx + r < a.g.G0 - 1) bd = fminf(bd, (a.g.lo0 + (float)(cx + r + 1) * h) - qx);
                if (cy - r > 0) bd = fminf(bd, qy - (a.g.lo1 + (float)(cy - r) * h));
                if (cy + r < a.g.G1 - 1) bd = fminf(bd, (a.g.lo1 + (float)(cy + r + 1) * h) - qy);
                if (cz - r > 0) bd = fminf(bd, qz - (a.g.lo2 + (float)(cz - r) * h));
                if (cz + r < a.g.G2 - 1) bd = fminf(bd, (a.g.lo2 + (float)(cz + r + 1) * h) - qz);
                bd -= eps;
                if (bd > 0.f && __uint_as_float((unsigned)(top.mx >> 32)) < bd * bd * 0.9999f) break;
            }
            if (r == 1 && a.levels > 0) {
                if (!knn_pyramid<KMAX>(a, qx, qy, qz, cx, cy, cz, top)) {
                    // at most once per query: the list holds nq.  The walk's
                    // current maximum (its k-th key, or the initial bound)
                    // bounds the k-th squared distance
                    const int pos = atomicAdd(a.deep_count, 1);
                    a.deep[pos] = (int)qi;
                    a.deep_bound[pos] = top.mx == NONE ? INFINITY : __uint_as_float((unsigned)(top.mx >> 32));
                    deferred = true;
                }
                break;
            }
        }
        if (deferred) continue;
        top.sort();
        // slots >= k hold 0 (below every key) and sort first; results start at KMAX - k
#pragma unroll
        for (int t = 0; t < KMAX; ++t) {
            const int o = t - (KMAX - k);
            if (o >= 0) a.out[qi * k + o] = top.e[t] == NONE ? -1 : (int)(unsigned)(top.e[t] & 0xffffffffu);
        }
    }
}

// ------------------------------------------------------ cell-grouped path --
// Queries with k <= 16 and no exclusion are grouped by the grid cell they fall
// in (clamped to the grid).  For cell c with centre x_c, kb[c] bounds the
// distance from x_c to its 16th nearest point from above, and m_c is the
// largest |q - x_c| over the cell's queries.  By the triangle inequality the
// k nearest points of every such query lie within R_c = kb[c] + 2 m_c of x_c,
// so one warp gathers that candidate set once (occupancy pyramid, then
// cells, then points, all 32 lanes in step) into shared memory and every lane
// then ranks the same candidates for its own query: no divergence, one search
// per cell instead of one per query.  A cell whose candidate set does not fit
// (or has no finite bound) sends its queries to the per-thread search.
constexpr int kCqWarps = 4;
constexpr int kCqNodes = 1024;  // frontier capacity per warp (ping-pong pair, shared memory), at level >= 1
constexpr int kCqChunk = 256;   // candidates staged in shared memory at a time

__device__ __forceinline__ float cell_mid(float lo, int i, float h) { return lo + ((float)i + 0.5f) * h; }

// kb from the 3x3x3 block around each cell: the 16th smallest distance, or
// +inf when the block holds fewer than 16 points
__global__ void k_kb_local(KnnGrid g, const int* __restrict__ cell_start, const float4* __restrict__ pts,
                           const unsigned char* __restrict__ occ1, int D0, int D1, float* __restrict__ kb) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= (long long)g.G0 * g.G1 * g.G2) return;
    const int i = (int)(c % g.G0), j = (int)((c / g.G0) % g.G1), k = (int)(c / ((long long)g.G0 * g.G1));
    if (occ1) {
        // the 3x3x3 block lies in at most 2x2x2 nodes of pyramid level 1:
        // when they are all empty the bound stays +inf (cheap for empty space)
        bool any = false;
        for (int z = max(k - 1, 0) >> 1; z <= min(k + 1, g.G2 - 1) >> 1 && !any; ++z)
            for (int y = max(j - 1, 0) >> 1; y <= min(j + 1, g.G1 - 1) >> 1 && !any; ++y)
                for (int x = max(i - 1, 0) >> 1; x <= min(i + 1, g.G0 - 1) >> 1; ++x)
                    if (occ1[x + (long long)D0 * (y + (long long)D1 * z)]) {
                        any = true;
                        break;
                    }
        if (!any) {
            kb[c] = INFINITY;
            return;
        }
    }
    const float x = cell_mid(g.lo0, i, g.h), y = cell_mid(g.lo1, j, g.h), z = cell_mid(g.lo2, k, g.h);
    float d[kKnnBoundK];
#pragma unroll
    for (int t = 0; t < kKnnBoundK; ++t) d[t] = INFINITY;
    float mx = INFINITY;
    int mpos = 0, cnt = 0;
    for (int dz = -1; dz <= 1; ++dz) {
        const int zz = k + dz;
        if (zz < 0 || zz >= g.G2) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int yy = j + dy;
            if (yy < 0 || yy >= g.G1) continue;
            for (int dx = -1; dx <= 1; ++dx) {
                const int xx = i + dx;
                if (xx < 0 || xx >= g.G0) continue;
                const int cc = xx + g.G0 * (yy + g.G1 * zz);
                const int e = cell_start[cc + 1];
                for (int t = cell_start[cc]; t < e; ++t) {
                    const float4 p = pts[t];
                    const float ex = p.x - x, ey = p.y - y, ez = p.z - z;
                    const float d2 = ex * ex + ey * ey + ez * ez;
                    if (cnt < kKnnBoundK) {  // the first keys fill the slots; the maximum once they are full
#pragma unroll
                        for (int q = 0; q < kKnnBoundK; ++q)
                            if (q == cnt) d[q] = d2;
                        if (cnt == kKnnBoundK - 1) {
                            tour_max<0, kKnnBoundK>(d, mx, mpos);
                        }
                    } else if (d2 < mx) {
#pragma unroll
                        for (int q = 0; q < kKnnBoundK; ++q)
                            if (q == mpos) d[q] = d2;
                        tour_max<0, kKnnBoundK>(d, mx, mpos);
                    }
                    ++cnt;
                }
            }
        }
    }
    kb[c] = cnt >= kKnnBoundK ? sqrtf(mx) * 1.00002f + 1e-7f : INFINITY;
}

// kb for the cells that hold queries: the 16th smallest distance from the
// cell centre over the cells within Chebyshev radius r, r = 1, 2, 3 until 16
// points are found (any 16 points bound the 16th nearest from above), +inf
// when the radius-3 block holds fewer (those queries take the per-thread
// search, which needs no bound) or when every query of the cell has a seed
constexpr int kKbActiveRadius = 3;
__global__ void k_kb_active(KnnGrid g, const int* __restrict__ cell_start, const float4* __restrict__ pts,
                            const unsigned char* __restrict__ occ1, int D0, int D1, const int* __restrict__ active,
                            const int* __restrict__ misc, const unsigned int* __restrict__ sbits,
                            float* __restrict__ kb) {
    const int na = misc[0];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < na; t += gridDim.x * blockDim.x) {
        const int c = active[t];
        // a cell whose queries all have seeds takes its radius from them
        if (sbits && isfinite(__uint_as_float(sbits[c]))) {
            kb[c] = INFINITY;
            continue;
        }
        const int i = c % g.G0, j = (c / g.G0) % g.G1, k = c / (g.G0 * g.G1);
        const float x = cell_mid(g.lo0, i, g.h), y = cell_mid(g.lo1, j, g.h), z = cell_mid(g.lo2, k, g.h);
        float d[kKnnBoundK];
#pragma unroll
        for (int q = 0; q < kKnnBoundK; ++q) d[q] = INFINITY;
        float mx = INFINITY;
        int mpos = 0, cnt = 0;
        for (int r = 0; r <= kKbActiveRadius; ++r) {
            for (int dz = -r; dz <= r; ++dz) {
                const int zz = k + dz;
                if (zz < 0 || zz >= g.G2) continue;
                for (int dy = -r; dy <= r; ++dy) {
                    const int yy = j + dy;
                    if (yy < 0 || yy >= g.G1) continue;
                    for (int dx = -r; dx <= r; ++dx) {
                        // the shell of radius r only
                        if (max(abs(dx), max(abs(dy), abs(dz))) != r) continue;
                        const int xx = i + dx;
                        if (xx < 0 || xx >= g.G0) continue;
                        // an empty cell by its bit in the level-1 child mask
                        // (8 cells share a byte): no range loads
                        if (occ1 && !((occ1[(xx >> 1) + (long long)D0 * ((yy >> 1) + (long long)D1 * (zz >> 1))] >>
                                       ((xx & 1) | ((yy & 1) << 1) | ((zz & 1) << 2))) &
                                      1))
                            continue;
                        const int cc = xx + g.G0 * (yy + g.G1 * zz);
                        const int e = cell_start[cc + 1];
                        for (int s = cell_start[cc]; s < e; ++s) {
                            const float4 p = pts[s];
                            const float ex = p.x - x, ey = p.y - y, ez = p.z - z;
                            const float d2 = ex * ex + ey * ey + ez * ez;
                            if (cnt < kKnnBoundK) {  // fill, then the maximum once
#pragma unroll
                                for (int q = 0; q < kKnnBoundK; ++q)
                                    if (q == cnt) d[q] = d2;
                                if (cnt == kKnnBoundK - 1) {
                                    tour_max<0, kKnnBoundK>(d, mx, mpos);
                                }
                            } else if (d2 < mx) {
#pragma unroll
                                for (int q = 0; q < kKnnBoundK; ++q)
                                    if (q == mpos) d[q] = d2;
                                tour_max<0, kKnnBoundK>(d, mx, mpos);
                            }
                            ++cnt;
                        }
                    }
                }
            }
            if (r >= 1 && cnt >= kKnnBoundK) break;
        }
        kb[c] = cnt >= kKnnBoundK ? sqrtf(mx) * 1.00002f + 1e-7f : INFINITY;
    }
}

// one min-plus pass with the 26 neighbours at distance `step` cells:
// kb[c] <= kb[c'] + |x_c - x_c'| (triangle inequality); len1..3 are the
// neighbour distances rounded up
__global__ void k_kb_jfa(KnnGrid g, const float* __restrict__ in, float* __restrict__ out, int step, float len1,
                         float len2, float len3) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= (long long)g.G0 * g.G1 * g.G2) return;
    const int i = (int)(c % g.G0), j = (int)((c / g.G0) % g.G1), k = (int)(c / ((long long)g.G0 * g.G1));
    float v = in[c];
    for (int dz = -1; dz <= 1; ++dz) {
        const int zz = k + dz * step;
        if (zz < 0 || zz >= g.G2) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int yy = j + dy * step;
            if (yy < 0 || yy >= g.G1) continue;
            for (int dx = -1; dx <= 1; ++dx) {
                const int xx = i + dx * step;
                if (xx < 0 || xx >= g.G0) continue;
                const int nz = (dx != 0) + (dy != 0) + (dz != 0);
                if (nz == 0) continue;
                const float len = nz == 1 ? len1 : (nz == 2 ? len2 : len3);
                v = fminf(v, __fadd_ru(in[xx + (long long)g.G0 * (yy + (long long)g.G1 * zz)], len));
            }
        }
    }
    out[c] = v;
}

static int build_kbound(const KnnIndex& ix, cudaStream_t s) {
    const long long ncell = (long long)ix.G[0] * ix.G[1] * ix.G[2];
    KnnGrid g{ix.G[0], ix.G[1], ix.G[2], ix.lo[0], ix.lo[1], ix.lo[2], ix.h, ix.inv_h};
    DWG_TRY(ix.kb.reserve(ncell));
    DWG_TRY(ix.kb_tmp.reserve(ncell));
    const unsigned char* occ1 = ix.levels >= 1 ? ix.occ.ptr + ix.loff[1] : nullptr;
    k_kb_local<<<div_up(ncell, 128), 128, 0, s>>>(g, ix.cell_start.ptr, ix.pts.ptr, occ1, ix.ldim[1][0], ix.ldim[1][1],
                                                   ix.kb.ptr);
    DWG_CHECK_LAUNCH();
    const int gmax = max(ix.G[0], max(ix.G[1], ix.G[2]));
    int step = 1;
    while (step * 2 < gmax) step *= 2;
    std::vector<int> steps;
    for (int st = step; st >= 1; st /= 2) steps.push_back(st);
    steps.push_back(1);
    steps.push_back(1);
    float* a = ix.kb.ptr;
    float* b = ix.kb_tmp.ptr;
    for (int st : steps) {
        const double hs = (double)st * (double)ix.h;
        const float l1 = nextafterf((float)hs, INFINITY);
        const float l2 = nextafterf((float)(hs * 1.4142135623730951), INFINITY);
        const float l3 = nextafterf((float)(hs * 1.7320508075688772), INFINITY);
        k_kb_jfa<<<div_up(ncell, 256), 256, 0, s>>>(g, a, b, st, l1, l2, l3);
        DWG_CHECK_LAUNCH();
        std::swap(a, b);
    }
    if (a != ix.kb.ptr)
        DWG_CHECK_CUDA(cudaMemcpyAsync(ix.kb.ptr, a, sizeof(float) * ncell, cudaMemcpyDeviceToDevice, s));
    ix.kb_ready = true;
    return DWG_OK;
}

// cell of every query, queries per cell, largest |q - x_c| per cell
// with seeds, sbits[c] gets the largest |q - x_c| + seed radius over the
// cell's queries (+inf when one has no seed): the k nearest of every query of
// the cell lie within it of the centre
__global__ void k_cq_key(KnnArgs a, int* __restrict__ key, int* __restrict__ count, unsigned int* __restrict__ mbits,
                         unsigned int* __restrict__ sbits) {
    if (a.gate_count && *a.gate_count <= a.gate_min) return;
    const long long nq = knn_count(a);
    for (long long qi = blockIdx.x * (long long)blockDim.x + threadIdx.x; qi < nq;
         qi += (long long)gridDim.x * blockDim.x) {
        float qx, qy, qz;
        knn_load_query(a, qi, qx, qy, qz);
        const int cx = cell_coord(qx, a.g.lo0, a.g.inv_h, a.g.G0);
        const int cy = cell_coord(qy, a.g.lo1, a.g.inv_h, a.g.G1);
        const int cz = cell_coord(qz, a.g.lo2, a.g.inv_h, a.g.G2);
        const int c = cx + a.g.G0 * (cy + a.g.G1 * cz);
        const float ex = qx - cell_mid(a.g.lo0, cx, a.g.h), ey = qy - cell_mid(a.g.lo1, cy, a.g.h),
                    ez = qz - cell_mid(a.g.lo2, cz, a.g.h);
        const float m = sqrtf(ex * ex + ey * ey + ez * ez) * 1.00002f + 1e-7f;
        key[qi] = c;
        atomicAdd(&count[c], 1);
        atomicMax(&mbits[c], __float_as_uint(m));  // non-negative floats order as their bits
        if (sbits) atomicMax(&sbits[c], __float_as_uint((m + seed_radius(a.seed[qi])) * 1.00002f));
    }
}

__global__ void k_cq_active(const int* __restrict__ count, long long ncell, int* __restrict__ active,
                            int* __restrict__ nactive) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= ncell || count[c] == 0) return;
    active[atomicAdd(nactive, 1)] = (int)c;
}

__global__ void k_cq_scatter(KnnArgs a, const int* __restrict__ key, int* __restrict__ fill, int* __restrict__ order) {
    if (a.gate_count && *a.gate_count <= a.gate_min) return;
    const long long nq = knn_count(a);
    for (long long qi = blockIdx.x * (long long)blockDim.x + threadIdx.x; qi < nq;
         qi += (long long)gridDim.x * blockDim.x)
        order[atomicAdd(&fill[key[qi]], 1)] = (int)qi;
}

// is the node (ni, nj, nk) of level l non-empty and within R of (x, y, z)?
__device__ __forceinline__ bool cq_node_hit(const KnnArgs& a, int l, int ni, int nj, int nk, float x, float y,
                                            float z, float R2, float eps) {
    const int* D = a.ldim[l];
    if (ni < 0 || nj < 0 || nk < 0 || ni >= D[0] || nj >= D[1] || nk >= D[2]) return false;
    const float h = a.g.h;
    const float x0 = a.g.lo0 + (float)(ni << l) * h - eps, x1 = a.g.lo0 + (float)((ni + 1) << l) * h + eps;
    const float y0 = a.g.lo1 + (float)(nj << l) * h - eps, y1 = a.g.lo1 + (float)((nj + 1) << l) * h + eps;
    const float z0 = a.g.lo2 + (float)(nk << l) * h - eps, z1 = a.g.lo2 + (float)((nk + 1) << l) * h + eps;
    const float ddx = fmaxf(0.f, fmaxf(x0 - x, x - x1));
    const float ddy = fmaxf(0.f, fmaxf(y0 - y, y - y1));
    const float ddz = fmaxf(0.f, fmaxf(z0 - z, z - z1));
    if (ddx * ddx + ddy * ddy + ddz * ddz > R2) return false;
    if (l == 0) {
        const int c = ni + a.g.G0 * (nj + a.g.G1 * nk);
        return a.cell_start[c + 1] > a.cell_start[c];
    }
    return a.occ[a.loff[l] + ni + (long long)D[0] * (nj + (long long)D[1] * nk)] != 0;
}

template <int KMAX>
__global__ void __launch_bounds__(kCqWarps * 32) k_knn_cells(KnnArgs a, const int* __restrict__ active,
                                                             const int* __restrict__ misc,
                                                             const int* __restrict__ cstart,
                                                             const int* __restrict__ ccount,
                                                             const unsigned int* __restrict__ mbits,
                                                             const unsigned int* __restrict__ sbits,
                                                             const float* __restrict__ kb,
                                                             const int* __restrict__ order,
                                                             int* __restrict__ work, int* __restrict__ fb) {
    __shared__ int nodes[kCqWarps][2][kCqNodes];
    __shared__ float4 stage[kCqWarps][kCqChunk];
    if (a.gate_count && *a.gate_count <= a.gate_min) return;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    const int nactive = misc[0];
    const unsigned long long NONE = ~0ull;
    const float h = a.g.h;
    const float eps = 1e-4f * h + 1e-6f;
    const int k = a.k;
    for (;;) {
        int wi = 0;
        if (lane == 0) wi = atomicAdd(&work[0], 1);
        wi = __shfl_sync(FULL, wi, 0);
        if (wi >= nactive) break;
        const int c = active[wi];
        const int ci = c % a.g.G0, cj = (c / a.g.G0) % a.g.G1, ck = c / (a.g.G0 * a.g.G1);
        const float x = cell_mid(a.g.lo0, ci, h), y = cell_mid(a.g.lo1, cj, h), z = cell_mid(a.g.lo2, ck, h);
        const int qs = cstart[c], qn = ccount[c];
        float R = (kb[c] + 2.0f * __uint_as_float(mbits[c])) * 1.00002f + 1e-6f * h;
        if (sbits) R = fminf(R, __uint_as_float(sbits[c]) * 1.00002f + 1e-6f * h);
        bool ok = isfinite(R);
        int* cur = nodes[w][0];
        int nf = 0;
        int l = 0;   // the level the frontier starts at
        int fl = 0;  // the level it ends at (cells are streamed from there)
        if (ok) {
            const float R2 = R * R;
            // the ball's box in cells
            const int x0 = cell_coord(x - R, a.g.lo0, a.g.inv_h, a.g.G0), x1 = cell_coord(x + R, a.g.lo0, a.g.inv_h, a.g.G0);
            const int y0 = cell_coord(y - R, a.g.lo1, a.g.inv_h, a.g.G1), y1 = cell_coord(y + R, a.g.lo1, a.g.inv_h, a.g.G1);
            const int z0 = cell_coord(z - R, a.g.lo2, a.g.inv_h, a.g.G2), z1 = cell_coord(z + R, a.g.lo2, a.g.inv_h, a.g.G2);
            // coarsest-enough level: the nodes covering the box fit the frontier
            for (;;) {
                const long long nn = (long long)((x1 >> l) - (x0 >> l) + 1) * ((y1 >> l) - (y0 >> l) + 1) *
                                     ((z1 >> l) - (z0 >> l) + 1);
                if (nn <= kCqNodes || l >= a.levels) break;
                ++l;
            }
            const int bx = (x1 >> l) - (x0 >> l) + 1, by = (y1 >> l) - (y0 >> l) + 1, bz = (z1 >> l) - (z0 >> l) + 1;
            const int tot = bx * by * bz;
            int* nxt = nodes[w][1];
            // stage A: the nodes of level l covering the box
            for (int b = 0; b < tot; b += 32) {
                const int t = b + lane;
                bool keep = false;
                int id = 0;
                if (t < tot) {
                    const int ni = (x0 >> l) + t % bx, nj = (y0 >> l) + (t / bx) % by, nk = (z0 >> l) + t / (bx * by);
                    keep = cq_node_hit(a, l, ni, nj, nk, x, y, z, R2, eps);
                    id = ni + a.ldim[l][0] * (nj + a.ldim[l][1] * nk);
                }
                const unsigned bal = __ballot_sync(FULL, keep);
                const int pos = nf + __popc(bal & below);
                if (keep && pos < kCqNodes) cur[pos] = id;
                nf += __popc(bal);
            }
            ok = nf <= kCqNodes;
            // stage B: down to level 1 (the cells are expanded while
            // streaming); when the next level would not fit, the frontier
            // stays at the coarser level and its nodes' cells are streamed
            fl = l;
            for (int lv = l; lv >= 2 && ok; --lv) {
                __syncwarp();
                const int* D = a.ldim[lv];
                int nn = 0;
                for (int b = 0; b < nf * 8; b += 32) {
                    const int t = b + lane;
                    bool keep = false;
                    int id = 0;
                    if (t < nf * 8) {
                        const int node = cur[t >> 3], oc = t & 7;
                        const int ni = node % D[0], nj = (node / D[0]) % D[1], nk = node / (D[0] * D[1]);
                        const int ui = 2 * ni + (oc & 1), uj = 2 * nj + ((oc >> 1) & 1), uk = 2 * nk + (oc >> 2);
                        keep = cq_node_hit(a, lv - 1, ui, uj, uk, x, y, z, R2, eps);
                        id = ui + a.ldim[lv - 1][0] * (uj + a.ldim[lv - 1][1] * uk);
                    }
                    const unsigned bal = __ballot_sync(FULL, keep);
                    const int pos = nn + __popc(bal & below);
                    if (keep && pos < kCqNodes) nxt[pos] = id;
                    nn += __popc(bal);
                }
                if (nn > kCqNodes) break;  // keep the level-lv frontier
                int* tmp = cur;
                cur = nxt;
                nxt = tmp;
                nf = nn;
                fl = lv - 1;
            }
            __syncwarp();
        }
        // a ball so large that the frontier stayed coarse, for a handful of
        // queries: the per-thread search, seeded with each query's own bound,
        // prunes it faster than the warp streams it
        if (ok && fl >= 2 && qn < 8) ok = false;
        if (!ok) {  // the per-thread search takes this cell's queries
            for (int t = lane; t < qn; t += 32) fb[atomicAdd(&work[1], 1)] = order[qs + t];
            continue;
        }
        // stages C + D, per chunk of up to 32 queries: the points of the
        // frontier cells within R of the centre are streamed through shared
        // memory and ranked for every query, starting from the bound
        // kb[c] + |q - x_c| on its 16th distance.  A chunk of nb queries gives
        // each query G lanes (the largest power of two with nb * G <= 32): a
        // lane ranks every G-th staged point for its query, and the G lanes'
        // sets are merged at the end.  Cells hold a few queries, so this
        // keeps the lanes busy instead of ranking for absent queries.
        const float kbc = kb[c];
        const float R2 = R * R;
        for (int base = 0; base < qn; base += 32) {
            const int nb = qn - base < 32 ? qn - base : 32;
            const int lg = nb > 16 ? 0 : nb > 8 ? 1 : nb > 4 ? 2 : nb > 2 ? 3 : nb > 1 ? 4 : 5;
            const int G = 1 << lg;
            const int u = lane >> lg, sl = lane & (G - 1);
            const bool has = u < nb;
            long long qi = 0;
            float qx = x, qy = y, qz = z;
            if (has) {
                qi = order[qs + base + u];
                knn_load_query(a, qi, qx, qy, qz);
            }
            const float ex = qx - x, ey = qy - y, ez = qz - z;
            const float rq = (kbc + sqrtf(ex * ex + ey * ey + ez * ez) * 1.00002f) * 1.00002f + 1e-7f;
            unsigned long long T = ((unsigned long long)__float_as_uint(rq * rq * 1.00002f) << 32) | 0xffffffffull;
            if (a.seed && has) {
                const unsigned long long sd = a.seed[qi];
                T = sd < T ? sd : T;
            }
            TopK<KMAX> top;
            top.init_bound(k, T);
            int staged = 0;
            auto rank = [&]() {
                __syncwarp();
                if (has) {
                    for (int t = sl; t < staged; t += G) {
                        const float4 pp = stage[w][t];
                        const float d2 = sq3_rn(__fsub_rn(pp.x, qx), __fsub_rn(pp.y, qy), __fsub_rn(pp.z, qz));
                        const unsigned long long v = ((unsigned long long)__float_as_uint(d2) << 32) |
                                                     (unsigned)__float_as_int(pp.w);
                        if (v < top.mx) top.push(v, k);
                    }
                }
                __syncwarp();
                staged = 0;
            };
            // frontier entries are cells (level 0) or nodes of level fl,
            // cubes of side 2^fl cells
            const int side = 1 << fl;
            const long long per = (long long)side * side * side;
            const long long total = (long long)nf * per;
            for (long long b = 0; b < total; b += 32) {
                const long long t = b + lane;
                int s0 = 0, cnt = 0;
                if (t < total) {
                    int cell;
                    bool hit = true;
                    if (fl == 0) {
                        cell = cur[t];
                    } else {
                        const int* D = a.ldim[fl];
                        const int node = cur[t / per];
                        const int o = (int)(t % per);
                        const int ni = node % D[0], nj = (node / D[0]) % D[1], nk = node / (D[0] * D[1]);
                        const int ui = ni * side + o % side, uj = nj * side + (o / side) % side,
                                  uk = nk * side + o / (side * side);
                        hit = cq_node_hit(a, 0, ui, uj, uk, x, y, z, R2, eps);
                        cell = ui + a.g.G0 * (uj + a.g.G1 * uk);
                    }
                    if (hit) {
                        s0 = a.cell_start[cell];
                        cnt = a.cell_start[cell + 1] - s0;
                    }
                }
                // the points of the 32 cells as one list that the lanes walk
                // together, a lane per point (not a lane per cell, which
                // would idle the warp on the fullest cell)
                int incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += v;
                }
                const int excl = incl - cnt;
                const int tot = __shfl_sync(FULL, incl, 31);
                for (int pb = 0; pb < tot; pb += 32) {
                    const int tp = pb + lane;
                    // owner of list position tp: the last lane whose range starts at or before it
                    int own = 0;
#pragma unroll
                    for (int st = 16; st > 0; st >>= 1) {
                        const int e = __shfl_sync(FULL, excl, own + st);
                        if (e <= tp) own += st;
                    }
                    const int os0 = __shfl_sync(FULL, s0, own);
                    const int oex = __shfl_sync(FULL, excl, own);
                    bool keep = false;
                    float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (tp < tot) {
                        p = a.pts[os0 + (tp - oex)];
                        const float px = p.x - x, py = p.y - y, pz = p.z - z;
                        keep = px * px + py * py + pz * pz <= R2;
                    }
                    const unsigned bal = __ballot_sync(FULL, keep);
                    if (keep) stage[w][staged + __popc(bal & below)] = p;
                    staged += __popc(bal);
                    if (staged > kCqChunk - 32) rank();
                }
            }
            if (staged > 0) rank();
            top.sort();
            if (G == 1) {
                if (has) {
#pragma unroll
                    for (int t = 0; t < KMAX; ++t) {
                        const int o = t - (KMAX - k);
                        if (o >= 0)
                            a.out[qi * k + o] = top.e[t] == NONE ? -1 : (int)(unsigned)(top.e[t] & 0xffffffffu);
                    }
                }
            } else {
                // slots >= k hold 0 and sort first: drop them, then k rounds
                // of the minimum over the G lanes' smallest keys (aligned
                // groups, so the butterfly stays inside the group); the lane
                // holding it drops it.  Keys are unique (one index each), the
                // initial key T and NONE aside, which give -1 as before.
#pragma unroll 1
                for (int z = 0; z < KMAX - k; ++z) top.shift_down();
#pragma unroll 1
                for (int r = 0; r < k; ++r) {
                    unsigned long long m = top.e[0];
                    for (int o = 1; o < G; o <<= 1) {
                        const unsigned long long v = __shfl_xor_sync(FULL, m, o);
                        m = v < m ? v : m;
                    }
                    if (top.e[0] == m) top.shift_down();
                    if (has && sl == 0) a.out[qi * k + r] = m == NONE ? -1 : (int)(unsigned)(m & 0xffffffffu);
                }
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------ deep queries --
// The queries whose per-thread walk ran past its budget (far from every
// point, so the walk's bound tightens late), one warp per query, level by
// level down the occupancy pyramid.  The frontier holds the nodes that may
// contain one of the k nearest; a level's children come from the nodes'
// child masks, and a child stays when its (eps-widened) box is within the
// bound U of the query.  After each level U is lowered to the k-th smallest,
// over the lanes, of each lane's smallest far-corner distance among the
// children it kept: those are k distinct occupied nodes, so k points lie
// within it.  At the cells, every lane ranks the points of its share of the
// cells within U, and the 32 lanes' sets are merged.  A level whose children
// do not fit the frontier is retried once with the lowered U; if they still
// do not fit, the cells under the current level's nodes are enumerated.
constexpr int kDeepWarps = 4;
constexpr int kDeepNodes = 1024;

// k-th smallest (1 <= k <= 32) of one value per lane, to every lane
__device__ __forceinline__ float warp_kth_smallest(float v, int k) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const float o = __shfl_xor_sync(0xffffffffu, v, stride);
            const bool asc = (lane & size) == 0 || size == 32;
            const bool low = (lane & stride) == 0;
            v = (low == asc) ? fminf(v, o) : fmaxf(v, o);
        }
    }
    return __shfl_sync(0xffffffffu, v, k - 1);
}

// squared distances from q to the nearest and the farthest point of the
// eps-widened box of node (ni, nj, nk) of level l
__device__ __forceinline__ void node_d2(const KnnArgs& a, int l, int ni, int nj, int nk, float qx, float qy, float qz,
                                        float eps, float& mind2, float& maxd2) {
    const float h = a.g.h;
    const float x0 = a.g.lo0 + (float)(ni << l) * h - eps, x1 = a.g.lo0 + (float)((ni + 1) << l) * h + eps;
    const float y0 = a.g.lo1 + (float)(nj << l) * h - eps, y1 = a.g.lo1 + (float)((nj + 1) << l) * h + eps;
    const float z0 = a.g.lo2 + (float)(nk << l) * h - eps, z1 = a.g.lo2 + (float)((nk + 1) << l) * h + eps;
    const float dx = fmaxf(0.f, fmaxf(x0 - qx, qx - x1)), fx = fmaxf(qx - x0, x1 - qx);
    const float dy = fmaxf(0.f, fmaxf(y0 - qy, qy - y1)), fy = fmaxf(qy - y0, y1 - qy);
    const float dz = fmaxf(0.f, fmaxf(z0 - qz, qz - z1)), fz = fmaxf(qz - z0, z1 - qz);
    mind2 = dx * dx + dy * dy + dz * dz;
    maxd2 = fx * fx + fy * fy + fz * fz;
}

__device__ __forceinline__ int pack3(int i, int j, int k) { return i | (j << 10) | (k << 20); }

template <int KMAX>
__global__ void __launch_bounds__(kDeepWarps * 32) k_knn_deep(KnnArgs a, const int* __restrict__ list,
                                                             const float* __restrict__ bound,
                                                             const int* __restrict__ count, int* __restrict__ work) {
    __shared__ int fco[kDeepWarps][2][kDeepNodes];
    __shared__ unsigned char fmk[kDeepWarps][2][kDeepNodes];
    if (a.gate_count && *a.gate_count <= a.gate_min) return;
    const unsigned FULL = 0xffffffffu;
    const unsigned long long NONE = ~0ull;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    const int nd = *count;
    const int k = a.k;
    const float eps = 1e-4f * a.g.h + 1e-6f;
    for (;;) {
        int j = 0;
        if (lane == 0) j = atomicAdd(work, 1);
        j = __shfl_sync(FULL, j, 0);
        if (j >= nd) break;
        const long long qi = list[j];
        float qx, qy, qz;
        knn_load_query(a, qi, qx, qy, qz);
        int* cur = fco[w][0];
        unsigned char* curm = fmk[w][0];
        int* nxt = fco[w][1];
        unsigned char* nxtm = fmk[w][1];
        int lvl = a.levels;
        if (lane == 0) {
            cur[0] = 0;
            curm[0] = a.occ[a.loff[lvl]];
        }
        int nf = 1;
        float U2 = bound[j];  // from the per-thread walk
        __syncwarp();
        while (lvl > 0) {
            const int nl = lvl - 1;
            const int* D = a.ldim[nl];
            int nn = 0;
            for (int pass = 0; pass < 2; ++pass) {
                float lmin = INFINITY;
                nn = 0;
                for (int b = 0; b < nf * 8; b += 32) {
                    const int t = b + lane;
                    bool keep = false;
                    int cc = 0;
                    unsigned char cm = 0;
                    if (t < nf * 8 && ((curm[t >> 3] >> (t & 7)) & 1)) {
                        const int pc = cur[t >> 3], oc = t & 7;
                        const int ni = ((pc & 1023) << 1) | (oc & 1), nj = (((pc >> 10) & 1023) << 1) | ((oc >> 1) & 1),
                                  nk = ((pc >> 20) << 1) | (oc >> 2);
                        float mind2, maxd2;
                        node_d2(a, nl, ni, nj, nk, qx, qy, qz, eps, mind2, maxd2);
                        if (mind2 <= U2) {
                            keep = true;
                            lmin = fminf(lmin, maxd2);
                            cc = pack3(ni, nj, nk);
                            if (nl > 0) cm = a.occ[a.loff[nl] + ni + (long long)D[0] * (nj + (long long)D[1] * nk)];
                        }
                    }
                    const unsigned bal = __ballot_sync(FULL, keep);
                    const int pos = nn + __popc(bal & below);
                    if (keep && pos < kDeepNodes) {
                        nxt[pos] = cc;
                        nxtm[pos] = cm;
                    }
                    nn += __popc(bal);
                }
                const float kth = warp_kth_smallest(lmin, k);
                if (kth < INFINITY) U2 = fminf(U2, kth * 1.0001f);
                if (nn <= kDeepNodes) break;
            }
            __syncwarp();
            if (nn > kDeepNodes) break;  // the cells under this level's nodes are enumerated below
            int* ti = cur;
            cur = nxt;
            nxt = ti;
            unsigned char* tm = curm;
            curm = nxtm;
            nxtm = tm;
            nf = nn;
            lvl = nl;
        }
        // rank the points of the cells within U (cells of the frontier, or
        // under its nodes of level lvl), a lane per point of 32 cells at a time
        TopK<KMAX> top;
        if (U2 < INFINITY)
            top.init_bound(k, ((unsigned long long)__float_as_uint(U2) << 32) | 0xffffffffull);
        else
            top.init(k);
        const int side = 1 << lvl;
        const long long per = (long long)side * side * side;
        const long long total = (long long)nf * per;
        for (long long b = 0; b < total; b += 32) {
            const long long t = b + lane;
            int s0 = 0, cnt = 0;
            if (t < total) {
                const int pc = cur[t / per];
                const int o = (int)(t % per);
                const int ci = (pc & 1023) * side + o % side, cj = ((pc >> 10) & 1023) * side + (o / side) % side,
                          ck = (pc >> 20) * side + o / (side * side);
                if (ci < a.g.G0 && cj < a.g.G1 && ck < a.g.G2) {
                    float mind2, maxd2;
                    node_d2(a, 0, ci, cj, ck, qx, qy, qz, eps, mind2, maxd2);
                    if (mind2 <= U2) {
                        const int cell = ci + a.g.G0 * (cj + a.g.G1 * ck);
                        s0 = a.cell_start[cell];
                        cnt = a.cell_start[cell + 1] - s0;
                    }
                }
            }
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += v;
            }
            const int excl = incl - cnt;
            const int tot = __shfl_sync(FULL, incl, 31);
            for (int pb = 0; pb < tot; pb += 32) {
                const int tp = pb + lane;
                int own = 0;
#pragma unroll
                for (int st = 16; st > 0; st >>= 1) {
                    const int e = __shfl_sync(FULL, excl, own + st);
                    if (e <= tp) own += st;
                }
                const int os0 = __shfl_sync(FULL, s0, own);
                const int oex = __shfl_sync(FULL, excl, own);
                if (tp < tot) {
                    const float4 pp = a.pts[os0 + (tp - oex)];
                    const float d2 = sq3_rn(__fsub_rn(pp.x, qx), __fsub_rn(pp.y, qy), __fsub_rn(pp.z, qz));
                    const unsigned long long v = ((unsigned long long)__float_as_uint(d2) << 32) |
                                                 (unsigned)__float_as_int(pp.w);
                    if (v < top.mx) top.push(v, k);
                }
            }
        }
        // merge the 32 lanes' sets (as in k_knn_cells)
        top.sort();
#pragma unroll 1
        for (int z = 0; z < KMAX - k; ++z) top.shift_down();
#pragma unroll 1
        for (int r = 0; r < k; ++r) {
            unsigned long long m = top.e[0];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long v = __shfl_xor_sync(FULL, m, o);
                m = v < m ? v : m;
            }
            if (top.e[0] == m) top.shift_down();
            if (lane == 0) a.out[qi * k + r] = m == NONE ? -1 : (int)(unsigned)(m & 0xffffffffu);
        }
        __syncwarp();
    }
}

template <int KMAX>
static int knn_launch(const KnnArgs& a, long long nq, cudaStream_t s) {
    static int bps = 0;
    if (!bps) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_knn_thread<KMAX>, 128, 0);
        if (bps <= 0) bps = 1;
    }
    long long blocks = (nq + 127) / 128;
    long long cap = (long long)num_sms() * bps;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    k_knn_thread<KMAX><<<(unsigned)blocks, 128, 0, s>>>(a);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

template <int KMAX>
static int cells_launch(const KnnIndex& ix, const KnnArgs& a, long long nq, const unsigned int* sbits,
                        cudaStream_t s) {
    static int bps = 0;
    if (!bps) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_knn_cells<KMAX>, kCqWarps * 32, 0);
        if (bps <= 0) bps = 1;
    }
    const long long grid = (long long)num_sms() * bps;
    k_knn_cells<KMAX><<<(unsigned)grid, kCqWarps * 32, 0, s>>>(
        a, ix.c_active.ptr, ix.c_misc.ptr, ix.c_start.ptr, ix.c_count.ptr, ix.c_m.ptr, sbits, ix.kb.ptr, ix.q_order.ptr,
        ix.c_misc.ptr + 1, ix.c_fb.ptr);
    DWG_CHECK_LAUNCH();
    // the queries of cells whose candidate sets did not fit, per thread;
    // those far from every point finish one warp each
    KnnArgs f = a;
    f.order = ix.c_fb.ptr;
    f.nq_dev_i32 = ix.c_misc.ptr + 2;
    f.kb = ix.kb.ptr;
    f.deep = ix.levels > 0 ? ix.c_deep.ptr : nullptr;
    f.deep_bound = ix.c_deep_bound.ptr;
    f.deep_count = ix.c_misc.ptr + 3;
    DWG_TRY(knn_launch<KMAX>(f, nq, s));
    if (f.deep) {
        static int dbps = 0;
        if (!dbps) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&dbps, k_knn_deep<KMAX>, kDeepWarps * 32, 0);
            if (dbps <= 0) dbps = 1;
        }
        k_knn_deep<KMAX><<<(unsigned)(num_sms() * dbps), kDeepWarps * 32, 0, s>>>(
            f, ix.c_deep.ptr, ix.c_deep_bound.ptr, ix.c_misc.ptr + 3, ix.c_misc.ptr + 4);
        DWG_CHECK_LAUNCH();
    }
    return DWG_OK;
}

// queries grouped by cell (k <= 16, no exclusion), see k_knn_cells
static int knn_query_cells(const KnnIndex& ix, const KnnArgs& a0, long long nq, cudaStream_t s) {
    if (!ix.kb_per_query && !ix.kb_ready) DWG_TRY(build_kbound(ix, s));
    const long long ncell = (long long)ix.G[0] * ix.G[1] * ix.G[2];
    DWG_TRY(ix.c_count.reserve(ncell + 1));
    DWG_TRY(ix.c_start.reserve(ncell + 1));
    DWG_TRY(ix.c_fill.reserve(ncell + 1));
    DWG_TRY(ix.c_m.reserve(ncell));
    DWG_TRY(ix.c_active.reserve(ncell));
    DWG_TRY(ix.c_misc.reserve(8));
    DWG_TRY(ix.q_key.reserve(nq));
    DWG_TRY(ix.q_order.reserve(nq));
    DWG_TRY(ix.c_fb.reserve(nq));
    DWG_TRY(ix.c_deep.reserve(nq));
    DWG_TRY(ix.c_deep_bound.reserve(nq));
    DWG_CHECK_CUDA(cudaMemsetAsync(ix.c_count.ptr, 0, sizeof(int) * (ncell + 1), s));
    DWG_CHECK_CUDA(cudaMemsetAsync(ix.c_m.ptr, 0, sizeof(unsigned int) * ncell, s));
    unsigned int* sbits = nullptr;
    if (a0.seed) {
        DWG_TRY(ix.c_s.reserve(ncell));
        DWG_CHECK_CUDA(cudaMemsetAsync(ix.c_s.ptr, 0, sizeof(unsigned int) * ncell, s));
        sbits = ix.c_s.ptr;
    }
    DWG_CHECK_CUDA(cudaMemsetAsync(ix.c_misc.ptr, 0, sizeof(int) * 8, s));
    KnnArgs a = a0;
    long long blocks = (nq + 255) / 256;
    const long long cap = (long long)num_sms() * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    k_cq_key<<<(unsigned)blocks, 256, 0, s>>>(a, ix.q_key.ptr, ix.c_count.ptr, ix.c_m.ptr, sbits);
    DWG_CHECK_LAUNCH();
    size_t bytes = 0;
    int* cin = ix.c_count.ptr;
    int* cout = ix.c_start.ptr;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cin, cout, (int)(ncell + 1), s));
    DWG_TRY(ix.c_scratch.reserve(bytes + 256));
    bytes = ix.c_scratch.n;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(ix.c_scratch.ptr, bytes, cin, cout, (int)(ncell + 1), s));
    DWG_CHECK_CUDA(cudaMemcpyAsync(ix.c_fill.ptr, ix.c_start.ptr, sizeof(int) * (ncell + 1), cudaMemcpyDeviceToDevice, s));
    k_cq_active<<<div_up(ncell, 256), 256, 0, s>>>(ix.c_count.ptr, ncell, ix.c_active.ptr, ix.c_misc.ptr);
    if (ix.kb_per_query) {
        DWG_TRY(ix.kb.reserve(ncell));
        KnnGrid g{ix.G[0], ix.G[1], ix.G[2], ix.lo[0], ix.lo[1], ix.lo[2], ix.h, ix.inv_h};
        const unsigned char* occ1 = ix.levels >= 1 ? ix.occ.ptr + ix.loff[1] : nullptr;
        k_kb_active<<<num_sms() * 4, 128, 0, s>>>(g, ix.cell_start.ptr, ix.pts.ptr, occ1, ix.ldim[1][0],
                                                  ix.ldim[1][1], ix.c_active.ptr, ix.c_misc.ptr, sbits, ix.kb.ptr);
    }
    k_cq_scatter<<<(unsigned)blocks, 256, 0, s>>>(a, ix.q_key.ptr, ix.c_fill.ptr, ix.q_order.ptr);
    DWG_CHECK_LAUNCH();
    // k = 15 (the triangle queries) keeps 15 slots per lane instead of 16 and
    // k <= 10 (the zero repair) 10: every maximum search and the final sort
    // are shorter, and the lanes hold fewer registers
    if (a.k == 15) return cells_launch<15>(ix, a, nq, sbits, s);
    if (a.k <= 10) return cells_launch<10>(ix, a, nq, sbits, s);
    return cells_launch<16>(ix, a, nq, sbits, s);
}

// ------------------------------------------------------------- subsets --
__global__ void k_sub_count(long long ncell, const int* __restrict__ cs, const float4* __restrict__ pts,
                            const unsigned char* __restrict__ exclude, int* __restrict__ count) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c > ncell) return;
    int m = 0;
    if (c < ncell) {
        const int e = cs[c + 1];
        for (int t = cs[c]; t < e; ++t) m += exclude[__float_as_int(pts[t].w)] ? 0 : 1;
    }
    count[c] = m;  // count[ncell] = 0 closes the scan
}

__global__ void k_sub_fill(long long ncell, const int* __restrict__ cs, const float4* __restrict__ pts,
                           const unsigned char* __restrict__ exclude, const int* __restrict__ sub_start,
                           float4* __restrict__ sub_pts) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    int o = sub_start[c];
    const int e = cs[c + 1];
    for (int t = cs[c]; t < e; ++t) {
        const float4 p = pts[t];
        if (!exclude[__float_as_int(p.w)]) sub_pts[o++] = p;
    }
}

int knn_build_subset(const KnnIndex& full, const unsigned char* exclude, KnnIndex& sub, cudaStream_t s) {
    DWG_REQUIRE(exclude && full.n >= 1, "knn subset: bad arguments");
    const long long ncell = (long long)full.G[0] * full.G[1] * full.G[2];
    if (sub.n != full.n || sub.G[0] != full.G[0] || sub.G[1] != full.G[1] || sub.G[2] != full.G[2]) {
        sub.n = full.n;  // an upper bound; the kept count stays on the device
        for (int d = 0; d < 3; ++d) {
            sub.G[d] = full.G[d];
            sub.lo[d] = full.lo[d];
        }
        sub.h = full.h;
        sub.inv_h = full.inv_h;
        sub.morton_shift = full.morton_shift;
        DWG_TRY(sub.cell_start.reserve(ncell + 1));
        DWG_TRY(sub.cell_fill.reserve(ncell + 1));
        DWG_TRY(sub.pts.reserve(full.n));
        DWG_TRY(sub.bbox.reserve(6));
        DWG_CHECK_CUDA(cudaMemcpyAsync(sub.bbox.ptr, full.bbox.ptr, sizeof(float) * 6, cudaMemcpyDeviceToDevice, s));
        DWG_TRY(pyramid_dims(sub));
        size_t bytes = 0;
        DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, sub.cell_fill.ptr, sub.cell_start.ptr,
                                                     (int)(ncell + 1), s));
        DWG_TRY(sub.scratch.reserve(bytes + 256));
    }
    k_sub_count<<<div_up(ncell + 1, 256), 256, 0, s>>>(ncell, full.cell_start.ptr, full.pts.ptr, exclude,
                                                       sub.cell_fill.ptr);
    DWG_CHECK_LAUNCH();
    size_t bytes = sub.scratch.n;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(sub.scratch.ptr, bytes, sub.cell_fill.ptr, sub.cell_start.ptr,
                                                 (int)(ncell + 1), s));
    k_sub_fill<<<div_up(ncell, 256), 256, 0, s>>>(ncell, full.cell_start.ptr, full.pts.ptr, exclude,
                                                  sub.cell_start.ptr, sub.pts.ptr);
    DWG_CHECK_LAUNCH();
    DWG_TRY(pyramid_fill(sub, s));
    // the subset changes between queries.  The whole-grid bound (local blocks
    // plus min-plus passes) costs in proportion to the grid, empty space
    // included; past 2^22 cells the bounds of the queried cells alone are
    // cheaper, at the price of sending the queries of sparse neighbourhoods
    // to the per-thread search
    sub.kb_ready = false;
    sub.kb_per_query = ncell > (1ll << 22);
    if (!sub.kb_per_query) return build_kbound(sub, s);
    return DWG_OK;
}

constexpr int kKnnBuckets = 1 << 15;

int knn_query(const KnnIndex& ix, const KnnQuery& q, int k, int* out, cudaStream_t s) {
    DWG_REQUIRE(k >= 1 && k <= 64, "knn: k must be in [1, 64] (got %d)", k);
    DWG_REQUIRE(out != nullptr, "knn: output is null");
    DWG_REQUIRE(q.q || (q.q_index && q.q_source), "knn: no queries");
    if (q.nq <= 0) return DWG_OK;
    KnnArgs a;
    a.g = KnnGrid{ix.G[0], ix.G[1], ix.G[2], ix.lo[0], ix.lo[1], ix.lo[2], ix.h, ix.inv_h};
    a.pts = ix.pts.ptr;
    a.cell_start = ix.cell_start.ptr;
    a.q = q.q;
    a.q_index = q.q_index;
    a.q_source = q.q_source;
    a.nq = q.nq;
    a.nq_dev = q.nq_dev;
    a.nq_dev_i32 = q.nq_dev_i32;
    a.exclude = q.exclude;
    a.gate_count = q.gate_count;
    a.gate_min = q.gate_min;
    a.k = k;
    a.out = out;
    a.morton_shift = ix.morton_shift;
    a.occ = ix.occ.ptr;
    a.levels = ix.levels;
    for (int l = 0; l < KnnIndex::kMaxLevels; ++l) {
        a.loff[l] = ix.loff[l];
        for (int t = 0; t < 3; ++t) a.ldim[l][t] = ix.ldim[l][t];
    }
    a.order = nullptr;
    a.kb = nullptr;
    a.deep = nullptr;
    a.deep_bound = nullptr;
    a.deep_count = nullptr;
    a.seed = q.seed;
    if (k <= kKnnBoundK && !q.exclude && ix.n >= kKnnBoundK && q.use_cells) return knn_query_cells(ix, a, q.nq, s);
    // bucket the queries spatially (counting sort on device counts, no host sync)
    DWG_TRY(ix.q_key.reserve(q.nq));
    DWG_TRY(ix.q_order.reserve(q.nq));
    DWG_TRY(ix.q_hist.reserve(kKnnBuckets));
    DWG_TRY(ix.q_fill.reserve(kKnnBuckets));
    a.q_key = ix.q_key.ptr;
    a.q_hist = ix.q_hist.ptr;
    a.order = nullptr;
    DWG_CHECK_CUDA(cudaMemsetAsync(ix.q_hist.ptr, 0, sizeof(int) * kKnnBuckets, s));
    long long blocks = (q.nq + 255) / 256;
    long long cap = (long long)num_sms() * 8;
    if (blocks > cap) blocks = cap;
    k_knn_qkey<<<(unsigned)blocks, 256, 0, s>>>(a);
    DWG_CHECK_LAUNCH();
    size_t bytes = 0;
    int* hin = ix.q_hist.ptr;
    int* hout = ix.q_fill.ptr;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, hin, hout, kKnnBuckets, s));
    DWG_TRY(ix.q_scratch.reserve(bytes + 256));
    bytes = ix.q_scratch.n;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(ix.q_scratch.ptr, bytes, hin, hout, kKnnBuckets, s));
    k_knn_qscatter<<<(unsigned)blocks, 256, 0, s>>>(a, ix.q_fill.ptr, ix.q_order.ptr);
    DWG_CHECK_LAUNCH();
    a.order = ix.q_order.ptr;
    if (k <= 10) return knn_launch<10>(a, q.nq, s);
    if (k <= 16) return knn_launch<16>(a, q.nq, s);
    if (k <= 32) return knn_launch<32>(a, q.nq, s);
    return knn_launch<64>(a, q.nq, s);
}

}  // namespace dwg
