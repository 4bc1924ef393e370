// mc.cu -- marching cubes, two passes with cell-ordered (deterministic) output.
//
// The reference (src/TurboMC.cu:383-478) launches one 12-thread block per cell
// and appends triangles at atomicAdd slots.  Here pass 1 classifies 256 cells
// per block and reduces the triangle counts; a scan over blocks gives every
// block its output offset; pass 2 re-classifies, scans counts inside the block
// and writes each triangle at its final position, so the triangle order is
// the cell order (x fastest) -- identical from run to run.
//
// Conventions kept from the reference: corner c of cell (x,y,z) sits at
// (x + (b0 != b1), y + b1, z + !b2) (src/TurboMC.cu:408-413); bit c of the case
// index is set when the corner value is above the iso value (:418-425); edge e
// joins corners (e & 7, e<4 ? (e+1)&3 : e<8 ? 4+((e-3)&3) : e-4) (:433-434);
// vertex = P1 - l (P2 - P1), l = (v1 - iso)/(v2 - v1 + 1e-10) (:373-381);
// centroid = mean of the vertices; normal = -cross/(|cross| + 1e-8) (:453-470).
// The case table is generated (mc_tables_host), not transcribed.
#include <cub/cub.cuh>

#include <mutex>

#include "mc.cuh"

namespace dwg {

__constant__ signed char c_tri[256][16];
__constant__ unsigned char c_ntri[256];
__constant__ unsigned short c_edges[256];

static const int kCorner[8][3] = {{0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1},
                                  {0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}};
static int edge_a(int e) { return e & 7; }
static int edge_b(int e) { return e < 4 ? ((e + 1) & 3) : (e < 8 ? 4 + ((e - 3) & 3) : e - 4); }

// Case table from the cube geometry: on each face the crossing edges pair up
// into segments (an ambiguous face cuts off its two corners above the iso
// value); segments are oriented so that, looking at the face from outside with
// its corners counter-clockwise, a segment starts at the crossing entered from
// a corner below the iso value; the closed loops are fanned from their lowest
// edge.  These loops and per-case triangle counts equal the reference table's.
void mc_tables_host(int* edge_table, signed char* tri_table) {
    int face[6][4];
    int nf = 0;
    for (int axis = 0; axis < 3; ++axis)
        for (int val = 0; val < 2; ++val) {
            int cs[4], k = 0;
            for (int c = 0; c < 8; ++c)
                if (kCorner[c][axis] == val) cs[k++] = c;
            int o[4] = {cs[0], -1, -1, -1};
            for (int i = 1; i < 4; ++i)
                for (int j = 0; j < 4; ++j) {
                    int c = cs[j];
                    bool used = false;
                    for (int u = 0; u < i; ++u) used |= (o[u] == c);
                    int dist = 0;
                    for (int d = 0; d < 3; ++d) dist += abs(kCorner[c][d] - kCorner[o[i - 1]][d]);
                    if (!used && dist == 1) {
                        o[i] = c;
                        break;
                    }
                }
            // (o1 - o0) x (o2 - o1) must point along the outward normal
            int a[3], b[3];
            for (int d = 0; d < 3; ++d) {
                a[d] = kCorner[o[1]][d] - kCorner[o[0]][d];
                b[d] = kCorner[o[2]][d] - kCorner[o[1]][d];
            }
            int cr[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
            if (cr[axis] * (val ? 1 : -1) < 0) {
                int tmp = o[1];
                o[1] = o[3];
                o[3] = tmp;
            }
            for (int i = 0; i < 4; ++i) face[nf][i] = o[i];
            ++nf;
        }
    auto edge_of = [](int p, int q) {
        for (int e = 0; e < 12; ++e)
            if ((edge_a(e) == p && edge_b(e) == q) || (edge_a(e) == q && edge_b(e) == p)) return e;
        return -1;
    };
    for (int ci = 0; ci < 256; ++ci) {
        int above[8];
        for (int c = 0; c < 8; ++c) above[c] = (ci >> c) & 1;
        int mask = 0;
        for (int e = 0; e < 12; ++e)
            if (above[edge_a(e)] != above[edge_b(e)]) mask |= 1 << e;
        edge_table[ci] = mask;
        int next[12];
        for (int e = 0; e < 12; ++e) next[e] = -1;
        for (int f = 0; f < 6; ++f) {
            int ce[4], from_above[4], n = 0;
            for (int k = 0; k < 4; ++k) {
                int p = face[f][k], q = face[f][(k + 1) & 3];
                if (above[p] != above[q]) {
                    ce[n] = edge_of(p, q);
                    from_above[n] = above[p];
                    ++n;
                }
            }
            int seg[2][2], ns = 0;
            if (n == 2) {
                seg[0][0] = 0;
                seg[0][1] = 1;
                ns = 1;
            } else if (n == 4) {
                if (above[face[f][0]]) {
                    seg[0][0] = 3; seg[0][1] = 0;
                    seg[1][0] = 1; seg[1][1] = 2;
                } else {
                    seg[0][0] = 0; seg[0][1] = 1;
                    seg[1][0] = 2; seg[1][1] = 3;
                }
                ns = 2;
            }
            for (int k = 0; k < ns; ++k) {
                int x = seg[k][0], y = seg[k][1];
                if (!from_above[x])
                    next[ce[x]] = ce[y];
                else
                    next[ce[y]] = ce[x];
            }
        }
        signed char* row = tri_table + ci * 16;
        int wpos = 0;
        bool seen[12] = {false};
        for (int e = 0; e < 12; ++e) {
            if (next[e] < 0 || seen[e]) continue;
            int loop[12], len = 0, c = e;
            do {
                loop[len++] = c;
                seen[c] = true;
                c = next[c];
            } while (c != e && len < 12);
            for (int k = 1; k + 1 < len; ++k) {
                row[wpos] = (signed char)loop[0];
                row[wpos + 1] = (signed char)loop[k];
                row[wpos + 2] = (signed char)loop[k + 1];
                wpos += 3;
            }
        }
        for (; wpos < 16; ++wpos) row[wpos] = -1;
    }
}

int mc_upload_tables() {
    static bool done[64] = {false};
    int dev = 0;
    DWG_CHECK_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && done[dev]) return DWG_OK;
    int et[256];
    signed char tt[256 * 16];
    mc_tables_host(et, tt);
    unsigned char nt[256];
    unsigned short es[256];
    for (int i = 0; i < 256; ++i) {
        int k = 0;
        while (k < 16 && tt[i * 16 + k] >= 0) k += 3;
        nt[i] = (unsigned char)(k / 3);
        es[i] = (unsigned short)et[i];
    }
    DWG_CHECK_CUDA(cudaMemcpyToSymbol(c_tri, tt, sizeof(tt)));
    DWG_CHECK_CUDA(cudaMemcpyToSymbol(c_ntri, nt, sizeof(nt)));
    DWG_CHECK_CUDA(cudaMemcpyToSymbol(c_edges, es, sizeof(es)));
    if (dev >= 0 && dev < 64) done[dev] = true;
    return DWG_OK;
}

constexpr int kMcThreads = 256;

struct McArgs {
    const float* __restrict__ field;
    const float* __restrict__ pos;
    int rx, ry, rz;
    long long ncell;
    float ox, oy, oz, h;
    int zoff;  // global z index of local sample 0
    float iso;
    const float* iso_dev;
};

__device__ __forceinline__ int mc_case(const McArgs& a, long long cell, int& x, int& y, int& z,
                                       float v[8], float iso) {
    const long long cx = a.rx - 1, cy = a.ry - 1;
    x = (int)(cell % cx);
    long long t = cell / cx;
    y = (int)(t % cy);
    z = (int)(t / cy);
    int ci = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int ox = ((c & 1) != ((c >> 1) & 1)) ? 1 : 0;
        const int oy = (c >> 1) & 1;
        const int oz = (c & 4) ? 0 : 1;
        v[c] = a.field[(long long)(x + ox) + (long long)a.rx * ((long long)(y + oy) + (long long)a.ry * (z + oz))];
        if (v[c] > iso) ci |= 1 << c;
    }
    return ci;
}

__global__ void __launch_bounds__(kMcThreads) k_mc_count(McArgs a, unsigned int* __restrict__ counts) {
    const float iso = a.iso_dev ? *a.iso_dev : a.iso;
    long long cell = (long long)blockIdx.x * kMcThreads + threadIdx.x;
    unsigned n = 0;
    if (cell < a.ncell) {
        int x, y, z;
        float v[8];
        n = c_ntri[mc_case(a, cell, x, y, z, v, iso)];
    }
    typedef cub::BlockReduce<unsigned, kMcThreads> BR;
    __shared__ typename BR::TempStorage tmp;
    unsigned tot = BR(tmp).Sum(n);
    if (threadIdx.x == 0) counts[blockIdx.x] = tot;
}

__global__ void k_mc_total(const unsigned int* __restrict__ counts, const unsigned int* __restrict__ offs,
                           long long nb, unsigned long long* __restrict__ total) {
    *total = (unsigned long long)offs[nb - 1] + counts[nb - 1];
}

__global__ void __launch_bounds__(kMcThreads)
    k_mc_emit(McArgs a, const unsigned int* __restrict__ offs, long long cap, float* __restrict__ tris,
              float* __restrict__ cen, float* __restrict__ nrm) {
    const float iso = a.iso_dev ? *a.iso_dev : a.iso;
    long long cell = (long long)blockIdx.x * kMcThreads + threadIdx.x;
    int x = 0, y = 0, z = 0, ci = 0;
    float v[8];
    unsigned n = 0;
    if (cell < a.ncell) {
        ci = mc_case(a, cell, x, y, z, v, iso);
        n = c_ntri[ci];
    }
    typedef cub::BlockScan<unsigned, kMcThreads> BS;
    __shared__ typename BS::TempStorage tmp;
    unsigned local;
    BS(tmp).ExclusiveSum(n, local);
    if (!n) return;
    unsigned long long base = (unsigned long long)offs[blockIdx.x] + local;
    float p[8][3];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int ox = ((c & 1) != ((c >> 1) & 1)) ? 1 : 0;
        const int oy = (c >> 1) & 1;
        const int oz = (c & 4) ? 0 : 1;
        const int gx = x + ox, gy = y + oy, gz = z + oz;
        if (a.pos) {
            long long gi = (long long)gx + (long long)a.rx * ((long long)gy + (long long)a.ry * gz);
            p[c][0] = a.pos[gi * 3];
            p[c][1] = a.pos[gi * 3 + 1];
            p[c][2] = a.pos[gi * 3 + 2];
        } else {
            p[c][0] = __fadd_rn(a.ox, __fmul_rn((float)gx, a.h));
            p[c][1] = __fadd_rn(a.oy, __fmul_rn((float)gy, a.h));
            p[c][2] = __fadd_rn(a.oz, __fmul_rn((float)(gz + a.zoff), a.h));
        }
    }
    const unsigned emask = c_edges[ci];
    float vl[12][3];
#pragma unroll
    for (int e = 0; e < 12; ++e) {
        if (!(emask & (1u << e))) continue;
        const int ia = e & 7;
        const int ib = e < 4 ? ((e + 1) & 3) : (e < 8 ? 4 + ((e - 3) & 3) : e - 4);
        float num = __fsub_rn(v[ia], iso);
        float den = __double2float_rn(__dadd_rn((double)__fsub_rn(v[ib], v[ia]), 1e-10));
        float ell = __fdiv_rn(num, den);
#pragma unroll
        for (int d = 0; d < 3; ++d) vl[e][d] = __fsub_rn(p[ia][d], __fmul_rn(ell, __fsub_rn(p[ib][d], p[ia][d])));
    }
    for (unsigned k = 0; k < n; ++k) {
        unsigned long long t = base + k;
        if ((long long)t >= cap) break;
        const int e0 = c_tri[ci][3 * k], e1 = c_tri[ci][3 * k + 1], e2 = c_tri[ci][3 * k + 2];
        float P0[3], P1[3], P2[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            P0[d] = vl[e0][d];
            P1[d] = vl[e1][d];
            P2[d] = vl[e2][d];
        }
        if (tris) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                tris[t * 9 + d] = P0[d];
                tris[t * 9 + 3 + d] = P1[d];
                tris[t * 9 + 6 + d] = P2[d];
            }
        }
        if (cen) {
#pragma unroll
            for (int d = 0; d < 3; ++d) cen[t * 3 + d] = __fdiv_rn(__fadd_rn(__fadd_rn(P0[d], P1[d]), P2[d]), 3.0f);
        }
        if (nrm) {
            float u[3], w[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                u[d] = __fsub_rn(P1[d], P0[d]);
                w[d] = __fsub_rn(P2[d], P0[d]);
            }
            float cx = __fsub_rn(__fmul_rn(u[1], w[2]), __fmul_rn(u[2], w[1]));
            float cy = __fsub_rn(__fmul_rn(u[2], w[0]), __fmul_rn(u[0], w[2]));
            float cz = __fsub_rn(__fmul_rn(u[0], w[1]), __fmul_rn(u[1], w[0]));
            float sc = -inv_len_eps(__fsqrt_rn(sq3_rn(cx, cy, cz)));
            nrm[t * 3] = __fmul_rn(cx, sc);
            nrm[t * 3 + 1] = __fmul_rn(cy, sc);
            nrm[t * 3 + 2] = __fmul_rn(cz, sc);
        }
    }
}

int mc_run(const float* field, const McGrid& g, float iso, const float* iso_dev, float* tris,
           float* centroids, float* normals, long long cap, unsigned long long* num_tris_dev,
           McWorkspace& ws, cudaStream_t s) {
    DWG_REQUIRE(field && num_tris_dev, "marching cubes: null field or count pointer");
    DWG_REQUIRE(g.res[0] >= 2 && g.res[1] >= 2 && g.res[2] >= 2, "marching cubes: resolution must be >= 2");
    DWG_TRY(mc_upload_tables());
    McArgs a;
    a.field = field;
    a.pos = g.positions;
    a.rx = g.res[0];
    a.ry = g.res[1];
    a.rz = g.res[2];
    a.ncell = (long long)(g.res[0] - 1) * (g.res[1] - 1) * (g.res[2] - 1);
    a.ox = g.origin[0];
    a.oy = g.origin[1];
    a.oz = g.origin[2];
    a.zoff = g.zoff;
    a.h = g.spacing;
    a.iso = iso;
    a.iso_dev = iso_dev;
    long long nb = (a.ncell + kMcThreads - 1) / kMcThreads;
    DWG_REQUIRE(nb < (1ll << 31), "marching cubes: grid too large");
    DWG_TRY(ws.block_counts.reserve(nb));
    DWG_TRY(ws.block_offsets.reserve(nb));
    k_mc_count<<<(unsigned)nb, kMcThreads, 0, s>>>(a, ws.block_counts.ptr);
    DWG_CHECK_LAUNCH();
    size_t bytes = 0;
    unsigned* cin = ws.block_counts.ptr;
    unsigned* cout = ws.block_offsets.ptr;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cin, cout, (int)nb, s));
    DWG_TRY(ws.scratch.reserve(bytes + 256));
    bytes = ws.scratch.n;
    DWG_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(ws.scratch.ptr, bytes, cin, cout, (int)nb, s));
    k_mc_total<<<1, 1, 0, s>>>(cin, cout, nb, num_tris_dev);
    k_mc_emit<<<(unsigned)nb, kMcThreads, 0, s>>>(a, cout, cap, tris, centroids, normals);
    DWG_CHECK_LAUNCH();
    return DWG_OK;
}

}  // namespace dwg

// ----------------------------------------------------------------------------
// Marching cubes without any device allocation.
//
// Some callers cannot allocate device memory when they mesh: a host that is
// recording a CUDA graph in global capture mode (cudaMalloc is not permitted
// while such a capture is open), a real-time loop that must not allocate after
// start-up, or an application that owns every byte of device memory through
// its own pool.  dwg_marching_cubes_noalloc serves them with the same two
// kernels as dwg_marching_cubes; its scratch (per-block triangle counts, their
// offsets and the total) lives in the file-scope device array below, which
// every GPU that loads this library holds until the process exits.
// ----------------------------------------------------------------------------
namespace dwg {

// 2^19 blocks of 256 cells: grids up to 134,217,728 cells (e.g. 512^3)
constexpr long long kMcNoAllocMaxBlocks = 1ll << 19;
constexpr long long kMcNoAllocMaxCells = kMcNoAllocMaxBlocks * kMcThreads;
// [0, max) block counts, [max, 2 max) block offsets, then the 64-bit total
static __device__ __align__(256) unsigned int g_mc_noalloc_scratch[2 * kMcNoAllocMaxBlocks + 64];

// exclusive scan of the block counts by one block, in chunks, with a carry;
// writes every offset and the total, so no slot has to start at zero
constexpr int kMcScanThreads = 1024;
__global__ void __launch_bounds__(kMcScanThreads)
    k_mc_noalloc_scan(const unsigned int* __restrict__ counts, unsigned int* __restrict__ offs, long long nb,
                      unsigned long long* __restrict__ total) {
    typedef cub::BlockScan<unsigned long long, kMcScanThreads> BS;
    __shared__ typename BS::TempStorage tmp;
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < nb; base += kMcScanThreads) {
        const long long i = base + threadIdx.x;
        const unsigned long long v = i < nb ? counts[i] : 0ull;
        unsigned long long ex, agg;
        BS(tmp).ExclusiveSum(v, ex, agg);
        if (i < nb) offs[i] = (unsigned int)(carry + ex);
        __syncthreads();
        if (threadIdx.x == 0) carry += agg;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// device address of the scratch array, looked up once per device with that
// device current (the host-side symbol is not a device address)
static int mc_noalloc_scratch(unsigned int** out) {
    static std::mutex mu;
    static unsigned int* addr[64] = {nullptr};
    int dev = 0;
    DWG_CHECK_CUDA(cudaGetDevice(&dev));
    DWG_REQUIRE(dev >= 0 && dev < 64, "marching_cubes_noalloc: device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_mc_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error("marching_cubes_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return DWG_ERR_CUDA;
        }
        addr[dev] = (unsigned int*)p;
    }
    *out = addr[dev];
    return DWG_OK;
}

}  // namespace dwg

extern "C" int dwg_marching_cubes_noalloc(const float* field_dev, const int res[3], const float* positions_dev,
                                          const float origin[3], float spacing, float iso, float* tris_dev,
                                          float* centroids_dev, float* normals_dev, long long capacity,
                                          long long* num_tris_host, void* stream) {
    using namespace dwg;
    DWG_REQUIRE(field_dev && res && num_tris_host, "marching_cubes_noalloc: null field, resolution or count");
    DWG_REQUIRE(origin || positions_dev, "marching_cubes_noalloc: grid undefined (no origin, no positions)");
    DWG_REQUIRE(res[0] >= 2 && res[1] >= 2 && res[2] >= 2, "marching_cubes_noalloc: resolution must be >= 2");
    DWG_REQUIRE(capacity >= 0, "marching_cubes_noalloc: negative capacity");
    const long long ncell = (long long)(res[0] - 1) * (res[1] - 1) * (res[2] - 1);
    DWG_REQUIRE(ncell <= kMcNoAllocMaxCells,
                "marching_cubes_noalloc: %lld cells exceed the allocation-free limit of %lld cells; use "
                "dwg_marching_cubes",
                ncell, kMcNoAllocMaxCells);
    DWG_TRY(mc_upload_tables());
    unsigned int* scratch = nullptr;
    DWG_TRY(mc_noalloc_scratch(&scratch));
    unsigned int* counts = scratch;
    unsigned int* offs = scratch + kMcNoAllocMaxBlocks;
    unsigned long long* total = reinterpret_cast<unsigned long long*>(scratch + 2 * kMcNoAllocMaxBlocks);
    cudaStream_t s = (cudaStream_t)stream;
    McArgs a;
    a.field = field_dev;
    a.pos = positions_dev;
    a.rx = res[0];
    a.ry = res[1];
    a.rz = res[2];
    a.ncell = ncell;
    a.ox = origin ? origin[0] : 0.f;
    a.oy = origin ? origin[1] : 0.f;
    a.oz = origin ? origin[2] : 0.f;
    a.zoff = 0;
    a.h = spacing;
    a.iso = iso;
    a.iso_dev = nullptr;
    const long long nb = (ncell + kMcThreads - 1) / kMcThreads;
    k_mc_count<<<(unsigned)nb, kMcThreads, 0, s>>>(a, counts);
    k_mc_noalloc_scan<<<1, kMcScanThreads, 0, s>>>(counts, offs, nb, total);
    k_mc_emit<<<(unsigned)nb, kMcThreads, 0, s>>>(a, offs, capacity, tris_dev, centroids_dev, normals_dev);
    DWG_CHECK_LAUNCH();
    unsigned long long T = 0;
    DWG_CHECK_CUDA(cudaMemcpyAsync(&T, total, sizeof(T), cudaMemcpyDeviceToHost, s));
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    *num_tris_host = (long long)T;
    if ((long long)T > capacity) {
        set_error("marching_cubes_noalloc: %llu triangles exceed capacity %lld", T, capacity);
        return DWG_ERR_OVERFLOW;
    }
    return DWG_OK;
}
