// io.cu -- point-cloud and mesh files: the .xyz reader, the binary STL and
// oriented .xyz writers (include/DWGProcess.h:53-97, src/TurboMC.cu:333-371,
// src/TurboDWG.cu:903-923).
//
// The reference reads and writes one line / one record at a time on one host
// thread.  Here the reader loads the file once and parses newline-aligned
// chunks on all host cores with exact decimal conversion (std::from_chars,
// the same doubles as scanf's %lf); the STL writer packs the 50-byte records
// on the GPU, chunk by chunk into two pinned buffers, while the host writes
// the previous chunk; the text writer formats chunks in parallel and writes
// them in order.
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace dwg {

static int io_threads(size_t work, size_t per_thread) {
    unsigned hc = std::thread::hardware_concurrency();
    size_t t = hc ? hc : 4;
    if (t > 64) t = 64;
    size_t want = work / per_thread + 1;
    return (int)(want < t ? want : t);
}

// up to 6 numbers of one line, as sscanf("%lf %lf ...") reads them: leading
// whitespace is skipped before every number and reading stops at the first
// token that is not a number.  Returns how many were read.
static int parse_numbers(const char* b, const char* e, double v[6]) {
    int k = 0;
    while (k < 6) {
        while (b < e && (*b == ' ' || *b == '\t' || *b == '\r' || *b == '\v' || *b == '\f')) ++b;
        if (b >= e) break;
        const char* s = b;
        bool neg = false;
        if (*s == '+' || *s == '-') {  // from_chars takes no '+'; a sign before inf / nan too
            neg = *s == '-';
            ++s;
        }
        double x = 0;
        auto r = std::from_chars(s, e, x, std::chars_format::general);
        if (r.ec != std::errc() && r.ec != std::errc::result_out_of_range) break;
        if (r.ec == std::errc::result_out_of_range) {
            // scanf gives +-HUGE_VAL on overflow and a (signed) zero or a
            // subnormal on underflow; strtod agrees with it on both
            x = std::strtod(std::string(s, r.ptr).c_str(), nullptr);
        }
        v[k++] = neg ? -x : x;
        b = r.ptr;
    }
    return k;
}

struct XyzChunk {
    std::vector<double> P, N;
    long long lines = 0;      // lines in the chunk
    long long bad_line = -1;  // first malformed line (chunk-local, 1-based)
    int bad_count = 0;
    bool bad_value = false;
};

static void parse_chunk(const char* b, const char* e, XyzChunk& c) {
    while (b < e) {
        const char* nl = static_cast<const char*>(memchr(b, '\n', (size_t)(e - b)));
        const char* le = nl ? nl : e;
        ++c.lines;
        double v[6];
        const int k = parse_numbers(b, le, v);
        b = nl ? nl + 1 : e;
        if (k <= 0) continue;  // blank line
        if (k < 3 || !std::isfinite(v[0]) || !std::isfinite(v[1]) || !std::isfinite(v[2])) {
            c.bad_line = c.lines;
            c.bad_count = k;
            c.bad_value = k >= 3;
            return;
        }
        for (int d = 0; d < 3; ++d) c.P.push_back(v[d]);
        for (int d = 3; d < 6; ++d) c.N.push_back(k == 6 ? v[d] : 0.0);
    }
}

// records of save_binary_STL: facet normal (cross / |cross|, 0 when the
// cross product is 0; get_normal, src/TurboMC.cu:333-340), three vertices,
// a zero attribute.  Single-precision operations each rounded once, so the
// host and the GPU packers write the same bytes.
__host__ __device__ inline void stl_record(const float* v, unsigned char* rec) {
#ifdef __CUDA_ARCH__
    const float e1[3] = {__fsub_rn(v[3], v[0]), __fsub_rn(v[4], v[1]), __fsub_rn(v[5], v[2])};
    const float e2[3] = {__fsub_rn(v[6], v[0]), __fsub_rn(v[7], v[1]), __fsub_rn(v[8], v[2])};
    const float c[3] = {__fsub_rn(__fmul_rn(e1[1], e2[2]), __fmul_rn(e1[2], e2[1])),
                        __fsub_rn(__fmul_rn(e1[2], e2[0]), __fmul_rn(e1[0], e2[2])),
                        __fsub_rn(__fmul_rn(e1[0], e2[1]), __fmul_rn(e1[1], e2[0]))};
    const float len =
        __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(c[0], c[0]), __fmul_rn(c[1], c[1])), __fmul_rn(c[2], c[2])));
    float n[3] = {0.f, 0.f, 0.f};
    if (len > 0.f)
        for (int d = 0; d < 3; ++d) n[d] = __fdiv_rn(c[d], len);
#else
    const float e1[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
    const float e2[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
    const float c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    const float len = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    float n[3] = {0.f, 0.f, 0.f};
    if (len > 0.f)
        for (int d = 0; d < 3; ++d) n[d] = c[d] / len;
#endif
    // 50-byte records start 2-byte aligned: copy as 16-bit halves
    unsigned short w[25];
    memcpy(w, n, 12);
    memcpy(w + 6, v, 36);
    w[24] = 0;
    unsigned short* r = reinterpret_cast<unsigned short*>(rec);
    for (int i = 0; i < 25; ++i) r[i] = w[i];
}

__global__ void k_stl_pack(const float* __restrict__ tris, long long T, unsigned char* __restrict__ out) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= T) return;
    float v[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) v[i] = tris[t * 9 + i];
    stl_record(v, out + t * 50);
}

static bool write_stl_header(FILE* f, long long T) {
    char header[80] = {0};
    const uint32_t cnt = (uint32_t)T;
    return fwrite(header, 1, 80, f) == 80 && fwrite(&cnt, 4, 1, f) == 1;
}

}  // namespace dwg

using namespace dwg;

#define IO_GUARD(...)                                            \
    try {                                                        \
        __VA_ARGS__                                              \
    } catch (const std::bad_alloc&) {                            \
        set_error("host allocation failed");                     \
        return DWG_ERR_NOMEM;                                    \
    } catch (...) {                                              \
        set_error("unexpected exception");                       \
        return DWG_ERR_INVALID;                                  \
    }

extern "C" {

// ReadPointandNormals (include/DWGProcess.h:53-97)
int dwg_read_xyz(const char* path, int normalize, float** points, float** normals, int* n) {
    IO_GUARD({
        DWG_REQUIRE(path && points && n, "read_xyz: null argument");
        FILE* f = fopen(path, "rb");
        DWG_REQUIRE(f != nullptr, "read_xyz: cannot open '%s'", path);
        std::vector<char> buf;
        {
            char tmp[1 << 16];
            size_t got;
            while ((got = fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
        }
        fclose(f);
        // newline-aligned chunks, parsed concurrently
        const size_t size = buf.size();
        const int nt = io_threads(size, (size_t)1 << 20);
        std::vector<size_t> cut(nt + 1, size);
        cut[0] = 0;
        for (int t = 1; t < nt; ++t) {
            size_t c = size * (size_t)t / (size_t)nt;
            if (c < cut[t - 1]) c = cut[t - 1];
            const void* nl = c < size ? memchr(buf.data() + c, '\n', size - c) : nullptr;
            cut[t] = nl ? (size_t)(static_cast<const char*>(nl) - buf.data()) + 1 : size;
        }
        std::vector<XyzChunk> ch(nt);
        {
            std::vector<std::thread> th;
            for (int t = 0; t < nt; ++t)
                th.emplace_back([&, t] { parse_chunk(buf.data() + cut[t], buf.data() + cut[t + 1], ch[t]); });
            for (auto& x : th) x.join();
        }
        long long line0 = 0;
        size_t total = 0;
        for (int t = 0; t < nt; ++t) {
            if (ch[t].bad_line >= 0) {
                if (ch[t].bad_value)
                    set_error("read_xyz: non-finite coordinate on line %lld of '%s'", line0 + ch[t].bad_line, path);
                else
                    set_error("read_xyz: line %lld of '%s' has %d values (need 3 or 6)", line0 + ch[t].bad_line,
                              path, ch[t].bad_count);
                return DWG_ERR_INVALID;
            }
            line0 += ch[t].lines;
            total += ch[t].P.size();
        }
        const int cnt = (int)(total / 3);
        DWG_REQUIRE(cnt > 0, "read_xyz: no points in '%s'", path);
        std::vector<double> P;
        P.reserve(total);
        for (auto& c : ch) P.insert(P.end(), c.P.begin(), c.P.end());
        if (normalize) {
            // centre on the mean, divide by max 2|x| (:69-92), in FP64
            double c[3] = {0, 0, 0};
            for (int i = 0; i < cnt; ++i)
                for (int d = 0; d < 3; ++d) c[d] += P[(size_t)i * 3 + d];
            for (int d = 0; d < 3; ++d) c[d] /= (1.0 * cnt);
            double scale = 0;
            for (int i = 0; i < cnt; ++i)
                for (int d = 0; d < 3; ++d) {
                    P[(size_t)i * 3 + d] -= c[d];
                    scale = std::max(2.0 * std::fabs(P[(size_t)i * 3 + d]), scale);
                }
            if (scale == 0) scale = 1;
            for (auto& x : P) x /= scale;
        }
        float* po = (float*)malloc(sizeof(float) * 3 * cnt);
        float* no = normals ? (float*)malloc(sizeof(float) * 3 * cnt) : nullptr;
        if (!po || (normals && !no)) {
            free(po);
            free(no);
            set_error("read_xyz: host allocation failed");
            return DWG_ERR_NOMEM;
        }
        for (size_t i = 0; i < P.size(); ++i) po[i] = (float)P[i];
        if (no) {
            size_t o = 0;
            for (auto& c : ch)
                for (double x : c.N) no[o++] = (float)x;
        }
        *points = po;
        if (normals) *normals = no;
        *n = cnt;
        return DWG_OK;
    })
}

void dwg_free_host(void* p) { free(p); }

// save_binary_STL (src/TurboMC.cu:344-371): 80-byte header, uint32 count,
// per triangle normal (cross / |cross|, 0 if degenerate), 3 vertices, uint16 0
int dwg_write_stl(const char* path, const float* tris, long long T) {
    IO_GUARD({
        DWG_REQUIRE(path && (tris || T == 0) && T >= 0 && T <= 0xffffffffll, "write_stl: bad arguments");
        std::vector<unsigned char> body((size_t)T * 50);
        const int nt = io_threads((size_t)T, 1 << 16);
        {
            std::vector<std::thread> th;
            for (int t = 0; t < nt; ++t)
                th.emplace_back([&, t] {
                    for (long long i = T * t / nt; i < T * (t + 1) / nt; ++i) stl_record(tris + i * 9, &body[i * 50]);
                });
            for (auto& x : th) x.join();
        }
        FILE* f = fopen(path, "wb");
        DWG_REQUIRE(f != nullptr, "write_stl: cannot create '%s'", path);
        bool ok = write_stl_header(f, T) && (T == 0 || fwrite(body.data(), 1, body.size(), f) == body.size());
        ok = (fclose(f) == 0) && ok;
        DWG_REQUIRE(ok, "write_stl: cannot write '%s'", path);
        return DWG_OK;
    })
}

// the same file from triangles in device memory: records packed on the GPU
// in chunks, copied into two pinned buffers in turn and written while the
// next chunk is packed
int dwg_write_stl_device(const char* path, const float* tris_dev, long long T, void* stream) {
    IO_GUARD({
        DWG_REQUIRE(path && (tris_dev || T == 0) && T >= 0 && T <= 0xffffffffll, "write_stl: bad arguments");
        cudaStream_t s = (cudaStream_t)stream;
        FILE* f = fopen(path, "wb");
        DWG_REQUIRE(f != nullptr, "write_stl: cannot create '%s'", path);
        bool ok = write_stl_header(f, T);
        const long long kChunk = 1 << 20;  // triangles per chunk (50 MB)
        const long long per = T < kChunk ? T : kChunk;
        unsigned char* host[2] = {nullptr, nullptr};
        cudaEvent_t done[2] = {nullptr, nullptr};
        DevBuf<unsigned char> dev[2];
        int rc = DWG_OK;
        if (ok && T > 0) {
            for (int b = 0; b < 2 && rc == DWG_OK; ++b) {
                if (cudaMallocHost(&host[b], (size_t)per * 50) != cudaSuccess ||
                    cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming) != cudaSuccess) {
                    set_error("write_stl: pinned buffer or event creation failed");
                    rc = DWG_ERR_CUDA;
                } else {
                    rc = dev[b].reserve((size_t)per * 50);
                }
            }
            long long sizes[2] = {0, 0};
            long long k = 0;
            for (long long t0 = 0; rc == DWG_OK && t0 < T; t0 += per, ++k) {
                const int b = (int)(k & 1);
                const long long cnt = T - t0 < per ? T - t0 : per;
                k_stl_pack<<<div_up(cnt, 256), 256, 0, s>>>(tris_dev + t0 * 9, cnt, dev[b].ptr);
                cudaError_t e = cudaGetLastError();
                if (e == cudaSuccess) e = cudaMemcpyAsync(host[b], dev[b].ptr, (size_t)cnt * 50, cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaEventRecord(done[b], s);
                if (e != cudaSuccess) {
                    set_error("write_stl: %s", cudaGetErrorString(e));
                    rc = DWG_ERR_CUDA;
                    break;
                }
                sizes[b] = cnt;
                if (k > 0) {  // write the previous chunk while this one is packed
                    const int pb = 1 - b;
                    if (cudaEventSynchronize(done[pb]) != cudaSuccess) {
                        rc = DWG_ERR_CUDA;
                        break;
                    }
                    ok = ok && fwrite(host[pb], 1, (size_t)sizes[pb] * 50, f) == (size_t)sizes[pb] * 50;
                }
            }
            if (rc == DWG_OK && k > 0) {
                const int lb = (int)((k - 1) & 1);
                if (cudaEventSynchronize(done[lb]) != cudaSuccess) rc = DWG_ERR_CUDA;
                else ok = ok && fwrite(host[lb], 1, (size_t)sizes[lb] * 50, f) == (size_t)sizes[lb] * 50;
            }
            cudaStreamSynchronize(s);  // no copy in flight before the buffers go
        }
        for (int b = 0; b < 2; ++b) {
            if (host[b]) cudaFreeHost(host[b]);
            if (done[b]) cudaEventDestroy(done[b]);
        }
        ok = (fclose(f) == 0) && ok;
        if (rc != DWG_OK) return rc;
        DWG_REQUIRE(ok, "write_stl: cannot write '%s'", path);
        return DWG_OK;
    })
}

// oriented point cloud output (src/TurboDWG.cu:903-923): "x y z nx ny nz"
// with six significant digits (the ostream default), or "x y z"
int dwg_write_xyz(const char* path, const float* P, const float* N, int n) {
    IO_GUARD({
        DWG_REQUIRE(path && P && n >= 0, "write_xyz: bad arguments");
        const int nt = io_threads((size_t)n, 1 << 15);
        std::vector<std::string> part(nt);
        {
            std::vector<std::thread> th;
            for (int t = 0; t < nt; ++t)
                th.emplace_back([&, t] {
                    std::string& o = part[t];
                    char line[192];
                    for (long long i = (long long)n * t / nt; i < (long long)n * (t + 1) / nt; ++i) {
                        int len;
                        if (N)
                            len = snprintf(line, sizeof(line), "%g %g %g %g %g %g\n", P[i * 3], P[i * 3 + 1],
                                           P[i * 3 + 2], N[i * 3], N[i * 3 + 1], N[i * 3 + 2]);
                        else
                            len = snprintf(line, sizeof(line), "%g %g %g\n", P[i * 3], P[i * 3 + 1], P[i * 3 + 2]);
                        o.append(line, (size_t)len);
                    }
                });
            for (auto& x : th) x.join();
        }
        FILE* f = fopen(path, "w");
        DWG_REQUIRE(f != nullptr, "write_xyz: cannot create '%s'", path);
        bool ok = true;
        for (auto& s : part) ok = ok && fwrite(s.data(), 1, s.size(), f) == s.size();
        ok = (fclose(f) == 0) && ok;
        DWG_REQUIRE(ok, "write_xyz: cannot write '%s'", path);
        return DWG_OK;
    })
}

}  // extern "C"
