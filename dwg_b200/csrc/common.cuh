// common.cuh -- shared helpers of the dwg_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/dwg_b200.h"

namespace dwg {

// ---------------------------------------------------------------- errors --
void set_error(const char* fmt, ...);

struct Status {
    int code = DWG_OK;
};

#define DWG_CHECK_CUDA(expr)                                                     \
    do {                                                                         \
        cudaError_t _e = (expr);                                                 \
        if (_e != cudaSuccess) {                                                 \
            ::dwg::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), \
                             __FILE__, __LINE__);                                \
            return _e == cudaErrorMemoryAllocation ? DWG_ERR_NOMEM : DWG_ERR_CUDA; \
        }                                                                        \
    } while (0)

#define DWG_CHECK_LAUNCH() DWG_CHECK_CUDA(cudaGetLastError())

#define DWG_REQUIRE(cond, ...)              \
    do {                                    \
        if (!(cond)) {                      \
            ::dwg::set_error(__VA_ARGS__);  \
            return DWG_ERR_INVALID;         \
        }                                   \
    } while (0)

#define DWG_TRY(...)               \
    do {                           \
        int _s = (__VA_ARGS__);    \
        if (_s != DWG_OK) return _s; \
    } while (0)

// ------------------------------------------------------ device buffers --
// Device memory comes from the device's stream-ordered pool, which keeps
// freed blocks mapped (release threshold = unlimited): building and tearing
// down a pipeline per cloud then costs no page-table work.  An allocation is
// made on a private stream of the device and is complete when it is returned
// (no other stream waits).  A release made while a FreeScope of the calling
// thread is alive is ordered on the scope's stream (after the work queued
// there: the owner's stream, which is the only one that used the block) or,
// for an idle scope, made at once (the owner's stream was drained); any
// other release first waits for the device to finish its work, like cudaFree.
int pool_alloc(void** p, size_t bytes);
void pool_free(void* p);
struct FreeScope {
    FreeScope(cudaStream_t stream, bool idle);
    ~FreeScope();
    FreeScope(const FreeScope&) = delete;
    FreeScope& operator=(const FreeScope&) = delete;

  private:
    bool prev_active_, prev_idle_;
    cudaStream_t prev_stream_;
};

// Device memory this library can still count on: the free memory it first
// saw on the current device (plus what it held then) minus the blocks it
// holds now.  Freed blocks stay in its pool, so they count as available; no
// driver query runs after the first call.
size_t device_free_bytes();

// Streams and events recycled across pipelines (creating them per cloud
// costs driver calls that other processes' monitoring can hold up).
cudaStream_t stream_acquire();
void stream_release(cudaStream_t s);
cudaEvent_t event_acquire();
void event_release(cudaEvent_t e);

// An executable graph for g: a released executable of the same topology is
// updated in place (cudaGraphExecUpdate: new buffers and arguments, no new
// instantiation), otherwise g is instantiated.  release() keeps it for the
// next pipeline of the same shape; it must be idle.
int graph_exec_acquire(cudaGraph_t g, cudaGraphExec_t* out);
void graph_exec_release(cudaGraphExec_t e);

// Grow-only device buffer; owner frees.
template <typename T>
struct DevBuf {
    T* ptr = nullptr;
    size_t n = 0;
    int reserve(size_t count) {
        if (count <= n && ptr) return DWG_OK;
        release();
        size_t bytes = (count ? count : 1) * sizeof(T);
        void* p = nullptr;
        int st = pool_alloc(&p, bytes);
        if (st != DWG_OK) return st;
        ptr = (T*)p;
        n = count ? count : 1;
        return DWG_OK;
    }
    void release() {
        if (ptr) pool_free(ptr);
        ptr = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

inline int num_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

inline unsigned div_up(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

// ------------------------------------------- exact single-precision ops --
// The discrete decisions (opening test, kNN keys, marching-cubes geometry)
// use round-to-nearest intrinsics so that they cannot be contracted into
// FMAs and match the CPU oracle operation for operation.
__device__ __forceinline__ float sq3_rn(float dx, float dy, float dz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

__device__ __forceinline__ float inv_len_eps(float len) {
    // 1 / (len + 1e-8), the sum taken in double and rounded to float, like the
    // reference's __frcp_rn(length + 1e-8)
    return __frcp_rn(__double2float_rn(__dadd_rn((double)len, 1e-8)));
}

}  // namespace dwg
