// Shared device/host helpers for the qsdvr_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "qsdvr_b200.h"

namespace qsdvr {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// ---- host-side status plumbing (capi.cu) ------------------------------------------------
int set_error(int code, const char *fmt, ...);
int check_launch(const char *what);
int check_cuda(cudaError_t e, const char *what);

// ---- device error word -------------------------------------------------------------------
// Each translation unit owns one word (internal linkage, no relocatable device code);
// QSDVR_ERROR_WORD_ACCESSOR(name) gives capi.cu a host function that reads/clears it.
static __device__ unsigned int g_device_error;

__device__ __forceinline__ void flag_error(unsigned bits) { atomicOr(&g_device_error, bits); }

// ---- bounds-checked build ------------------------------------------------------------------
// Compiled with -DQSDVR_DEBUG_BOUNDS (libqsdvr_b200_debug.so), every global gather, store and
// RED whose index a kernel derives from geometry or caller data goes through QSDVR_AT, which
// checks [index, index + width) against the buffer's extent (all in elements).  A range
// outside it sets QSDVR_DEVERR_BOUNDS, records the first such (source line, index, extent) of
// the translation unit and is redirected to a 256-byte sink, so the launch completes and
// nothing traps.  Without the macro QSDVR_AT is the plain address: the product library's
// code is unchanged.
#ifdef QSDVR_DEBUG_BOUNDS
static __device__ unsigned long long g_bounds_record[3];
static __device__ __align__(16) unsigned char g_bounds_sink[256];

static __device__ __noinline__ void *bounds_fail(uint64_t index, uint64_t extent, uint32_t line) {
    flag_error(QSDVR_DEVERR_BOUNDS);
    if (atomicCAS(&g_bounds_record[0], 0ull, (unsigned long long)line) == 0ull) {
        g_bounds_record[1] = index;
        g_bounds_record[2] = extent;
    }
    return g_bounds_sink;
}

// (an access through QSDVR_AT spans at most 256 bytes, the sink's size)
template <typename T>
static __device__ __forceinline__ T *checked_at(T *base, uint64_t index, uint64_t width, uint64_t extent, uint32_t line) {
    if (index < extent && width <= extent - index) return base + index;
    return static_cast<T *>(bounds_fail(index, extent, line));
}
// A wider range (a whole row stash, say) is checked with QSDVR_IN_RANGE, which records a
// violation the same way and returns false, and the caller skips the access.
static __device__ __forceinline__ bool checked_range(uint64_t index, uint64_t width, uint64_t extent, uint32_t line) {
    if (index < extent && width <= extent - index) return true;
    bounds_fail(index, extent, line);
    return false;
}
#define QSDVR_AT(base, index, width, extent) \
    ::qsdvr::checked_at((base), (uint64_t)(index), (uint64_t)(width), (uint64_t)(extent), __LINE__)
#define QSDVR_IN_RANGE(index, width, extent) \
    ::qsdvr::checked_range((uint64_t)(index), (uint64_t)(width), (uint64_t)(extent), __LINE__)
#define QSDVR_BOUNDS_CHECKED 1
#else
#define QSDVR_AT(base, index, width, extent) ((base) + (index))
#define QSDVR_IN_RANGE(index, width, extent) true
#define QSDVR_BOUNDS_CHECKED 0
#endif

#if QSDVR_BOUNDS_CHECKED
#define QSDVR_BOUNDS_RECORD_READ(rec, clear, stream, e)                                              \
    do {                                                                                           \
        if (e == cudaSuccess) e = cudaMemcpyFromSymbolAsync(rec, g_bounds_record, 3 * sizeof(uint64_t), 0, \
                                                            cudaMemcpyDeviceToHost, stream);       \
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);                                   \
        if (e == cudaSuccess && clear && rec[0]) {                                                 \
            const unsigned long long zero[3] = {0, 0, 0};                                          \
            e = cudaMemcpyToSymbolAsync(g_bounds_record, zero, sizeof(zero), 0,                    \
                                        cudaMemcpyHostToDevice, stream);                           \
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);                               \
        }                                                                                          \
    } while (0)
#else
#define QSDVR_BOUNDS_RECORD_READ(rec, clear, stream, e) \
    do {                                                \
        rec[0] = rec[1] = rec[2] = 0;                   \
    } while (0)
#endif

// Per translation unit: error_word_<name> reads (and clears) its error word;
// bounds_record_<name> its first out-of-range record {line, index, extent} (zeros when none
// or in the product build).
#define QSDVR_ERROR_WORD_ACCESSOR(name)                                                              \
    cudaError_t error_word_##name(unsigned *word, int clear, cudaStream_t stream) {                \
        unsigned v = 0;                                                                            \
        cudaError_t e = cudaMemcpyFromSymbolAsync(&v, g_device_error, sizeof(v), 0,                \
                                                  cudaMemcpyDeviceToHost, stream);                 \
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);                                   \
        if (e == cudaSuccess && clear && v) {                                                      \
            const unsigned zero = 0;                                                               \
            e = cudaMemcpyToSymbolAsync(g_device_error, &zero, sizeof(zero), 0,                    \
                                        cudaMemcpyHostToDevice, stream);                           \
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);                               \
        }                                                                                          \
        *word |= v;                                                                                \
        return e;                                                                                  \
    }                                                                                              \
    cudaError_t bounds_record_##name(uint64_t *rec, int clear, cudaStream_t stream) {              \
        cudaError_t e = cudaSuccess;                                                               \
        QSDVR_BOUNDS_RECORD_READ(rec, clear, stream, e);                                           \
        return e;                                                                                  \
    }

// ---- small vector helpers ----------------------------------------------------------------
struct f3 {
    float x, y, z;
};

__device__ __forceinline__ f3 load3(const float *p) { return f3{p[0], p[1], p[2]}; }
__device__ __forceinline__ void store3(float *p, f3 v) {
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
}

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }

// 16-byte vector reduction into global memory (returns nothing, so it lowers to a RED).
__device__ __forceinline__ void red4(float *p, float4 v) { atomicAdd(reinterpret_cast<float4 *>(p), v); }

// True when all four values are +0 or -0.  Adding such a vector to a gradient accumulator
// that starts at +0 changes no bit of it (x + 0 = x for x != 0; +0 + -0 = +0 in round to
// nearest, so the accumulator never holds -0), and NaN or inf never compares equal to 0, so
// skipping the RED of a zero vector leaves the sum exactly as it was.
__device__ __forceinline__ bool is_zero4(float4 v) {
    return v.x == 0.0f && v.y == 0.0f && v.z == 0.0f && v.w == 0.0f;
}

inline unsigned grid_for(uint64_t threads, unsigned block) {
    uint64_t g = (threads + block - 1) / block;
    return g == 0 ? 1u : (unsigned)(g > 0x7fffffffull ? 0x7fffffffull : g);
}

inline bool aligned(const void *p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

}  // namespace qsdvr
