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

inline unsigned grid_for(uint64_t threads, unsigned block) {
    uint64_t g = (threads + block - 1) / block;
    return g == 0 ? 1u : (unsigned)(g > 0x7fffffffull ? 0x7fffffffull : g);
}

inline bool aligned(const void *p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

}  // namespace qsdvr
