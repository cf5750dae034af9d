// Proposal network: a small MLP (32-d positional encoding -> 64 -> 64 -> 1, BF16 weights,
// FP32 accumulation) that bounds the renderer's density so that 32 fine samples per ray,
// placed by inverse-CDF sampling of 64 coarse MLP evaluations, replace the uniform march.
// No counterpart in the reference.
//
// GEMMs run on the 5th-generation tensor cores (tcgen05): a CTA of 128 threads owns a tile of
// 128 points (thread t <-> point t <-> TMEM lane t); operands are staged in shared memory in
// canonical no-swizzle layouts, one thread issues the MMAs, accumulators live in TMEM.  The
// training kernel keeps the weight-gradient accumulators in TMEM across all of its tiles.
//
// Parameter vector (fp32 master, bf16 copy read by the kernels), QSDVR_MLP_PARAMS floats:
//   [0, 2048)    W1[o][i], 64 x 32 (input feature 27 is the constant 1: the layer-1 bias)
//   [2048, 6144) W2[o][i], 64 x 64
//   [6144, 6208) b2[64]   [6208, 6272) w3[64]   [6272] b3   (padded to 6280)
// Encoding of p in [-1,1]^3: f0..2 = p, f(3 + 6l + 2c) = sin(pi 2^l p_c), f(4 + 6l + 2c) =
// cos(pi 2^l p_c) for l = 0..3, f27 = 1, f28..31 = 0.  Density bound = softplus(w3 . h2 + b3).
// b2 rides in the layer-2 GEMM: the staged H1 has a constant feature 64 = 1 and the staged
// W2 a column 64 = b2 (K = 80), so in training the dW2 GEMM also yields db2 (its column 64).
#include <cuda_bf16.h>

#include "common.cuh"
#include "raygen.cuh"
#include "tcgen05.cuh"

namespace qsdvr {

QSDVR_ERROR_WORD_ACCESSOR(proposal)

namespace {

constexpr int kTile = 128;
constexpr int kF = 32, kH = 64;
constexpr int kOffW2 = 2048, kOffB2 = 6144, kOffW3 = 6208, kOffB3 = 6272;
constexpr uint32_t kSpins = 1u << 26;  // bounded mbarrier waits (~ seconds), then give up
constexpr uint32_t kInferCols = 64;    // TMEM columns of an inference CTA (both layers)
constexpr uint32_t kTrainCols = 256;   // of a training CTA: forward 0..63, dW2 128..191, dW1 192..223

// shared-memory operand layouts (bytes): element (row, feature) of an activation buffer with
// point-group stride SP sits at (row/8)*SP + (f/8)*128 + (row%8)*16 + (f%8)*2
constexpr uint32_t kSpX = 512, kSpH = 1280, kSpG = 2048;  // X (32 f), H1 (64 f + bias 1 + 15 zero),
                                                           // grads (64 f + 64 zero)
constexpr uint32_t kSoW1 = 512, kSoW2 = 1280;              // W1 (32 inputs), W2 (64 inputs + b2 + 15 zero)
constexpr uint32_t kK2 = 80;                               // layer-2 K with the bias feature
constexpr uint32_t kBytesX = 16 * kSpX, kBytesH = 16 * kSpH, kBytesG = 16 * kSpG;
constexpr uint32_t kBytesW1 = 8 * kSoW1, kBytesW2 = 8 * kSoW2;

__device__ __forceinline__ uint32_t act_off(uint32_t row, uint32_t f, uint32_t sp) {
    return (row >> 3) * sp + (f >> 3) * 128 + (row & 7) * 16 + (f & 7) * 2;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ float bf16f(const __nv_bfloat16 *p, int i) { return __bfloat162float(p[i]); }

// Two floats -> bf16x2 with ReLU applied, one instruction (cvt.rn.relu.bf16x2.f32).
__device__ __forceinline__ uint32_t pack_relu_bf16(float a, float b) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
    return r;
}

// Write 8 consecutive features [8g, 8g+8) of one row, ReLU applied, as one 16-byte store.
__device__ __forceinline__ void store_relu_row8(uint8_t *buf, uint32_t row, uint32_t g, uint32_t sp, const float *v) {
    uint4 q;
    q.x = pack_relu_bf16(v[0], v[1]);
    q.y = pack_relu_bf16(v[2], v[3]);
    q.z = pack_relu_bf16(v[4], v[5]);
    q.w = pack_relu_bf16(v[6], v[7]);
    *reinterpret_cast<uint4 *>(buf + act_off(row, 8 * g, sp)) = q;
}

// Write 8 consecutive features [8g, 8g+8) of one row as one 16-byte store.
__device__ __forceinline__ void store_row8(uint8_t *buf, uint32_t row, uint32_t g, uint32_t sp, const float *v) {
    uint4 q;
    q.x = pack_bf16(v[0], v[1]);
    q.y = pack_bf16(v[2], v[3]);
    q.z = pack_bf16(v[4], v[5]);
    q.w = pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4 *>(buf + act_off(row, 8 * g, sp)) = q;
}

// The base octave uses the hardware sine/cosine (absolute error about 2^-21 on [-pi, pi]); the
// octaves 2^l (l = 1..3) follow by the double-angle identities sin 2a = 2 sin a cos a,
// cos 2a = 1 - 2 sin^2 a.  Both errors (~1e-6) are far below the bf16 rounding that follows.
__device__ __forceinline__ void encode(f3 p, float *f) {
    constexpr float kPi = 3.14159265358979f;
    f[0] = p.x;
    f[1] = p.y;
    f[2] = p.z;
    const float c[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float sn = __sinf(kPi * c[k]), cs = __cosf(kPi * c[k]);
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            f[3 + 6 * l + 2 * k] = sn;
            f[4 + 6 * l + 2 * k] = cs;
            const float s2 = 2.0f * sn * cs;
            cs = fmaf(-2.0f * sn, sn, 1.0f);
            sn = s2;
        }
    }
    f[27] = 1.0f;
    f[28] = f[29] = f[30] = f[31] = 0.0f;
}

__device__ __forceinline__ float softplus(float y) { return y > 20.0f ? y : __logf(1.0f + __expf(y)); }
__device__ __forceinline__ float sigmoid(float y) { return 1.0f / (1.0f + __expf(-y)); }

// Stage W1 / W2 (bf16) in their canonical K-major layouts: element (o, i) at
// (o/8)*SO + (i/8)*128 + (o%8)*16 + (i%8)*2 with SO = kSoW1 (W1) or kSoW2 (W2; its column 64
// is b2, columns 65..79 zero).  Also the constant features 64..79 (1, 0, ..) of H1 row t.
__device__ void stage_weights(const __nv_bfloat16 *w, uint8_t *w1s, uint8_t *w2s, uint8_t *hs) {
    for (int idx = threadIdx.x; idx < 64 * 4; idx += blockDim.x) {  // W1: 64 rows x 4 groups
        const int o = idx >> 2, g = idx & 3;
        *reinterpret_cast<uint4 *>(w1s + act_off(o, 8 * g, kSoW1)) =
            *reinterpret_cast<const uint4 *>(w + o * 32 + 8 * g);
    }
    for (int idx = threadIdx.x; idx < 64 * 10; idx += blockDim.x) {  // W2: 64 rows x 10 groups
        const int o = idx / 10, g = idx % 10;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (g < 8) v = *reinterpret_cast<const uint4 *>(w + kOffW2 + o * 64 + 8 * g);
        else if (g == 8) v.x = (uint32_t)__bfloat16_as_ushort(w[kOffB2 + o]);  // (b2[o], 0)
        *reinterpret_cast<uint4 *>(w2s + act_off(o, 8 * g, kSoW2)) = v;
    }
    const uint32_t one = (uint32_t)__bfloat16_as_ushort(__float2bfloat16(1.0f));
    *reinterpret_cast<uint4 *>(hs + act_off(threadIdx.x, 64, kSpH)) = make_uint4(one, 0, 0, 0);
    *reinterpret_cast<uint4 *>(hs + act_off(threadIdx.x, 72, kSpH)) = make_uint4(0, 0, 0, 0);
}

struct Sync {
    uint64_t *mbar;
    uint32_t phase;
    bool ok;
    // commit the MMAs issued by thread 0 and wait for them on every thread; a wait that gave
    // up stops the whole CTA (the flag is made block-uniform so every thread leaves the tile
    // loop at the same barrier)
    __device__ __forceinline__ void complete() {
        if (threadIdx.x == 0) tc::commit(mbar);
        const bool done = tc::mbar_wait(mbar, phase, kSpins);
        if (!done) flag_error(QSDVR_DEVERR_TIMEOUT);
        if (__syncthreads_or(!done)) ok = false;
        phase ^= 1u;
        tc::fence_after_sync();
    }
};

// smem staging -> visible to the tensor core, and everyone past their TMEM reads
__device__ __forceinline__ void handoff() {
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
}

// Forward of one tile: X (staged) -> H1 (staged, returns the relu mask) -> z2 = W2 h1 + b2
// (this thread's row, in registers; b2 through H1's constant feature).  Both layers
// accumulate in the same 64 TMEM columns at d1: every thread has read layer 1's result before
// the barrier that precedes layer 2.
__device__ __forceinline__ uint64_t forward_tile(uint8_t *xs, uint8_t *hs, uint8_t *w1s, uint8_t *w2s, uint32_t d1,
                                                 Sync &sync, float *z2) {
    const uint32_t t = threadIdx.x, warp = t >> 5;
    constexpr uint32_t i1 = tc::idesc_bf16(128, 64, false, false);
    handoff();
    if (t == 0) {
        for (int s = 0; s < 2; ++s)
            tc::mma_bf16(d1, tc::smem_desc(tc::smem_addr(xs) + 256 * s, 128, kSpX),
                         tc::smem_desc(tc::smem_addr(w1s) + 256 * s, 128, kSoW1), i1, s > 0);
    }
    sync.complete();
    uint64_t mask = 0;
    {
        float v[64];
        tc::tmem_ld64(tc::tmem_at(d1, 32 * warp, 0), v);
#pragma unroll
        for (int q = 0; q < 64; ++q)
            if (v[q] > 0.0f) mask |= 1ull << q;  // only the training kernel uses the mask
#pragma unroll
        for (int g = 0; g < 8; ++g) store_relu_row8(hs, t, g, kSpH, v + 8 * g);
    }
    handoff();
    if (t == 0) {
        for (int s = 0; s < (int)kK2 / 16; ++s)
            tc::mma_bf16(d1, tc::smem_desc(tc::smem_addr(hs) + 256 * s, 128, kSpH),
                         tc::smem_desc(tc::smem_addr(w2s) + 256 * s, 128, kSoW2), i1, s > 0);
    }
    sync.complete();
    tc::tmem_ld64(tc::tmem_at(d1, 32 * warp, 0), z2);
    return mask;
}

// Inference forward of one tile with X and H1 in the same buffer (X is dead once layer 1
// has run) and the TMEM results read in halves of 32 columns, so that a CTA needs ~35 KB of
// shared memory and at most 80 registers a thread: six CTAs per SM.  Returns the head's
// pre-activation w3 . relu(z2) + b3.
__device__ __forceinline__ float infer_tile(uint8_t *buf, uint8_t *w1s, uint8_t *w2s, uint32_t d1, Sync &sync,
                                            const float *w3, float b3) {
    const uint32_t t = threadIdx.x, warp = t >> 5;
    constexpr uint32_t i1 = tc::idesc_bf16(128, 64, false, false);
    handoff();
    if (t == 0) {
        for (int s = 0; s < 2; ++s)
            tc::mma_bf16(d1, tc::smem_desc(tc::smem_addr(buf) + 256 * s, 128, kSpX),
                         tc::smem_desc(tc::smem_addr(w1s) + 256 * s, 128, kSoW1), i1, s > 0);
    }
    sync.complete();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        float v[32];
        tc::tmem_ld32(tc::tmem_at(d1, 32 * warp, 32 * h), v);
#pragma unroll
        for (int g = 0; g < 4; ++g) store_relu_row8(buf, t, 4 * h + g, kSpH, v + 8 * g);
    }
    // H1's constant features (the layer-2 bias input): X covered them
    const uint32_t one = (uint32_t)__bfloat16_as_ushort(__float2bfloat16(1.0f));
    *reinterpret_cast<uint4 *>(buf + act_off(t, 64, kSpH)) = make_uint4(one, 0, 0, 0);
    *reinterpret_cast<uint4 *>(buf + act_off(t, 72, kSpH)) = make_uint4(0, 0, 0, 0);
    handoff();
    if (t == 0) {
        for (int s = 0; s < (int)kK2 / 16; ++s)
            tc::mma_bf16(d1, tc::smem_desc(tc::smem_addr(buf) + 256 * s, 128, kSpH),
                         tc::smem_desc(tc::smem_addr(w2s) + 256 * s, 128, kSoW2), i1, s > 0);
    }
    sync.complete();
    float y = b3;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        float z[32];
        tc::tmem_ld32(tc::tmem_at(d1, 32 * warp, 32 * h), z);
#pragma unroll
        for (int o = 0; o < 32; ++o) y += w3[32 * h + o] * fmaxf(z[o], 0.0f);
    }
    return y;
}

// ---- training -------------------------------------------------------------------------------

struct TrainSmem {
    float w3[64], dw3[64], db3, loss;
    uint64_t mbar;
    uint32_t tmem;
};

// points [P][4] = (x, y, z, target density).  Loss per point (mean over P):
// w (log1p(s) - log1p(t))^2 with s = softplus(y) the bound and w = under_weight when s < t;
// a point with a negative target is ignored (no loss, no gradient; it still counts in P).
__global__ void __launch_bounds__(128) mlp_train_kernel(const float4 *__restrict__ pts, uint32_t P,
                                                        const __nv_bfloat16 *__restrict__ w, float under_weight,
                                                        float *__restrict__ grad, float *__restrict__ loss_out) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *xs = smem;
    uint8_t *hs = xs + kBytesX;
    uint8_t *g2 = hs + kBytesH;
    uint8_t *g1 = g2 + kBytesG;
    uint8_t *w1s = g1 + kBytesG;
    uint8_t *w2s = w1s + kBytesW1;
    TrainSmem &S = *reinterpret_cast<TrainSmem *>(w2s + kBytesW2);
    const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31;
    // zero the gradient operand buffers (their upper 64 feature columns stay zero: rows
    // 64..127 of the padded M = 128 weight-gradient GEMMs)
    for (uint32_t i = t; i < 2 * kBytesG / 16; i += 128) reinterpret_cast<uint4 *>(g2)[i] = make_uint4(0, 0, 0, 0);
    stage_weights(w, w1s, w2s, hs);
    if (t < 64) {
        S.w3[t] = bf16f(w, kOffW3 + t);
        S.dw3[t] = 0.0f;
    }
    if (t == 0) {
        S.db3 = 0.0f;
        S.loss = 0.0f;
        tc::mbar_init(&S.mbar, 1);
    }
    if (warp == 0) tc::tmem_alloc(&S.tmem, kTrainCols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = S.tmem;
    const float b3 = bf16f(w, kOffB3);
    Sync sync{&S.mbar, 0u, true};
    constexpr uint32_t kD1 = 0, kDW2 = 128, kDW1 = 224;  // dW2: 80 columns (64 + db2 + pad), dW1: 32
    const uint32_t tiles = (P + kTile - 1) / kTile;
    bool first = true;
    float my_db3 = 0.0f, my_loss = 0.0f;
    for (uint32_t tile = blockIdx.x; tile < tiles && sync.ok; tile += gridDim.x) {
        const uint32_t g = tile * kTile + t;
        float4 pt = g < P ? *QSDVR_AT(pts, g, 1, P) : make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        const bool valid = pt.w >= 0.0f;
        {
            float f[kF];
            encode(f3{pt.x, pt.y, pt.z}, f);
            if (!valid) f[27] = 0.0f;
#pragma unroll
            for (int q = 0; q < 4; ++q) store_row8(xs, t, q, kSpX, f + 8 * q);
        }
        float z2[kH];
        const uint64_t mask1 = forward_tile(xs, hs, w1s, w2s, tmem + kD1, sync, z2);
        if (!sync.ok) break;
        // head, loss and its gradient
        float y = b3;
#pragma unroll
        for (int o = 0; o < kH; ++o) y += S.w3[o] * fmaxf(z2[o], 0.0f);
        const float s = softplus(y);
        const float e = log1pf(s) - log1pf(pt.w);
        const float wgt = e < 0.0f ? under_weight : 1.0f;
        float dy = 0.0f;
        if (valid) {
            my_loss += wgt * e * e;
            dy = 2.0f * wgt * e / (1.0f + s) * sigmoid(y) / (float)P;
        }
        my_db3 += dy;
        float dh2[kH];
#pragma unroll
        for (int o = 0; o < kH; ++o) {
            const float h2 = fmaxf(z2[o], 0.0f);
            dh2[o] = z2[o] > 0.0f ? dy * S.w3[o] : 0.0f;
            // warp-reduce this output's dw3 partial, one shared add per warp
            float a = dy * h2;
#pragma unroll
            for (int off = 16; off; off >>= 1) a += __shfl_xor_sync(kFull, a, off);
            if (lane == 0) atomicAdd(&S.dw3[o], a);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) store_row8(g2, t, q, kSpG, dh2 + 8 * q);
        handoff();
        if (t == 0) {
            // dH1 = dH2 W2  (A: dH2 K-major over o;  B: W2 viewed MN-major, N = i, K = o)
            constexpr uint32_t i_dh1 = tc::idesc_bf16(128, 64, false, true);
            for (int s4 = 0; s4 < 4; ++s4)
                tc::mma_bf16(tmem + kD1, tc::smem_desc(tc::smem_addr(g2) + 256 * s4, 128, kSpG),
                             tc::smem_desc(tc::smem_addr(w2s) + 2 * kSoW2 * s4, kSoW2, 128), i_dh1, s4 > 0);
            // dW2 += dH2^T H1 (A: dH2 MN-major, M = o padded to 128;  B: H1 MN-major, N = i
            // including the constant feature 64, whose column is db2;  K = points)
            constexpr uint32_t i_dw2 = tc::idesc_bf16(128, kK2, true, true);
            for (int s8 = 0; s8 < 8; ++s8)
                tc::mma_bf16(tmem + kDW2, tc::smem_desc(tc::smem_addr(g2) + 2 * kSpG * s8, kSpG, 128),
                             tc::smem_desc(tc::smem_addr(hs) + 2 * kSpH * s8, kSpH, 128), i_dw2, !(first && s8 == 0));
        }
        sync.complete();
        if (!sync.ok) break;
        {
            float v[64];
            tc::tmem_ld64(tc::tmem_at(tmem, 32 * warp, kD1), v);
#pragma unroll
            for (int q = 0; q < 64; ++q)
                if (!((mask1 >> q) & 1ull)) v[q] = 0.0f;
#pragma unroll
            for (int gq = 0; gq < 8; ++gq) store_row8(g1, t, gq, kSpG, v + 8 * gq);
        }
        handoff();
        if (t == 0) {
            // dW1 += dH1^T X  (A: dH1 MN-major, M = o padded;  B: X MN-major, N = i = 32;  K = points)
            constexpr uint32_t i_dw1 = tc::idesc_bf16(128, 32, true, true);
            for (int s8 = 0; s8 < 8; ++s8)
                tc::mma_bf16(tmem + kDW1, tc::smem_desc(tc::smem_addr(g1) + 2 * kSpG * s8, kSpG, 128),
                             tc::smem_desc(tc::smem_addr(xs) + 2 * kSpX * s8, kSpX, 128), i_dw1, !(first && s8 == 0));
        }
        sync.complete();
        first = false;
    }
    // flush: per-CTA weight gradients from TMEM (rows o = lanes 0..63: warps 0 and 1)
    if (sync.ok && !first) {
        if (warp < 2) {
            const uint32_t o = t;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float v[16];
                tc::tmem_ld16(tc::tmem_at(tmem, 32 * warp, kDW2 + 16 * j), v);
#pragma unroll
                for (int q = 0; q < 16; ++q) atomicAdd(&grad[kOffW2 + o * 64 + 16 * j + q], v[q]);
            }
            {
                float v[16];
                tc::tmem_ld16(tc::tmem_at(tmem, 32 * warp, kDW2 + 64), v);
                atomicAdd(&grad[kOffB2 + o], v[0]);
            }
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                float v[16];
                tc::tmem_ld16(tc::tmem_at(tmem, 32 * warp, kDW1 + 16 * j), v);
#pragma unroll
                for (int q = 0; q < 16; ++q) atomicAdd(&grad[o * 32 + 16 * j + q], v[q]);
            }
        }
        for (int off = 16; off; off >>= 1) {
            my_db3 += __shfl_xor_sync(kFull, my_db3, off);
            my_loss += __shfl_xor_sync(kFull, my_loss, off);
        }
        if (lane == 0) {
            atomicAdd(&S.db3, my_db3);
            atomicAdd(&S.loss, my_loss);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (sync.ok && !first) {
        if (t < 64) atomicAdd(&grad[kOffW3 + t], S.dw3[t]);
        if (t == 0) {
            atomicAdd(&grad[kOffB3], S.db3);
            atomicAdd(loss_out, S.loss / (float)P);
        }
    }
    if (warp == 0) tc::tmem_dealloc(tmem, kTrainCols);
}

// ---- inference --------------------------------------------------------------------------

struct InferSmem {
    float w3[64];
    uint64_t mbar;
    uint32_t tmem;
};

// Point g of the inference input: points[g].xyz, or coarse point g % 64 of ray g / 64 at
// t = (j + 0.5) L / 64, L = (sdf_count - 1) interval.
__device__ __forceinline__ f3 infer_input(const float4 *__restrict__ pts, const qsdvr_ray_info *__restrict__ rays,
                                          const float *__restrict__ origin, const float *__restrict__ dir,
                                          float interval, uint32_t g, [[maybe_unused]] uint64_t extent) {
    if (rays) {  // extent = rays
        const uint32_t r = g >> 6, j = g & 63;
        const uint32_t ns = QSDVR_AT(rays, r, 1, extent)->sdf_count;
        const float L = ns > 1 ? (float)(ns - 1) * interval : 0.0f;
        const float tt = ((float)j + 0.5f) * (L / 64.0f);
        const f3 o = load3(QSDVR_AT(origin, 3ull * r, 3, 3 * extent)), d = load3(QSDVR_AT(dir, 3ull * r, 3, 3 * extent));
        return f3{fmaf(d.x, tt, o.x), fmaf(d.y, tt, o.y), fmaf(d.z, tt, o.z)};
    }
    const float4 q = *QSDVR_AT(pts, g, 1, extent);  // extent = points
    return f3{q.x, q.y, q.z};
}

// Density bound at points [P][4] (xyz used), or — when rays is non-null — at the 64 coarse
// points of every ray (0 for rays with fewer than 2 SDF samples; a tile of two such rays
// skips the MMAs).  Persistent: each CTA walks tiles of 128 points and fetches the next
// tile's input before waiting on this tile's MMAs.
__global__ void __launch_bounds__(128, 6) mlp_infer_kernel(const float4 *__restrict__ pts, uint32_t P,
                                                        const qsdvr_ray_info *__restrict__ rays,
                                                        const float *__restrict__ origin,
                                                        const float *__restrict__ dir, uint32_t nrays,
                                                        float interval, const __nv_bfloat16 *__restrict__ w,
                                                        float *__restrict__ out) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *xs = smem;  // X, then H1 over it (infer_tile)
    uint8_t *w1s = xs + kBytesH;
    uint8_t *w2s = w1s + kBytesW1;
    InferSmem &S = *reinterpret_cast<InferSmem *>(w2s + kBytesW2);
    const uint32_t t = threadIdx.x, warp = t >> 5;
    stage_weights(w, w1s, w2s, xs);
    if (t < 64) S.w3[t] = bf16f(w, kOffW3 + t);
    if (t == 0) tc::mbar_init(&S.mbar, 1);
    if (warp == 0) tc::tmem_alloc(&S.tmem, kInferCols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = S.tmem;
    const float b3 = bf16f(w, kOffB3);
    Sync sync{&S.mbar, 0u, true};
    const uint32_t total = rays ? nrays * 64u : P;
    const uint32_t tiles = (total + kTile - 1) / kTile;
    uint32_t tile = blockIdx.x;
    uint32_t g = tile * kTile + t;
    [[maybe_unused]] const uint64_t extent = rays ? nrays : P;
    f3 p = g < total ? infer_input(pts, rays, origin, dir, interval, g, extent) : f3{0.0f, 0.0f, 0.0f};
    bool live = g < total && (!rays || QSDVR_AT(rays, g >> 6, 1, nrays)->sdf_count > 1);
    while (tile < tiles && sync.ok) {
        const bool valid = g < total, cur_live = live;
        const uint32_t next = tile + gridDim.x;
        const uint32_t gn = next * kTile + t;
        if (!__syncthreads_or(live)) {
            // every ray of the tile misses the volume: its densities are never used
            if (valid) *QSDVR_AT(out, g, 1, total) = 0.0f;
            if (next < tiles && gn < total) p = infer_input(pts, rays, origin, dir, interval, gn, extent);
            live = next < tiles && gn < total && (!rays || QSDVR_AT(rays, gn >> 6, 1, nrays)->sdf_count > 1);
            tile = next;
            g = gn;
            continue;
        }
        {
            float f[kF];
            encode(p, f);
#pragma unroll
            for (int q = 0; q < 4; ++q) store_row8(xs, t, q, kSpX, f + 8 * q);
        }
        // the next tile's input is in flight while this tile runs on the tensor cores
        if (next < tiles && gn < total) p = infer_input(pts, rays, origin, dir, interval, gn, extent);
        live = next < tiles && gn < total && (!rays || QSDVR_AT(rays, gn >> 6, 1, nrays)->sdf_count > 1);
        const float y = infer_tile(xs, w1s, w2s, tmem, sync, S.w3, b3);
        if (valid && sync.ok) *QSDVR_AT(out, g, 1, total) = cur_live ? softplus(y) : 0.0f;
        tile = next;
        g = gn;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kInferCols);
}

// ---- coarse-to-fine sampling ---------------------------------------------------------------
// One warp per kSampleRays rays, processed in lockstep so that their memory and shuffle
// latencies overlap: coarse opacity a_j = 1 - exp(-s_j L/64), weights T_j a_j, a pdf mixed
// with the fraction uniform_mix of uniform, and the 33 fine SDF positions at the CDF
// quantiles k/32 (t_0 = 0, t_32 = L).
constexpr int kSampleRays = 4;

__global__ void __launch_bounds__(256) proposal_sample_kernel(const qsdvr_ray_info *__restrict__ rays,
                                                              uint32_t nrays, float interval, float uniform_mix,
                                                              const float *__restrict__ dens,
                                                              float *__restrict__ tlist) {
    constexpr int kR = kSampleRays;
    __shared__ float cdf_s[8][kR][65];
    const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t r0 = (blockIdx.x * 8 + w) * kR;
    if (r0 >= nrays) return;
    float L[kR], delta[kR], t0[kR], t1[kR];
#pragma unroll
    for (int q = 0; q < kR; ++q) {
        const uint32_t r = r0 + q;
        const bool have = r < nrays;  // warp-uniform
        const uint32_t ns = have ? rays[r].sdf_count : 0u;
        L[q] = ns > 1 ? (float)(ns - 1) * interval : 0.0f;
        delta[q] = L[q] / 64.0f;
        // two coarse bins per lane: j = 2 lane, 2 lane + 1
        const float s0 = have ? *QSDVR_AT(dens, 64ull * r + 2 * lane, 2, 64ull * nrays) : 0.0f,
                    s1 = have ? *QSDVR_AT(dens, 64ull * r + 2 * lane + 1, 1, 64ull * nrays) : 0.0f;
        t0[q] = expf(-fmaxf(s0, 0.0f) * delta[q]);  // 1 - alpha
        t1[q] = expf(-fmaxf(s1, 0.0f) * delta[q]);
    }
    float incl[kR];
#pragma unroll
    for (int q = 0; q < kR; ++q) incl[q] = t0[q] * t1[q];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
        for (int q = 0; q < kR; ++q) {
            const float v = __shfl_up_sync(kFull, incl[q], o);
            if ((int)lane >= o) incl[q] *= v;
        }
    }
    float w0[kR], w1[kR], sum[kR];
#pragma unroll
    for (int q = 0; q < kR; ++q) {
        float T = __shfl_up_sync(kFull, incl[q], 1);
        if (lane == 0) T = 1.0f;
        w0[q] = T * (1.0f - t0[q]);
        w1[q] = T * t0[q] * (1.0f - t1[q]);
        sum[q] = w0[q] + w1[q];
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
#pragma unroll
        for (int q = 0; q < kR; ++q) sum[q] += __shfl_xor_sync(kFull, sum[q], o);
    }
    const float mix = uniform_mix / 64.0f, keep = 1.0f - uniform_mix;
    float p1[kR], c[kR];
#pragma unroll
    for (int q = 0; q < kR; ++q) {
        const float p0 = sum[q] > 0.0f ? keep * w0[q] / sum[q] + mix : 1.0f / 64.0f;
        p1[q] = sum[q] > 0.0f ? keep * w1[q] / sum[q] + mix : 1.0f / 64.0f;
        c[q] = p0 + p1[q];
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
        for (int q = 0; q < kR; ++q) {
            const float v = __shfl_up_sync(kFull, c[q], o);
            if ((int)lane >= o) c[q] += v;
        }
    }
#pragma unroll
    for (int q = 0; q < kR; ++q) {
        const float total = __shfl_sync(kFull, c[q], 31);
        float *cdf = cdf_s[w][q];
        cdf[2 * lane + 1] = (c[q] - p1[q]) / total;
        cdf[2 * lane + 2] = c[q] / total;
        if (lane == 0) cdf[0] = 0.0f;
    }
    __syncwarp();
    // quantile k = lane (k = 0 is t = 0) and, on lane 0, k = 32 (t = L); the bisection
    // cdf[lo] <= k/32 < cdf[lo + 1] over 64 bins takes exactly 6 halvings
#pragma unroll
    for (int q = 0; q < kR; ++q) {
        const uint32_t r = r0 + q;
        if (r >= nrays) break;
        const float *cdf = cdf_s[w][q];
        float tk = 0.0f;
        if (lane > 0) {
            const float qk = (float)lane / 32.0f;
            int lo = 0;
#pragma unroll
            for (int step = 32; step >= 1; step >>= 1)
                if (cdf[lo + step] <= qk) lo += step;
            const float span = cdf[lo + 1] - cdf[lo];
            const float frac = span > 0.0f ? (qk - cdf[lo]) / span : 0.5f;
            tk = fminf(((float)lo + fminf(fmaxf(frac, 0.0f), 1.0f)) * delta[q], L[q]);
        }
        *QSDVR_AT(tlist, 33ull * r + lane, 1, 33ull * nrays) = tk;
        if (lane == 0) *QSDVR_AT(tlist, 33ull * r + 32, 1, 33ull * nrays) = L[q];
    }
}

// ---- check of the bounded waits -------------------------------------------------------------
// One wait, with the tensor-core kernels' own mbar_wait, on an mbarrier that no arrival ever
// completes: it must give up after limit_ns, record QSDVR_DEVERR_TIMEOUT and return.
__global__ void wait_check_kernel(uint64_t limit_ns, uint32_t *completed) {
    __shared__ uint64_t mbar;
    if (threadIdx.x == 0) tc::mbar_init(&mbar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        const bool done = tc::mbar_wait(&mbar, 0, kSpins, limit_ns);
        if (!done) flag_error(QSDVR_DEVERR_TIMEOUT);
        *completed = done ? 1u : 0u;
    }
}

// ---- training targets from the renderer ------------------------------------------------------
// One warp per ray: render sample i of ray r (position midpoint(o, d, i, interval), the
// reference's render sample) with the renderer's alpha gives the target density
// -log(1 - alpha) / interval.
__global__ void __launch_bounds__(256) proposal_targets_kernel(const qsdvr_ray_info *__restrict__ rays,
                                                               const float *__restrict__ origin,
                                                               const float *__restrict__ dir, uint32_t nrays,
                                                               float interval, const float *__restrict__ alpha,
                                                               uint64_t capacity, float4 *__restrict__ pts) {
    const uint32_t r = (blockIdx.x * 256u + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (r >= nrays) return;
    const qsdvr_ray_info info = rays[r];
    if ((uint64_t)info.render_offset + info.render_count > capacity) {
        if (lane == 0) flag_error(QSDVR_DEVERR_CAPACITY);
        return;
    }
    const f3 o = load3(origin + 3ull * r), d = load3(dir + 3ull * r);
    for (uint32_t i = lane; i < info.render_count; i += 32) {
        const uint64_t m = (uint64_t)info.render_offset + i;
        const f3 p = midpoint(o, d, i, interval);
        const float a = fminf(fmaxf(*QSDVR_AT(alpha, m, 1, capacity), 0.0f), 1.0f - 1e-6f);
        *QSDVR_AT(pts, m, 1, capacity) = make_float4(p.x, p.y, p.z, -log1pf(-a) / interval);
    }
}

// ---- training points drawn straight from the renderer's alphas ----------------------------
// Point j: a ray r and render sample i < render_count(r) chosen by a counter-based hash of
// (seed, j) — rays uniformly, then samples uniformly within the ray, up to 16 draws to find a
// ray with samples — at position midpoint(o, d, i) with target -log(1 - alpha) / interval,
// alpha read at rays[r].render_offset + i.  A point that finds no such ray gets target -1
// (ignored by the training kernel).
__device__ __forceinline__ uint32_t mix32(uint32_t x) {  // a 32-bit finaliser hash
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__global__ void __launch_bounds__(256) proposal_draw_kernel(const qsdvr_ray_info *__restrict__ rays,
                                                            const float *__restrict__ origin,
                                                            const float *__restrict__ dir, uint32_t nrays,
                                                            float interval, const float *__restrict__ alpha,
                                                            uint64_t capacity, uint32_t count, uint32_t seed,
                                                            float4 *__restrict__ pts) {
    const uint32_t j = blockIdx.x * 256u + threadIdx.x;
    if (j >= count) return;
    float4 out = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    uint32_t h = mix32(j * 0x9e3779b9u ^ mix32(seed));
    for (int attempt = 0; attempt < 16; ++attempt) {
        const uint32_t r = (uint32_t)(((uint64_t)h * nrays) >> 32);
        const qsdvr_ray_info info = *QSDVR_AT(rays, r, 1, nrays);
        h = mix32(h + 0x632be5abu);
        if (info.render_count == 0) continue;
        const uint32_t i = (uint32_t)(((uint64_t)h * info.render_count) >> 32);
        const uint64_t m = (uint64_t)info.render_offset + i;
        if (m >= capacity) {
            flag_error(QSDVR_DEVERR_CAPACITY);
            break;
        }
        const f3 p = midpoint(load3(QSDVR_AT(origin, 3ull * r, 3, 3ull * nrays)),
                              load3(QSDVR_AT(dir, 3ull * r, 3, 3ull * nrays)), i, interval);
        const float a = fminf(fmaxf(*QSDVR_AT(alpha, m, 1, capacity), 0.0f), 1.0f - 1e-6f);
        out = make_float4(p.x, p.y, p.z, -log1pf(-a) / interval);
        break;
    }
    pts[j] = out;
}

constexpr size_t train_smem() { return kBytesX + kBytesH + 2 * kBytesG + kBytesW1 + kBytesW2 + sizeof(TrainSmem); }
constexpr size_t infer_smem() { return kBytesH + kBytesW1 + kBytesW2 + sizeof(InferSmem); }
// Shared memory alone keeps every resident CTA's TMEM columns free (2 training CTAs x 256
// columns, at most 6 inference CTAs x 64), so tcgen05.alloc never has to wait in practice.
static_assert(2 * train_smem() <= 228 * 1024 && 3 * (train_smem() + 1024) > 228 * 1024,
              "training CTAs: exactly two per SM");
static_assert((228 * 1024 / (infer_smem() + 1024)) * kInferCols <= 512, "inference CTAs: TMEM oversubscribed");
static_assert(6 * (infer_smem() + 1024) <= 228 * 1024, "inference CTAs: six fit per SM");

// Persistent grid: resident CTAs per SM x SMs, capped at the tile count.  The occupancy API
// answers 1 CTA per SM for kernels that use tensor memory (it cannot know how many columns a
// CTA allocates), so residency is computed from the limits themselves: registers (allocated
// per warp in units of 256), shared memory (plus the per-CTA reservation), threads, and the
// 512 TMEM columns over the columns each CTA allocates.  Launching that many is safe either
// way: a CTA whose tcgen05.alloc finds too few free columns waits for a resident CTA to exit,
// and no CTA waits on another.
cudaError_t persistent_blocks(const void *fn, size_t smem, uint32_t tmem_cols, uint32_t tiles, unsigned *blocks,
                              int *per_sm_out) {
    int dev = 0, sms = 0, regs_sm = 0, smem_sm = 0, reserved = 0, threads_sm = 0, blocks_sm = 0;
    cudaFuncAttributes fa;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&blocks_sm, cudaDevAttrMaxBlocksPerMultiprocessor, dev);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
    if (e != cudaSuccess) return e;
    const int warps = kTile / 32;
    const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;
    int per_sm = regs_sm / (regs_warp * warps);
    per_sm = min(per_sm, smem_sm / (int)(smem + fa.sharedSizeBytes + reserved));
    per_sm = min(per_sm, threads_sm / kTile);
    per_sm = min(per_sm, blocks_sm);
    per_sm = min(per_sm, (int)(512 / tmem_cols));
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t b = (uint64_t)sms * (uint64_t)per_sm;
    if (b > tiles) b = tiles;
    *blocks = (unsigned)(b ? b : 1);
    if (per_sm_out) *per_sm_out = per_sm;
    return cudaSuccess;
}

// Opt each kernel in to its dynamic shared memory once per process.
int configure(const void *fn, size_t smem, bool *done, const char *what) {
    if (*done) return QSDVR_OK;
    const int st = check_cuda(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), what);
    if (st == QSDVR_OK) *done = true;
    return st;
}

bool g_train_configured = false, g_infer_configured = false;

}  // namespace
}  // namespace qsdvr

using namespace qsdvr;

extern "C" int qsdvr_mlp_train(const float *points, uint32_t count, const void *params_bf16, float under_weight,
                               float *grad, float *loss, cudaStream_t stream) {
    if (count == 0) return QSDVR_OK;
    if (!points || !params_bf16 || !grad || !loss)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_mlp_train: null pointer");
    if (!aligned(points, 16) || !aligned(params_bf16, 16))
        return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_mlp_train: points and params need 16-byte alignment");
    const void *fn = (const void *)mlp_train_kernel;
    int st = configure(fn, train_smem(), &g_train_configured, "qsdvr_mlp_train: smem attribute");
    if (st != QSDVR_OK) return st;
    unsigned blocks = 0;
    st = check_cuda(persistent_blocks(fn, train_smem(), kTrainCols, (count + kTile - 1) / kTile, &blocks, nullptr),
                    "qsdvr_mlp_train: occupancy");
    if (st != QSDVR_OK) return st;
    mlp_train_kernel<<<blocks, kTile, train_smem(), stream>>>(reinterpret_cast<const float4 *>(points), count,
                                                              static_cast<const __nv_bfloat16 *>(params_bf16),
                                                              under_weight, grad, loss);
    return check_launch("qsdvr_mlp_train");
}

extern "C" int qsdvr_mlp_density(const float *points, uint32_t count, const qsdvr_ray_info *rays, const float *origin,
                                 const float *dir, uint32_t ray_count, float interval, const void *params_bf16,
                                 float *out, cudaStream_t stream) {
    const uint32_t total = rays ? ray_count * 64u : count;
    if (total == 0) return QSDVR_OK;
    if (!params_bf16 || !out || (rays ? (!origin || !dir) : !points))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_mlp_density: null pointer");
    if ((points && !aligned(points, 16)) || !aligned(params_bf16, 16))
        return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_mlp_density: points and params need 16-byte alignment");
    if (rays && ray_count > (1u << 25))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_mlp_density: too many rays");
    const void *fn = (const void *)mlp_infer_kernel;
    int st = configure(fn, infer_smem(), &g_infer_configured, "qsdvr_mlp_density: smem attribute");
    if (st != QSDVR_OK) return st;
    unsigned blocks = 0;
    st = check_cuda(persistent_blocks(fn, infer_smem(), kInferCols, (total + kTile - 1) / kTile, &blocks, nullptr),
                    "qsdvr_mlp_density: occupancy");
    if (st != QSDVR_OK) return st;
    mlp_infer_kernel<<<blocks, kTile, infer_smem(), stream>>>(reinterpret_cast<const float4 *>(points), count, rays,
                                                              origin, dir, ray_count, interval,
                                                              static_cast<const __nv_bfloat16 *>(params_bf16), out);
    return check_launch("qsdvr_mlp_density");
}

extern "C" int qsdvr_mlp_launch_shape(int kernel, uint32_t count, uint32_t *blocks, int *blocks_per_sm) {
    if (!blocks || !blocks_per_sm || (kernel != 0 && kernel != 1))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_mlp_launch_shape: bad arguments");
    const void *fn = kernel == 0 ? (const void *)mlp_infer_kernel : (const void *)mlp_train_kernel;
    const size_t smem = kernel == 0 ? infer_smem() : train_smem();
    int st = configure(fn, smem, kernel == 0 ? &g_infer_configured : &g_train_configured,
                       "qsdvr_mlp_launch_shape: smem attribute");
    if (st != QSDVR_OK) return st;
    unsigned b = 0;
    st = check_cuda(persistent_blocks(fn, smem, kernel == 0 ? kInferCols : kTrainCols, (count + kTile - 1) / kTile, &b,
                                      blocks_per_sm),
                    "qsdvr_mlp_launch_shape: occupancy");
    *blocks = b;
    return st;
}

extern "C" int qsdvr_proposal_sample(const qsdvr_ray_info *rays, uint32_t ray_count, float interval,
                                     float uniform_mix, const float *coarse_density, float *tlist,
                                     cudaStream_t stream) {
    if (ray_count == 0) return QSDVR_OK;
    if (!rays || !coarse_density || !tlist)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_proposal_sample: null pointer");
    if (!(uniform_mix > 0.0f && uniform_mix <= 1.0f))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_proposal_sample: uniform_mix must be in (0, 1]");
    proposal_sample_kernel<<<grid_for(ray_count, 8 * kSampleRays), 256, 0, stream>>>(rays, ray_count, interval,
                                                                                     uniform_mix, coarse_density,
                                                                                     tlist);
    return check_launch("qsdvr_proposal_sample");
}

extern "C" int qsdvr_check_bounded_wait(uint64_t limit_ns, uint32_t *completed, cudaStream_t stream) {
    if (!completed) return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_check_bounded_wait: null pointer");
    if (limit_ns == 0 || limit_ns > 2000000000ull)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_check_bounded_wait: limit must be in (0, 2 s]");
    wait_check_kernel<<<1, 32, 0, stream>>>(limit_ns, completed);
    return check_launch("qsdvr_check_bounded_wait");
}

extern "C" int qsdvr_proposal_targets(const qsdvr_ray_info *rays, const float *origin, const float *dir,
                                      uint32_t ray_count, float interval, const float *alpha, uint64_t sample_count,
                                      float *points, cudaStream_t stream) {
    if (ray_count == 0) return QSDVR_OK;
    if (!rays || !origin || !dir || !alpha || !points)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_proposal_targets: null pointer");
    if (!aligned(points, 16)) return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_proposal_targets: points alignment");
    proposal_targets_kernel<<<grid_for((uint64_t)ray_count * 32, 256), 256, 0, stream>>>(
        rays, origin, dir, ray_count, interval, alpha, sample_count, reinterpret_cast<float4 *>(points));
    return check_launch("qsdvr_proposal_targets");
}

extern "C" int qsdvr_proposal_draw(const qsdvr_ray_info *rays, const float *origin, const float *dir,
                                   uint32_t ray_count, float interval, const float *alpha, uint64_t sample_count,
                                   uint32_t count, uint32_t seed, float *points, cudaStream_t stream) {
    if (count == 0) return QSDVR_OK;
    if (ray_count == 0 || !rays || !origin || !dir || !alpha || !points)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_proposal_draw: null pointer or no rays");
    if (!aligned(points, 16)) return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_proposal_draw: points alignment");
    proposal_draw_kernel<<<grid_for(count, 256), 256, 0, stream>>>(rays, origin, dir, ray_count, interval, alpha,
                                                                  sample_count, count, seed,
                                                                  reinterpret_cast<float4 *>(points));
    return check_launch("qsdvr_proposal_draw");
}
