// Fused grid optimizer: Adam on the FP32 master grids in one pass over HBM, optionally
// refreshing the BF16 storage copy the render kernels read and zeroing the gradient for
// the next step (the reference runs torch.optim.Adam then zero_grad, test.py:34-35).
//
// Per element: m = m + (1 - b1)(g - m); v = b2 v + (1 - b2) g^2;
// p -= (lr / (1 - b1^t)) m / (sqrt(v) / sqrt(1 - b2^t) + eps)   (torch.optim.Adam's formula).
//
// BF16 quadric cells.  A cell's SDF sample is f(u) / |grad_u f| / R, invariant to a common
// scale of its 7 coefficients; rounding a3..a5 to bf16 each by up to 2^-9 rescales |grad f|
// and so the whole cell's SDF by ~2^-9.  Far from the surface that is ~1e-3 of absolute SDF,
// more than the SDF changes between two samples of a ray that runs nearly along a level set,
// and the NeuS alpha max((E1 - E0) / (1 + E1), 0) then flips between active and inactive
// there: the SDF-coefficient gradient of those samples jumps.  The storage copy therefore
// keeps a0..a5 rounded to nearest and replaces a6 by a6 |bf16(a3..a5)| / |a3..a5|, which
// makes the cell-centre SDF of the stored cell equal the master's, and stores it as two bf16
// (hi = bf16(a6'), lo = bf16(a6' - hi)) in slots 6 and 7 (slot 7 is the fp32 layout's pad);
// the render kernels read a6 = hi + lo (exact in fp32).  A copy made by plain rounding (lo =
// 0) is read the same way.
#include <cuda_bf16.h>

#include "common.cuh"

namespace qsdvr {

QSDVR_ERROR_WORD_ACCESSOR(optim)

namespace {

struct AdamParams {
    float *param, *grad, *m, *v;  // grad holds bf16 values in the kBf16Grad kernel
    __nv_bfloat16 *copy;
    uint64_t n;
    float b1, b2, one_minus_b1, one_minus_b2, step_size, bc2_sqrt, eps;
    bool zero_grad, skip_zero;
    bool state_bf16;  // m and v hold bf16 values, stochastically rounded after each update
    uint32_t seed;    // per-step seed of the stochastic rounding
};

// Stochastic rounding of the bf16 moments (QSDVR_ADAM_STATE_BF16).  Adam's second moment
// decays by beta2 = 0.999 per step, a relative change below half a bf16 ulp (2^-9), so round
// to nearest would leave it frozen; rounding up with probability equal to the discarded
// fraction keeps every moment unbiased.  The random bits come from a counter-based integer
// hash (the "lowbias32" xorshift-multiply mixer) of the element group and the step.
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ uint32_t sr_bf16(float x, uint32_t r16) {
    uint32_t u = __float_as_uint(x);
    if ((u & 0x7f800000u) != 0x7f800000u) u += r16 & 0xffffu;  // inf and NaN keep their bits
    return u >> 16;
}
__device__ __forceinline__ float4 bf16x4(uint2 r) {
    return make_float4(__uint_as_float(r.x << 16), __uint_as_float(r.x & 0xffff0000u), __uint_as_float(r.y << 16),
                       __uint_as_float(r.y & 0xffff0000u));
}
__device__ __forceinline__ uint2 sr_bf16x4(float4 v, uint32_t ra, uint32_t rb) {
    return make_uint2(sr_bf16(v.x, ra) | (sr_bf16(v.y, ra >> 16) << 16), sr_bf16(v.z, rb) | (sr_bf16(v.w, rb >> 16) << 16));
}

__device__ __forceinline__ uint32_t bf16_bits(float x) { return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf16_value(uint32_t b) { return __uint_as_float(b << 16); }

// The 16-byte bf16 form of one fp32 cell (a0..a3 in lo, a4..a6 + pad in hi), as described above.
__device__ __forceinline__ uint4 encode_sdf_cell(float4 lo, float4 hi) {
    const uint32_t r0 = bf16_bits(lo.x), r1 = bf16_bits(lo.y), r2 = bf16_bits(lo.z), r3 = bf16_bits(lo.w),
                   r4 = bf16_bits(hi.x), r5 = bf16_bits(hi.y);
    const float a3 = lo.w, a4 = hi.x, a5 = hi.y, a6 = hi.z;
    const float b3 = bf16_value(r3), b4 = bf16_value(r4), b5 = bf16_value(r5);
    const float n0 = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(a3, a3), __fmul_rn(a4, a4)), __fmul_rn(a5, a5)));
    const float n1 = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(b3, b3), __fmul_rn(b4, b4)), __fmul_rn(b5, b5)));
    float c6 = a6;
    if (n0 > 0.0f && isfinite(n0) && isfinite(n1)) c6 = __fmul_rn(a6, __fdiv_rn(n1, n0));
    const uint32_t h6 = bf16_bits(c6);
    const uint32_t l6 = isfinite(c6) ? bf16_bits(__fsub_rn(c6, bf16_value(h6))) : 0u;
    return make_uint4(r0 | (r1 << 16), r2 | (r3 << 16), r4 | (r5 << 16), h6 | (l6 << 16));
}

__global__ void __launch_bounds__(256) sdf_cells_bf16_kernel(const float *__restrict__ cells, uint4 *__restrict__ out,
                                                             uint64_t count) {
    const uint64_t stride = (uint64_t)gridDim.x * 256;
    for (uint64_t c = blockIdx.x * 256ull + threadIdx.x; c < count; c += stride)
        out[c] = encode_sdf_cell(ld4(cells + 8 * c), ld4(cells + 8 * c + 4));
}

__device__ __forceinline__ void adam_one(float &p, float g, float &m, float &v, const AdamParams &a) {
    m = m + a.one_minus_b1 * (g - m);       // lerp(m, g, 1 - b1)
    v = __fmul_rn(v, a.b2);                  // v *= b2, then v += (1 - b2) g g
    v = v + a.one_minus_b2 * g * g;
    const float denom = sqrtf(v) / a.bc2_sqrt + a.eps;
    p = p - a.step_size * (m / denom);
}

// Gradient elements [4i, 4i + 4) as floats, and their zeroing, for fp32 or bf16 gradients.
template <bool kBf16Grad>
__device__ __forceinline__ float4 grad4(const AdamParams &a, uint64_t i) {
    if (!kBf16Grad) return ld4(a.grad + 4 * i);
    const uint2 r = reinterpret_cast<const uint2 *>(a.grad)[i];
    return make_float4(__uint_as_float(r.x << 16), __uint_as_float(r.x & 0xffff0000u), __uint_as_float(r.y << 16),
                       __uint_as_float(r.y & 0xffff0000u));
}
template <bool kBf16Grad>
__device__ __forceinline__ void zero_grad4(const AdamParams &a, uint64_t i) {
    if (kBf16Grad) reinterpret_cast<uint2 *>(a.grad)[i] = make_uint2(0u, 0u);
    else st4(a.grad + 4 * i, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
}
template <bool kBf16Grad>
__device__ __forceinline__ float grad1(const AdamParams &a, uint64_t i) {
    if (!kBf16Grad) return a.grad[i];
    return __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(a.grad)[i]);
}

// One group of 4 elements: loads the gradient and, unless every element is skipped, updates
// p, m and v in place (stored back) and zeroes the gradient.  Returns whether p changed; p
// holds the group's parameters whenever it did, or when `load` asks for them anyway.
template <bool kBf16Grad>
__device__ __forceinline__ bool adam_group(const AdamParams &a, uint64_t i, float4 &p, bool load) {
    float4 g = grad4<kBf16Grad>(a, i);
    if (a.skip_zero && g.x == 0.0f && g.y == 0.0f && g.z == 0.0f && g.w == 0.0f) {
        if (load) p = ld4(a.param + 4 * i);
        return false;
    }
    p = ld4(a.param + 4 * i);
    float4 m, v;
    if (a.state_bf16) {
        m = bf16x4(reinterpret_cast<const uint2 *>(a.m)[i]);
        v = bf16x4(reinterpret_cast<const uint2 *>(a.v)[i]);
    } else {
        m = ld4(a.m + 4 * i);
        v = ld4(a.v + 4 * i);
    }
    if (!a.skip_zero || g.x != 0.0f) adam_one(p.x, g.x, m.x, v.x, a);
    if (!a.skip_zero || g.y != 0.0f) adam_one(p.y, g.y, m.y, v.y, a);
    if (!a.skip_zero || g.z != 0.0f) adam_one(p.z, g.z, m.z, v.z, a);
    if (!a.skip_zero || g.w != 0.0f) adam_one(p.w, g.w, m.w, v.w, a);
    st4(a.param + 4 * i, p);
    if (a.state_bf16) {
        const uint32_t h0 = mix32((uint32_t)i ^ mix32((uint32_t)(i >> 32) ^ a.seed)), h1 = mix32(h0), h2 = mix32(h1),
                       h3 = mix32(h2);
        reinterpret_cast<uint2 *>(a.m)[i] = sr_bf16x4(m, h0, h1);
        reinterpret_cast<uint2 *>(a.v)[i] = sr_bf16x4(v, h2, h3);
    } else {
        st4(a.m + 4 * i, m);
        st4(a.v + 4 * i, v);
    }
    if (a.zero_grad) zero_grad4<kBf16Grad>(a, i);
    return true;
}

template <bool kBf16Grad>
__global__ void __launch_bounds__(256) adam_kernel(const AdamParams a) {
    const uint64_t n4 = a.n / 4;
    const uint64_t stride = (uint64_t)gridDim.x * 256;
    for (uint64_t i = blockIdx.x * 256ull + threadIdx.x; i < n4; i += stride) {
        float4 p;
        if (!adam_group<kBf16Grad>(a, i, p, false) || !a.copy) continue;
        __nv_bfloat162 lo = __floats2bfloat162_rn(p.x, p.y), hi = __floats2bfloat162_rn(p.z, p.w);
        uint2 packed;
        packed.x = *reinterpret_cast<uint32_t *>(&lo);
        packed.y = *reinterpret_cast<uint32_t *>(&hi);
        *reinterpret_cast<uint2 *>(a.copy + 4 * i) = packed;
    }
    // tail (n not a multiple of 4)
    for (uint64_t i = 4 * n4 + blockIdx.x * 256ull + threadIdx.x; i < a.n; i += stride) {
        const float g = grad1<kBf16Grad>(a, i);
        if (a.skip_zero && g == 0.0f) continue;
        __nv_bfloat16 *mb = reinterpret_cast<__nv_bfloat16 *>(a.m), *vb = reinterpret_cast<__nv_bfloat16 *>(a.v);
        float p = a.param[i];
        float m = a.state_bf16 ? __bfloat162float(mb[i]) : a.m[i], v = a.state_bf16 ? __bfloat162float(vb[i]) : a.v[i];
        adam_one(p, g, m, v, a);
        a.param[i] = p;
        if (a.state_bf16) {
            const uint32_t h = mix32(mix32((uint32_t)i ^ a.seed) ^ 0x51ed270bu);
            mb[i] = __ushort_as_bfloat16((unsigned short)sr_bf16(m, h));
            vb[i] = __ushort_as_bfloat16((unsigned short)sr_bf16(v, h >> 16));
        } else {
            a.m[i] = m;
            a.v[i] = v;
        }
        if (a.zero_grad) {
            if (kBf16Grad) reinterpret_cast<__nv_bfloat16 *>(a.grad)[i] = __float2bfloat16_rn(0.0f);
            else a.grad[i] = 0.0f;
        }
        if (a.copy) a.copy[i] = __float2bfloat16_rn(p);
    }
}

// QSDVR_ADAM_SDF_CELLS: the parameters are quadric cells [n/8][8] with an fp32 gradient; one
// thread per cell, so the bf16 copy is written in the compensated cell form.
__global__ void __launch_bounds__(256) adam_cells_kernel(const AdamParams a) {
    const uint64_t cells = a.n / 8;
    const uint64_t stride = (uint64_t)gridDim.x * 256;
    for (uint64_t c = blockIdx.x * 256ull + threadIdx.x; c < cells; c += stride) {
        float4 lo, hi;
        const bool ch_lo = adam_group<false>(a, 2 * c, lo, a.copy != nullptr);
        const bool ch_hi = adam_group<false>(a, 2 * c + 1, hi, a.copy != nullptr);
        if (a.copy && (ch_lo || ch_hi)) reinterpret_cast<uint4 *>(a.copy)[c] = encode_sdf_cell(lo, hi);
    }
}

}  // namespace
}  // namespace qsdvr

using namespace qsdvr;

static uint32_t mix32_host(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

extern "C" int qsdvr_adam_step(const qsdvr_adam_args *args, cudaStream_t stream) {
    if (!args) return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_adam_step: null args");
    if (args->count == 0) return QSDVR_OK;
    if (!args->param || !args->grad || !args->exp_avg || !args->exp_avg_sq)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_adam_step: null pointer");
    if (!aligned(args->param, 16) || !aligned(args->grad, 16) || !aligned(args->exp_avg, 16) ||
        !aligned(args->exp_avg_sq, 16) || (args->param_bf16 && !aligned(args->param_bf16, 8)))
        return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_adam_step: buffers need 16-byte (copy 8-byte) alignment");
    if (args->step == 0 || !(args->beta1 >= 0.0 && args->beta1 < 1.0) || !(args->beta2 >= 0.0 && args->beta2 < 1.0))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_adam_step: step must be >= 1 and betas in [0,1)");
    AdamParams a;
    a.param = args->param;
    a.grad = args->grad;
    a.m = args->exp_avg;
    a.v = args->exp_avg_sq;
    a.copy = static_cast<__nv_bfloat16 *>(args->param_bf16);
    a.n = args->count;
    // constants rounded once from double, as torch.optim.Adam's scalars are
    a.b1 = (float)args->beta1;
    a.b2 = (float)args->beta2;
    a.one_minus_b1 = (float)(1.0 - args->beta1);
    a.one_minus_b2 = (float)(1.0 - args->beta2);
    const double bc1 = 1.0 - pow(args->beta1, (double)args->step);
    const double bc2 = 1.0 - pow(args->beta2, (double)args->step);
    a.step_size = (float)(args->lr / bc1);
    a.bc2_sqrt = (float)sqrt(bc2);
    a.eps = (float)args->eps;
    a.zero_grad = (args->flags & QSDVR_ADAM_ZERO_GRAD) != 0;
    a.skip_zero = (args->flags & QSDVR_ADAM_SKIP_ZERO_GRAD) != 0;
    a.state_bf16 = (args->flags & QSDVR_ADAM_STATE_BF16) != 0;
    a.seed = mix32_host(args->step);
    const uint64_t work = (args->count + 3) / 4;
    unsigned blocks = grid_for(work, 256);
    const unsigned cap = 148u * 16;  // a few waves of resident blocks, grid-stride beyond
    if (blocks > cap) blocks = cap;
    if (args->flags & QSDVR_ADAM_SDF_CELLS) {
        if (args->flags & QSDVR_ADAM_GRAD_BF16)
            return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_adam_step: SDF cells take an fp32 gradient");
        if (args->count % 8 != 0 || (args->param_bf16 && !aligned(args->param_bf16, 16)))
            return set_error(QSDVR_ERR_INVALID_ARGUMENT,
                             "qsdvr_adam_step: SDF cells need a multiple of 8 elements and a 16-byte aligned copy");
        unsigned cblocks = grid_for(args->count / 8, 256);
        if (cblocks > cap) cblocks = cap;
        adam_cells_kernel<<<cblocks, 256, 0, stream>>>(a);
    } else if (args->flags & QSDVR_ADAM_GRAD_BF16) {
        adam_kernel<true><<<blocks, 256, 0, stream>>>(a);
    } else {
        adam_kernel<false><<<blocks, 256, 0, stream>>>(a);
    }
    return check_launch("qsdvr_adam_step");
}

extern "C" int qsdvr_sdf_cells_bf16(const float *cells, void *out, uint64_t cell_count, cudaStream_t stream) {
    if (cell_count == 0) return QSDVR_OK;
    if (!cells || !out) return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_sdf_cells_bf16: null pointer");
    if (!aligned(cells, 16) || !aligned(out, 16))
        return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_sdf_cells_bf16: buffers need 16-byte alignment");
    unsigned blocks = grid_for(cell_count, 256);
    if (blocks > 148u * 16) blocks = 148u * 16;
    sdf_cells_bf16_kernel<<<blocks, 256, 0, stream>>>(cells, static_cast<uint4 *>(out), cell_count);
    return check_launch("qsdvr_sdf_cells_bf16");
}
