// Per-op appearance fetch, shading and compositing (kernel/render.cu), the drop-in
// equivalents of the reference's six render kernels.  The fused path lives in fused.cu.
#include "common.cuh"
#include "shading.cuh"

namespace qsdvr {

QSDVR_ERROR_WORD_ACCESSOR(render)

namespace {

constexpr int kC = 32;  // channels per vertex (kernel/render.cu:3)

// ---- trilinear fetch (kernel/render.cu:93-152) ---------------------------------------------
// Eight lanes per sample, each owning one float4 of the 32 channels, so every load and
// every vector RED of a warp covers four whole 128-byte vertex rows.

__device__ __forceinline__ float lerp_ref(float a, float b, float x) { return a * (1 - x) + b * x; }

__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float x) {
    return make_float4(lerp_ref(a.x, b.x, x), lerp_ref(a.y, b.y, x), lerp_ref(a.z, b.z, x), lerp_ref(a.w, b.w, x));
}

__device__ __forceinline__ bool corners_ok(int32_t idx, uint32_t reso, uint64_t vertices) {
    if (idx < 0 || (uint64_t)idx + (uint64_t)reso * reso + reso + 1 >= vertices) {
        flag_error(QSDVR_DEVERR_INDEX);
        return false;
    }
    return true;
}

__global__ void __launch_bounds__(256) interp_forward_kernel(const float *__restrict__ data,
                                                             const float *__restrict__ pts,
                                                             const int32_t *__restrict__ index,
                                                             float *__restrict__ out, uint64_t n, uint32_t reso,
                                                             uint64_t vertices) {
    const uint64_t t = blockIdx.x * 256ull + threadIdx.x;
    const uint64_t s = t >> 3;
    const int q = (int)(t & 7);
    if (s >= n) return;
    const int32_t idx = index[s];
    if (!corners_ok(idx, reso, vertices)) {
        st4(out + s * kC + 4 * q, make_float4(0, 0, 0, 0));
        return;
    }
    const float px = (pts[3 * s] + 1.0f) / 2.0f, py = (pts[3 * s + 1] + 1.0f) / 2.0f,
                pz = (pts[3 * s + 2] + 1.0f) / 2.0f;
    const uint64_t dy = (uint64_t)reso * kC, dz = (uint64_t)reso * reso * kC;
    const float *b = data + (uint64_t)idx * kC + 4 * q;
    const float4 v000 = ld4(b), v001 = ld4(b + kC), v010 = ld4(b + dy), v011 = ld4(b + dy + kC);
    const float4 v100 = ld4(b + dz), v101 = ld4(b + dz + kC), v110 = ld4(b + dz + dy), v111 = ld4(b + dz + dy + kC);
    const float4 a0 = lerp4(lerp4(v000, v001, px), lerp4(v010, v011, px), py);
    const float4 a1 = lerp4(lerp4(v100, v101, px), lerp4(v110, v111, px), py);
    st4(out + s * kC + 4 * q, lerp4(a0, a1, pz));
}

__global__ void __launch_bounds__(256) interp_backward_kernel(float *__restrict__ grad_data,
                                                              const float *__restrict__ pts,
                                                              const int32_t *__restrict__ index,
                                                              const float *__restrict__ gout, uint64_t n,
                                                              uint32_t reso, uint64_t vertices) {
    const uint64_t t = blockIdx.x * 256ull + threadIdx.x;
    const uint64_t s = t >> 3;
    const int q = (int)(t & 7);
    if (s >= n) return;
    const int32_t idx = index[s];
    if (!corners_ok(idx, reso, vertices)) return;
    const float px = (pts[3 * s] + 1.0f) / 2.0f, py = (pts[3 * s + 1] + 1.0f) / 2.0f,
                pz = (pts[3 * s + 2] + 1.0f) / 2.0f;
    const float4 g = ld4(gout + s * kC + 4 * q);
    // a zero gradient quad (a sample with alpha = 0 or T = 0) adds nothing: its eight REDs,
    // each an L2 read-modify-write, are skipped and the sums stay bit-identical (is_zero4)
    if (is_zero4(g)) return;
    const float dx = 1 - px, dy = 1 - py;
    // kernel/render.cu:136-151: weights applied in the reference's order.
    auto scale = [](float4 v, float w) { return make_float4(v.x * w, v.y * w, v.z * w, v.w * w); };
    const float4 a0 = scale(g, 1 - pz), a1 = scale(g, pz);
    const float4 a00 = scale(a0, dy), a01 = scale(a0, py), a10 = scale(a1, dy), a11 = scale(a1, py);
    const uint64_t sy = (uint64_t)reso * kC, sz = (uint64_t)reso * reso * kC;
    float *b = grad_data + (uint64_t)idx * kC + 4 * q;
    red4(b, scale(a00, dx));
    red4(b + kC, scale(a00, px));
    red4(b + sy, scale(a01, dx));
    red4(b + sy + kC, scale(a01, px));
    red4(b + sz, scale(a10, dx));
    red4(b + sz + kC, scale(a10, px));
    red4(b + sz + sy, scale(a11, dx));
    red4(b + sz + sy + kC, scale(a11, px));
}

// ---- shader (kernel/render.cu:154-221) -------------------------------------------------------

__device__ __forceinline__ void load_row(const float *p, float *d) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float4 v = ld4(p + 4 * k);
        d[4 * k] = v.x;
        d[4 * k + 1] = v.y;
        d[4 * k + 2] = v.z;
        d[4 * k + 3] = v.w;
    }
}

template <bool kCompat>
__global__ void __launch_bounds__(128) shader_forward_kernel(float *__restrict__ out, const float *__restrict__ nrm,
                                                             const float *__restrict__ view,
                                                             const float *__restrict__ data,
                                                             float *__restrict__ spec_out, uint64_t n) {
    const uint64_t id = blockIdx.x * 128ull + threadIdx.x;
    if (id >= n) return;
    float d[kC];
    load_row(data + id * kC, d);
    f3 spec;
    const f3 rgb = shade<kCompat>(load3(nrm + 3 * id), load3(view + 3 * id), d, &spec);
    store3(out + 3 * id, rgb);
    store3(spec_out + 3 * id, spec);
}

template <bool kCompat>
__global__ void __launch_bounds__(128) shader_backward_kernel(const float *__restrict__ gout,
                                                              const float *__restrict__ nrm,
                                                              const float *__restrict__ view,
                                                              const float *__restrict__ data,
                                                              const float *__restrict__ spec,
                                                              float *__restrict__ ngrad, float *__restrict__ dgrad,
                                                              uint64_t n) {
    const uint64_t id = blockIdx.x * 128ull + threadIdx.x;
    if (id >= n) return;
    float d[kC], g[kC];
    load_row(data + id * kC, d);
    const f3 ng = shade_backward<kCompat>(load3(gout + 3 * id), load3(nrm + 3 * id), load3(view + 3 * id), d,
                                          load3(spec + 3 * id), g);
    store3(ngrad + 3 * id, ng);
#pragma unroll
    for (int k = 0; k < 8; ++k) st4(dgrad + id * kC + 4 * k, make_float4(g[4 * k], g[4 * k + 1], g[4 * k + 2], g[4 * k + 3]));
}

// ---- compositing (kernel/render.cu:223-315) ----------------------------------------------
// One warp per ray, 32 render samples per step; transmittance is an exclusive prefix
// product by warp shuffles, carried across steps.

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ bool ray_ok(const qsdvr_ray_info &r, uint64_t sdf_cap, uint64_t render_cap) {
    const bool counts = r.sdf_count == 0 || r.render_count + 1 == r.sdf_count;
    if (!counts || (uint64_t)r.sdf_offset + r.sdf_count > sdf_cap ||
        (uint64_t)r.render_offset + r.render_count > render_cap) {
        flag_error(counts ? QSDVR_DEVERR_CAPACITY : QSDVR_DEVERR_RAY);
        return false;
    }
    return true;
}

__global__ void __launch_bounds__(256) aggregate_forward_kernel(float *__restrict__ out,
                                                                const float *__restrict__ rgb,
                                                                const float *__restrict__ sdf,
                                                                const qsdvr_ray_info *__restrict__ rays,
                                                                float *__restrict__ alpha_out,
                                                                float *__restrict__ t_out, uint32_t n, float k,
                                                                uint64_t sdf_cap, uint64_t render_cap) {
    const uint64_t r = (blockIdx.x * 256ull + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    const qsdvr_ray_info info = rays[r];
    f3 color{0.0f, 0.0f, 0.0f};
    if (info.sdf_count != 0 && ray_ok(info, sdf_cap, render_cap)) {
        float carry = 1.0f;
        for (uint32_t base = 0; base < info.render_count; base += kWarp) {
            const uint32_t i = base + lane;
            const bool valid = i < info.render_count;
            float a = 0.0f;
            if (valid) {
                const float e0 = expf(-k * *QSDVR_AT(sdf, (uint64_t)info.sdf_offset + i, 2, sdf_cap));
                const float e1 = expf(-k * *QSDVR_AT(sdf, (uint64_t)info.sdf_offset + i + 1, 1, sdf_cap));
                a = fmaxf((e1 - e0) / (1.0f + e1), 0.0f);
            }
            float incl = valid ? 1.0f - a : 1.0f;
#pragma unroll
            for (int o = 1; o < kWarp; o <<= 1) {
                const float v = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl *= v;
            }
            float excl = __shfl_up_sync(kFull, incl, 1);
            if (lane == 0) excl = 1.0f;
            const float T = carry * excl;
            f3 c{0.0f, 0.0f, 0.0f};
            if (valid) {
                const uint64_t m = (uint64_t)info.render_offset + i;
                *QSDVR_AT(alpha_out, m, 1, render_cap) = a;
                *QSDVR_AT(t_out, m, 1, render_cap) = T;
                const f3 v = load3(QSDVR_AT(rgb, 3 * m, 3, 3 * render_cap));
                c = f3{v.x * a * T, v.y * a * T, v.z * a * T};
            }
            color.x += warp_sum(c.x);
            color.y += warp_sum(c.y);
            color.z += warp_sum(c.z);
            carry *= __shfl_sync(kFull, incl, kWarp - 1);
        }
    }
    if (lane == 0) store3(out + 3 * r, color);
}

// Reverse pass: suffix sums of T a c (the reference's Tac) by a reverse warp scan, the
// derivative formulas of kernel/render.cu:266-313 per render sample, and the two
// contributions to each SDF sample combined by one shuffle.
__global__ void __launch_bounds__(256) aggregate_backward_kernel(
    const float *__restrict__ gout, const float *__restrict__ rgb, const float *__restrict__ sdf,
    const qsdvr_ray_info *__restrict__ rays, const float *__restrict__ alpha, const float *__restrict__ tr,
    float *__restrict__ rgb_grad, float *__restrict__ sdf_grad, uint32_t n, float k, uint64_t sdf_cap,
    uint64_t render_cap) {
    const uint64_t r = (blockIdx.x * 256ull + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    const qsdvr_ray_info info = rays[r];
    if (info.sdf_count == 0 || !ray_ok(info, sdf_cap, render_cap)) return;
    const uint32_t nr = info.render_count;
    if (nr == 0) {
        if (lane == 0) *QSDVR_AT(sdf_grad, info.sdf_offset, 1, sdf_cap) = 0.0f;
        return;
    }
    const f3 g = load3(gout + 3 * r);
    f3 tac_carry{0.0f, 0.0f, 0.0f};  // sum of T a c over samples after this chunk
    float next_this = 0.0f;          // d_this contribution of the first sample of the next chunk
    const uint32_t chunks = (nr + kWarp - 1) / kWarp;
    for (int ch = (int)chunks - 1; ch >= 0; --ch) {
        const uint32_t i = (uint32_t)ch * kWarp + lane;
        const bool valid = i < nr;
        float a = 0.0f, T = 0.0f, e0 = 0.0f, e1 = 0.0f;
        f3 c{0.0f, 0.0f, 0.0f};
        if (valid) {
            const uint64_t m = (uint64_t)info.render_offset + i;
            a = *QSDVR_AT(alpha, m, 1, render_cap);
            T = *QSDVR_AT(tr, m, 1, render_cap);
            c = load3(QSDVR_AT(rgb, 3 * m, 3, 3 * render_cap));
            e0 = expf(-k * *QSDVR_AT(sdf, (uint64_t)info.sdf_offset + i, 2, sdf_cap));
            e1 = expf(-k * *QSDVR_AT(sdf, (uint64_t)info.sdf_offset + i + 1, 1, sdf_cap));
        }
        const f3 v{T * a * c.x, T * a * c.y, T * a * c.z};
        // inclusive suffix sum within the chunk
        f3 s = v;
#pragma unroll
        for (int o = 1; o < kWarp; o <<= 1) {
            const float x = __shfl_down_sync(kFull, s.x, o), y = __shfl_down_sync(kFull, s.y, o),
                        z = __shfl_down_sync(kFull, s.z, o);
            if (lane + o < kWarp) {
                s.x += x;
                s.y += y;
                s.z += z;
            }
        }
        f3 after{__shfl_down_sync(kFull, s.x, 1), __shfl_down_sync(kFull, s.y, 1), __shfl_down_sync(kFull, s.z, 1)};
        if (lane == kWarp - 1) after = f3{0.0f, 0.0f, 0.0f};
        after.x += tac_carry.x;
        after.y += tac_carry.y;
        after.z += tac_carry.z;
        float d_this = 0.0f, d_next = 0.0f, dl = 0.0f;
        if (valid) {
            const float inv = 1.0f / (1.0f + e1);
            if (a != 0.0f) {
                d_next = -k * e1 * (1.0f + e0) * inv * inv;
                d_this = k * e0 * inv;
            }
            const f3 dc{T * c.x + after.x / (a - 1), T * c.y + after.y / (a - 1), T * c.z + after.z / (a - 1)};
            dl = g.x * dc.x + g.y * dc.y + g.z * dc.z;
            store3(QSDVR_AT(rgb_grad, 3 * ((uint64_t)info.render_offset + i), 3, 3 * render_cap),
                   f3{g.x * T * a, g.y * T * a, g.z * T * a});
        }
        const float mine_this = dl * d_this;
        float from_next = __shfl_down_sync(kFull, mine_this, 1);
        if (lane == kWarp - 1) from_next = next_this;
        if (valid) {
            // SDF sample i+1 gets this sample's d_next term and the next sample's d_this term.
            *QSDVR_AT(sdf_grad, (uint64_t)info.sdf_offset + i + 1, 1, sdf_cap) =
                dl * d_next + (i + 1 < nr ? from_next : 0.0f);
            if (i == 0) *QSDVR_AT(sdf_grad, info.sdf_offset, 1, sdf_cap) = mine_this;
        }
        next_this = __shfl_sync(kFull, mine_this, 0);
        tac_carry.x += __shfl_sync(kFull, s.x, 0);
        tac_carry.y += __shfl_sync(kFull, s.y, 0);
        tac_carry.z += __shfl_sync(kFull, s.z, 0);
    }
}

}  // namespace
}  // namespace qsdvr

using namespace qsdvr;

extern "C" int qsdvr_grid_interpolation_forward(const float *data, const float *points, const int32_t *index,
                                                float *out, uint64_t count, uint32_t reso, uint64_t vertex_count,
                                                cudaStream_t stream) {
    if (count == 0) return QSDVR_OK;
    if (!data || !points || !index || !out)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_grid_interpolation_forward: null pointer");
    if (!aligned(data, 16) || !aligned(out, 16))
        return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_grid_interpolation_forward: data/out need 16-byte alignment");
    interp_forward_kernel<<<grid_for(count * 8, 256), 256, 0, stream>>>(data, points, index, out, count, reso,
                                                                        vertex_count);
    return check_launch("qsdvr_grid_interpolation_forward");
}

extern "C" int qsdvr_grid_interpolation_backward(float *data_grad, const float *points, const int32_t *index,
                                                 const float *grad_out, uint64_t count, uint32_t reso,
                                                 uint64_t vertex_count, cudaStream_t stream) {
    if (count == 0) return QSDVR_OK;
    if (!data_grad || !points || !index || !grad_out)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_grid_interpolation_backward: null pointer");
    if (!aligned(data_grad, 16) || !aligned(grad_out, 16))
        return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_grid_interpolation_backward: buffers need 16-byte alignment");
    interp_backward_kernel<<<grid_for(count * 8, 256), 256, 0, stream>>>(data_grad, points, index, grad_out, count,
                                                                         reso, vertex_count);
    return check_launch("qsdvr_grid_interpolation_backward");
}

extern "C" int qsdvr_shader_forward(float *out, const float *normal, const float *view, const float *data,
                                    float *specular, uint64_t count, int mode, cudaStream_t stream) {
    if (count == 0) return QSDVR_OK;
    if (!out || !normal || !view || !data || !specular)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_shader_forward: null pointer");
    if (mode != QSDVR_MODE_COMPAT && mode != QSDVR_MODE_FIXED)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_shader_forward: bad mode %d", mode);
    if (!aligned(data, 16)) return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_shader_forward: data needs 16-byte alignment");
    if (mode == QSDVR_MODE_COMPAT)
        shader_forward_kernel<true><<<grid_for(count, 128), 128, 0, stream>>>(out, normal, view, data, specular, count);
    else
        shader_forward_kernel<false><<<grid_for(count, 128), 128, 0, stream>>>(out, normal, view, data, specular, count);
    return check_launch("qsdvr_shader_forward");
}

extern "C" int qsdvr_shader_backward(const float *grad_out, const float *normal, const float *view, const float *data,
                                     const float *specular, float *normal_grad, float *data_grad, uint64_t count,
                                     int mode, cudaStream_t stream) {
    if (count == 0) return QSDVR_OK;
    if (!grad_out || !normal || !view || !data || !specular || !normal_grad || !data_grad)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_shader_backward: null pointer");
    if (mode != QSDVR_MODE_COMPAT && mode != QSDVR_MODE_FIXED)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_shader_backward: bad mode %d", mode);
    if (!aligned(data, 16) || !aligned(data_grad, 16))
        return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_shader_backward: data buffers need 16-byte alignment");
    if (mode == QSDVR_MODE_COMPAT)
        shader_backward_kernel<true><<<grid_for(count, 128), 128, 0, stream>>>(grad_out, normal, view, data, specular,
                                                                              normal_grad, data_grad, count);
    else
        shader_backward_kernel<false><<<grid_for(count, 128), 128, 0, stream>>>(grad_out, normal, view, data, specular,
                                                                               normal_grad, data_grad, count);
    return check_launch("qsdvr_shader_backward");
}

extern "C" int qsdvr_ray_aggregate_forward(float *out, const float *rgb, const float *sdf, const qsdvr_ray_info *rays,
                                           float *alpha, float *transmittance, uint32_t ray_count,
                                           float logistic_coef, uint64_t sdf_capacity, uint64_t render_capacity,
                                           cudaStream_t stream) {
    if (ray_count == 0) return QSDVR_OK;
    if (!out || !rays || (render_capacity && (!rgb || !alpha || !transmittance)) || (sdf_capacity && !sdf))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_ray_aggregate_forward: null pointer");
    aggregate_forward_kernel<<<grid_for((uint64_t)ray_count * kWarp, 256), 256, 0, stream>>>(
        out, rgb, sdf, rays, alpha, transmittance, ray_count, logistic_coef, sdf_capacity, render_capacity);
    return check_launch("qsdvr_ray_aggregate_forward");
}

extern "C" int qsdvr_ray_aggregate_backward(const float *grad_out, const float *rgb, const float *sdf,
                                            const qsdvr_ray_info *rays, const float *alpha, const float *transmittance,
                                            float *rgb_grad, float *sdf_grad, uint32_t ray_count, float logistic_coef,
                                            uint64_t sdf_capacity, uint64_t render_capacity, cudaStream_t stream) {
    if (ray_count == 0) return QSDVR_OK;
    if (!grad_out || !rays || (render_capacity && (!rgb || !alpha || !transmittance || !rgb_grad)) ||
        (sdf_capacity && (!sdf || !sdf_grad)))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_ray_aggregate_backward: null pointer");
    aggregate_backward_kernel<<<grid_for((uint64_t)ray_count * kWarp, 256), 256, 0, stream>>>(
        grad_out, rgb, sdf, rays, alpha, transmittance, rgb_grad, sdf_grad, ray_count, logistic_coef, sdf_capacity,
        render_capacity);
    return check_launch("qsdvr_ray_aggregate_backward");
}
