// Quadric surface grid: separable layers -> 7-coefficient cells (forward/backward) and the
// SDF / normal samples of a cell (kernel/surface.cu).
//
// Cell layout [R^3][7] fp32, index x + yR + zR^2; coefficients a0..a6 of
// f(u) = a0 ux^2 + a1 uy^2 + a2 uz^2 + a3 ux + a4 uy + a5 uz + a6 in local u in [-1,1)^3.
#include "common.cuh"

namespace qsdvr {

QSDVR_ERROR_WORD_ACCESSOR(surface)

namespace {

// ---- LayerToGrid ------------------------------------------------------------------------

// kernel/surface.cu:161-178: the per-axis prefix recurrences (three threads, one axis each),
// evaluated with the same unfused float operations as the reference's host code.
__global__ void layer_tables_kernel(const float *__restrict__ x0, const float *__restrict__ y1,
                                    const float *__restrict__ z2, const float *__restrict__ offset, uint32_t R,
                                    float *__restrict__ tables /* [6][R]: x3 y4 z5 x6 y6 z6 */) {
    const int axis = threadIdx.x;
    if (axis >= 3) return;
    const float *a0 = axis == 0 ? x0 : (axis == 1 ? y1 : z2);
    float *a3 = tables + axis * R;
    float *a6 = tables + (3 + axis) * R;
    float p3 = offset[axis], p6 = 0.0f;
    a3[0] = p3;
    a6[0] = p6;
    for (uint32_t i = 1; i < R; ++i) {
        const float c3 = __fadd_rn(__fadd_rn(__fmul_rn(2.0f, a0[i - 1]), __fmul_rn(2.0f, a0[i])), p3);
        a3[i] = c3;
        const float c6 =
            __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(3.0f, a0[i - 1]), a0[i]), __fmul_rn(2.0f, p3)), p6);
        a6[i] = c6;
        p3 = c3;
        p6 = c6;
    }
}

// kernel/surface.cu:3-24: one thread per output float (coalesced writes).
__global__ void __launch_bounds__(256) layer_expand_kernel(float *__restrict__ grid7, const float *__restrict__ x0,
                                                           const float *__restrict__ y1,
                                                           const float *__restrict__ z2,
                                                           const float *__restrict__ tables,
                                                           const float *__restrict__ offset, uint32_t R) {
    const uint64_t total = (uint64_t)R * R * R * 7;
    const float off3 = offset[3];
    for (uint64_t i = blockIdx.x * 256ull + threadIdx.x; i < total; i += (uint64_t)gridDim.x * 256) {
        const uint64_t cell = i / 7;
        const int comp = (int)(i - cell * 7);
        const uint32_t x = (uint32_t)(cell % R), y = (uint32_t)((cell / R) % R), z = (uint32_t)(cell / ((uint64_t)R * R));
        float v;
        switch (comp) {
            case 0: v = x0[x]; break;
            case 1: v = y1[y]; break;
            case 2: v = z2[z]; break;
            case 3: v = tables[x]; break;
            case 4: v = tables[R + y]; break;
            case 5: v = tables[2 * R + z]; break;
            default:
                v = __fadd_rn(__fadd_rn(__fadd_rn(tables[3 * R + x], tables[4 * R + y]), tables[5 * R + z]), off3);
        }
        grid7[i] = v;
    }
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// kernel/surface.cu:26-52 as a reduction: one block per z slab.  Per-x sums over y stay in
// registers, per-y sums over x are warp-reduced then added in shared memory, and the slab
// sum is a block reduction, so the layer arrays see O(R^2) atomics instead of 10 R^3.
// acc layout: [0..R) x0  [R..2R) y1  [2R..3R) z2  then (workspace) x3 y4 z5 x6 y6 z6, off3.
__global__ void __launch_bounds__(256) layer_grad_reduce_kernel(const float *__restrict__ g7, uint32_t R,
                                                                float *__restrict__ xg, float *__restrict__ yg,
                                                                float *__restrict__ zg, float *__restrict__ acc,
                                                                float *__restrict__ off3) {
    extern __shared__ float ysum[];  // [3][R]: comps 1, 4, 6 summed over x
    const uint32_t z = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t i = threadIdx.x; i < 3 * R; i += 256) ysum[i] = 0.0f;
    __syncthreads();
    float zs2 = 0.0f, zs5 = 0.0f, zs6 = 0.0f;
    for (uint32_t xb = 0; xb < R; xb += 256) {
        const uint32_t x = xb + threadIdx.x;
        const bool on = x < R;
        float s0 = 0.0f, s3 = 0.0f, s6 = 0.0f;
        for (uint32_t y = 0; y < R; ++y) {
            float v[7] = {0, 0, 0, 0, 0, 0, 0};
            if (on) {
                const float *c = g7 + (((uint64_t)z * R + y) * R + x) * 7;
#pragma unroll
                for (int k = 0; k < 7; ++k) v[k] = c[k];
            }
            s0 += v[0];
            s3 += v[3];
            s6 += v[6];
            zs2 += v[2];
            zs5 += v[5];
            zs6 += v[6];
            const float w1 = warp_sum(v[1]), w4 = warp_sum(v[4]), w6 = warp_sum(v[6]);
            if (lane == 0 && (xb + warp * 32) < R) {
                atomicAdd(&ysum[y], w1);
                atomicAdd(&ysum[R + y], w4);
                atomicAdd(&ysum[2 * R + y], w6);
            }
        }
        if (on) {
            atomicAdd(&xg[x], s0);
            atomicAdd(&acc[x], s3);           // x3
            atomicAdd(&acc[3 * R + x], s6);   // x6
        }
    }
    __syncthreads();
    for (uint32_t y = threadIdx.x; y < R; y += 256) {
        atomicAdd(&yg[y], ysum[y]);
        atomicAdd(&acc[R + y], ysum[R + y]);      // y4
        atomicAdd(&acc[4 * R + y], ysum[2 * R + y]);  // y6
    }
    __shared__ float red[3][8];
    zs2 = warp_sum(zs2);
    zs5 = warp_sum(zs5);
    zs6 = warp_sum(zs6);
    if (lane == 0) {
        red[0][warp] = zs2;
        red[1][warp] = zs5;
        red[2][warp] = zs6;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        float s = 0.0f;
        for (int w = 0; w < 8; ++w) s += red[threadIdx.x][w];
        if (threadIdx.x == 0) zg[z] = s;
        if (threadIdx.x == 1) acc[2 * R + z] = s;  // z5
        if (threadIdx.x == 2) {
            acc[5 * R + z] = s;  // z6
            atomicAdd(off3, s);
        }
    }
}

// kernel/surface.cu:301-334: reverse recurrences (one thread per axis), unfused as on the host.
__global__ void layer_grad_reverse_kernel(float *__restrict__ xg, float *__restrict__ yg, float *__restrict__ zg,
                                          float *__restrict__ acc, float *__restrict__ offset_grad, uint32_t R) {
    const int axis = threadIdx.x;
    if (axis >= 3) return;
    float *a0 = axis == 0 ? xg : (axis == 1 ? yg : zg);
    float *a3 = acc + axis * R;
    float *a6 = acc + (3 + axis) * R;
    for (uint32_t i = R - 1; i > 0; --i) {
        a0[i] = __fadd_rn(a0[i], a6[i]);
        a0[i - 1] = __fadd_rn(a0[i - 1], __fmul_rn(3.0f, a6[i]));
        a3[i - 1] = __fadd_rn(a3[i - 1], __fmul_rn(2.0f, a6[i]));
        a6[i - 1] = __fadd_rn(a6[i - 1], a6[i]);
    }
    for (uint32_t i = R - 1; i > 0; --i) {
        a0[i] = __fadd_rn(a0[i], __fmul_rn(2.0f, a3[i]));
        a0[i - 1] = __fadd_rn(a0[i - 1], __fmul_rn(2.0f, a3[i]));
        a3[i - 1] = __fadd_rn(a3[i - 1], a3[i]);
    }
    offset_grad[axis] = a3[0];
}

// ---- separable SDF tables for the fused renderer ---------------------------------------------
// tables [3R+1] float4: axis a, index i -> (a0, a3, a6, 0) of the per-axis recurrences (the
// same arithmetic as layer_tables_kernel), then (off3, 0, 0, 0).
__global__ void separable_tables_kernel(const float *__restrict__ x0, const float *__restrict__ y1,
                                        const float *__restrict__ z2, const float *__restrict__ offset, uint32_t R,
                                        float4 *__restrict__ tables) {
    const int axis = threadIdx.x;
    if (axis == 3) tables[3 * R] = make_float4(offset[3], 0.0f, 0.0f, 0.0f);
    if (axis >= 3) return;
    const float *a0 = axis == 0 ? x0 : (axis == 1 ? y1 : z2);
    float4 *t = tables + axis * R;
    float p3 = offset[axis], p6 = 0.0f;
    t[0] = make_float4(a0[0], p3, p6, 0.0f);
    for (uint32_t i = 1; i < R; ++i) {
        const float c3 = __fadd_rn(__fadd_rn(__fmul_rn(2.0f, a0[i - 1]), __fmul_rn(2.0f, a0[i])), p3);
        const float c6 =
            __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(3.0f, a0[i - 1]), a0[i]), __fmul_rn(2.0f, p3)), p6);
        t[i] = make_float4(a0[i], c3, c6, 0.0f);
        p3 = c3;
        p6 = c6;
    }
}

// Adjoint (kernel/surface.cu:301-334 on the per-axis sums the fused renderer accumulated):
// reverse recurrences in place over the table gradient, then the layer and offset gradients.
// offset[3]'s gradient is the sum of every cell's g6 = the x axis' a6 chain summed to index 0.
__global__ void separable_grad_kernel(float4 *__restrict__ tg, uint32_t R, float *__restrict__ x_grad,
                                      float *__restrict__ y_grad, float *__restrict__ z_grad,
                                      float *__restrict__ offset_grad) {
    const int axis = threadIdx.x;
    if (axis >= 3) return;
    float4 *t = tg + axis * R;  // (.x a0, .y a3, .z a6)
    for (uint32_t i = R - 1; i > 0; --i) {
        const float a6 = t[i].z;
        t[i].x = __fadd_rn(t[i].x, a6);
        t[i - 1].x = __fadd_rn(t[i - 1].x, __fmul_rn(3.0f, a6));
        t[i - 1].y = __fadd_rn(t[i - 1].y, __fmul_rn(2.0f, a6));
        t[i - 1].z = __fadd_rn(t[i - 1].z, a6);
    }
    for (uint32_t i = R - 1; i > 0; --i) {
        const float a3 = t[i].y;
        t[i].x = __fadd_rn(t[i].x, __fmul_rn(2.0f, a3));
        t[i - 1].x = __fadd_rn(t[i - 1].x, __fmul_rn(2.0f, a3));
        t[i - 1].y = __fadd_rn(t[i - 1].y, a3);
    }
    float *out = axis == 0 ? x_grad : (axis == 1 ? y_grad : z_grad);
    for (uint32_t i = 0; i < R; ++i) out[i] = t[i].x;
    offset_grad[axis] = t[0].y;
    if (axis == 0) offset_grad[3] = t[0].z;
}

// ---- SDF / normal samples ------------------------------------------------------------------

__device__ __forceinline__ bool cell_ok(int32_t idx, uint64_t cells) {
    if (idx < 0 || (uint64_t)idx >= cells) {
        flag_error(QSDVR_DEVERR_INDEX);
        return false;
    }
    return true;
}

// Scalar gradient accumulation that sends no atomic for an exact zero (bit-identical: the
// accumulator starts at +0 and never holds -0; NaN and inf are still added).
__device__ __forceinline__ void add_nonzero(float *p, float v) {
    if (v != 0.0f) atomicAdd(p, v);
}

// kernel/surface.cu:54-72.
__global__ void __launch_bounds__(256) sdf_forward_kernel(float *__restrict__ out, const float *__restrict__ g,
                                                          const float *__restrict__ pts,
                                                          const int32_t *__restrict__ index, uint64_t n,
                                                          float reso, uint64_t cells) {
    const uint64_t id = blockIdx.x * 256ull + threadIdx.x;
    if (id >= n) return;
    const int32_t idx = index[id];
    if (!cell_ok(idx, cells)) {
        out[id] = 0.0f;
        return;
    }
    const float *c = g + (uint64_t)idx * 7;
    const float px = pts[3 * id], py = pts[3 * id + 1], pz = pts[3 * id + 2];
    const float a0 = c[0] * px, a1 = c[1] * py, a2 = c[2] * pz;
    const float a3 = c[3], a4 = c[4], a5 = c[5], a6 = c[6];
    const float nx = 2 * a0 + a3, ny = 2 * a1 + a4, nz = 2 * a2 + a5;
    out[id] = ((a0 + a3) * px + (a1 + a4) * py + (a2 + a5) * pz + a6) / sqrtf(nx * nx + ny * ny + nz * nz) / reso;
}

// kernel/surface.cu:74-102.
__global__ void __launch_bounds__(256) sdf_backward_kernel(const float *__restrict__ gout,
                                                           const float *__restrict__ g,
                                                           const float *__restrict__ pts,
                                                           const int32_t *__restrict__ index,
                                                           float *__restrict__ gg, uint64_t n, float reso,
                                                           uint64_t cells) {
    const uint64_t id = blockIdx.x * 256ull + threadIdx.x;
    if (id >= n) return;
    const int32_t idx = index[id];
    if (!cell_ok(idx, cells)) return;
    const float *c = g + (uint64_t)idx * 7;
    float *d = gg + (uint64_t)idx * 7;
    const float px = pts[3 * id], py = pts[3 * id + 1], pz = pts[3 * id + 2];
    const float a0 = c[0] * px, a1 = c[1] * py, a2 = c[2] * pz;
    const float a3 = c[3], a4 = c[4], a5 = c[5], a6 = c[6];
    const float value = (a0 + a3) * px + (a1 + a4) * py + (a2 + a5) * pz + a6;
    const float nx = 2 * a0 + a3, ny = 2 * a1 + a4, nz = 2 * a2 + a5;
    const float norm = 1.0f / sqrtf(nx * nx + ny * ny + nz * nz);
    const float norm3 = value * norm * norm * norm;
    const float go = gout[id] / reso;
    add_nonzero(d + 0, go * px * (px * norm - 2 * nx * norm3));
    add_nonzero(d + 1, go * py * (py * norm - 2 * ny * norm3));
    add_nonzero(d + 2, go * pz * (pz * norm - 2 * nz * norm3));
    add_nonzero(d + 3, go * (px * norm - nx * norm3));
    add_nonzero(d + 4, go * (py * norm - ny * norm3));
    add_nonzero(d + 5, go * (pz * norm - nz * norm3));
    add_nonzero(d + 6, go * norm);
}

// kernel/surface.cu:104-115.
__global__ void __launch_bounds__(256) normal_forward_kernel(float *__restrict__ out, const float *__restrict__ g,
                                                             const float *__restrict__ pts,
                                                             const int32_t *__restrict__ index, uint64_t n,
                                                             uint64_t cells) {
    const uint64_t id = blockIdx.x * 256ull + threadIdx.x;
    if (id >= n) return;
    const int32_t idx = index[id];
    if (!cell_ok(idx, cells)) {
        store3(out + 3 * id, f3{0.0f, 0.0f, 0.0f});
        return;
    }
    const float *c = g + (uint64_t)idx * 7;
    const float px = pts[3 * id], py = pts[3 * id + 1], pz = pts[3 * id + 2];
    const float vx = 2 * c[0] * px + c[3], vy = 2 * c[1] * py + c[4], vz = 2 * c[2] * pz + c[5];
    const float nrm = sqrtf(vx * vx + vy * vy + vz * vz);
    store3(out + 3 * id, f3{vx / nrm, vy / nrm, vz / nrm});
}

// kernel/surface.cu:117-146.
__global__ void __launch_bounds__(256) normal_backward_kernel(const float *__restrict__ gout,
                                                              const float *__restrict__ g,
                                                              const float *__restrict__ pts,
                                                              const int32_t *__restrict__ index,
                                                              float *__restrict__ gg, uint64_t n, uint64_t cells) {
    const uint64_t id = blockIdx.x * 256ull + threadIdx.x;
    if (id >= n) return;
    const int32_t idx = index[id];
    if (!cell_ok(idx, cells)) return;
    const float *c = g + (uint64_t)idx * 7;
    float *d = gg + (uint64_t)idx * 7;
    const float px = pts[3 * id], py = pts[3 * id + 1], pz = pts[3 * id + 2];
    const float a0 = 2 * c[0] * px, a1 = 2 * c[1] * py, a2 = 2 * c[2] * pz;
    const float a3 = c[3], a4 = c[4], a5 = c[5];
    const float vx = a0 + a3, vy = a1 + a4, vz = a2 + a5;
    const float norm = 1.0f / sqrtf(vx * vx + vy * vy + vz * vz);
    const float norm3 = norm * norm * norm;
    const float ox = gout[3 * id], oy = gout[3 * id + 1], oz = gout[3 * id + 2];
    const float gx = ox * (norm - norm3 * vx * vx) - oy * vy * norm3 * vx - oz * vz * norm3 * vx;
    const float gy = oy * (norm - norm3 * vy * vy) - ox * vx * norm3 * vy - oz * vz * norm3 * vy;
    const float gz = oz * (norm - norm3 * vz * vz) - oy * vy * norm3 * vz - ox * vx * norm3 * vz;
    add_nonzero(d + 0, 2.0f * px * gx);
    add_nonzero(d + 1, 2.0f * py * gy);
    add_nonzero(d + 2, 2.0f * pz * gz);
    add_nonzero(d + 3, gx);
    add_nonzero(d + 4, gy);
    add_nonzero(d + 5, gz);
}

}  // namespace
}  // namespace qsdvr

using namespace qsdvr;

static constexpr uint32_t kMaxReso = 1290;  // (R+1)^3 * 32 floats must stay addressable

extern "C" size_t qsdvr_layer_to_grid_workspace_size(uint32_t reso) { return (size_t)6 * reso * sizeof(float); }

extern "C" int qsdvr_layer_to_grid_forward(float *grid7, const float *x_layer, const float *y_layer,
                                           const float *z_layer, const float *offset, uint32_t reso,
                                           void *workspace, size_t workspace_bytes, cudaStream_t stream) {
    if (!grid7 || !x_layer || !y_layer || !z_layer || !offset)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_layer_to_grid_forward: null pointer");
    if (reso == 0 || reso > kMaxReso)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_layer_to_grid_forward: reso %u out of range", reso);
    if (!workspace || workspace_bytes < qsdvr_layer_to_grid_workspace_size(reso) || !aligned(workspace, 4))
        return set_error(QSDVR_ERR_WORKSPACE, "qsdvr_layer_to_grid_forward: workspace too small");
    float *tables = static_cast<float *>(workspace);
    layer_tables_kernel<<<1, 32, 0, stream>>>(x_layer, y_layer, z_layer, offset, reso, tables);
    const uint64_t total = (uint64_t)reso * reso * reso * 7;
    layer_expand_kernel<<<grid_for(total, 256) > 148u * 64 ? 148u * 64 : grid_for(total, 256), 256, 0, stream>>>(
        grid7, x_layer, y_layer, z_layer, tables, offset, reso);
    return check_launch("qsdvr_layer_to_grid_forward");
}

extern "C" int qsdvr_layer_to_grid_backward(const float *grad7, uint32_t reso, float *x_grad, float *y_grad,
                                            float *z_grad, float *offset_grad, void *workspace,
                                            size_t workspace_bytes, cudaStream_t stream) {
    if (!grad7 || !x_grad || !y_grad || !z_grad || !offset_grad)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_layer_to_grid_backward: null pointer");
    if (reso == 0 || reso > kMaxReso)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_layer_to_grid_backward: reso %u out of range", reso);
    if (!workspace || workspace_bytes < qsdvr_layer_to_grid_workspace_size(reso) || !aligned(workspace, 4))
        return set_error(QSDVR_ERR_WORKSPACE, "qsdvr_layer_to_grid_backward: workspace too small");
    float *acc = static_cast<float *>(workspace);
    int st = check_cuda(cudaMemsetAsync(acc, 0, qsdvr_layer_to_grid_workspace_size(reso), stream), "memset");
    if (st == QSDVR_OK) st = check_cuda(cudaMemsetAsync(x_grad, 0, reso * sizeof(float), stream), "memset");
    if (st == QSDVR_OK) st = check_cuda(cudaMemsetAsync(y_grad, 0, reso * sizeof(float), stream), "memset");
    if (st == QSDVR_OK) st = check_cuda(cudaMemsetAsync(z_grad, 0, reso * sizeof(float), stream), "memset");
    if (st == QSDVR_OK) st = check_cuda(cudaMemsetAsync(offset_grad, 0, 4 * sizeof(float), stream), "memset");
    if (st != QSDVR_OK) return st;
    layer_grad_reduce_kernel<<<reso, 256, 3 * reso * sizeof(float), stream>>>(grad7, reso, x_grad, y_grad, z_grad,
                                                                             acc, offset_grad + 3);
    layer_grad_reverse_kernel<<<1, 32, 0, stream>>>(x_grad, y_grad, z_grad, acc, offset_grad, reso);
    return check_launch("qsdvr_layer_to_grid_backward");
}

extern "C" int qsdvr_separable_sdf_tables(const float *x_layer, const float *y_layer, const float *z_layer,
                                          const float *offset, uint32_t reso, float *tables, cudaStream_t stream) {
    if (!x_layer || !y_layer || !z_layer || !offset || !tables)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_separable_sdf_tables: null pointer");
    if (reso == 0 || reso > kMaxReso)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_separable_sdf_tables: reso %u out of range", reso);
    if (!aligned(tables, 16)) return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_separable_sdf_tables: tables alignment");
    separable_tables_kernel<<<1, 32, 0, stream>>>(x_layer, y_layer, z_layer, offset, reso,
                                                  reinterpret_cast<float4 *>(tables));
    return check_launch("qsdvr_separable_sdf_tables");
}

extern "C" int qsdvr_separable_sdf_grad(float *table_grad, uint32_t reso, float *x_grad, float *y_grad,
                                        float *z_grad, float *offset_grad, cudaStream_t stream) {
    if (!table_grad || !x_grad || !y_grad || !z_grad || !offset_grad)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_separable_sdf_grad: null pointer");
    if (reso == 0 || reso > kMaxReso)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_separable_sdf_grad: reso %u out of range", reso);
    if (!aligned(table_grad, 16)) return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_separable_sdf_grad: alignment");
    separable_grad_kernel<<<1, 32, 0, stream>>>(reinterpret_cast<float4 *>(table_grad), reso, x_grad, y_grad, z_grad,
                                                offset_grad);
    return check_launch("qsdvr_separable_sdf_grad");
}

extern "C" int qsdvr_sample_sdf_forward(float *out, const float *grid7, const float *points, const int32_t *index,
                                        uint64_t count, float reso, uint64_t cell_count, cudaStream_t stream) {
    if (count == 0) return QSDVR_OK;
    if (!out || !grid7 || !points || !index)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_sample_sdf_forward: null pointer");
    sdf_forward_kernel<<<grid_for(count, 256), 256, 0, stream>>>(out, grid7, points, index, count, reso, cell_count);
    return check_launch("qsdvr_sample_sdf_forward");
}

extern "C" int qsdvr_sample_sdf_backward(const float *grad_out, const float *grid7, const float *points,
                                         const int32_t *index, float *grid7_grad, uint64_t count, float reso,
                                         uint64_t cell_count, cudaStream_t stream) {
    if (count == 0) return QSDVR_OK;
    if (!grad_out || !grid7 || !points || !index || !grid7_grad)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_sample_sdf_backward: null pointer");
    sdf_backward_kernel<<<grid_for(count, 256), 256, 0, stream>>>(grad_out, grid7, points, index, grid7_grad, count,
                                                                  reso, cell_count);
    return check_launch("qsdvr_sample_sdf_backward");
}

extern "C" int qsdvr_sample_normal_forward(float *out, const float *grid7, const float *points,
                                           const int32_t *index, uint64_t count, uint64_t cell_count,
                                           cudaStream_t stream) {
    if (count == 0) return QSDVR_OK;
    if (!out || !grid7 || !points || !index)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_sample_normal_forward: null pointer");
    normal_forward_kernel<<<grid_for(count, 256), 256, 0, stream>>>(out, grid7, points, index, count, cell_count);
    return check_launch("qsdvr_sample_normal_forward");
}

extern "C" int qsdvr_sample_normal_backward(const float *grad_out, const float *grid7, const float *points,
                                            const int32_t *index, float *grid7_grad, uint64_t count,
                                            uint64_t cell_count, cudaStream_t stream) {
    if (count == 0) return QSDVR_OK;
    if (!grad_out || !grid7 || !points || !index || !grid7_grad)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_sample_normal_backward: null pointer");
    normal_backward_kernel<<<grid_for(count, 256), 256, 0, stream>>>(grad_out, grid7, points, index, grid7_grad,
                                                                     count, cell_count);
    return check_launch("qsdvr_sample_normal_backward");
}
