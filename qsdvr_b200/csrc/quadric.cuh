// Quadric cell evaluation (kernel/surface.cu:54-146) as device functions shared by the
// per-op kernels and the fused render kernels.  a[0..6] are the cell's coefficients of
// f(u) = a0 ux^2 + a1 uy^2 + a2 uz^2 + a3 ux + a4 uy + a5 uz + a6.
#pragma once

#include "common.cuh"

namespace qsdvr {

// kernel/surface.cu:61-71: first-order distance f / |grad_u f| / R.
__device__ __forceinline__ float quad_sdf(const float *a, f3 u, float reso) {
    const float a0 = a[0] * u.x, a1 = a[1] * u.y, a2 = a[2] * u.z;
    const float nx = 2 * a0 + a[3], ny = 2 * a1 + a[4], nz = 2 * a2 + a[5];
    return ((a0 + a[3]) * u.x + (a1 + a[4]) * u.y + (a2 + a[5]) * u.z + a[6]) / sqrtf(nx * nx + ny * ny + nz * nz) /
           reso;
}

// kernel/surface.cu:81-101: d sdf / d a (times gout), written to g[0..6].
__device__ __forceinline__ void quad_sdf_grad(const float *a, f3 u, float reso, float gout, float *g) {
    const float a0 = a[0] * u.x, a1 = a[1] * u.y, a2 = a[2] * u.z;
    const float value = (a0 + a[3]) * u.x + (a1 + a[4]) * u.y + (a2 + a[5]) * u.z + a[6];
    const float nx = 2 * a0 + a[3], ny = 2 * a1 + a[4], nz = 2 * a2 + a[5];
    const float norm = 1.0f / sqrtf(nx * nx + ny * ny + nz * nz);
    const float norm3 = value * norm * norm * norm;
    const float go = gout / reso;
    g[0] = go * u.x * (u.x * norm - 2 * nx * norm3);
    g[1] = go * u.y * (u.y * norm - 2 * ny * norm3);
    g[2] = go * u.z * (u.z * norm - 2 * nz * norm3);
    g[3] = go * (u.x * norm - nx * norm3);
    g[4] = go * (u.y * norm - ny * norm3);
    g[5] = go * (u.z * norm - nz * norm3);
    g[6] = go * norm;
}

// kernel/surface.cu:111-114: normalize(2 a_k u_k + a_{k+3}).
__device__ __forceinline__ f3 quad_normal(const float *a, f3 u) {
    const float vx = 2 * a[0] * u.x + a[3], vy = 2 * a[1] * u.y + a[4], vz = 2 * a[2] * u.z + a[5];
    const float nrm = sqrtf(vx * vx + vy * vy + vz * vz);
    return f3{vx / nrm, vy / nrm, vz / nrm};
}

// kernel/surface.cu:124-145: d normal / d a (contracted with gout), written to g[0..5].
__device__ __forceinline__ void quad_normal_grad(const float *a, f3 u, f3 o, float *g) {
    const float a0 = 2 * a[0] * u.x, a1 = 2 * a[1] * u.y, a2 = 2 * a[2] * u.z;
    const float vx = a0 + a[3], vy = a1 + a[4], vz = a2 + a[5];
    const float norm = 1.0f / sqrtf(vx * vx + vy * vy + vz * vz);
    const float norm3 = norm * norm * norm;
    const float gx = o.x * (norm - norm3 * vx * vx) - o.y * vy * norm3 * vx - o.z * vz * norm3 * vx;
    const float gy = o.y * (norm - norm3 * vy * vy) - o.x * vx * norm3 * vy - o.z * vz * norm3 * vy;
    const float gz = o.z * (norm - norm3 * vz * vz) - o.y * vy * norm3 * vz - o.x * vx * norm3 * vz;
    g[0] = 2.0f * u.x * gx;
    g[1] = 2.0f * u.y * gy;
    g[2] = 2.0f * u.z * gz;
    g[3] = gx;
    g[4] = gy;
    g[5] = gz;
}

}  // namespace qsdvr
