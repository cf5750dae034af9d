// Sample positions along a ray and their quadric cells, bit-exact with the reference's
// GenerateRayPoints (kernel/camera.cu:60-96).  Shared by the per-op sample generator and
// the fused render kernels, so both produce identical samples.
#pragma once

#include "common.cuh"

namespace qsdvr {

// SDF sample j: ori + (dir * j) * interval (kernel/camera.cu:45, :73), with the product
// that feeds the addition fused as the reference's build evaluates it.
__device__ __forceinline__ f3 march(f3 o, f3 d, float jf, float interval) {
    return f3{__fmaf_rn(__fmul_rn(d.x, jf), interval, o.x), __fmaf_rn(__fmul_rn(d.y, jf), interval, o.y),
              __fmaf_rn(__fmul_rn(d.z, jf), interval, o.z)};
}

// Render sample j: ori + dir * ((j + 0.5) * interval) (kernel/camera.cu:86).
__device__ __forceinline__ f3 midpoint(f3 o, f3 d, uint32_t j, float interval) {
    const float t = __fmul_rn(__fadd_rn((float)j, 0.5f), interval);
    return f3{__fmaf_rn(d.x, t, o.x), __fmaf_rn(d.y, t, o.y), __fmaf_rn(d.z, t, o.z)};
}

struct CellPoint {
    f3 u;           // local coordinates in [-1,1)^3
    int cx, cy, cz; // cell coordinates
    int32_t index;  // cx + cy R + cz R^2 (unsigned arithmetic, as the reference)
};

// World point -> cell and local coordinates (kernel/camera.cu:73-78, :86-91).
__device__ __forceinline__ CellPoint to_cell(f3 p, float volume_offset, uint32_t reso) {
    const float qx = __fmul_rn(__fadd_rn(p.x, 1.0f), volume_offset);
    const float qy = __fmul_rn(__fadd_rn(p.y, 1.0f), volume_offset);
    const float qz = __fmul_rn(__fadd_rn(p.z, 1.0f), volume_offset);
    CellPoint c;
    c.cx = (int)floorf(qx);
    c.cy = (int)floorf(qy);
    c.cz = (int)floorf(qz);
    c.u.x = __fsub_rn(__fmul_rn(qx, 2.0f), __fadd_rn((float)(2 * c.cx), 1.0f));
    c.u.y = __fsub_rn(__fmul_rn(qy, 2.0f), __fadd_rn((float)(2 * c.cy), 1.0f));
    c.u.z = __fsub_rn(__fmul_rn(qz, 2.0f), __fadd_rn((float)(2 * c.cz), 1.0f));
    c.index = (int32_t)((uint32_t)c.cx + (uint32_t)c.cy * reso + (uint32_t)c.cz * (reso * reso));
    return c;
}

}  // namespace qsdvr
