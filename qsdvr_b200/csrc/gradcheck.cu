// FP64 loss of the render path, for central finite-difference checks of the fused
// backward.  This is the only FP64 arithmetic on the GPU: one thread per ray, every
// quantity in double, sample positions from the same float32 generator as every other
// kernel (bit-exact with GenerateRayPoints), packed-SH (fixed mode) shading.
#include "common.cuh"
#include "raygen.cuh"

namespace qsdvr {

QSDVR_ERROR_WORD_ACCESSOR(gradcheck)

namespace {

struct d3 {
    double x, y, z;
};

__device__ __forceinline__ bool in_grid(const CellPoint &c, uint32_t R) {
    return (unsigned)c.cx < R && (unsigned)c.cy < R && (unsigned)c.cz < R;
}

// kernel/surface.cu:61-71 in double
__device__ double sdf64(const double *a, d3 u, double reso) {
    const double a0 = a[0] * u.x, a1 = a[1] * u.y, a2 = a[2] * u.z;
    const double nx = 2 * a0 + a[3], ny = 2 * a1 + a[4], nz = 2 * a2 + a[5];
    return ((a0 + a[3]) * u.x + (a1 + a[4]) * u.y + (a2 + a[5]) * u.z + a[6]) / sqrt(nx * nx + ny * ny + nz * nz) / reso;
}

// kernel/surface.cu:111-114 in double
__device__ d3 normal64(const double *a, d3 u) {
    const double vx = 2 * a[0] * u.x + a[3], vy = 2 * a[1] * u.y + a[4], vz = 2 * a[2] * u.z + a[5];
    const double n = sqrt(vx * vx + vy * vy + vz * vz);
    return d3{vx / n, vy / n, vz / n};
}

// kernel/render.cu:154-179 with the packed SH layout, in double
__device__ d3 shade64(d3 n, d3 v, const double *d) {
    const double vdotn = v.x * n.x + v.y * n.y + v.z * n.z;
    const d3 r{v.x - n.x * (2.0 * vdotn), v.y - n.y * (2.0 * vdotn), v.z - n.z * (2.0 * vdotn)};
    const double f[9] = {0.28209479177387814347403972578039, 0.48860251190291992158638462283835,
                         0.48860251190291992158638462283835, 0.48860251190291992158638462283835,
                         1.0925484305920790705433857058027,  1.0925484305920790705433857058027,
                         0.31539156525252000603089369029571, 1.0925484305920790705433857058027,
                         0.54627421529603953527169285290135};
    const double b[9] = {f[0],
                         f[1] * r.x,
                         f[2] * r.y,
                         f[3] * r.z,
                         f[4] * r.x * r.z,
                         f[5] * r.x * r.y,
                         f[6] * (2.0 * r.y * r.y - r.z * r.z - r.x * r.x),
                         f[7] * r.y * r.z,
                         f[8] * (r.z * r.z - r.x * r.x)};
    d3 s{0.0, 0.0, 0.0};
    for (int i = 0; i < 9; ++i) {
        s.x += b[i] * d[3 * i];
        s.y += b[i] * d[3 * i + 1];
        s.z += b[i] * d[3 * i + 2];
    }
    const double m = d[30], ao = d[31];
    return d3{(d[27] * (1.0 - m) + s.x * m) * ao, (d[28] * (1.0 - m) + s.y * m) * ao, (d[29] * (1.0 - m) + s.z * m) * ao};
}

// SDF sample j and whether fixed mode trusts it (|grad f|^2 >= 1e-30 and |sdf| <= 4, the
// rule of the fused kernels); an interval with an untrusted end is empty.
__device__ double sample_sdf(const double *g8, f3 o, f3 dir, uint32_t j, float interval, float vo, uint32_t R,
                             bool *ok, bool *trusted) {
    const CellPoint c = to_cell(march(o, dir, (float)j, interval), vo, R);
    if (!in_grid(c, R)) {
        *ok = false;
        *trusted = false;
        return 0.0;
    }
    const double *a = g8 + 8ull * (uint32_t)c.index;
    const d3 u{c.u.x, c.u.y, c.u.z};
    const double nx = 2 * a[0] * u.x + a[3], ny = 2 * a[1] * u.y + a[4], nz = 2 * a[2] * u.z + a[5];
    const double s = sdf64(a, u, (double)R);
    *trusted = nx * nx + ny * ny + nz * nz >= 1e-30 && fabs(s) <= 4.0;
    return *trusted ? s : 0.0;
}

__global__ void __launch_bounds__(128) loss64_kernel(const qsdvr_ray_info *__restrict__ rays,
                                                     const float *__restrict__ origin, const float *__restrict__ dir,
                                                     uint32_t n, uint32_t R, float interval, double k,
                                                     const double *__restrict__ g8, const double *__restrict__ data,
                                                     const double *__restrict__ target, double *__restrict__ out) {
    const uint32_t r = blockIdx.x * 128u + threadIdx.x;
    if (r >= n) return;
    const uint32_t ns = rays[r].sdf_count;
    const uint32_t nr = ns > 1 ? ns - 1 : 0;
    const f3 o = load3(origin + 3ull * r), dv = load3(dir + 3ull * r);
    const float vo = (float)R / 2.0f;
    const uint32_t R1 = R + 1;
    bool ok = true;
    d3 C{0.0, 0.0, 0.0};
    double T = 1.0;
    bool t0 = false, t1 = false;
    double e0 = nr ? exp(-k * sample_sdf(g8, o, dv, 0, interval, vo, R, &ok, &t0)) : 0.0;
    for (uint32_t i = 0; i < nr && ok; ++i) {
        const double e1 = exp(-k * sample_sdf(g8, o, dv, i + 1, interval, vo, R, &ok, &t1));
        const double x = (e1 - e0) / (1.0 + e1);
        const double alpha = (t0 && t1 && x > 0.0) ? x : 0.0;
        const CellPoint c = to_cell(midpoint(o, dv, i, interval), vo, R);
        if (!in_grid(c, R)) {
            ok = false;
            break;
        }
        const d3 u{c.u.x, c.u.y, c.u.z};
        const d3 nrm = normal64(g8 + 8ull * (uint32_t)c.index, u);
        // trilinear fetch at the fixed-mode base vertex (kernel/render.cu:98-119)
        const uint64_t b = (uint64_t)c.cx + (uint64_t)c.cy * R1 + (uint64_t)c.cz * R1 * R1;
        const double px = (u.x + 1.0) / 2.0, py = (u.y + 1.0) / 2.0, pz = (u.z + 1.0) / 2.0;
        double row[32];
        for (int ch = 0; ch < 32; ++ch) {
            auto at = [&](uint64_t dx, uint64_t dy, uint64_t dz) {
                return data[(b + dx + dy * R1 + dz * (uint64_t)R1 * R1) * 32 + ch];
            };
            const double a00 = at(0, 0, 0) * (1 - px) + at(1, 0, 0) * px;
            const double a01 = at(0, 1, 0) * (1 - px) + at(1, 1, 0) * px;
            const double a10 = at(0, 0, 1) * (1 - px) + at(1, 0, 1) * px;
            const double a11 = at(0, 1, 1) * (1 - px) + at(1, 1, 1) * px;
            row[ch] = (a00 * (1 - py) + a01 * py) * (1 - pz) + (a10 * (1 - py) + a11 * py) * pz;
        }
        const d3 rgb = shade64(nrm, d3{dv.x, dv.y, dv.z}, row);
        C.x += rgb.x * alpha * T;
        C.y += rgb.y * alpha * T;
        C.z += rgb.z * alpha * T;
        T *= (1.0 - alpha);
        e0 = e1;
        t0 = t1;
    }
    if (!ok) flag_error(QSDVR_DEVERR_INDEX);
    const double ex = C.x - target[3 * r], ey = C.y - target[3 * r + 1], ez = C.z - target[3 * r + 2];
    out[r] = ex * ex + ey * ey + ez * ez;
}

}  // namespace
}  // namespace qsdvr

using namespace qsdvr;

extern "C" int qsdvr_render_loss_f64(const qsdvr_ray_info *rays, const float *origin, const float *dir,
                                     uint32_t ray_count, uint32_t reso, float interval, double logistic_coef,
                                     const double *sdf_grid, const double *data, const double *target,
                                     double *loss_per_ray, cudaStream_t stream) {
    if (ray_count == 0) return QSDVR_OK;
    if (!rays || !origin || !dir || !sdf_grid || !data || !target || !loss_per_ray)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_render_loss_f64: null pointer");
    if (reso == 0 || reso > 1290 || !(interval > 0.0f))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_render_loss_f64: bad reso or interval");
    loss64_kernel<<<grid_for(ray_count, 128), 128, 0, stream>>>(rays, origin, dir, ray_count, reso, interval,
                                                              logistic_coef, sdf_grid, data, target, loss_per_ray);
    return check_launch("qsdvr_render_loss_f64");
}
