// Reflection SH-2 shader (kernel/render.cu:5-91, :154-221) as register-resident device
// functions shared by the per-op and the fused kernels.
//
// Channel layout of a 32-float appearance row: 0..26 specular SH (9 coefficients x RGB),
// 27..29 diffuse RGB, 30 metallic, 31 ambient occlusion.  kCompat selects the reference's
// read of coefficient i from channels i, i+1, i+2 (overlapping); otherwise 3i..3i+2.  The
// data gradient of the SH block is written packed at 3i..3i+2 in both modes, exactly as
// kernel/render.cu:212 does.
#pragma once

#include "common.cuh"

namespace qsdvr {

// kernel/render.cu:5-15 (real SH normalisation constants, degree 2).
#define QSDVR_SH0 0.28209479177387814347403972578039f
#define QSDVR_SH1 0.48860251190291992158638462283835f
#define QSDVR_SH4 1.0925484305920790705433857058027f
#define QSDVR_SH6 0.31539156525252000603089369029571f
#define QSDVR_SH8 0.54627421529603953527169285290135f

template <bool kCompat>
__device__ __forceinline__ f3 sh_coef(const float *d, int i) {
    const int o = kCompat ? i : 3 * i;
    return f3{d[o], d[o + 1], d[o + 2]};
}

// kernel/render.cu:17-59: specular radiance SH_2(v; coef), one colour channel at a time.
template <bool kCompat>
__device__ __forceinline__ f3 sh_eval(f3 v, const float *d) {
    const float x4 = v.x * v.z, zz = v.z * v.z, xx = v.x * v.x, x5 = v.x * v.y;
    const float x6 = 2.0f * v.y * v.y - zz - xx;
    const float x7 = v.y * v.z, x8 = zz - xx;
    const f3 c0 = sh_coef<kCompat>(d, 0), c1 = sh_coef<kCompat>(d, 1), c2 = sh_coef<kCompat>(d, 2),
             c3 = sh_coef<kCompat>(d, 3), c4 = sh_coef<kCompat>(d, 4), c5 = sh_coef<kCompat>(d, 5),
             c6 = sh_coef<kCompat>(d, 6), c7 = sh_coef<kCompat>(d, 7), c8 = sh_coef<kCompat>(d, 8);
    f3 r;
    r.x = QSDVR_SH0 * c0.x + QSDVR_SH1 * c1.x * v.x + QSDVR_SH1 * c2.x * v.y + QSDVR_SH1 * c3.x * v.z +
          QSDVR_SH4 * c4.x * x4 + QSDVR_SH4 * c5.x * x5 + QSDVR_SH6 * c6.x * x6 + QSDVR_SH4 * c7.x * x7 +
          QSDVR_SH8 * c8.x * x8;
    r.y = QSDVR_SH0 * c0.y + QSDVR_SH1 * c1.y * v.x + QSDVR_SH1 * c2.y * v.y + QSDVR_SH1 * c3.y * v.z +
          QSDVR_SH4 * c4.y * x4 + QSDVR_SH4 * c5.y * x5 + QSDVR_SH6 * c6.y * x6 + QSDVR_SH4 * c7.y * x7 +
          QSDVR_SH8 * c8.y * x8;
    r.z = QSDVR_SH0 * c0.z + QSDVR_SH1 * c1.z * v.x + QSDVR_SH1 * c2.z * v.y + QSDVR_SH1 * c3.z * v.z +
          QSDVR_SH4 * c4.z * x4 + QSDVR_SH4 * c5.z * x5 + QSDVR_SH6 * c6.z * x6 + QSDVR_SH4 * c7.z * x7 +
          QSDVR_SH8 * c8.z * x8;
    return r;
}

__device__ __forceinline__ f3 reflect_dir(f3 view, f3 n) {
    const float vdotn = view.x * n.x + view.y * n.y + view.z * n.z;
    const float s = 2.0f * vdotn;
    return f3{view.x - n.x * s, view.y - n.y * s, view.z - n.z * s};
}

// kernel/render.cu:161-178: returns rgb, writes the specular radiance to *spec.
template <bool kCompat>
__device__ __forceinline__ f3 shade(f3 n, f3 view, const float *d, f3 *spec) {
    const f3 r = reflect_dir(view, n);
    const f3 s = sh_eval<kCompat>(r, d);
    const float m = d[30], ao = d[31];
    const float om = 1.0f - m;
    *spec = s;
    return f3{(d[27] * om + s.x * m) * ao, (d[28] * om + s.y * m) * ao, (d[29] * om + s.z * m) * ao};
}

// kernel/render.cu:188-220 and :61-91.  g receives the 32-channel data gradient; returns the
// normal gradient.  spec is the specular radiance the forward produced.
template <bool kCompat>
__device__ __forceinline__ f3 shade_backward(f3 og, f3 n, f3 view, const float *d, f3 spec, float *g) {
    const f3 r = reflect_dir(view, n);
    const float m = d[30], ao = d[31];
    const f3 color{d[27] * (1.0f - m) + spec.x * m, d[28] * (1.0f - m) + spec.y * m, d[29] * (1.0f - m) + spec.z * m};
    g[31] = og.x * color.x + og.y * color.y + og.z * color.z;
    const f3 o{og.x * ao, og.y * ao, og.z * ao};
    g[30] = o.x * (spec.x - d[27]) + o.y * (spec.y - d[28]) + o.z * (spec.z - d[29]);
    g[27] = o.x * (1.0f - m);
    g[28] = o.y * (1.0f - m);
    g[29] = o.z * (1.0f - m);
    const f3 w{o.x * m, o.y * m, o.z * m};  // gradient of the specular radiance
    // kernel/render.cu:61-91
    const float x4 = r.x * r.z, zz = r.z * r.z, xx = r.x * r.x, x5 = r.x * r.y;
    const float x6 = 2.0f * r.y * r.y - zz - xx;
    const float x7 = r.y * r.z, x8 = zz - xx;
    float gc[8];
    const float fac[8] = {QSDVR_SH1, QSDVR_SH1, QSDVR_SH1, QSDVR_SH4, QSDVR_SH4, QSDVR_SH6, QSDVR_SH4, QSDVR_SH8};
#pragma unroll
    for (int i = 1; i < 9; ++i) {
        const f3 c = sh_coef<kCompat>(d, i);
        gc[i - 1] = fac[i - 1] * (c.x * w.x + c.y * w.y + c.z * w.z);
    }
    const f3 rg{gc[0] + r.z * gc[3] + r.y * gc[4] - 2 * r.x * (gc[5] + gc[7]),
                gc[1] + r.z * gc[6] + r.x * gc[4] + 4 * r.y * gc[5],
                gc[2] + r.x * gc[3] + r.y * gc[6] + 2 * r.z * (gc[7] - gc[5])};
    const float basis[9] = {QSDVR_SH0,      QSDVR_SH1 * r.x, QSDVR_SH1 * r.y, QSDVR_SH1 * r.z, QSDVR_SH4 * x4,
                            QSDVR_SH4 * x5, QSDVR_SH6 * x6,  QSDVR_SH4 * x7,  QSDVR_SH8 * x8};
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        g[3 * i] = w.x * basis[i];
        g[3 * i + 1] = w.y * basis[i];
        g[3 * i + 2] = w.z * basis[i];
    }
    // kernel/render.cu:213-219: gradient through reflect = v - 2 (v.n) n.
    const float ax = n.x * view.x, ay = n.y * view.y, az = n.z * view.z;
    return f3{-2.0f * (rg.x * (2 * ax + ay + az) + view.x * (rg.y * n.y + rg.z * n.z)),
              -2.0f * (rg.y * (ax + 2 * ay + az) + view.y * (rg.x * n.x + rg.z * n.z)),
              -2.0f * (rg.z * (ax + ay + 2 * az) + view.z * (rg.x * n.x + rg.y * n.y))};
}

// shade_backward with the data gradient written over the data row d itself (d may live
// in shared memory): all reads of a channel happen before any write that overlaps it.
template <bool kCompat>
__device__ __forceinline__ f3 shade_backward_inplace(f3 og, f3 n, f3 view, float *d, f3 spec) {
    const f3 r = reflect_dir(view, n);
    const float m = d[30], ao = d[31];
    const float d27 = d[27], d28 = d[28], d29 = d[29];
    const f3 o{og.x * ao, og.y * ao, og.z * ao};
    const f3 w{o.x * m, o.y * m, o.z * m};
    float gc[8];
    const float fac[8] = {QSDVR_SH1, QSDVR_SH1, QSDVR_SH1, QSDVR_SH4, QSDVR_SH4, QSDVR_SH6, QSDVR_SH4, QSDVR_SH8};
#pragma unroll
    for (int i = 1; i < 9; ++i) {
        const f3 c = sh_coef<kCompat>(d, i);
        gc[i - 1] = fac[i - 1] * (c.x * w.x + c.y * w.y + c.z * w.z);
    }
    const f3 rg{gc[0] + r.z * gc[3] + r.y * gc[4] - 2 * r.x * (gc[5] + gc[7]),
                gc[1] + r.z * gc[6] + r.x * gc[4] + 4 * r.y * gc[5],
                gc[2] + r.x * gc[3] + r.y * gc[6] + 2 * r.z * (gc[7] - gc[5])};
    // every channel has been read: write the gradient (kernel/render.cu:207-212)
    const f3 color{d27 * (1.0f - m) + spec.x * m, d28 * (1.0f - m) + spec.y * m, d29 * (1.0f - m) + spec.z * m};
    d[31] = og.x * color.x + og.y * color.y + og.z * color.z;
    d[30] = o.x * (spec.x - d27) + o.y * (spec.y - d28) + o.z * (spec.z - d29);
    d[27] = o.x * (1.0f - m);
    d[28] = o.y * (1.0f - m);
    d[29] = o.z * (1.0f - m);
    const float x4 = r.x * r.z, zz = r.z * r.z, xx = r.x * r.x, x5 = r.x * r.y;
    const float x6 = 2.0f * r.y * r.y - zz - xx;
    const float x7 = r.y * r.z, x8 = zz - xx;
    const float basis[9] = {QSDVR_SH0,      QSDVR_SH1 * r.x, QSDVR_SH1 * r.y, QSDVR_SH1 * r.z, QSDVR_SH4 * x4,
                            QSDVR_SH4 * x5, QSDVR_SH6 * x6,  QSDVR_SH4 * x7,  QSDVR_SH8 * x8};
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        d[3 * i] = w.x * basis[i];
        d[3 * i + 1] = w.y * basis[i];
        d[3 * i + 2] = w.z * basis[i];
    }
    const float ax = n.x * view.x, ay = n.y * view.y, az = n.z * view.z;
    return f3{-2.0f * (rg.x * (2 * ax + ay + az) + view.x * (rg.y * n.y + rg.z * n.z)),
              -2.0f * (rg.y * (ax + 2 * ay + az) + view.y * (rg.x * n.x + rg.z * n.z)),
              -2.0f * (rg.z * (ax + ay + 2 * az) + view.z * (rg.x * n.x + rg.y * n.y))};
}

// ---- SH degree 3 (not in the reference, which hard-codes degree 2) ---------------------
// Row layout: 16 coefficients x RGB packed at 3i..3i+2 (48 channels), diffuse 48..50,
// metallic 51, ao 52, channels 53..63 unused (64-float rows = two 128-byte lines).
// Band 3 extends the reference's degree-2 basis in its own axis convention: y is the polar
// axis and (z, x) span the azimuthal plane (its l=2 terms are xz, xy, 2y^2-z^2-x^2, yz,
// z^2-x^2); constants are the real-SH normalisations sqrt(35/(32 pi)), sqrt(105/(4 pi)),
// sqrt(21/(32 pi)), sqrt(7/(16 pi)), sqrt(105/(16 pi)).
#define QSDVR_SH3_A 0.59004358992664351034f
#define QSDVR_SH3_B 2.89061144264055405538f
#define QSDVR_SH3_C 0.45704579946446573616f
#define QSDVR_SH3_D 0.37317633259011539141f
#define QSDVR_SH3_E 1.44530572132027702769f

template <int kDeg>
struct ShLayout {
    static constexpr int kBasis = (kDeg + 1) * (kDeg + 1);
    static constexpr int kDiffuse = 3 * kBasis;
    static constexpr int kMetal = kDiffuse + 3;
    static constexpr int kAO = kDiffuse + 4;
    static constexpr int kChannels = kDeg == 2 ? 32 : 64;
};

// The 16 basis values (constants included) at direction v, and their gradients.
__device__ __forceinline__ void sh3_basis(f3 v, float *b) {
    const float x = v.x, y = v.y, z = v.z;
    b[0] = QSDVR_SH0;
    b[1] = QSDVR_SH1 * x;
    b[2] = QSDVR_SH1 * y;
    b[3] = QSDVR_SH1 * z;
    b[4] = QSDVR_SH4 * x * z;
    b[5] = QSDVR_SH4 * x * y;
    b[6] = QSDVR_SH6 * (2.0f * y * y - z * z - x * x);
    b[7] = QSDVR_SH4 * y * z;
    b[8] = QSDVR_SH8 * (z * z - x * x);
    b[9] = QSDVR_SH3_A * x * (3.0f * z * z - x * x);
    b[10] = QSDVR_SH3_B * x * y * z;
    b[11] = QSDVR_SH3_C * x * (4.0f * y * y - z * z - x * x);
    b[12] = QSDVR_SH3_D * y * (2.0f * y * y - 3.0f * z * z - 3.0f * x * x);
    b[13] = QSDVR_SH3_C * z * (4.0f * y * y - z * z - x * x);
    b[14] = QSDVR_SH3_E * y * (z * z - x * x);
    b[15] = QSDVR_SH3_A * z * (z * z - 3.0f * x * x);
}

// sum_i w_i grad(b_i)(v) for basis weights w[0..15]
__device__ __forceinline__ f3 sh3_basis_grad_dot(f3 v, const float *w) {
    const float x = v.x, y = v.y, z = v.z;
    f3 g{QSDVR_SH1 * w[1], QSDVR_SH1 * w[2], QSDVR_SH1 * w[3]};
    g.x += QSDVR_SH4 * (z * w[4] + y * w[5]) - 2.0f * QSDVR_SH6 * x * w[6] - 2.0f * QSDVR_SH8 * x * w[8];
    g.y += QSDVR_SH4 * (x * w[5] + z * w[7]) + 4.0f * QSDVR_SH6 * y * w[6];
    g.z += QSDVR_SH4 * (x * w[4] + y * w[7]) - 2.0f * QSDVR_SH6 * z * w[6] + 2.0f * QSDVR_SH8 * z * w[8];
    // band 3
    g.x += QSDVR_SH3_A * (3.0f * z * z - 3.0f * x * x) * w[9] + QSDVR_SH3_B * y * z * w[10] +
           QSDVR_SH3_C * (4.0f * y * y - z * z - 3.0f * x * x) * w[11] - 6.0f * QSDVR_SH3_D * x * y * w[12] -
           2.0f * QSDVR_SH3_C * x * z * w[13] - 2.0f * QSDVR_SH3_E * x * y * w[14] - 6.0f * QSDVR_SH3_A * x * z * w[15];
    g.y += QSDVR_SH3_B * x * z * w[10] + 8.0f * QSDVR_SH3_C * x * y * w[11] +
           QSDVR_SH3_D * (6.0f * y * y - 3.0f * z * z - 3.0f * x * x) * w[12] + 8.0f * QSDVR_SH3_C * y * z * w[13] +
           QSDVR_SH3_E * (z * z - x * x) * w[14];
    g.z += 6.0f * QSDVR_SH3_A * x * z * w[9] + QSDVR_SH3_B * x * y * w[10] - 2.0f * QSDVR_SH3_C * x * z * w[11] -
           6.0f * QSDVR_SH3_D * y * z * w[12] + QSDVR_SH3_C * (4.0f * y * y - 3.0f * z * z - x * x) * w[13] +
           2.0f * QSDVR_SH3_E * y * z * w[14] + QSDVR_SH3_A * (3.0f * z * z - 3.0f * x * x) * w[15];
    return g;
}

// Degree-3 shading (packed layout): returns rgb, writes the specular radiance.
__device__ __forceinline__ f3 shade_sh3(f3 n, f3 view, const float *d, f3 *spec) {
    const f3 r = reflect_dir(view, n);
    float b[16];
    sh3_basis(r, b);
    f3 s{0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        s.x += b[i] * d[3 * i];
        s.y += b[i] * d[3 * i + 1];
        s.z += b[i] * d[3 * i + 2];
    }
    const float m = d[51], ao = d[52];
    const float om = 1.0f - m;
    *spec = s;
    return f3{(d[48] * om + s.x * m) * ao, (d[49] * om + s.y * m) * ao, (d[50] * om + s.z * m) * ao};
}

// Degree-3 backward, data gradient written over the row in place; returns the normal gradient.
__device__ __forceinline__ f3 shade_sh3_backward_inplace(f3 og, f3 n, f3 view, float *d, f3 spec) {
    const f3 r = reflect_dir(view, n);
    const float m = d[51], ao = d[52];
    const float d48 = d[48], d49 = d[49], d50 = d[50];
    const f3 o{og.x * ao, og.y * ao, og.z * ao};
    const f3 w{o.x * m, o.y * m, o.z * m};
    float gc[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) gc[i] = d[3 * i] * w.x + d[3 * i + 1] * w.y + d[3 * i + 2] * w.z;
    const f3 rg = sh3_basis_grad_dot(r, gc);
    const f3 color{d48 * (1.0f - m) + spec.x * m, d49 * (1.0f - m) + spec.y * m, d50 * (1.0f - m) + spec.z * m};
    d[52] = og.x * color.x + og.y * color.y + og.z * color.z;
    d[51] = o.x * (spec.x - d48) + o.y * (spec.y - d49) + o.z * (spec.z - d50);
    d[48] = o.x * (1.0f - m);
    d[49] = o.y * (1.0f - m);
    d[50] = o.z * (1.0f - m);
    float b[16];
    sh3_basis(r, b);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        d[3 * i] = w.x * b[i];
        d[3 * i + 1] = w.y * b[i];
        d[3 * i + 2] = w.z * b[i];
    }
    // gradient through reflect = v - 2 (v.n) n (kernel/render.cu:213-219)
    const float ax = n.x * view.x, ay = n.y * view.y, az = n.z * view.z;
    return f3{-2.0f * (rg.x * (2 * ax + ay + az) + view.x * (rg.y * n.y + rg.z * n.z)),
              -2.0f * (rg.y * (ax + 2 * ay + az) + view.y * (rg.x * n.x + rg.z * n.z)),
              -2.0f * (rg.z * (ax + ay + 2 * az) + view.z * (rg.x * n.x + rg.y * n.y))};
}

// Dispatch on the SH degree (degree 3 exists only in the packed layout).
template <bool kCompat, int kDeg>
__device__ __forceinline__ f3 shade_any(f3 n, f3 view, const float *d, f3 *spec) {
    if constexpr (kDeg == 3) return shade_sh3(n, view, d, spec);
    else return shade<kCompat>(n, view, d, spec);
}
template <bool kCompat, int kDeg>
__device__ __forceinline__ f3 shade_any_backward_inplace(f3 og, f3 n, f3 view, float *d, f3 spec) {
    if constexpr (kDeg == 3) return shade_sh3_backward_inplace(og, n, view, d, spec);
    else return shade_backward_inplace<kCompat>(og, n, view, d, spec);
}

}  // namespace qsdvr
