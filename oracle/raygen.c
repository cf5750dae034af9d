/*
 * ORACLE (test infrastructure only, never the product path).
 *
 * Plain-C float32 restatement of the reference's ray generation:
 *   kernel/camera.cu:3-10    TransCameraToWorld
 *   kernel/camera.cu:12-58   RayCutKernel (per-pixel march and in-box count)
 *   kernel/camera.cu:98-130  RayCut host part (mask, <2 zeroing, exclusive scan)
 *   kernel/camera.cu:60-96   GenerateRayPointsKernel (sample points, cell index)
 *
 * Sample counts and cell indices must be bit-exact, so every float operation is
 * written out with the rounding the reference's nvcc build (default --fmad=true)
 * performs: products that feed an addition are fused (fmaf), divisions and square
 * roots are IEEE round-to-nearest.  Build with -ffp-contract=off so that gcc adds
 * no contraction of its own.  The fused forms are pinned against sample lists the
 * reference itself produced on a B200 (tests/golden).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef struct {
    uint32_t width, height;
    float rotation[9];   /* row-major camera-to-world rotation */
    float translation[3];
    float fx, fy, cx, cy, near_, far_;
} oracle_camera;

/* camera.cu:3-10 — pixel (px,py) at camera depth pz to world space. */
static void trans_camera_to_world(const oracle_camera *c, float p[3])
{
    const float x = ((p[0] + c->cx) / c->fx) * p[2];
    const float y = ((p[1] + c->cy) / c->fy) * p[2];
    const float z = p[2];
    const float *r = c->rotation;
    p[0] = fmaf(r[2], z, fmaf(r[0], x, r[1] * y)) + c->translation[0];
    p[1] = fmaf(r[5], z, fmaf(r[3], x, r[4] * y)) + c->translation[1];
    p[2] = fmaf(r[8], z, fmaf(r[6], x, r[7] * y)) + c->translation[2];
}

static int in_box(const float p[3])
{
    return p[0] < 0.9999f && p[0] > -0.9999f && p[1] < 0.9999f && p[1] > -0.9999f &&
           p[2] < 0.9999f && p[2] > -0.9999f;
}

/* camera.cu:12-58 for one pixel: world direction, first in-box sample, count. */
static uint32_t ray_cut_pixel(const oracle_camera *c, uint32_t id, float interval, float dir[3],
                              float origin[3])
{
    const float px = (float)(id % c->width) + 0.5f;
    const float py = (float)(id / c->width) + 0.5f;
    float n[3] = {px, py, c->near_};
    float f[3] = {px, py, c->far_};
    trans_camera_to_world(c, n);
    trans_camera_to_world(c, f);
    float d[3] = {f[0] - n[0], f[1] - n[1], f[2] - n[2]};
    const float norm = sqrtf(fmaf(d[2], d[2], fmaf(d[0], d[0], d[1] * d[1])));
    d[0] = d[0] / norm;
    d[1] = d[1] / norm;
    d[2] = d[2] / norm;
    float end;
    if (d[0] != 0.0f)
        end = (f[0] - n[0]) / d[0];
    else if (d[1] != 0.0f)
        end = (f[1] - n[1]) / d[1];
    else
        end = (f[2] - n[2]) / d[2];
    const float steps = end / interval;
    /* float -> unsigned conversion truncates; negative and NaN map to 0 as on the GPU. */
    const uint32_t count = (steps > 0.0f) ? (steps >= 4294967040.0f ? 0xffffffffu : (uint32_t)steps) : 0u;
    uint32_t hits = 0;
    origin[0] = origin[1] = origin[2] = 0.0f;
    for (uint32_t j = 0; j < count; ++j) {
        const float jf = (float)j;
        float p[3];
        for (int k = 0; k < 3; ++k) p[k] = fmaf(d[k] * jf, interval, n[k]);
        if (in_box(p)) {
            if (hits == 0) memcpy(origin, p, sizeof(p));
            ++hits;
        }
    }
    memcpy(dir, d, sizeof(d));
    return hits;
}

/*
 * camera.cu:98-130.  rays is [pixel_count][4] = {sdfCount, sdfOffset, renderCount,
 * renderOffset}; fields 1..3 of unmasked pixels keep their previous contents, as in the
 * reference (only sdfCount is written for them).  totals[0..1] = sdfCount, renderCount.
 */
void oracle_ray_cut(const oracle_camera *cam, const uint8_t *mask, uint32_t pixel_count, float interval,
                    uint32_t *rays, float *origin, float *dir, uint32_t *totals)
{
    uint32_t sdf_total = 0, render_total = 0;
    for (uint32_t i = 0; i < pixel_count; ++i) {
        uint32_t cnt = ray_cut_pixel(cam, i, interval, dir + 3 * i, origin + 3 * i);
        uint32_t *r = rays + 4 * i;
        r[0] = cnt;
        if (mask[i]) {
            if (cnt < 2) cnt = 0;
            r[0] = cnt;
            r[1] = sdf_total;
            sdf_total += cnt;
            r[3] = render_total;
            r[2] = cnt > 1 ? cnt - 1 : 0;
            render_total += r[2];
        }
    }
    totals[0] = sdf_total;
    totals[1] = render_total;
}

/* The records of a list of pixels (each marched as camera.cu:12-58 does), with packed
 * exclusive-scan offsets in list order: the host-side ray batch of the benchmark's CPU arm
 * (a random sample of pixels over many views) without marching every pixel of a view. */
void oracle_ray_cut_pixels(const oracle_camera *cam, const uint32_t *pixels, uint32_t count, float interval,
                           uint32_t *rays, float *origin, float *dir)
{
    uint32_t sdf_total = 0, render_total = 0;
    for (uint32_t i = 0; i < count; ++i) {
        uint32_t cnt = ray_cut_pixel(cam, pixels[i], interval, dir + 3 * i, origin + 3 * i);
        if (cnt < 2) cnt = 0;
        uint32_t *r = rays + 4 * i;
        r[0] = cnt;
        r[1] = sdf_total;
        sdf_total += cnt;
        r[2] = cnt > 1 ? cnt - 1 : 0;
        r[3] = render_total;
        render_total += r[2];
    }
}

/* camera.cu:73-80 / 86-93: world point to (local coords in [-1,1), cell index). */
static void to_cell(const float p_in[3], float volume_offset, uint32_t reso, float local[3], int32_t *index)
{
    int32_t c[3];
    for (int k = 0; k < 3; ++k) {
        const float p = (p_in[k] + 1.0f) * volume_offset;
        c[k] = (int32_t)floorf(p);
        local[k] = p * 2.0f - ((float)(2 * c[k]) + 1.0f);
    }
    *index = (int32_t)((uint32_t)c[0] + (uint32_t)c[1] * reso + (uint32_t)c[2] * (reso * reso));
}

/* camera.cu:60-96 and host wrapper :132-147. */
void oracle_generate_ray_points(const uint32_t *rays, const float *origin, const float *dir, uint32_t nrays,
                                float interval, uint32_t reso, float *sdf_pts, int32_t *sdf_idx,
                                float *render_pts, int32_t *render_idx, float *view_dir)
{
    const float volume_offset = (float)reso / 2.0f;
    for (uint32_t r = 0; r < nrays; ++r) {
        const float *o = origin + 3 * r;
        const float *d = dir + 3 * r;
        const uint32_t sc = rays[4 * r + 0], so = rays[4 * r + 1];
        const uint32_t rc = rays[4 * r + 2], ro = rays[4 * r + 3];
        for (uint32_t j = 0; j < sc; ++j) {
            const float jf = (float)j;
            float p[3];
            for (int k = 0; k < 3; ++k) p[k] = fmaf(d[k] * jf, interval, o[k]);
            to_cell(p, volume_offset, reso, sdf_pts + 3 * (size_t)(so + j), sdf_idx + (so + j));
        }
        for (uint32_t j = 0; j < rc; ++j) {
            const float s = ((float)j + 0.5f) * interval;
            float p[3];
            for (int k = 0; k < 3; ++k) p[k] = fmaf(d[k], s, o[k]);
            to_cell(p, volume_offset, reso, render_pts + 3 * (size_t)(ro + j), render_idx + (ro + j));
            memcpy(view_dir + 3 * (size_t)(ro + j), d, 3 * sizeof(float));
        }
    }
}

/*
 * List sampling (the proposal path of the fused renderer; no reference counterpart): ray r
 * with sdf_count >= 2 gets the 33 SDF samples fmaf(d, t_j, o) for t_j = tlist[33 r + j] and
 * the 32 render samples at 0.5 (t_j + t_{j+1}), converted to cells like camera.cu:73-80.
 * Outputs are packed 33 / 32 per such ray in ray order; rays with fewer samples get none.
 */
void oracle_list_points(const uint32_t *rays, const float *origin, const float *dir, uint32_t nrays,
                        const float *tlist, uint32_t reso, float *sdf_pts, int32_t *sdf_idx, float *render_pts,
                        int32_t *render_idx, float *view_dir)
{
    const float volume_offset = (float)reso / 2.0f;
    size_t k = 0;
    for (uint32_t r = 0; r < nrays; ++r) {
        if (rays[4 * r] < 2) continue;
        const float *o = origin + 3 * r;
        const float *d = dir + 3 * r;
        const float *t = tlist + 33 * (size_t)r;
        for (uint32_t j = 0; j < 33; ++j) {
            float p[3];
            for (int c = 0; c < 3; ++c) p[c] = fmaf(d[c], t[j], o[c]);
            to_cell(p, volume_offset, reso, sdf_pts + 3 * (33 * k + j), sdf_idx + 33 * k + j);
        }
        for (uint32_t j = 0; j < 32; ++j) {
            const float s = 0.5f * (t[j] + t[j + 1]);
            float p[3];
            for (int c = 0; c < 3; ++c) p[c] = fmaf(d[c], s, o[c]);
            to_cell(p, volume_offset, reso, render_pts + 3 * (32 * k + j), render_idx + 32 * k + j);
            memcpy(view_dir + 3 * (32 * k + j), d, 3 * sizeof(float));
        }
        ++k;
    }
}
