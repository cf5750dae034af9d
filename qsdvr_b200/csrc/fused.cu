// Fused render path: for every ray, sample generation -> quadric SDF and normal ->
// trilinear 32-channel fetch -> reflection shading -> NeuS alpha -> transmittance ->
// colour, and the whole backward, in one kernel.  Nothing per-sample is stored in global
// memory: the backward recomputes each sample (memory stays O(rays)).
//
// Work mapping (one warp per ray, 32 render samples per "chunk"):
//   * lane i owns render sample i of the chunk: its positions (bit-exact with
//     GenerateRayPoints), quadric cells, SDF values, normal, alpha and shading;
//   * the 32-channel appearance rows are gathered with 16-byte loads by groups of 8 lanes
//     (one float4 each) or 4 lanes (bf16 x 8 each), so every load covers whole 128-byte
//     (64-byte bf16) vertex rows, interpolated and staged in a per-warp shared-memory
//     tile [32][36] floats
//     (row stride 36 keeps both the row-wise and the lane-wise float4 accesses
//     conflict-free);
//   * transmittance is an exclusive prefix product (or a compensated prefix sum of
//     log(1 - alpha)) by warp shuffles, carried across chunks;
//   * the backward walks the chunks in reverse, carrying the suffix state, and
//     scatters the data gradient back through the same tile with 16-byte vector REDs
//     that cover whole vertex rows.
#include <cuda.h>  // CUtensorMap (the driver is reached through cudaGetDriverEntryPoint)
#include <cuda_bf16.h>

#include <mutex>

#include "common.cuh"
#include "quadric.cuh"
#include "raygen.cuh"
#include "shading.cuh"
#include "tcgen05.cuh"

namespace qsdvr {

QSDVR_ERROR_WORD_ACCESSOR(fused)

namespace {

// Tunables (compile-time).  One ray per warp; with one warp per block the block scheduler
// balances ray lengths by itself.
#ifndef QSDVR_FUSED_WARPS
#define QSDVR_FUSED_WARPS 1
#endif
#ifndef QSDVR_FUSED_MIN_BLOCKS
#define QSDVR_FUSED_MIN_BLOCKS 16
#endif
#ifndef QSDVR_GATHER_UNROLL
#define QSDVR_GATHER_UNROLL 2
#endif
constexpr int kWarpsPerBlock = QSDVR_FUSED_WARPS;
constexpr int kGatherUnroll = QSDVR_GATHER_UNROLL;
constexpr int kThreads = kWarpsPerBlock * kWarp;
// Per SH degree: channels per row (32 or 64), staged row stride (+4 floats keeps both the
// row-wise and the lane-wise float4 accesses bank-conflict free), lanes per sample in the
// gather/scatter (one float4 each) and samples per warp instruction.
template <int kDeg>
struct Rows {
    static constexpr int kC = ShLayout<kDeg>::kChannels;
    static constexpr int kStride = kC + 4;
    static constexpr int kLanes = kC / 4;
    static constexpr int kPerStep = kWarp / kLanes;
};
constexpr uint32_t kMaxChunks = 256;  // render samples per ray <= 8192
// Each staged tile row carries 4 floats of padding (the row stride keeps the row-wise and
// lane-wise float4 accesses bank-conflict free); the gather and the scatter keep there the
// sample's (base vertex, wx, wy, wz), the vertex kNoVertex for a sample without a row, so a
// step reads one sample's parameters with one 16-byte shared load instead of 5 shuffles.
constexpr uint32_t kNoVertex = 0xffffffffu;

enum Pass { kForward = 0, kBackward = 1, kTrain = 2 };

// Persistent train mode: each warp stashes the interpolated rows of the kSlotChunks chunks
// before a ray's last one (the last stays in shared memory) so that the backward reloads
// them from L2 instead of re-gathering 8 corner rows per sample from HBM.
#ifndef QSDVR_SLOT_CHUNKS
#define QSDVR_SLOT_CHUNKS 5
#endif
constexpr uint32_t kSlotChunks = QSDVR_SLOT_CHUNKS;
#ifndef QSDVR_STASH_DISCARD
#define QSDVR_STASH_DISCARD 1
#endif
// Latency: the gather walks a chunk's samples a few at a time, and each round of its loads
// waited for DRAM.  With QSDVR_GATHER_PREFETCH every shaded sample beyond the first round
// requests its 8 corner rows into L2 (four bulk prefetches of two adjacent rows) as soon as
// the chunk's alpha is known, so the later rounds find them there: SH degree 2 only (1, the
// default: with 64-channel rows the prefetches measured slower), every degree (2), none (0).
#ifndef QSDVR_GATHER_PREFETCH
#define QSDVR_GATHER_PREFETCH 1
#endif
template <int kDeg>
__host__ __device__ constexpr uint32_t chunk_floats() { return kWarp * Rows<kDeg>::kC; }  // rows of one chunk

// L2 evict_last for the stash: it is re-read shortly and must survive the streaming gathers.
__device__ __forceinline__ uint64_t evict_last_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ void st4_keep(float *p, float4 v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "f"(v.x), "f"(v.y),
                 "f"(v.z), "f"(v.w), "l"(pol)
                 : "memory");
}
// 16 bytes global -> shared without passing through registers (completed by cp_async_wait)
__device__ __forceinline__ void cp_async16_keep(float *dst, const float *src, uint64_t pol) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// A hint to bring [p, p + bytes) into L2 (16-byte aligned, a multiple of 16 bytes); nothing
// waits for it.
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

struct Params {
    const qsdvr_ray_info *rays;
    const float *origin;
    const float *dir;
    uint32_t n;
    uint32_t R;
    float interval, k, volume_offset;
    const void *sdf;   // [R^3][8], or null with sep
    const float4 *sep; // separable SDF: [3][R] (a0, a3, a6, 0) per axis index, then (off3, 0, 0, 0)
    float4 *sep_grad;  // its gradient, same layout (the last entry unused)
    const void *data;  // [(R+1)^3][32]
    float *color;
    const float *target;
    const float *grad_color;
    float *sdf_grad;
    float *data_grad;
    float *loss;
    float grad_scale;
    uint32_t *ray_counter;  // persistent mode: next ray to take (zeroed before the launch)
    float *slots;           // persistent train mode: per-warp row stash, kSlotChunks chunks each
    const float *tlist;     // list sampling: per ray kListT SDF positions (t from origin), or null
    float *sample_alpha;    // optional per-render-sample alpha output (forward, train)
    uint64_t sample_capacity;
    const uint32_t *order;  // optional: the i-th ray taken is order[i]
    bool grad_bf16;         // data_grad holds bf16 values
};

constexpr uint32_t kListT = 33;  // list sampling: 33 SDF positions, 32 render samples per ray

// SDF sample j and render sample j of ray r: the reference's uniform march, or positions
// o + d t from the ray's list (render samples at interval midpoints).
__device__ __forceinline__ f3 at_t(f3 o, f3 d, float t) {
    return f3{fmaf(d.x, t, o.x), fmaf(d.y, t, o.y), fmaf(d.z, t, o.z)};
}

// ---- storage access --------------------------------------------------------------------

__device__ __forceinline__ float bf_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf_hi(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

template <typename S>
struct Store;

template <>
struct Store<float> {
    __device__ static void cell(const void *g, uint32_t c, float *a, uint64_t cells) {
        const float *p = QSDVR_AT(static_cast<const float *>(g), 8ull * c, 8, 8 * cells);
        const float4 lo = ld4(p), hi = ld4(p + 4);
        a[0] = lo.x; a[1] = lo.y; a[2] = lo.z; a[3] = lo.w;
        a[4] = hi.x; a[5] = hi.y; a[6] = hi.z;
    }
    __device__ static float4 quad(const void *d, uint32_t v, int q, int C, uint64_t verts) {
        return ld4(QSDVR_AT(static_cast<const float *>(d), (uint64_t)C * v + 4 * q, 4, (uint64_t)C * verts));
    }
};

template <>
struct Store<__nv_bfloat16> {
    __device__ static void cell(const void *g, uint32_t c, float *a, uint64_t cells) {
        const uint4 r =
            *reinterpret_cast<const uint4 *>(QSDVR_AT(static_cast<const __nv_bfloat16 *>(g), 8ull * c, 8, 8 * cells));
        a[0] = bf_lo(r.x); a[1] = bf_hi(r.x); a[2] = bf_lo(r.y); a[3] = bf_hi(r.y);
        // a6 as the sum of slots 6 and 7 (qsdvr_sdf_cells_bf16: the compensated value split
        // into two bf16; exact in fp32)
        a[4] = bf_lo(r.z); a[5] = bf_hi(r.z); a[6] = bf_lo(r.w) + bf_hi(r.w);
    }
    // channels [8q, 8q + 8) of vertex v: one 16-byte load (bf16 x 8)
    __device__ static uint4 oct(const void *d, uint32_t v, int q, int C, uint64_t verts) {
        return *reinterpret_cast<const uint4 *>(
            QSDVR_AT(static_cast<const __nv_bfloat16 *>(d), (uint64_t)C * v + 8 * q, 8, (uint64_t)C * verts));
    }
};

// Lanes of the appearance gather: each lane loads 16 bytes of a vertex row per corner (a
// float4 of fp32 storage, 8 x bf16 of bf16 storage), so kLanes lanes cover one row and a warp
// instruction fetches kPerStep samples' rows.
template <typename S, int kDeg>
struct GatherLanes {
    static constexpr int kC = ShLayout<kDeg>::kChannels;
    static constexpr int kCh = 16 / (int)sizeof(S);  // channels per lane
    static constexpr int kLanes = kC / kCh;
    static constexpr int kPerStep = kWarp / kLanes;
};


__device__ __forceinline__ void red_cell(float *g8, uint32_t cell, const float *g, uint64_t cells) {
    float *b = QSDVR_AT(g8, 8ull * cell, 8, 8 * cells);
    const float4 lo = make_float4(g[0], g[1], g[2], g[3]), hi = make_float4(g[4], g[5], g[6], 0.0f);
    // a zero half (e.g. a sample whose SDF gradient vanishes with its alpha) is not sent
    if (!is_zero4(lo)) red4(b, lo);
    if (!is_zero4(hi)) red4(b + 4, hi);
}

// Separable SDF (models/render.py:172-207): cell (x, y, z) has coefficients
// (x0[x], y1[y], z2[z], x3[x], y4[y], z5[z], ((x6[x] + y6[y]) + z6[z]) + off3), the sum in the
// order kernel/surface.cu:3-24 materialises it, so a cell is bit-identical to the dense grid
// LayerToGrid would write.  The per-axis rows are O(R) and stay in L1/L2.
__device__ __forceinline__ void sep_cell(const float4 *sep, uint32_t R, const CellPoint &c, float *a) {
    [[maybe_unused]] const uint64_t n = 3ull * R + 1;
    const float4 x = *QSDVR_AT(sep, c.cx, 1, n), y = *QSDVR_AT(sep, R + c.cy, 1, n),
                 z = *QSDVR_AT(sep, 2 * R + c.cz, 1, n);
    const float off3 = sep[3 * R].x;
    a[0] = x.x; a[1] = y.x; a[2] = z.x;
    a[3] = x.y; a[4] = y.y; a[5] = z.y;
    a[6] = __fadd_rn(__fadd_rn(__fadd_rn(x.z, y.z), z.z), off3);
}

// Its adjoint: one 16-byte RED per axis row.  The off3 gradient (the sum of every cell's g6)
// is recovered from the x rows' g6 sums by the reverse recurrence, so it needs no atomics.
__device__ __forceinline__ void sep_red(float4 *sg, uint32_t R, const CellPoint &c, const float *g) {
    [[maybe_unused]] const uint64_t n = 3ull * R + 1;
    const float4 x = make_float4(g[0], g[3], g[6], 0.0f), y = make_float4(g[1], g[4], g[6], 0.0f),
                 z = make_float4(g[2], g[5], g[6], 0.0f);
    if (!is_zero4(x)) red4(reinterpret_cast<float *>(QSDVR_AT(sg, c.cx, 1, n)), x);
    if (!is_zero4(y)) red4(reinterpret_cast<float *>(QSDVR_AT(sg, R + c.cy, 1, n)), y);
    if (!is_zero4(z)) red4(reinterpret_cast<float *>(QSDVR_AT(sg, 2 * R + c.cz, 1, n)), z);
}

// Kernel variants (a template parameter, so each instance holds only the code it runs: the
// kernel's code size sets how often its warps wait for instruction fetch).
constexpr int kVarSep = 1;    // separable SDF tables instead of the dense cell grid
constexpr int kVarMerge = 2;  // same-cell merged appearance scatter

template <typename S, int kVar>
__device__ __forceinline__ void load_cell(const Params &p, const CellPoint &c, float *a) {
    if constexpr ((kVar & kVarSep) != 0) sep_cell(p.sep, p.R, c, a);
    else Store<S>::cell(p.sdf, (uint32_t)c.index, a, (uint64_t)p.R * p.R * p.R);
}

template <int kVar>
__device__ __forceinline__ void scatter_cell(const Params &p, const CellPoint &c, const float *g) {
    if constexpr ((kVar & kVarSep) != 0) sep_red(p.sep_grad, p.R, c, g);
    else red_cell(p.sdf_grad, (uint32_t)c.index, g, (uint64_t)p.R * p.R * p.R);
}

__device__ __forceinline__ float4 scale4(float4 v, float w) { return make_float4(v.x * w, v.y * w, v.z * w, v.w * w); }
// Trilinear interpolation as a weighted sum of the 8 corner rows (kernel/render.cu:98-119
// interpolates the same weights as nested lerps in x, y, z; the sum differs from the nested
// form only by float rounding).  Corner c = 4z + 2y + x has weight
// (z ? gz : 1 - gz)(y ? gy : 1 - gy)(x ? gx : 1 - gx): 8 FMAs per channel instead of 7 lerps,
// issued two channels at a time as packed fma.rn.f32x2.
__device__ __forceinline__ void corner_weights(float gx, float gy, float gz, float *w) {
    const float ox = 1.0f - gx, oy = 1.0f - gy, oz = 1.0f - gz;
    const float a = oy * oz, b = gy * oz, c = oy * gz, d = gy * gz;
    w[0] = ox * a;
    w[1] = gx * a;
    w[2] = ox * b;
    w[3] = gx * b;
    w[4] = ox * c;
    w[5] = gx * c;
    w[6] = ox * d;
    w[7] = gx * d;
}
// (a0, a1) += w * (x0, x1) as one packed fma.rn.f32x2 (sm_100)
__device__ __forceinline__ void ffma2(float &a0, float &a1, float w, float x0, float x1) {
    asm("{\n\t.reg .b64 acc, ww, xx;\n\t"
        "mov.b64 acc, {%0, %1};\n\t"
        "mov.b64 ww, {%2, %2};\n\t"
        "mov.b64 xx, {%3, %4};\n\t"
        "fma.rn.f32x2 acc, ww, xx, acc;\n\t"
        "mov.b64 {%0, %1}, acc;\n\t}"
        : "+f"(a0), "+f"(a1)
        : "f"(w), "f"(x0), "f"(x1));
}
__device__ __forceinline__ void fma4(float4 &v, float4 a, float w) {
    ffma2(v.x, v.y, w, a.x, a.y);
    ffma2(v.z, v.w, w, a.z, a.w);
}
// v = w * (8 bf16 channels of r), and v += w * (...)
__device__ __forceinline__ void first_bf8(uint4 r, float w, float *v) {
    const uint32_t rv[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        v[2 * t] = w * bf_lo(rv[t]);
        v[2 * t + 1] = w * bf_hi(rv[t]);
    }
}
__device__ __forceinline__ void fma_bf8(uint4 r, float w, float *v) {
    const uint32_t rv[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
    for (int t = 0; t < 4; ++t) ffma2(v[2 * t], v[2 * t + 1], w, bf_lo(rv[t]), bf_hi(rv[t]));
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ bool cell_in_grid(const CellPoint &c, uint32_t R) {
    return (unsigned)c.cx < R && (unsigned)c.cy < R && (unsigned)c.cz < R;
}

// The two per-sample terms of an interval's alpha.  compat: E = exp(-k sdf), the
// reference's (kernel/render.cu:239-244).  fixed: L = softplus(-k sdf) = -log sigmoid(k sdf),
// finite for every finite sdf, so no intermediate overflows however deep a sample lies.
template <bool kCompat>
__device__ __forceinline__ float alpha_term(float k, float sdf) {
    const float x = -k * sdf;
    if (kCompat) return expf(x);
    return fmaxf(x, 0.0f) + log1pf(expf(-fabsf(x)));
}

// alpha of one interval (kernel/render.cu:244).  compat: the reference's expression
// max((E1 - E0) / (1 + E1), 0).  fixed: the same quantity 1 - sigmoid(k s1) / sigmoid(k s0)
// = -expm1(L0 - L1), clamped at 0.
template <bool kCompat>
__device__ __forceinline__ float interval_alpha(float t0, float t1) {
    if (kCompat) return fmaxf((t1 - t0) / (1.0f + t1), 0.0f);
    return t0 < t1 ? -expm1f(t0 - t1) : 0.0f;
}

// d alpha / d sdf_{i+1} and d alpha / d sdf_i where alpha > 0 (kernel/render.cu:271-273).
// fixed: with 1 - alpha = exp(L0 - L1) and sigmoid(-k s) = -expm1(-L),
//   d alpha / d s0 = (1 - alpha) k sigmoid(-k s0),  d alpha / d s1 = -(1 - alpha) k sigmoid(-k s1),
// both bounded by k.
template <bool kCompat>
__device__ __forceinline__ void interval_dalpha(float t0, float t1, float k, float *d_next, float *d_this) {
    if (kCompat) {
        const float inv = 1.0f / (1.0f + t1);
        *d_next = -k * t1 * (1.0f + t0) * inv * inv;
        *d_this = k * t0 * inv;
    } else {
        const float keep = k * expf(t0 - t1);
        *d_next = keep * expm1f(-t1);
        *d_this = -keep * expm1f(-t0);
    }
}

// fixed mode: a first-order distance is trusted only where |grad f| does not vanish and the
// distance is on the volume's scale (|sdf| <= 4; the box diagonal is 2 sqrt 3); elsewhere the
// quadric is degenerate at that point and the sample is treated as empty.
constexpr float kMaxSdf = 4.0f;
constexpr float kMinGrad2 = 1e-30f;
template <bool kCompat>
__device__ __forceinline__ float checked_sdf(const float *a, f3 u, float reso) {
    const float s = quad_sdf(a, u, reso);
    if (kCompat) return s;
    const float nx = 2 * a[0] * u.x + a[3], ny = 2 * a[1] * u.y + a[4], nz = 2 * a[2] * u.z + a[5];
    const float len2 = nx * nx + ny * ny + nz * nz;
    return (len2 >= kMinGrad2 && fabsf(s) <= kMaxSdf) ? s : __int_as_float(0x7fc00000);
}

// The render sample's normal and its gradient.  fixed mode: where grad f vanishes the normal
// is undefined; it is taken as +z and passes no gradient back.
template <bool kCompat>
__device__ __forceinline__ f3 sample_normal(const float *a, f3 u) {
    if (!kCompat) {
        const float nx = 2 * a[0] * u.x + a[3], ny = 2 * a[1] * u.y + a[4], nz = 2 * a[2] * u.z + a[5];
        if (!(nx * nx + ny * ny + nz * nz >= kMinGrad2)) return f3{0.0f, 0.0f, 1.0f};
    }
    return quad_normal(a, u);
}
template <bool kCompat>
__device__ __forceinline__ void sample_normal_grad(const float *a, f3 u, f3 gn, float *g) {
    if (!kCompat) {
        const float nx = 2 * a[0] * u.x + a[3], ny = 2 * a[1] * u.y + a[4], nz = 2 * a[2] * u.z + a[5];
        if (!(nx * nx + ny * ny + nz * nz >= kMinGrad2)) {
#pragma unroll
            for (int t = 0; t < 6; ++t) g[t] = 0.0f;
            return;
        }
    }
    quad_normal_grad(a, u, gn, g);
}

// Per-lane state of one render sample of a chunk.
struct Sample {
    bool valid;      // sample exists and all its cells are inside the grid
    bool shaded;     // valid and its colour matters: its row is gathered and shaded
    float alpha;
    float e0, e1;    // alpha_term of sdf_i and sdf_{i+1}
    f3 rgb, spec, nrm;
    CellPoint c1;    // SDF sample i+1
    CellPoint cr;    // render sample i
    uint32_t vbase;  // base vertex of the trilinear fetch
    float wx, wy, wz;
};

// Forward evaluation of render sample i = chunk*32 + lane (kernel/camera.cu:60-96,
// kernel/surface.cu:54-115, kernel/render.cu:98-179, :239-244).  Leaves the sample's
// interpolated 32 channels in the warp's tile.
template <bool kCompat, typename S, int kDeg, int kVar>
__device__ __forceinline__ void eval_chunk(const Params &p, uint32_t r, f3 o, f3 d, uint32_t nr, uint32_t chunk,
                                           int lane, float *tile, Sample &s, const float *from_slot = nullptr,
                                           float *to_slot = nullptr) {
    using RW = Rows<kDeg>;
    constexpr int kC = RW::kC, kRow = RW::kStride, kL = RW::kLanes, kPS = RW::kPerStep;
    const uint32_t R = p.R;
    const uint32_t i = chunk * kWarp + lane;
    const bool live = i < nr;
    bool ok = live;
    const float *tl = p.tlist ? QSDVR_AT(p.tlist, (uint64_t)kListT * r, kListT, (uint64_t)kListT * p.n) : nullptr;
    // SDF sample i+1 (this lane's interval end); sample i comes from the previous lane.
    s.c1 = to_cell(tl ? at_t(o, d, live ? tl[i + 1] : 0.0f) : march(o, d, (float)(i + 1), p.interval),
                   p.volume_offset, R);
    float a1[7];
    float s1 = 0.0f;
    if (live) {
        if (cell_in_grid(s.c1, R)) {
            load_cell<S, kVar>(p, s.c1, a1);
            s1 = checked_sdf<kCompat>(a1, s.c1.u, (float)R);
        } else {
            ok = false;
        }
    }
    float s0 = __shfl_up_sync(kFull, s1, 1);
    if (lane == 0 && live) {
        const CellPoint c0 =
            to_cell(tl ? at_t(o, d, tl[i]) : march(o, d, (float)i, p.interval), p.volume_offset, R);
        if (cell_in_grid(c0, R)) {
            float a0[7];
            load_cell<S, kVar>(p, c0, a0);
            s0 = checked_sdf<kCompat>(a0, c0.u, (float)R);
        } else {
            ok = false;
        }
    }
    const bool ok_prev = __shfl_up_sync(kFull, ok, 1);
    if (lane > 0) ok = ok && ok_prev;  // sdf_i is only valid if the previous lane's cell was
    // render sample i
    s.cr = to_cell(tl ? at_t(o, d, live ? 0.5f * (tl[i] + tl[i + 1]) : 0.0f) : midpoint(o, d, i, p.interval),
                   p.volume_offset, R);
    float ar[7];
    if (live && cell_in_grid(s.cr, R)) {
        load_cell<S, kVar>(p, s.cr, ar);
        s.nrm = sample_normal<kCompat>(ar, s.cr.u);
    } else {
        ok = false;
        s.nrm = f3{0.0f, 0.0f, 1.0f};
    }
    if (live && !ok) flag_error(QSDVR_DEVERR_INDEX);
    // fixed mode: a sample whose first-order distance is not finite (|grad f| = 0 in a cell)
    // is empty; compat keeps the reference's arithmetic, non-finite values included
    if (!kCompat && !(isfinite(s0) && isfinite(s1))) ok = false;
    s.valid = ok;
    s.e0 = alpha_term<kCompat>(p.k, s0);
    s.e1 = alpha_term<kCompat>(p.k, s1);
    s.alpha = ok ? interval_alpha<kCompat>(s.e0, s.e1) : 0.0f;
    // A valid sample with alpha = 0 (the SDF does not fall across its interval: about half
    // of a ray's samples) adds alpha T c = 0 to the colour, and every backward term of its
    // colour is a product with alpha or with dalpha/dsdf, both 0 there.  Its row is neither
    // gathered nor shaded (rgb = 0), which leaves every output bit-identical for finite
    // appearance rows.  A non-finite normal keeps the full path, so the NaN colour of a
    // degenerate cell propagates as in the reference.
    s.shaded = ok && (s.alpha != 0.0f || !(isfinite(s.nrm.x) && isfinite(s.nrm.y) && isfinite(s.nrm.z)));
    // trilinear weights and base vertex (kernel/render.cu:107-111)
    s.wx = (s.cr.u.x + 1.0f) / 2.0f;
    s.wy = (s.cr.u.y + 1.0f) / 2.0f;
    s.wz = (s.cr.u.z + 1.0f) / 2.0f;
    const uint32_t R1 = R + 1;
    s.vbase = kCompat ? (uint32_t)s.cr.index
                      : (uint32_t)s.cr.cx + (uint32_t)s.cr.cy * R1 + (uint32_t)s.cr.cz * (R1 * R1);
    const int q = lane % kL;
    const uint32_t sy = R1, sz = R1 * R1;
    [[maybe_unused]] const uint64_t nv = (uint64_t)R1 * R1 * R1;  // vertex rows
#if QSDVR_GATHER_PREFETCH
    if constexpr (QSDVR_GATHER_PREFETCH == 2 || kDeg == 2) {
        // samples of the gather's first round of loads (issued right below) are not prefetched
        constexpr int kRound = (sizeof(S) == 2 ? GatherLanes<S, kDeg>::kPerStep : kPS) * kGatherUnroll;
        if (!from_slot && s.shaded && lane >= kRound) {
            constexpr uint32_t kPair = 2u * kC * sizeof(S);  // rows v and v + 1 are adjacent
            const S *base = static_cast<const S *>(p.data);
            const uint32_t pv[4] = {s.vbase, s.vbase + sy, s.vbase + sz, s.vbase + sz + sy};
#pragma unroll
            for (int t = 0; t < 4; ++t)
                prefetch_l2(QSDVR_AT(base, (uint64_t)kC * pv[t], 2 * kC, (uint64_t)kC * nv), kPair);
        }
    }
#endif
    if (!from_slot) {
        st4(tile + lane * kRow + kC, make_float4(__uint_as_float(s.shaded ? s.vbase : kNoVertex), s.wx, s.wy, s.wz));
        __syncwarp();
    }
    if (from_slot) {
        // rows stashed by the forward, one row per kL lanes per step, copied into the tile by
        // asynchronous 16-byte copies that are all in flight at once (one L2 round trip per
        // chunk instead of one per round of register loads)
        const uint64_t pol = evict_last_policy();
#pragma unroll
        for (int st = 0; st < kL; ++st) {
            const int j = st * kPS + lane / kL;
            cp_async16_keep(tile + j * kRow + 4 * q, from_slot + j * kC + 4 * q, pol);
        }
        cp_async_wait();
#if QSDVR_STASH_DISCARD
        // The stash is dead once read: drop its L2 lines without writing them back (they
        // would otherwise reach DRAM as dirty evictions) and free the room for the gathers.
        // Every lane's copies have completed (cp.async.wait_all before the warp barrier).
        __syncwarp();
        constexpr uint32_t kLines = kWarp * kC * sizeof(float) / 128;  // the chunk's 128-byte lines
        for (uint32_t l = lane; l < kLines; l += kWarp)
            asm volatile("discard.global.L2 [%0], 128;" ::"l"(from_slot + l * (128 / sizeof(float))) : "memory");
#endif
    } else if constexpr (sizeof(S) == 2) {
        // bf16 storage: groups of kGL lanes fetch one sample's 8 corner rows as 16-byte
        // (bf16 x 8) loads, kGPS samples per step; each lane stages 8 interpolated channels
        using GL = GatherLanes<S, kDeg>;
        constexpr int kGL = GL::kLanes, kGPS = GL::kPerStep;
        const int q8 = lane % kGL;
#pragma unroll kGatherUnroll
        for (int st = 0; st < kGL; ++st) {
            const int j = st * kGPS + lane / kGL;
            const float4 prm = ld4(tile + j * kRow + kC);
            const uint32_t vb = __float_as_uint(prm.x);
            const float gx = prm.y, gy = prm.z, gz = prm.w;
            const bool gok = vb != kNoVertex;
            float v[8];
            if (gok) {
                const uint4 v000 = Store<S>::oct(p.data, vb, q8, kC, nv), v001 = Store<S>::oct(p.data, vb + 1, q8, kC, nv);
                const uint4 v010 = Store<S>::oct(p.data, vb + sy, q8, kC, nv),
                            v011 = Store<S>::oct(p.data, vb + sy + 1, q8, kC, nv);
                const uint4 v100 = Store<S>::oct(p.data, vb + sz, q8, kC, nv),
                            v101 = Store<S>::oct(p.data, vb + sz + 1, q8, kC, nv);
                const uint4 v110 = Store<S>::oct(p.data, vb + sz + sy, q8, kC, nv),
                            v111 = Store<S>::oct(p.data, vb + sz + sy + 1, q8, kC, nv);
                float w[8];
                corner_weights(gx, gy, gz, w);
                first_bf8(v000, w[0], v);
                fma_bf8(v001, w[1], v);
                fma_bf8(v010, w[2], v);
                fma_bf8(v011, w[3], v);
                fma_bf8(v100, w[4], v);
                fma_bf8(v101, w[5], v);
                fma_bf8(v110, w[6], v);
                fma_bf8(v111, w[7], v);
            } else {
#pragma unroll
                for (int t = 0; t < 8; ++t) v[t] = 0.0f;
            }
            const float4 lo = make_float4(v[0], v[1], v[2], v[3]), hi = make_float4(v[4], v[5], v[6], v[7]);
            // with 8 lanes per row (64 channels) lanes 4..7 store their halves in the other
            // order, so each 8-lane phase of a store covers 32 distinct banks
            const bool swap = (q8 & 4) != 0;
            st4(tile + j * kRow + 8 * q8 + (swap ? 4 : 0), swap ? hi : lo);
            st4(tile + j * kRow + 8 * q8 + (swap ? 0 : 4), swap ? lo : hi);
            if (to_slot) {
                const uint64_t pol = evict_last_policy();
                st4_keep(to_slot + j * kC + 8 * q8, lo, pol);
                st4_keep(to_slot + j * kC + 8 * q8 + 4, hi, pol);
            }
        }
    } else {
    // gather: groups of kL lanes fetch one sample's 8 corner rows, kPS samples per step
#pragma unroll kGatherUnroll
    for (int st = 0; st < kL; ++st) {
        const int j = st * kPS + lane / kL;
        const float4 prm = ld4(tile + j * kRow + kC);
        const uint32_t vb = __float_as_uint(prm.x);
        const float gx = prm.y, gy = prm.z, gz = prm.w;
        const bool gok = vb != kNoVertex;
        float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (gok) {
            const float4 v000 = Store<S>::quad(p.data, vb, q, kC, nv), v001 = Store<S>::quad(p.data, vb + 1, q, kC, nv);
            const float4 v010 = Store<S>::quad(p.data, vb + sy, q, kC, nv),
                         v011 = Store<S>::quad(p.data, vb + sy + 1, q, kC, nv);
            const float4 v100 = Store<S>::quad(p.data, vb + sz, q, kC, nv),
                         v101 = Store<S>::quad(p.data, vb + sz + 1, q, kC, nv);
            const float4 v110 = Store<S>::quad(p.data, vb + sz + sy, q, kC, nv),
                         v111 = Store<S>::quad(p.data, vb + sz + sy + 1, q, kC, nv);
            float w[8];
            corner_weights(gx, gy, gz, w);
            v = scale4(v000, w[0]);
            fma4(v, v001, w[1]);
            fma4(v, v010, w[2]);
            fma4(v, v011, w[3]);
            fma4(v, v100, w[4]);
            fma4(v, v101, w[5]);
            fma4(v, v110, w[6]);
            fma4(v, v111, w[7]);
        }
        st4(tile + j * kRow + 4 * q, v);
        if (to_slot) st4_keep(to_slot + j * kC + 4 * q, v, evict_last_policy());
    }
    }
    // one shading call site for both the gathered and the stashed rows (the kernel's code
    // size sets how often its warps wait for instruction fetch)
    __syncwarp();
    if (s.shaded) {
        // the row stays in shared memory; the shader reads the channels it needs from it
        s.rgb = shade_any<kCompat, kDeg>(s.nrm, d, tile + lane * kRow, &s.spec);
    } else {
        s.rgb = f3{0.0f, 0.0f, 0.0f};
        s.spec = f3{0.0f, 0.0f, 0.0f};
    }
}

// Alpha only (no normal, gather or shading): what the backward-only pass needs to
// rebuild the transmittance at each chunk start.  Validity matches eval_chunk.
template <bool kCompat, typename S, int kVar>
__device__ __forceinline__ void eval_alpha(const Params &p, uint32_t r, f3 o, f3 d, uint32_t nr, uint32_t chunk,
                                           int lane, Sample &s) {
    const uint32_t R = p.R;
    const uint32_t i = chunk * kWarp + lane;
    const bool live = i < nr;
    bool ok = live;
    const float *tl = p.tlist ? QSDVR_AT(p.tlist, (uint64_t)kListT * r, kListT, (uint64_t)kListT * p.n) : nullptr;
    const CellPoint c1 = to_cell(tl ? at_t(o, d, live ? tl[i + 1] : 0.0f) : march(o, d, (float)(i + 1), p.interval),
                                 p.volume_offset, R);
    float s1 = 0.0f;
    if (live) {
        if (cell_in_grid(c1, R)) {
            float a1[7];
            load_cell<S, kVar>(p, c1, a1);
            s1 = checked_sdf<kCompat>(a1, c1.u, (float)R);
        } else {
            ok = false;
        }
    }
    float s0 = __shfl_up_sync(kFull, s1, 1);
    if (lane == 0 && live) {
        const CellPoint c0 =
            to_cell(tl ? at_t(o, d, tl[i]) : march(o, d, (float)i, p.interval), p.volume_offset, R);
        if (cell_in_grid(c0, R)) {
            float a0[7];
            load_cell<S, kVar>(p, c0, a0);
            s0 = checked_sdf<kCompat>(a0, c0.u, (float)R);
        } else {
            ok = false;
        }
    }
    const bool ok_prev = __shfl_up_sync(kFull, ok, 1);
    if (lane > 0) ok = ok && ok_prev;
    if (live && !cell_in_grid(to_cell(tl ? at_t(o, d, 0.5f * (tl[i] + tl[i + 1])) : midpoint(o, d, i, p.interval),
                                      p.volume_offset, R),
                              R))
        ok = false;
    if (!kCompat && !(isfinite(s0) && isfinite(s1))) ok = false;
    s.valid = ok;
    s.e0 = alpha_term<kCompat>(p.k, s0);
    s.e1 = alpha_term<kCompat>(p.k, s1);
    s.alpha = ok ? interval_alpha<kCompat>(s.e0, s.e1) : 0.0f;
}

// Transmittance at each lane's sample given the value at the chunk start.  kLogT uses the
// compensated running sum of log(1 - alpha) (carry = sum, comp = Kahan compensation).
template <bool kLogT>
struct Transmittance {
    float carry = kLogT ? 0.0f : 1.0f;
    float comp = 0.0f;

    // returns T_i for this lane and advances the carry past the chunk
    __device__ __forceinline__ float step(float alpha, bool valid, int lane) {
        if (kLogT) {
            float incl = valid ? log1pf(-alpha) : 0.0f;
#pragma unroll
            for (int o = 1; o < kWarp; o <<= 1) {
                const float v = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += v;
            }
            float excl = __shfl_up_sync(kFull, incl, 1);
            if (lane == 0) excl = 0.0f;
            const float T = expf(carry + excl);
            const float tot = __shfl_sync(kFull, incl, kWarp - 1);
            const float y = tot - comp;
            const float t = carry + y;
            // once alpha == 1 the sum is -inf for good: keep the compensation finite
            comp = isfinite(t) ? (t - carry) - y : 0.0f;
            carry = t;
            return T;
        } else {
            float incl = valid ? 1.0f - alpha : 1.0f;
#pragma unroll
            for (int o = 1; o < kWarp; o <<= 1) {
                const float v = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl *= v;
            }
            float excl = __shfl_up_sync(kFull, incl, 1);
            if (lane == 0) excl = 1.0f;
            const float T = carry * excl;
            carry *= __shfl_sync(kFull, incl, kWarp - 1);
            return T;
        }
    }
};

// 4 channels of the bf16 data gradient: one 8-byte vector RED (bf16x2 pairs, noftz).
__device__ __forceinline__ void red4_bf16(__nv_bfloat16 *p, float4 v) {
    const uint32_t lo = pack_bf16x2(v.x, v.y), hi = pack_bf16x2(v.z, v.w);
    asm volatile("red.global.add.noftz.v2.bf16x2 [%0], {%1, %2};" ::"l"(p), "r"(lo), "r"(hi) : "memory");
}

// The 8 corner contributions of one sample's gradient quad g at trilinear weights (px, py,
// pz), corner t = 4z + 2y + x (kernel/render.cu:136-151).
__device__ __forceinline__ void corner_grads(float4 g, float px, float py, float pz, float4 *v) {
    const float dx = 1 - px, dy = 1 - py;
    const float4 a0 = scale4(g, 1 - pz), a1 = scale4(g, pz);
    const float4 a00 = scale4(a0, dy), a01 = scale4(a0, py), a10 = scale4(a1, dy), a11 = scale4(a1, py);
    v[0] = scale4(a00, dx); v[1] = scale4(a00, px); v[2] = scale4(a01, dx); v[3] = scale4(a01, px);
    v[4] = scale4(a10, dx); v[5] = scale4(a10, px); v[6] = scale4(a11, dx); v[7] = scale4(a11, px);
}
__device__ __forceinline__ float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }

// Scatter the data-gradient tile (rows of 32 channels per lane's sample) through the
// trilinear weights: 8 lanes per sample, one 16-byte RED (8 bytes for a bf16 gradient) per
// lane and corner.  In the kVarMerge variant, samples of the chunk that lie in the same cell (same base
// vertex) are found with one match_any: the first of them sums the others' weighted
// contributions (their gradient rows and weights read from the tile) and sends one RED per
// corner row for all of them; the others send nothing.
template <int kDeg, int kVar>
__device__ __forceinline__ void scatter_tile(const Params &p, float *tile, const Sample &s, int lane) {
    using RW = Rows<kDeg>;
    constexpr int kC = RW::kC, kRow = RW::kStride, kL = RW::kLanes, kPS = RW::kPerStep;
    const uint32_t R1 = p.R + 1, sy = R1, sz = R1 * R1;
    [[maybe_unused]] const uint64_t ne = (uint64_t)kC * R1 * R1 * R1;  // gradient elements
    const int q = lane % kL;
    uint32_t others = 0;  // kVarMerge: the later samples of this lane's cell, summed into this one
    bool follower = false;
    if constexpr ((kVar & kVarMerge) != 0) {
        const uint32_t key = s.valid ? s.vbase : (0x80000000u | (uint32_t)lane);  // vertices < 2^31
        const uint32_t peers = __match_any_sync(kFull, key);
        follower = (peers & ((1u << lane) - 1u)) != 0;  // a lower lane of the same cell leads
        others = follower ? 0u : (peers & ~(1u << lane));
    }
    // the row pad: (base vertex, or kNoVertex for a sample that sends nothing, and weights)
    st4(tile + lane * kRow + kC,
        make_float4(__uint_as_float(s.valid && !follower ? s.vbase : kNoVertex), s.wx, s.wy, s.wz));
    __syncwarp();
// (one step per iteration: the REDs do not wait, and a smaller loop body keeps the kernel's
// code small; measured as fast as two steps per iteration)
#pragma unroll 1
    for (int st = 0; st < kL; ++st) {
        const int j = st * kPS + lane / kL;
        const uint32_t more = (kVar & kVarMerge) != 0 ? __shfl_sync(kFull, others, j) : 0u;
        const float4 w = ld4(tile + j * kRow + kC);
        const uint32_t vb = __float_as_uint(w.x);
        if (vb == kNoVertex) continue;
        // A sample with alpha = 0 (the SDF does not fall across its interval) or T = 0 has a
        // zero appearance gradient, as do channels its shader never reads: its 8 REDs would
        // add zeros, yet each costs an L2 read-modify-write of a row that is usually not
        // cached.  Skipped; the sums stay bit-identical (is_zero4).
        const float4 g = ld4(tile + j * kRow + 4 * q);
        if (is_zero4(g) && more == 0u) continue;
        float4 v[8];
        corner_grads(g, w.y, w.z, w.w, v);  // kernel/render.cu:136-151
        for (uint32_t m = more; m; m &= m - 1) {  // rare: the other samples of the same cell
            const int f = __ffs(m) - 1;
            const float4 gf = ld4(tile + f * kRow + 4 * q), wf = ld4(tile + f * kRow + kC);
            const float wx[2] = {1 - wf.y, wf.y}, wy[2] = {1 - wf.z, wf.z}, wz[2] = {1 - wf.w, wf.w};
#pragma unroll
            for (int t = 0; t < 8; ++t) v[t] = add4(v[t], scale4(gf, wz[t >> 2] * wy[(t >> 1) & 1] * wx[t & 1]));
        }
        const uint64_t o = (uint64_t)kC * vb + 4 * q;
        const uint64_t c[8] = {o, o + kC, o + (uint64_t)kC * sy, o + (uint64_t)kC * sy + kC, o + (uint64_t)kC * sz,
                               o + (uint64_t)kC * sz + kC, o + (uint64_t)kC * (sz + sy),
                               o + (uint64_t)kC * (sz + sy) + kC};
        if (p.grad_bf16) {
            __nv_bfloat16 *b = reinterpret_cast<__nv_bfloat16 *>(p.data_grad);
#pragma unroll
            for (int t = 0; t < 8; ++t) red4_bf16(QSDVR_AT(b, c[t], 4, ne), v[t]);
        } else {
#pragma unroll
            for (int t = 0; t < 8; ++t) red4(QSDVR_AT(p.data_grad, c[t], 4, ne), v[t]);
        }
    }
}


// Backward of one chunk given its per-sample state (eval_chunk) and transmittance T: the
// compositing backward (compat: the reference's Tac / (alpha - 1) form; fixed: the
// division-free reverse affine scan), dalpha/dsdf, the quadric-cell gradients and the
// appearance scatter.  suf and next_this carry the suffix state to the preceding chunk.
template <bool kCompat, typename S, int kDeg, int kVar>
__device__ __forceinline__ void backward_chunk(const Params &p, f3 o, f3 d, uint32_t nr, uint32_t c, int lane,
                                               float *tile, const Sample &s, float T, f3 g, f3 &suf,
                                               float &next_this) {
    constexpr int kRow = Rows<kDeg>::kStride;
    const float a = s.alpha;
    const uint32_t i = c * kWarp + lane;
    float dl = 0.0f;  // dL/dalpha_i
    if (kCompat) {
        // kernel/render.cu:279-313: Tac = sum over later samples of T a c
        f3 v = s.valid ? f3{s.rgb.x * T * a, s.rgb.y * T * a, s.rgb.z * T * a} : f3{0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int off = 1; off < kWarp; off <<= 1) {
            const float x = __shfl_down_sync(kFull, v.x, off), y = __shfl_down_sync(kFull, v.y, off),
                        z = __shfl_down_sync(kFull, v.z, off);
            if (lane + off < kWarp) {
                v.x += x;
                v.y += y;
                v.z += z;
            }
        }
        f3 after{__shfl_down_sync(kFull, v.x, 1), __shfl_down_sync(kFull, v.y, 1),
                 __shfl_down_sync(kFull, v.z, 1)};
        if (lane == kWarp - 1) after = f3{0.0f, 0.0f, 0.0f};
        after.x += suf.x;
        after.y += suf.y;
        after.z += suf.z;
        if (s.valid) {
            const f3 dc{s.rgb.x * T + after.x / (a - 1), s.rgb.y * T + after.y / (a - 1),
                        s.rgb.z * T + after.z / (a - 1)};
            dl = g.x * dc.x + g.y * dc.y + g.z * dc.z;
        }
        suf.x += __shfl_sync(kFull, v.x, 0);
        suf.y += __shfl_sync(kFull, v.y, 0);
        suf.z += __shfl_sync(kFull, v.z, 0);
    } else {
        // R_i = a_i c_i + (1 - a_i) R_{i+1}: reverse scan of affine maps, no division
        f3 A = s.valid ? f3{a * s.rgb.x, a * s.rgb.y, a * s.rgb.z} : f3{0.0f, 0.0f, 0.0f};
        float B = s.valid ? 1.0f - a : 1.0f;
#pragma unroll
        for (int off = 1; off < kWarp; off <<= 1) {
            const float x = __shfl_down_sync(kFull, A.x, off), y = __shfl_down_sync(kFull, A.y, off),
                        z = __shfl_down_sync(kFull, A.z, off), b = __shfl_down_sync(kFull, B, off);
            if (lane + off < kWarp) {
                A.x += B * x;
                A.y += B * y;
                A.z += B * z;
                B *= b;
            }
        }
        const f3 Ri{A.x + B * suf.x, A.y + B * suf.y, A.z + B * suf.z};
        f3 Rn{__shfl_down_sync(kFull, Ri.x, 1), __shfl_down_sync(kFull, Ri.y, 1),
              __shfl_down_sync(kFull, Ri.z, 1)};
        if (lane == kWarp - 1) Rn = suf;
        if (s.valid) dl = T * (g.x * (s.rgb.x - Rn.x) + g.y * (s.rgb.y - Rn.y) + g.z * (s.rgb.z - Rn.z));
        suf = f3{__shfl_sync(kFull, Ri.x, 0), __shfl_sync(kFull, Ri.y, 0), __shfl_sync(kFull, Ri.z, 0)};
    }
    // dalpha/dsdf (kernel/render.cu:271-278), zero where alpha == 0
    float d_this = 0.0f, d_next = 0.0f;
    if (s.valid && a != 0.0f) interval_dalpha<kCompat>(s.e0, s.e1, p.k, &d_next, &d_this);
    const float mine_this = dl * d_this;
    float from_next = __shfl_down_sync(kFull, mine_this, 1);
    if (lane == kWarp - 1) from_next = next_this;
    next_this = __shfl_sync(kFull, mine_this, 0);
    if (s.valid) {
        // SDF sample i+1 and, for the ray's first lane, SDF sample 0
        const float gs1 = dl * d_next + (i + 1 < nr ? from_next : 0.0f);
        float a1[7], gq[7];
        load_cell<S, kVar>(p, s.c1, a1);
        quad_sdf_grad(a1, s.c1.u, (float)p.R, gs1, gq);
        // rgb gradient; 0 for an unshaded sample (alpha = 0) unless the ray's colour
        // gradient is not finite (a NaN colour), which the reference spreads to
        // every sample of the ray: then the unshaded one takes the full path too
        // (its zero row gives the same NaN outputs as the real row would)
        const f3 grgb{g.x * T * a, g.y * T * a, g.z * T * a};
        if (s.shaded || !(isfinite(grgb.x) && isfinite(grgb.y) && isfinite(grgb.z))) {
            // rgb gradient -> shader backward (data gradient into the tile, normal gradient)
            // data gradient written over the data row (every read precedes its write)
            const f3 gn =
                shade_any_backward_inplace<kCompat, kDeg>(grgb, s.nrm, d, tile + lane * kRow, s.spec);
            float ar[7], gr[6];
            load_cell<S, kVar>(p, s.cr, ar);
            sample_normal_grad<kCompat>(ar, s.cr.u, gn, gr);
            if (s.cr.index == s.c1.index) {
#pragma unroll
                for (int t = 0; t < 6; ++t) gq[t] += gr[t];
                scatter_cell<kVar>(p, s.c1, gq);
            } else {
                scatter_cell<kVar>(p, s.c1, gq);
                const float g7[7] = {gr[0], gr[1], gr[2], gr[3], gr[4], gr[5], 0.0f};
                scatter_cell<kVar>(p, s.cr, g7);
            }
        } else {
            // alpha = 0: the colour's gradients (data row, normal) are 0 and the row
            // in the tile is the gather's zeros, which the scatter skips
            scatter_cell<kVar>(p, s.c1, gq);
        }
        if (i == 0) {
            const CellPoint c0 = to_cell(march(o, d, 0.0f, p.interval), p.volume_offset, p.R);
            float a0[7], g0[7];
            load_cell<S, kVar>(p, c0, a0);
            quad_sdf_grad(a0, c0.u, (float)p.R, mine_this, g0);
            scatter_cell<kVar>(p, c0, g0);
        }
    }
    __syncwarp();
    scatter_tile<kDeg, kVar>(p, tile, s, lane);
    __syncwarp();
}

template <bool kCompat, typename S, int kPass, bool kLogT, int kDeg, int kVar>
__global__ void __launch_bounds__(kThreads, QSDVR_FUSED_MIN_BLOCKS) render_kernel(const Params p) {
    constexpr int kRow = Rows<kDeg>::kStride;
    constexpr uint32_t kChunkFloats = chunk_floats<kDeg>();
    __shared__ __align__(16) float tiles[kWarpsPerBlock][kWarp * kRow];
    // the transmittance carry at each chunk start of the current ray, for the backward
    __shared__ float carries[kWarpsPerBlock][kMaxChunks];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float *tile = tiles[w];
    const uint32_t warp_id = blockIdx.x * kWarpsPerBlock + w;
    // Without a workspace each warp renders one ray (one warp per block: the block scheduler
    // balances ray lengths).  With one, the grid is persistent and warps take rays from a
    // counter; in train mode each warp also owns a row stash (slot).
    const bool persistent = p.ray_counter != nullptr;
    float *slot = (kPass == kTrain && p.slots &&
                   QSDVR_IN_RANGE((uint64_t)warp_id * kSlotChunks * kChunkFloats, kSlotChunks * kChunkFloats,
                                  (uint64_t)gridDim.x * kWarpsPerBlock * kSlotChunks * kChunkFloats))
                      ? p.slots + (uint64_t)warp_id * kSlotChunks * kChunkFloats
                      : nullptr;
    float sq = 0.0f;
    uint32_t r = persistent ? 0u : warp_id;
    for (;;) {
    if (persistent) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(p.ray_counter, 1u);
        r = __shfl_sync(kFull, t, 0);
    }
    if (r >= p.n) break;
    const uint32_t taken = r;  // the ray counter's index; the ray itself may come from an order
    if (p.order) {
        r = *QSDVR_AT(p.order, taken, 1, p.n);
        if (r >= p.n) {  // not a permutation of the batch: skip the entry
            if (lane == 0) flag_error(QSDVR_DEVERR_RAY);
            if (!persistent) break;
            continue;
        }
    }
    {
        const qsdvr_ray_info info = *QSDVR_AT(p.rays, r, 1, p.n);
        const uint32_t ns = info.sdf_count;
        const uint32_t nr = ns > 1 ? (p.tlist ? kListT - 1 : ns - 1) : 0;
        const uint32_t chunks = (nr + kWarp - 1) / kWarp;
        const f3 o = load3(QSDVR_AT(p.origin, 3ull * r, 3, 3ull * p.n)),
                 d = load3(QSDVR_AT(p.dir, 3ull * r, 3, 3ull * p.n));
        f3 C{0.0f, 0.0f, 0.0f};
        bool run = nr > 0;
        if (chunks > kMaxChunks) {
            if (lane == 0) flag_error(QSDVR_DEVERR_RAY);
            run = false;
        }
        Sample s;
        Transmittance<kLogT> tr;
        float *carry_at = carries[w];  // carry_at[c]: the transmittance carry at the start of chunk c
        float T_last = 0.0f;               // transmittance of this lane's sample in the last chunk
        // ---------------- forward (forward and backward-only passes)
        if (kPass == kForward || (kPass == kBackward && run)) {
            if (run) {
                f3 acc{0.0f, 0.0f, 0.0f};
                for (uint32_t c = 0; c < chunks; ++c) {
                    if (lane == 0) carry_at[c] = tr.carry;  // warp-uniform
                    if (kPass == kBackward) {
                        eval_alpha<kCompat, S, kVar>(p, r, o, d, nr, c, lane, s);
                        tr.step(s.alpha, s.valid, lane);
                    } else {
                        eval_chunk<kCompat, S, kDeg, kVar>(p, r, o, d, nr, c, lane, tile, s);
                        const float T = tr.step(s.alpha, s.valid, lane);
                        if (p.sample_alpha && c * kWarp + lane < nr) {
                            const uint64_t m = (uint64_t)info.render_offset + c * kWarp + lane;
                            if (m < p.sample_capacity) p.sample_alpha[m] = s.alpha;
                            else flag_error(QSDVR_DEVERR_CAPACITY);
                        }
                        acc.x += s.rgb.x * s.alpha * T;
                        acc.y += s.rgb.y * s.alpha * T;
                        acc.z += s.rgb.z * s.alpha * T;
                        __syncwarp();
                    }
                }
                C = f3{warp_sum(acc.x), warp_sum(acc.y), warp_sum(acc.z)};
            }
            if (kPass == kForward && lane == 0) store3(QSDVR_AT(p.color, 3ull * r, 3, 3ull * p.n), C);
        }
        if (kPass == kBackward && run) {
            const f3 g = load3(QSDVR_AT(p.grad_color, 3ull * r, 3, 3ull * p.n));
            f3 suf{0.0f, 0.0f, 0.0f};  // compat: sum_{m>chunk} T a c ; fixed: R after the chunk
            float next_this = 0.0f;    // d_this term of the first sample of the following chunk
            for (int c = (int)chunks - 1; c >= 0; --c) {
                __syncwarp();
                tr.carry = carry_at[c];
                eval_chunk<kCompat, S, kDeg, kVar>(p, r, o, d, nr, (uint32_t)c, lane, tile, s);
                const float T = tr.step(s.alpha, s.valid, lane);
                backward_chunk<kCompat, S, kDeg, kVar>(p, o, d, nr, (uint32_t)c, lane, tile, s, T, g, suf, next_this);
            }
        }
        // ---------------- train: the forward chunks, the MSE gradient, then the chunks in
        // reverse, as one loop with one chunk evaluation (one inlined copy of the gather and
        // shading code; the kernel's code size sets how often its warps wait for instruction
        // fetch).  The last forward chunk's rows and per-sample state stay in the tile and in
        // registers for the first backward step; stashed rows serve the chunks before it.
        if (kPass == kTrain) {
            f3 g{0.0f, 0.0f, 0.0f};
            f3 acc{0.0f, 0.0f, 0.0f};
            f3 suf{0.0f, 0.0f, 0.0f};
            float next_this = 0.0f;
            const uint32_t total = run ? 2 * chunks : 0;
            for (uint32_t it = 0;; ++it) {
                if (it == (run ? chunks : 0)) {
                    // end of the forward: colour, loss and its gradient
                    C = f3{warp_sum(acc.x), warp_sum(acc.y), warp_sum(acc.z)};
                    if (lane == 0) store3(QSDVR_AT(p.color, 3ull * r, 3, 3ull * p.n), C);
                    const f3 t = load3(QSDVR_AT(p.target, 3ull * r, 3, 3ull * p.n));
                    const f3 e{C.x - t.x, C.y - t.y, C.z - t.z};
                    if (lane == 0) sq += e.x * e.x + e.y * e.y + e.z * e.z;  // C is warp-uniform: count it once
                    g = f3{p.grad_scale * e.x, p.grad_scale * e.y, p.grad_scale * e.z};
                }
                if (it >= total) break;
                const bool fwd = it < chunks;
                const uint32_t c = fwd ? it : total - 1 - it;  // backward: chunks - 1 down to 0
                float T;
                if (fwd || c + 1 < chunks) {
                    if (fwd) {
                        if (lane == 0) carry_at[c] = tr.carry;  // warp-uniform
                    } else {
                        __syncwarp();
                        tr.carry = carry_at[c];
                    }
                    float *sl = (slot && c + 1 < chunks && c + 1 + kSlotChunks >= chunks)
                                    ? slot + (c % kSlotChunks) * kChunkFloats
                                    : nullptr;
                    eval_chunk<kCompat, S, kDeg, kVar>(p, r, o, d, nr, c, lane, tile, s, fwd ? nullptr : sl,
                                                 fwd ? sl : nullptr);
                    T = tr.step(s.alpha, s.valid, lane);
                } else {
                    // the forward just evaluated this chunk: its rows are still in the tile and
                    // its per-sample state in registers, so nothing is fetched again
                    T = T_last;
                }
                if (fwd) {
                    T_last = T;
                    if (p.sample_alpha && c * kWarp + lane < nr) {
                        const uint64_t m = (uint64_t)info.render_offset + c * kWarp + lane;
                        if (m < p.sample_capacity) p.sample_alpha[m] = s.alpha;
                        else flag_error(QSDVR_DEVERR_CAPACITY);
                    }
                    acc.x += s.rgb.x * s.alpha * T;
                    acc.y += s.rgb.y * s.alpha * T;
                    acc.z += s.rgb.z * s.alpha * T;
                    __syncwarp();
                } else {
                    backward_chunk<kCompat, S, kDeg, kVar>(p, o, d, nr, c, lane, tile, s, T, g, suf, next_this);
                }
            }
        }
    }
    if (!persistent) break;
    }  // ray loop
    if (kPass == kTrain && lane == 0 && sq != 0.0f) atomicAdd(p.loss, sq);
}

// ---- TMA brick staging for full frames (forward only, fixed mode, uniform march) --------
// A frame's rays listed tile by tile (8 x 8 pixels, Camera order "tiles"): one block of 64
// threads per tile, one thread per ray, each marching its render samples in order.  Rays of
// a tile cross neighbouring cells at similar depths, so the appearance rows their current
// samples need are staged in shared memory as one brick of kBrick^3 vertex rows, copied by
// one TMA tensor load (cp.async.bulk.tensor.4d, this GPU's grid only, no multicast) per
// round.  A round places the brick at the lowest corner of the tile's next samples, pulled
// toward the lowest-numbered ray that still marches so that it always advances; each thread
// then renders its samples while their cells stay inside the brick.  Per sample the arithmetic
// is the fused forward's (same cell validity, alpha, interpolation order and shading), with the
// compensated log-transmittance summed sample by sample.
constexpr int kBrick = 8;          // vertex rows per axis: a brick covers 7 cells per axis
constexpr int kBrickThreads = 64;  // rays per tile

template <typename S, int kDeg>
__global__ void __launch_bounds__(kBrickThreads) brick_frame_kernel(const __grid_constant__ CUtensorMap tmap,
                                                                    const Params p) {
    constexpr int kC = ShLayout<kDeg>::kChannels;
    constexpr int kRowBytes = kC * (int)sizeof(S);
    static_assert(kRowBytes == 128, "brick rows are 128-byte vertex rows");
    constexpr uint32_t kBrickBytes = kBrick * kBrick * kBrick * kRowBytes;
    constexpr int kPitch = kC + 1;  // per-thread row stride in floats (scalar reads conflict-free)
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // the brick at a 128-byte boundary of the dynamic shared memory (128 bytes of slack)
    unsigned char *smem = smem_raw + ((128u - (tc::smem_addr(smem_raw) & 127u)) & 127u);
    const S *brick = reinterpret_cast<const S *>(smem);
    float *row = reinterpret_cast<float *>(smem + kBrickBytes) + threadIdx.x * kPitch;
    __shared__ uint64_t mbar;
    __shared__ int box[7];  // min x, y, z, then the leader's cell x, y, z, then the leader thread
    const int t = threadIdx.x;
    const uint32_t R = p.R;
    const uint32_t r = blockIdx.x * kBrickThreads + t;
    // this thread's ray
    uint32_t nr = 0, i = 0;
    f3 o{0.0f, 0.0f, 0.0f}, d{0.0f, 0.0f, 1.0f};
    float s_prev = 0.0f, carry = 0.0f, comp = 0.0f;
    bool in_prev = false;
    f3 acc{0.0f, 0.0f, 0.0f};
    if (r < p.n) {
        const qsdvr_ray_info info = *QSDVR_AT(p.rays, r, 1, p.n);
        nr = info.sdf_count > 1 ? info.sdf_count - 1 : 0;
        o = load3(QSDVR_AT(p.origin, 3ull * r, 3, 3ull * p.n));
        d = load3(QSDVR_AT(p.dir, 3ull * r, 3, 3ull * p.n));
        if (nr > 0) {  // SDF sample 0
            const CellPoint c0 = to_cell(march(o, d, 0.0f, p.interval), p.volume_offset, R);
            in_prev = cell_in_grid(c0, R);
            if (in_prev) {
                float a0[7];
                load_cell<S, 0>(p, c0, a0);
                s_prev = checked_sdf<false>(a0, c0.u, (float)R);
            }
        }
    }
    if (t == 0) tc::mbar_init(&mbar, 1);
    __syncthreads();
    uint32_t parity = 0;
    bool failed = false;
    for (;;) {
        // the cell of this thread's next render sample
        CellPoint cr{};
        const bool active = i < nr;
        if (active) cr = to_cell(midpoint(o, d, i, p.interval), p.volume_offset, R);
        if (t == 0) {
            box[0] = box[1] = box[2] = 0x7fffffff;
            box[6] = kBrickThreads;
        }
        __syncthreads();
        if (active) {
            atomicMin(&box[0], cr.cx);
            atomicMin(&box[1], cr.cy);
            atomicMin(&box[2], cr.cz);
            atomicMin(&box[6], t);
        }
        __syncthreads();
        if (box[6] == kBrickThreads) break;  // every ray of the tile is done
        if (t == box[6]) {
            box[3] = cr.cx;
            box[4] = cr.cy;
            box[5] = cr.cz;
        }
        __syncthreads();
        int org[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) org[a] = min(max(box[a], box[3 + a] - (kBrick - 2)), box[3 + a]);
        if (t == 0) {
            // the previous round's reads of the brick are ordered before this copy by the
            // barriers above; the copy lands through the async proxy
            tc::fence_smem_to_async();
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_addr(&mbar)),
                         "r"(kBrickBytes)
                         : "memory");
            asm volatile(
                "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
                "%5}], [%6];" ::"r"(tc::smem_addr(smem)),
                "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(0), "r"(org[0]), "r"(org[1]), "r"(org[2]),
                "r"(tc::smem_addr(&mbar))
                : "memory");
        }
        if (!tc::mbar_wait(&mbar, parity, 1u << 30)) {
            if (t == 0) flag_error(QSDVR_DEVERR_TIMEOUT);
            failed = true;
        }
        if (__syncthreads_or(failed)) {
            tc::mbar_wait(&mbar, parity, 1u << 30);  // one more bounded wait for the copy in flight
            break;
        }
        parity ^= 1u;
        // render this thread's samples while their cell stays inside the brick
        while (i < nr) {
            cr = to_cell(midpoint(o, d, i, p.interval), p.volume_offset, R);
            const int lx = cr.cx - org[0], ly = cr.cy - org[1], lz = cr.cz - org[2];
            if (lx < 0 || ly < 0 || lz < 0 || lx > kBrick - 2 || ly > kBrick - 2 || lz > kBrick - 2) break;
            // SDF sample i + 1 and the interval's validity (eval_chunk, fixed mode)
            const CellPoint c1 = to_cell(march(o, d, (float)(i + 1), p.interval), p.volume_offset, R);
            bool ok = in_prev;
            float s1 = 0.0f;
            const bool in1 = cell_in_grid(c1, R);
            if (in1) {
                float a1[7];
                load_cell<S, 0>(p, c1, a1);
                s1 = checked_sdf<false>(a1, c1.u, (float)R);
            } else {
                ok = false;
            }
            f3 nrm{0.0f, 0.0f, 1.0f};
            if (cell_in_grid(cr, R)) {
                float ar[7];
                load_cell<S, 0>(p, cr, ar);
                nrm = sample_normal<false>(ar, cr.u);
            } else {
                ok = false;
            }
            if (!ok) flag_error(QSDVR_DEVERR_INDEX);
            if (!(isfinite(s_prev) && isfinite(s1))) ok = false;
            const float alpha = ok ? interval_alpha<false>(alpha_term<false>(p.k, s_prev), alpha_term<false>(p.k, s1))
                                   : 0.0f;
            const bool shaded = ok && (alpha != 0.0f || !(isfinite(nrm.x) && isfinite(nrm.y) && isfinite(nrm.z)));
            f3 rgb{0.0f, 0.0f, 0.0f};
            if (shaded) {
                // trilinear interpolation from the brick, corner order and FMA order of the
                // fused forward's gather
                float w[8];
                corner_weights((cr.u.x + 1.0f) / 2.0f, (cr.u.y + 1.0f) / 2.0f, (cr.u.z + 1.0f) / 2.0f, w);
                const int base = (lz * kBrick + ly) * kBrick + lx;
                const int off[8] = {0, 1, kBrick, kBrick + 1, kBrick * kBrick, kBrick * kBrick + 1,
                                    kBrick * kBrick + kBrick, kBrick * kBrick + kBrick + 1};
                for (int ch = 0; ch < kC; ch += 8) {
                    float v[8];
                    if constexpr (sizeof(S) == 2) {
                        first_bf8(*reinterpret_cast<const uint4 *>(brick + (base + off[0]) * kC + ch), w[0], v);
#pragma unroll
                        for (int q = 1; q < 8; ++q)
                            fma_bf8(*reinterpret_cast<const uint4 *>(brick + (base + off[q]) * kC + ch), w[q], v);
                    } else {
                        const float *b0 = reinterpret_cast<const float *>(brick) + (base + off[0]) * kC + ch;
                        float4 lo = scale4(ld4(b0), w[0]), hi = scale4(ld4(b0 + 4), w[0]);
#pragma unroll
                        for (int q = 1; q < 8; ++q) {
                            const float *bq = reinterpret_cast<const float *>(brick) + (base + off[q]) * kC + ch;
                            fma4(lo, ld4(bq), w[q]);
                            fma4(hi, ld4(bq + 4), w[q]);
                        }
                        v[0] = lo.x; v[1] = lo.y; v[2] = lo.z; v[3] = lo.w;
                        v[4] = hi.x; v[5] = hi.y; v[6] = hi.z; v[7] = hi.w;
                    }
#pragma unroll
                    for (int q = 0; q < 8; ++q) row[ch + q] = v[q];
                }
                f3 spec;
                rgb = shade_any<false, kDeg>(nrm, d, row, &spec);
            }
            // compensated log-transmittance, sample by sample
            const float T = expf(carry);
            acc.x += rgb.x * alpha * T;
            acc.y += rgb.y * alpha * T;
            acc.z += rgb.z * alpha * T;
            if (ok) {
                const float y = log1pf(-alpha) - comp;
                const float tt = carry + y;
                comp = isfinite(tt) ? (tt - carry) - y : 0.0f;
                carry = tt;
            }
            s_prev = s1;
            in_prev = in1;
            ++i;
        }
        __syncthreads();  // every read of this brick is done before the next copy overwrites it
    }
    if (r < p.n) store3(QSDVR_AT(p.color, 3ull * r, 3, 3ull * p.n), acc);
}

constexpr size_t kCounterBytes = 256;

// Calls f.template run<kCompat, S, kLogT, kDeg, kVar>() for the kernel configuration of `a`
// (degree 3 exists only in the packed, fixed-mode layout; the separable SDF only with degree
// 2 and without the merged scatter, which validate() enforces).
template <bool C, typename S, bool L, int D, typename F>
void with_variant(const qsdvr_render_args *a, F &f) {
    if (a->sdf_layers) {
        if constexpr (D == 2) f.template run<C, S, L, D, kVarSep>();
    } else if (a->merge_scatter) {
        f.template run<C, S, L, D, kVarMerge>();
    } else {
        f.template run<C, S, L, D, 0>();
    }
}

template <typename F>
void dispatch(const qsdvr_render_args *a, F &f) {
    const bool compat = a->mode == QSDVR_MODE_COMPAT;
    const bool bf16 = a->storage == QSDVR_STORAGE_BF16;
    const bool logt = a->transmittance == QSDVR_TRANSMITTANCE_LOG;
    const bool deg3 = a->sh_degree == 3;
    using B = __nv_bfloat16;
    if (deg3) {
        if (bf16) { if (logt) with_variant<false, B, true, 3>(a, f); else with_variant<false, B, false, 3>(a, f); }
        else { if (logt) with_variant<false, float, true, 3>(a, f); else with_variant<false, float, false, 3>(a, f); }
    } else if (compat) {
        if (bf16) { if (logt) with_variant<true, B, true, 2>(a, f); else with_variant<true, B, false, 2>(a, f); }
        else { if (logt) with_variant<true, float, true, 2>(a, f); else with_variant<true, float, false, 2>(a, f); }
    } else {
        if (bf16) { if (logt) with_variant<false, B, true, 2>(a, f); else with_variant<false, B, false, 2>(a, f); }
        else { if (logt) with_variant<false, float, true, 2>(a, f); else with_variant<false, float, false, 2>(a, f); }
    }
}

// The forward pass scatters nothing: its merged variant is the plain one.
template <int kPass, int kVar>
constexpr int pass_variant() { return kPass == kForward ? (kVar & ~kVarMerge) : kVar; }

// Persistent grid and workspace size for the current device: one block per resident slot
// of the train kernel (the heaviest instantiation, which bounds the others).
struct Layout {
    int error;
    unsigned blocks;
    size_t counter_bytes, train_bytes;
};

struct Occupancy {
    int pass = kTrain;
    int per_sm = 0, train_per_sm = 0;
    size_t chunk_bytes = 0;
    cudaError_t err = cudaSuccess;
    template <bool C, typename S, bool L, int D, int V>
    void run() {
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&train_per_sm, render_kernel<C, S, kTrain, L, D, V>, kThreads,
                                                            0);
        per_sm = train_per_sm;
        if (err == cudaSuccess && pass == kForward)
            err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, render_kernel<C, S, kForward, L, D, pass_variant<kForward, V>()>, kThreads, 0);
        if (err == cudaSuccess && pass == kBackward)
            err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_kernel<C, S, kBackward, L, D, V>,
                                                                kThreads, 0);
        chunk_bytes = chunk_floats<D>() * sizeof(float);
    }
};

// Persistent grid of a pass: as many one-warp blocks as are resident (each pass has its own
// register use, so the forward runs more warps per SM than the train kernel); the train
// pass's stash slots are sized by its own grid.
Layout layout_for(const qsdvr_render_args *a, int pass = kTrain) {
    Layout L{QSDVR_OK, 0, kCounterBytes, 0};
    int dev = 0, sms = 0;
    if (check_cuda(cudaGetDevice(&dev), "render: cudaGetDevice") != QSDVR_OK ||
        check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "render: SM count") != QSDVR_OK) {
        L.error = QSDVR_ERR_CUDA;
        return L;
    }
    Occupancy occ;
    occ.pass = pass;
    dispatch(a, occ);
    if (check_cuda(occ.err, "render: occupancy") != QSDVR_OK) {
        L.error = QSDVR_ERR_CUDA;
        return L;
    }
    L.blocks = (unsigned)(sms * (occ.per_sm > 0 ? occ.per_sm : 1));
    const size_t train_blocks = (size_t)sms * (occ.train_per_sm > 0 ? occ.train_per_sm : 1);
    L.train_bytes = kCounterBytes + train_blocks * kWarpsPerBlock * kSlotChunks * occ.chunk_bytes;
    return L;
}


template <int kPass>
struct Launcher {
    const Params *p;
    unsigned blocks;
    cudaStream_t stream;
    template <bool C, typename S, bool L, int D, int V>
    void run() {
        render_kernel<C, S, kPass, L, D, pass_variant<kPass, V>()><<<blocks, kThreads, 0, stream>>>(*p);
    }
};

template <int kPass>
int launch(const qsdvr_render_args *a, cudaStream_t stream) {
    Params p;
    p.rays = a->rays;
    p.origin = a->origin;
    p.dir = a->dir;
    p.n = a->ray_count;
    p.R = a->reso;
    p.interval = a->interval;
    p.k = a->logistic_coef;
    p.volume_offset = (float)a->reso / 2.0f;
    p.sdf = a->sdf_grid;
    p.sep = reinterpret_cast<const float4 *>(a->sdf_layers);
    p.sep_grad = a->sdf_layers ? reinterpret_cast<float4 *>(a->sdf_layers_grad) : nullptr;
    p.data = a->data;
    p.color = a->color;
    p.target = a->target;
    p.grad_color = a->grad_color;
    p.sdf_grad = a->sdf_grad;
    p.data_grad = a->data_grad;
    p.loss = a->loss;
    p.grad_scale = a->grad_scale;
    p.ray_counter = nullptr;
    p.slots = nullptr;
    p.tlist = a->tlist;
    p.sample_alpha = a->sample_alpha;
    p.sample_capacity = a->sample_capacity;
    p.order = a->order;
    p.grad_bf16 = a->data_grad_storage == QSDVR_STORAGE_BF16;
    unsigned blocks = grid_for(a->ray_count, kWarpsPerBlock);
    if (a->workspace) {
        const Layout L = layout_for(a, kPass);
        if (L.error != QSDVR_OK) return L.error;
        if (a->workspace_bytes < (kPass == kTrain ? L.train_bytes : L.counter_bytes))
            return set_error(QSDVR_ERR_WORKSPACE, "render: workspace %llu < %zu bytes",
                             (unsigned long long)a->workspace_bytes, kPass == kTrain ? L.train_bytes : L.counter_bytes);
        p.ray_counter = static_cast<uint32_t *>(a->workspace);
        if (kPass == kTrain) p.slots = reinterpret_cast<float *>(static_cast<char *>(a->workspace) + kCounterBytes);
        const int st = check_cuda(cudaMemsetAsync(p.ray_counter, 0, sizeof(uint32_t), stream), "render: memset");
        if (st != QSDVR_OK) return st;
        blocks = L.blocks;
    }
    Launcher<kPass> launcher{&p, blocks, stream};
    dispatch(a, launcher);
    return check_launch(kPass == kForward ? "qsdvr_render_forward"
                                          : (kPass == kBackward ? "qsdvr_render_backward" : "qsdvr_render_train"));
}

int validate(const qsdvr_render_args *a, int pass) {
    if (!a) return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: null args");
    const bool sep = a->sdf_layers != nullptr;
    if (a->ray_count && (!a->rays || !a->origin || !a->dir || !(a->sdf_grid || sep) || !a->data))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: null ray or grid pointer");
    if (a->reso == 0 || a->reso > 1290)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: reso %u out of range", a->reso);
    if (a->mode != QSDVR_MODE_COMPAT && a->mode != QSDVR_MODE_FIXED)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: bad mode %d", a->mode);
    if (a->storage != QSDVR_STORAGE_F32 && a->storage != QSDVR_STORAGE_BF16)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: bad storage %d", a->storage);
    if (a->sh_degree != 0 && a->sh_degree != 2 && a->sh_degree != 3)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: sh_degree %d not supported (2 or 3)", a->sh_degree);
    if (a->sh_degree == 3 && a->mode == QSDVR_MODE_COMPAT)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: SH degree 3 exists only in fixed mode");
    if (sep && a->sh_degree == 3)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: the separable SDF renders SH degree 2 only");
    if (sep && a->merge_scatter)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: merge_scatter is not available with sdf_layers");
    if (a->transmittance != QSDVR_TRANSMITTANCE_PRODUCT && a->transmittance != QSDVR_TRANSMITTANCE_LOG)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: bad transmittance form %d", a->transmittance);
    if (!(a->interval > 0.0f)) return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: interval must be > 0");
    if (!aligned(a->sdf_grid, 16) || !aligned(a->sdf_layers, 16) || !aligned(a->data, 16) || !aligned(a->rays, 16))
        return set_error(QSDVR_ERR_ALIGNMENT, "render: rays, SDF and data need 16-byte alignment");
    float *const sdf_g = sep ? a->sdf_layers_grad : a->sdf_grad;
    if (pass != kForward && a->ray_count &&
        (!sdf_g || !a->data_grad || !aligned(sdf_g, 16) || !aligned(a->data_grad, 16)))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: gradient buffers missing or not 16-byte aligned");
    if (pass != kBackward && a->ray_count && !a->color)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: null color output");
    if (pass == kBackward && a->ray_count && !a->grad_color)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: null grad_color");
    if (pass == kTrain && a->ray_count && (!a->target || !a->loss))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: null target or loss");
    if (a->data_grad_storage != QSDVR_STORAGE_F32 && a->data_grad_storage != QSDVR_STORAGE_BF16)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "render: bad data_grad_storage %d", a->data_grad_storage);
    if (a->workspace && !aligned(a->workspace, 256))
        return set_error(QSDVR_ERR_ALIGNMENT, "render: workspace needs 256-byte alignment");
    return QSDVR_OK;
}

}  // namespace
}  // namespace qsdvr

namespace qsdvr {
namespace {

// 10 bits of v spread to every third bit.
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__global__ void __launch_bounds__(256) ray_order_keys_kernel(const qsdvr_ray_info *__restrict__ rays,
                                                             const float *__restrict__ origin,
                                                             const float *__restrict__ dir, uint32_t n,
                                                             float interval, uint32_t *__restrict__ keys) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint32_t ns = rays[r].sdf_count;
    if (ns < 2) {
        keys[r] = 0x7fffffffu;  // after every ray with samples, also as a signed key
        return;
    }
    const float t = 0.5f * (float)(ns - 1) * interval;  // the in-box segment's midpoint
    const f3 o = load3(origin + 3ull * r), d = load3(dir + 3ull * r);
    const float c[3] = {fmaf(d.x, t, o.x), fmaf(d.y, t, o.y), fmaf(d.z, t, o.z)};
    uint32_t q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) q[a] = (uint32_t)fminf(fmaxf((c[a] + 1.0f) * 512.0f, 0.0f), 1023.0f);
    keys[r] = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
}

// Ray order by counting sort: the 15-bit Morton code of each ray's in-box midpoint (5 bits
// per axis, a 32^3 lattice of the volume; rays without samples in one extra last bucket),
// a histogram, its exclusive scan, and a scatter that lists each bucket's rays in the order
// the scatter reaches them.  Rays in one bucket lie within one 1/16-wide cube of the volume,
// the locality the render kernels need; finer keys order rays within such a cube, which does
// not change what the rays in flight share.
constexpr uint32_t kOrderBuckets = (1u << 15) + 1;

// With a sample list (list mode) the key point is each ray's median SDF position instead: the
// fine samples gather where the compositing weights are, so rays keyed there run beside the
// rays that hit the same patch of the surface and share its vertex rows and gradient lines.
__device__ __forceinline__ uint32_t ray_bucket(const qsdvr_ray_info *rays, const float *origin, const float *dir,
                                               uint32_t r, uint32_t n, float interval, const float *tlist) {
    const uint32_t ns = rays[r].sdf_count;
    if (ns < 2) return kOrderBuckets - 1;
    const float t = tlist ? *QSDVR_AT(tlist, (uint64_t)kListT * r + kListT / 2, 1, (uint64_t)kListT * n)
                          : 0.5f * (float)(ns - 1) * interval;
    const f3 o = load3(origin + 3ull * r), d = load3(dir + 3ull * r);
    const float c[3] = {fmaf(d.x, t, o.x), fmaf(d.y, t, o.y), fmaf(d.z, t, o.z)};
    uint32_t q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) q[a] = (uint32_t)fminf(fmaxf((c[a] + 1.0f) * 16.0f, 0.0f), 31.0f);
    return spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
}

__global__ void __launch_bounds__(256) ray_bucket_kernel(const qsdvr_ray_info *__restrict__ rays,
                                                         const float *__restrict__ origin,
                                                         const float *__restrict__ dir, uint32_t n, float interval,
                                                         const float *__restrict__ tlist, uint32_t *__restrict__ bucket,
                                                         uint32_t *__restrict__ hist) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint32_t b = ray_bucket(rays, origin, dir, r, n, interval, tlist);
    bucket[r] = b;
    atomicAdd(hist + b, 1u);
}

// Exclusive scan of the kOrderBuckets counts in place, one block of 1024 threads.  Each
// thread scans kPer consecutive counts; they pass through shared memory so that the global
// loads and stores are coalesced (thread t's run read straight from global memory touched a
// different sector per thread and step), and the stride-kPer shared accesses (kPer odd) fall
// in distinct banks.
constexpr uint32_t kScanPer = (kOrderBuckets + 1023) / 1024;
constexpr size_t kScanSmem = (size_t)kScanPer * 1024 * sizeof(uint32_t);
__global__ void __launch_bounds__(1024) bucket_scan_kernel(uint32_t *__restrict__ hist) {
    constexpr uint32_t kPer = kScanPer;
    static_assert(kPer % 2 == 1, "an odd run length keeps the shared accesses conflict-free");
    extern __shared__ uint32_t counts[];  // kPer * 1024
    __shared__ uint32_t warp_sums[32];
    const uint32_t t = threadIdx.x, lane = t & 31, w = t >> 5;
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
        const uint32_t i = k * 1024 + t;
        counts[i] = i < kOrderBuckets ? hist[i] : 0u;
    }
    __syncthreads();
    uint32_t v[kPer], sum = 0;
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
        v[k] = counts[t * kPer + k];
        sum += v[k];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t x = __shfl_up_sync(kFull, incl, o);
        if ((int)lane >= o) incl += x;
    }
    if (lane == 31) warp_sums[w] = incl;
    __syncthreads();
    if (w == 0) {
        uint32_t ws = warp_sums[lane], wi = ws;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t x = __shfl_up_sync(kFull, wi, o);
            if ((int)lane >= o) wi += x;
        }
        warp_sums[lane] = wi - ws;  // exclusive prefix of the warps
    }
    __syncthreads();
    uint32_t run = warp_sums[w] + incl - sum;
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
        counts[t * kPer + k] = run;
        run += v[k];
    }
    __syncthreads();
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
        const uint32_t i = k * 1024 + t;
        if (i < kOrderBuckets) hist[i] = counts[i];
    }
}

__global__ void __launch_bounds__(256) ray_scatter_kernel(const uint32_t *__restrict__ bucket, uint32_t n,
                                                          uint32_t *__restrict__ next, uint32_t *__restrict__ order) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint32_t pos = atomicAdd(next + bucket[r], 1u);
    if (pos < n) order[pos] = r;
    else flag_error(QSDVR_DEVERR_CAPACITY);
}

// Positive control of the bounds-checked build: element kBoundsProbe of a buffer declared to
// hold kBoundsDeclared elements, which physically holds kBoundsHeld, so the write is in
// bounds whether or not the check redirects it.
constexpr uint32_t kBoundsDeclared = 32, kBoundsProbe = 40, kBoundsHeld = 64;
static_assert(kBoundsDeclared <= kBoundsProbe && kBoundsProbe < kBoundsHeld, "probe inside the held buffer");

__global__ void bounds_check_kernel(float *buf) {
    *QSDVR_AT(buf, kBoundsProbe, 1, kBoundsDeclared) = 1.0f;
}

}  // namespace
}  // namespace qsdvr

using namespace qsdvr;

extern "C" int qsdvr_ray_order_keys(const qsdvr_ray_info *rays, const float *origin, const float *dir,
                                    uint32_t ray_count, float interval, uint32_t *keys, cudaStream_t stream) {
    if (ray_count == 0) return QSDVR_OK;
    if (!rays || !origin || !dir || !keys)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_ray_order_keys: null pointer");
    if (!(interval > 0.0f)) return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_ray_order_keys: interval must be > 0");
    ray_order_keys_kernel<<<grid_for(ray_count, 256), 256, 0, stream>>>(rays, origin, dir, ray_count, interval, keys);
    return check_launch("qsdvr_ray_order_keys");
}

extern "C" size_t qsdvr_ray_order_workspace_size(uint32_t ray_count) {
    return ((size_t)kOrderBuckets + (size_t)ray_count) * sizeof(uint32_t);
}

namespace qsdvr {
namespace {
int ray_order(const char *fn, const qsdvr_ray_info *rays, const float *origin, const float *dir, uint32_t ray_count,
              float interval, const float *tlist, uint32_t *order, void *workspace, size_t workspace_bytes,
              cudaStream_t stream) {
    if (ray_count == 0) return QSDVR_OK;
    if (!rays || !origin || !dir || !order) return set_error(QSDVR_ERR_INVALID_ARGUMENT, "%s: null pointer", fn);
    if (!tlist && !(interval > 0.0f)) return set_error(QSDVR_ERR_INVALID_ARGUMENT, "%s: interval must be > 0", fn);
    const size_t need = qsdvr_ray_order_workspace_size(ray_count);
    if (!workspace || workspace_bytes < need || !aligned(workspace, 4))
        return set_error(QSDVR_ERR_WORKSPACE, "%s: workspace %zu < %zu bytes (4-byte aligned)", fn, workspace_bytes,
                         need);
    uint32_t *hist = static_cast<uint32_t *>(workspace), *bucket = hist + kOrderBuckets;
    const int st = check_cuda(cudaMemsetAsync(hist, 0, kOrderBuckets * sizeof(uint32_t), stream), fn);
    if (st != QSDVR_OK) return st;
    // (the scan's shared memory is above the default 48 KB; the attribute is set on the
    // current device at every call: it is a host-side setting, not a stream operation)
    const int sa = check_cuda(
        cudaFuncSetAttribute(bucket_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kScanSmem), fn);
    if (sa != QSDVR_OK) return sa;
    const unsigned blocks = grid_for(ray_count, 256);
    ray_bucket_kernel<<<blocks, 256, 0, stream>>>(rays, origin, dir, ray_count, interval, tlist, bucket, hist);
    bucket_scan_kernel<<<1, 1024, kScanSmem, stream>>>(hist);
    ray_scatter_kernel<<<blocks, 256, 0, stream>>>(bucket, ray_count, hist, order);
    return check_launch(fn);
}
}  // namespace
}  // namespace qsdvr

extern "C" int qsdvr_ray_order(const qsdvr_ray_info *rays, const float *origin, const float *dir, uint32_t ray_count,
                               float interval, uint32_t *order, void *workspace, size_t workspace_bytes,
                               cudaStream_t stream) {
    return qsdvr::ray_order("qsdvr_ray_order", rays, origin, dir, ray_count, interval, nullptr, order, workspace,
                            workspace_bytes, stream);
}

extern "C" int qsdvr_ray_order_list(const qsdvr_ray_info *rays, const float *origin, const float *dir,
                                    uint32_t ray_count, const float *tlist, uint32_t *order, void *workspace,
                                    size_t workspace_bytes, cudaStream_t stream) {
    if (ray_count && !tlist) return qsdvr::set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_ray_order_list: null tlist");
    return qsdvr::ray_order("qsdvr_ray_order_list", rays, origin, dir, ray_count, 0.0f, tlist, order, workspace,
                            workspace_bytes, stream);
}

namespace {

using TensorMapEncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                            const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                            CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                            CUtensorMapFloatOOBfill);

TensorMapEncodeTiledFn tensor_map_encoder(int *status) {
    static TensorMapEncodeTiledFn fn = nullptr;
    static std::once_flag once;
    static cudaError_t err = cudaSuccess;
    static cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    std::call_once(once, [] {
        void *f = nullptr;
        err = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q);
        if (err == cudaSuccess && q == cudaDriverEntryPointSuccess) fn = reinterpret_cast<TensorMapEncodeTiledFn>(f);
    });
    *status = err != cudaSuccess ? check_cuda(err, "render bricks: cudaGetDriverEntryPoint")
                                 : (fn ? QSDVR_OK : set_error(QSDVR_ERR_UNSUPPORTED, "render bricks: no cuTensorMapEncodeTiled"));
    return fn;
}

template <typename S, int kDeg>
int launch_bricks(const qsdvr_render_args *a, cudaStream_t stream) {
    constexpr int kC = ShLayout<kDeg>::kChannels;
    int st = QSDVR_OK;
    TensorMapEncodeTiledFn encode = tensor_map_encoder(&st);
    if (st != QSDVR_OK) return st;
    const cuuint64_t R1 = a->reso + 1ull;
    const cuuint64_t dims[4] = {(cuuint64_t)kC, R1, R1, R1};
    const cuuint64_t strides[3] = {128ull, 128ull * R1, 128ull * R1 * R1};  // bytes, dims 1..3
    const cuuint32_t box[4] = {(cuuint32_t)kC, kBrick, kBrick, kBrick};
    const cuuint32_t estride[4] = {1, 1, 1, 1};
    CUtensorMap tmap;
    const CUresult cr = encode(&tmap, sizeof(S) == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                               4, const_cast<void *>(a->data), dims, strides, box, estride,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return set_error(QSDVR_ERR_CUDA, "render bricks: cuTensorMapEncodeTiled failed (%d)", (int)cr);
    Params p{};
    p.rays = a->rays;
    p.origin = a->origin;
    p.dir = a->dir;
    p.n = a->ray_count;
    p.R = a->reso;
    p.interval = a->interval;
    p.k = a->logistic_coef;
    p.volume_offset = (float)a->reso / 2.0f;
    p.sdf = a->sdf_grid;
    p.data = a->data;
    p.color = a->color;
    const size_t smem = (size_t)kBrick * kBrick * kBrick * 128 + (size_t)kBrickThreads * (kC + 1) * sizeof(float) + 128;
    st = check_cuda(cudaFuncSetAttribute(brick_frame_kernel<S, kDeg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem),
                    "render bricks: shared memory");
    if (st != QSDVR_OK) return st;
    brick_frame_kernel<S, kDeg><<<grid_for(a->ray_count, kBrickThreads), kBrickThreads, smem, stream>>>(tmap, p);
    return check_launch("qsdvr_render_forward_bricks");
}

}  // namespace

extern "C" int qsdvr_render_forward_bricks(const qsdvr_render_args *args, cudaStream_t stream) {
    int st = validate(args, kForward);
    if (st != QSDVR_OK || args->ray_count == 0) return st;
    if (args->mode != QSDVR_MODE_FIXED || args->tlist || args->sdf_layers || args->sample_alpha)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT,
                         "qsdvr_render_forward_bricks: fixed mode, uniform march and a dense SDF grid only");
    if (args->transmittance != QSDVR_TRANSMITTANCE_LOG)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_render_forward_bricks: log transmittance only");
    const bool bf16 = args->storage == QSDVR_STORAGE_BF16;
    const int deg = args->sh_degree == 3 ? 3 : 2;
    if (bf16 && deg == 3) return launch_bricks<__nv_bfloat16, 3>(args, stream);
    if (!bf16 && deg == 2) return launch_bricks<float, 2>(args, stream);
    return set_error(QSDVR_ERR_INVALID_ARGUMENT,
                     "qsdvr_render_forward_bricks: 128-byte vertex rows only (bf16 SH degree 3 or fp32 degree 2)");
}

extern "C" int qsdvr_check_bounds(float *buffer, cudaStream_t stream) {
    if (!buffer) return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_check_bounds: null buffer");
    bounds_check_kernel<<<1, 1, 0, stream>>>(buffer);
    return check_launch("qsdvr_check_bounds");
}

extern "C" size_t qsdvr_render_workspace_size(const qsdvr_render_args *args) {
    if (!args) return 0;
    const Layout L = layout_for(args);
    return L.error == QSDVR_OK ? L.train_bytes : 0;
}

extern "C" int qsdvr_render_forward(const qsdvr_render_args *args, cudaStream_t stream) {
    const int st = validate(args, kForward);
    if (st != QSDVR_OK || args->ray_count == 0) return st;
    return launch<kForward>(args, stream);
}

extern "C" int qsdvr_render_backward(const qsdvr_render_args *args, cudaStream_t stream) {
    const int st = validate(args, kBackward);
    if (st != QSDVR_OK || args->ray_count == 0) return st;
    return launch<kBackward>(args, stream);
}

extern "C" int qsdvr_render_train(const qsdvr_render_args *args, cudaStream_t stream) {
    const int st = validate(args, kTrain);
    if (st != QSDVR_OK || args->ray_count == 0) return st;
    return launch<kTrain>(args, stream);
}
