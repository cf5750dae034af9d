// Ray generation: RayCut (per-pixel ray + in-box sample count + masked exclusive scan, all
// on the device) and GenerateRayPoints (per-sample local coordinates and cell index).
//
// Counts and cell indices are bit-exact with the reference (kernel/camera.cu): every float
// operation uses an explicit round-to-nearest intrinsic in the fused/unfused form the
// reference's nvcc build (default --fmad=true) evaluates, so no compiler contraction
// choice can change a count or an index.
#include <cuda.h>  // CUcontext / CUresult types only; the driver is reached via cudaGetDriverEntryPoint

#include <mutex>

#include "common.cuh"
#include "raygen.cuh"

namespace qsdvr {

QSDVR_ERROR_WORD_ACCESSOR(camera)

namespace {

constexpr int kScanBlock = 256;
constexpr uint32_t kMaxMarchSteps = 1u << 20;  // samples per ray considered by RayCut

// kernel/camera.cu:3-10 (TransCameraToWorld).
__device__ __forceinline__ f3 camera_to_world(const qsdvr_camera &c, float px, float py, float z) {
    const float x = __fmul_rn(__fdiv_rn(__fadd_rn(px, c.cx), c.fx), z);
    const float y = __fmul_rn(__fdiv_rn(__fadd_rn(py, c.cy), c.fy), z);
    const float *r = c.rotation;
    f3 w;
    w.x = __fadd_rn(__fmaf_rn(r[2], z, __fmaf_rn(r[0], x, __fmul_rn(r[1], y))), c.translation[0]);
    w.y = __fadd_rn(__fmaf_rn(r[5], z, __fmaf_rn(r[3], x, __fmul_rn(r[4], y))), c.translation[1]);
    w.z = __fadd_rn(__fmaf_rn(r[8], z, __fmaf_rn(r[6], x, __fmul_rn(r[7], y))), c.translation[2]);
    return w;
}

__device__ __forceinline__ bool in_box(float x, float y, float z) {
    return x < 0.9999f && x > -0.9999f && y < 0.9999f && y > -0.9999f && z < 0.9999f && z > -0.9999f;
}

// Masked (sdf, render) contribution of a pixel with raw in-box count c (kernel/camera.cu:115-126).
__device__ __forceinline__ uint2 masked_counts(uint32_t c, bool m) {
    if (!m || c < 2) return make_uint2(0, 0);
    return make_uint2(c, c - 1);
}

__device__ __forceinline__ uint2 add2(uint2 a, uint2 b) { return make_uint2(a.x + b.x, a.y + b.y); }

// Exclusive scan of a uint2 across a kBlock-thread block; *total gets the block sum.
template <int kBlock>
__device__ __forceinline__ uint2 block_exclusive_scan(uint2 v, uint2 *total) {
    constexpr int kWarps = kBlock / kWarp;
    __shared__ uint2 warp_base[kWarps];
    __shared__ uint2 block_total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint2 inc = v;
#pragma unroll
    for (int off = 1; off < kWarp; off <<= 1) {
        uint2 n;
        n.x = __shfl_up_sync(kFull, inc.x, off);
        n.y = __shfl_up_sync(kFull, inc.y, off);
        if (lane >= off) inc = add2(inc, n);
    }
    if (lane == kWarp - 1) warp_base[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint2 w = lane < kWarps ? warp_base[lane] : make_uint2(0, 0);
        uint2 wi = w;
#pragma unroll
        for (int off = 1; off < kWarp; off <<= 1) {
            uint2 n;
            n.x = __shfl_up_sync(kFull, wi.x, off);
            n.y = __shfl_up_sync(kFull, wi.y, off);
            if (lane >= off) wi = add2(wi, n);
        }
        if (lane < kWarps) warp_base[lane] = make_uint2(wi.x - w.x, wi.y - w.y);
        if (lane == kWarps - 1) block_total = wi;
    }
    __syncthreads();
    const uint2 base = warp_base[warp];
    if (total) *total = block_total;
    __syncthreads();  // the shared arrays may be reused by the next call
    return make_uint2(base.x + inc.x - v.x, base.y + inc.y - v.y);
}

// Phase 1 — kernel/camera.cu:12-58: one thread per pixel.  Writes dir, first in-box point
// and the raw count (sdf_count), then the block's masked sums for the scan.
__global__ void __launch_bounds__(kScanBlock) ray_cut_kernel(qsdvr_camera cam, float interval,
                                                             uint32_t pixel_count, const uint8_t *__restrict__ mask,
                                                             qsdvr_ray_info *__restrict__ rays,
                                                             float *__restrict__ origin, float *__restrict__ dir,
                                                             uint2 *__restrict__ block_sums) {
    const uint32_t id = blockIdx.x * kScanBlock + threadIdx.x;
    uint2 contrib = make_uint2(0, 0);
    if (id < pixel_count) {
        const float px = __fadd_rn((float)(id % cam.width), 0.5f);
        const float py = __fadd_rn((float)(id / cam.width), 0.5f);
        const f3 n = camera_to_world(cam, px, py, cam.near_depth);
        const f3 f = camera_to_world(cam, px, py, cam.far_depth);
        f3 d{__fsub_rn(f.x, n.x), __fsub_rn(f.y, n.y), __fsub_rn(f.z, n.z)};
        const float nrm = __fsqrt_rn(__fmaf_rn(d.z, d.z, __fmaf_rn(d.x, d.x, __fmul_rn(d.y, d.y))));
        d.x = __fdiv_rn(d.x, nrm);
        d.y = __fdiv_rn(d.y, nrm);
        d.z = __fdiv_rn(d.z, nrm);
        float end;
        if (d.x != 0.0f)
            end = __fdiv_rn(__fsub_rn(f.x, n.x), d.x);
        else if (d.y != 0.0f)
            end = __fdiv_rn(__fsub_rn(f.y, n.y), d.y);
        else
            end = __fdiv_rn(__fsub_rn(f.z, n.z), d.z);
        // float -> unsigned truncation (cvt.rzi.u32 saturates: negative/NaN give 0).
        uint32_t steps = __float2uint_rz(__fdiv_rn(end, interval));
        if (steps > kMaxMarchSteps) {  // a degenerate interval: flag the ray instead of marching for ever
            flag_error(QSDVR_DEVERR_RAY);
            steps = 0;
        }
        // The in-box samples form one contiguous run of j (each coordinate is monotone in
        // j), so the march stops at the first sample that leaves the box after entering.
        uint32_t hits = 0;
        f3 first{0.0f, 0.0f, 0.0f};
        for (uint32_t j = 0; j < steps; ++j) {
            const f3 p = march(n, d, (float)j, interval);
            if (in_box(p.x, p.y, p.z)) {
                if (hits == 0) first = p;
                ++hits;
            } else if (hits) {
                break;
            }
        }
        store3(dir + 3ull * id, d);
        store3(origin + 3ull * id, first);
        rays[id].sdf_count = hits;
        contrib = masked_counts(hits, mask[id] != 0);
    }
    uint2 tot;
    block_exclusive_scan<kScanBlock>(contrib, &tot);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

// Phase 2 — exclusive scan of the per-block sums (one block, loops with a carry).
__global__ void __launch_bounds__(1024) scan_block_sums_kernel(uint2 *__restrict__ sums, uint32_t n,
                                                               uint32_t *__restrict__ totals) {
    __shared__ uint2 carry;
    if (threadIdx.x == 0) carry = make_uint2(0, 0);
    __syncthreads();
    for (uint32_t base = 0; base < n; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint2 v = i < n ? sums[i] : make_uint2(0, 0);
        uint2 tot;
        const uint2 ex = block_exclusive_scan<1024>(v, &tot);
        const uint2 c = carry;
        if (i < n) sums[i] = add2(ex, c);
        __syncthreads();
        if (threadIdx.x == 0) carry = add2(c, tot);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        totals[0] = carry.x;
        totals[1] = carry.y;
    }
}

// Phase 3 — kernel/camera.cu:113-127: masked pixels get counts (<2 zeroed) and offsets.
__global__ void __launch_bounds__(kScanBlock) ray_cut_apply_kernel(uint32_t pixel_count,
                                                                   const uint8_t *__restrict__ mask,
                                                                   qsdvr_ray_info *__restrict__ rays,
                                                                   const uint2 *__restrict__ block_offsets) {
    const uint32_t id = blockIdx.x * kScanBlock + threadIdx.x;
    const bool live = id < pixel_count;
    const bool m = live && mask[id] != 0;
    const uint32_t raw = live ? rays[id].sdf_count : 0u;
    const uint2 c = masked_counts(raw, m);
    const uint2 ex = block_exclusive_scan<kScanBlock>(c, nullptr);
    if (m) {
        const uint2 base = block_offsets[blockIdx.x];
        qsdvr_ray_info r;
        r.sdf_count = c.x;
        r.sdf_offset = base.x + ex.x;
        r.render_count = c.y;
        r.render_offset = base.y + ex.y;
        rays[id] = r;
    }
}

// kernel/camera.cu:60-96 — one warp per ray, lanes stride over the ray's samples so the
// sample lists are written contiguously.
__global__ void __launch_bounds__(256) generate_points_kernel(
    const qsdvr_ray_info *__restrict__ rays, const float *__restrict__ origin, const float *__restrict__ dir,
    uint32_t ray_count, float interval, uint32_t reso, float volume_offset, float *__restrict__ sdf_points,
    int32_t *__restrict__ sdf_index, float *__restrict__ render_points, int32_t *__restrict__ render_index,
    float *__restrict__ view_dir, uint64_t sdf_cap, uint64_t render_cap) {
    const uint64_t w = (blockIdx.x * 256ull + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= ray_count) return;
    const qsdvr_ray_info info = rays[w];
    const f3 o = load3(origin + 3 * w);
    const f3 d = load3(dir + 3 * w);
    if ((uint64_t)info.sdf_offset + info.sdf_count > sdf_cap ||
        (uint64_t)info.render_offset + info.render_count > render_cap) {
        if (lane == 0) flag_error(QSDVR_DEVERR_CAPACITY);
        return;
    }
    for (uint32_t j = lane; j < info.sdf_count; j += kWarp) {
        const uint64_t s = (uint64_t)info.sdf_offset + j;
        const CellPoint c = to_cell(march(o, d, (float)j, interval), volume_offset, reso);
        store3(QSDVR_AT(sdf_points, 3 * s, 3, 3 * sdf_cap), c.u);
        *QSDVR_AT(sdf_index, s, 1, sdf_cap) = c.index;
    }
    for (uint32_t j = lane; j < info.render_count; j += kWarp) {
        const uint64_t s = (uint64_t)info.render_offset + j;
        const CellPoint c = to_cell(midpoint(o, d, j, interval), volume_offset, reso);
        store3(QSDVR_AT(render_points, 3 * s, 3, 3 * render_cap), c.u);
        *QSDVR_AT(render_index, s, 1, render_cap) = c.index;
        store3(QSDVR_AT(view_dir, 3 * s, 3, 3 * render_cap), d);
    }
}

}  // namespace
}  // namespace qsdvr

using namespace qsdvr;

extern "C" size_t qsdvr_ray_cut_workspace_size(uint32_t pixel_count) {
    const size_t blocks = (pixel_count + kScanBlock - 1) / kScanBlock;
    return (blocks == 0 ? 1 : blocks) * sizeof(uint2);
}

extern "C" int qsdvr_ray_cut(const qsdvr_camera *camera, const uint8_t *mask, qsdvr_ray_info *rays, float *origin,
                             float *dir, float interval, uint32_t pixel_count, uint32_t *totals, void *workspace,
                             size_t workspace_bytes, cudaStream_t stream) {
    if (!camera || !mask || !rays || !origin || !dir || !totals)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_ray_cut: null pointer");
    if (camera->width == 0 || (uint64_t)camera->width * camera->height < pixel_count)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_ray_cut: pixel_count %u exceeds %u x %u", pixel_count,
                         camera->width, camera->height);
    if (!(interval > 0.0f))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_ray_cut: interval must be > 0");
    if (!aligned(rays, 16) || !aligned(workspace, 8))
        return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_ray_cut: rays need 16-byte, workspace 8-byte alignment");
    const size_t need = qsdvr_ray_cut_workspace_size(pixel_count);
    if (!workspace || workspace_bytes < need)
        return set_error(QSDVR_ERR_WORKSPACE, "qsdvr_ray_cut: workspace %zu < %zu bytes", workspace_bytes, need);
    if (pixel_count == 0) return check_cuda(cudaMemsetAsync(totals, 0, 2 * sizeof(uint32_t), stream), "memset");
    const uint32_t blocks = (pixel_count + kScanBlock - 1) / kScanBlock;
    uint2 *sums = static_cast<uint2 *>(workspace);
    ray_cut_kernel<<<blocks, kScanBlock, 0, stream>>>(*camera, interval, pixel_count, mask, rays, origin, dir, sums);
    scan_block_sums_kernel<<<1, 1024, 0, stream>>>(sums, blocks, totals);
    ray_cut_apply_kernel<<<blocks, kScanBlock, 0, stream>>>(pixel_count, mask, rays, sums);
    return check_launch("qsdvr_ray_cut");
}

extern "C" int qsdvr_generate_ray_points(const qsdvr_ray_info *rays, const float *origin, const float *dir,
                                         uint32_t ray_count, float interval, uint32_t base_volume_reso,
                                         float *sdf_points, int32_t *sdf_index, float *render_points,
                                         int32_t *render_index, float *view_dir, uint64_t sdf_capacity,
                                         uint64_t render_capacity, cudaStream_t stream) {
    if (ray_count == 0) return QSDVR_OK;
    if (!rays || !origin || !dir || (sdf_capacity && (!sdf_points || !sdf_index)) ||
        (render_capacity && (!render_points || !render_index || !view_dir)))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_generate_ray_points: null pointer");
    if (base_volume_reso == 0 || base_volume_reso > 1290)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_generate_ray_points: reso %u out of range",
                         base_volume_reso);
    const float volume_offset = (float)base_volume_reso / 2.0f;
    generate_points_kernel<<<grid_for((uint64_t)ray_count * kWarp, 256), 256, 0, stream>>>(
        rays, origin, dir, ray_count, interval, base_volume_reso, volume_offset, sdf_points, sdf_index,
        render_points, render_index, view_dir, sdf_capacity, render_capacity);
    return check_launch("qsdvr_generate_ray_points");
}

// ---- RayCut without any allocation -------------------------------------------------------
// Some callers cannot allocate device memory at all: an application whose device memory is
// owned up front by its own pool or arena (a cudaMalloc would fail or fragment it), or a host
// that hands a plugin only the buffers of its inputs and outputs.  Such a caller has no way to
// provide the workspace qsdvr_ray_cut asks for, so this variant keeps the scan's per-block
// sums in a fixed array in the library's device image instead.  Every GPU that loads the
// library holds the array (128 KiB) until the process exits.
namespace {

constexpr uint32_t kStaticScanBlocks = QSDVR_RAY_CUT_NOALLOC_MAX_PIXELS / kScanBlock;
static_assert(QSDVR_RAY_CUT_NOALLOC_MAX_PIXELS % kScanBlock == 0, "limit must be whole scan blocks");

// One slot per scan block.  Every call overwrites each slot it uses before reading it, so no
// slot has to start at zero; calls that overlap on the GPU share the array and race.
static __device__ __align__(256) uint2 g_ray_cut_scratch[kStaticScanBlocks];

// Device address of g_ray_cut_scratch per CUDA context.  In host code the symbol name is
// only a host-side stand-in; the array's device address belongs to the context that loaded
// the module, so it is looked up (cudaGetSymbolAddress) once per context, with that context
// current, and cached under the context's ID.  A context ID is never reused within a
// process: a context created after a device reset, or a host's own driver-API context on
// the same device, gets its own lookup.  The driver's context queries are reached through
// cudaGetDriverEntryPoint, so the library does not link libcuda.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

struct ScratchSlot {
    unsigned long long ctx_id;
    uint2 *addr;
};
constexpr int kScratchSlots = 64;
std::mutex g_scratch_mutex;
ScratchSlot g_scratch_slots[kScratchSlots] = {};
int g_scratch_used = 0, g_scratch_next = 0;

int current_context_id(unsigned long long *id, bool *have) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    static cudaError_t resolved = cudaSuccess;
    std::call_once(once, [] {
        void *f = nullptr, *g = nullptr;
        cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
        resolved = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q1);
        if (resolved == cudaSuccess) resolved = cudaGetDriverEntryPoint("cuCtxGetId", &g, cudaEnableDefault, &q2);
        if (resolved == cudaSuccess && q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
            get_id = reinterpret_cast<CtxGetIdFn>(g);
        }
    });
    if (resolved != cudaSuccess) return check_cuda(resolved, "qsdvr_ray_cut_noalloc: cudaGetDriverEntryPoint");
    if (!get_current || !get_id)
        return set_error(QSDVR_ERR_UNSUPPORTED, "qsdvr_ray_cut_noalloc: the driver lacks cuCtxGetCurrent/cuCtxGetId");
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS)
        return set_error(QSDVR_ERR_CUDA, "qsdvr_ray_cut_noalloc: cuCtxGetCurrent failed");
    *have = ctx != nullptr;
    if (ctx && get_id(ctx, id) != CUDA_SUCCESS)
        return set_error(QSDVR_ERR_CUDA, "qsdvr_ray_cut_noalloc: cuCtxGetId failed");
    return QSDVR_OK;
}

int scratch_address(uint2 **out) {
    unsigned long long id = 0;
    bool have = false;
    int st = current_context_id(&id, &have);
    if (st != QSDVR_OK) return st;
    if (have) {
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        for (int i = 0; i < g_scratch_used; ++i)
            if (g_scratch_slots[i].ctx_id == id) {
                *out = g_scratch_slots[i].addr;
                return QSDVR_OK;
            }
    }
    // First call in this context (or no context yet: the lookup makes the device's primary
    // context current, and its ID is read afterwards).
    void *addr = nullptr;
    st = check_cuda(cudaGetSymbolAddress(&addr, g_ray_cut_scratch), "qsdvr_ray_cut_noalloc: cudaGetSymbolAddress");
    if (st != QSDVR_OK) return st;
    if (!have) {
        st = current_context_id(&id, &have);
        if (st != QSDVR_OK) return st;
    }
    if (have) {
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        const int slot = g_scratch_used < kScratchSlots ? g_scratch_used++ : (g_scratch_next++ % kScratchSlots);
        g_scratch_slots[slot] = ScratchSlot{id, static_cast<uint2 *>(addr)};
    }
    *out = static_cast<uint2 *>(addr);
    return QSDVR_OK;
}

}  // namespace

extern "C" int qsdvr_ray_cut_noalloc(const qsdvr_camera *camera, const uint8_t *mask, qsdvr_ray_info *rays,
                                     float *origin, float *dir, float interval, uint32_t pixel_count, uint32_t *totals,
                                     cudaStream_t stream) {
    if (!camera || !mask || !rays || !origin || !dir || !totals)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_ray_cut_noalloc: null pointer");
    if (pixel_count > QSDVR_RAY_CUT_NOALLOC_MAX_PIXELS)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT,
                         "qsdvr_ray_cut_noalloc: pixel_count %u exceeds the fixed scratch limit of %u pixels; "
                         "use qsdvr_ray_cut with a caller workspace",
                         pixel_count, (unsigned)QSDVR_RAY_CUT_NOALLOC_MAX_PIXELS);
    if (camera->width == 0 || (uint64_t)camera->width * camera->height < pixel_count)
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_ray_cut_noalloc: pixel_count %u exceeds %u x %u",
                         pixel_count, camera->width, camera->height);
    if (!(interval > 0.0f))
        return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_ray_cut_noalloc: interval must be > 0");
    if (!aligned(rays, 16))
        return set_error(QSDVR_ERR_ALIGNMENT, "qsdvr_ray_cut_noalloc: rays need 16-byte alignment");
    uint2 *sums = nullptr;
    int st = scratch_address(&sums);
    if (st != QSDVR_OK) return st;
    if (pixel_count == 0)
        return check_cuda(cudaMemsetAsync(totals, 0, 2 * sizeof(uint32_t), stream), "qsdvr_ray_cut_noalloc: memset");
    const uint32_t blocks = (pixel_count + kScanBlock - 1) / kScanBlock;
    ray_cut_kernel<<<blocks, kScanBlock, 0, stream>>>(*camera, interval, pixel_count, mask, rays, origin, dir, sums);
    scan_block_sums_kernel<<<1, 1024, 0, stream>>>(sums, blocks, totals);
    ray_cut_apply_kernel<<<blocks, kScanBlock, 0, stream>>>(pixel_count, mask, rays, sums);
    return check_launch("qsdvr_ray_cut_noalloc");
}
