/*
 * qsdvr_b200 — C ABI of the B200-native QSDVR render path.
 *
 * Every entry point takes plain device pointers, element counts and the caller's CUDA
 * stream, returns a status code (QSDVR_OK on success) and never allocates: scratch
 * space is passed in by the caller (query its size with the *_workspace_size
 * functions).  Gradient buffers that receive atomic accumulation must be zeroed by the
 * caller, as in the reference.  Kernels check every grid / sample index they derive
 * from caller data and skip out-of-range accesses, recording the fact in a device
 * error word (qsdvr_device_error).
 *
 * Reference interface replaced by each entry point (paths within the reference project):
 *   qsdvr pybind module kernel/qsdvr.cpp:5-50, host wrappers in kernel/camera.cu,
 *   kernel/surface.cu, kernel/render.cu, declarations include/camera.h:57-59,
 *   include/surface.h:4-14, include/render.h:4-14.
 */
#ifndef QSDVR_B200_H
#define QSDVR_B200_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status ---------------------------------------------------------------------- */
enum {
    QSDVR_OK = 0,
    QSDVR_ERR_INVALID_ARGUMENT = 1, /* null pointer, zero/oversized extent, bad mode  */
    QSDVR_ERR_ALIGNMENT = 2,        /* pointer not aligned as the layout requires     */
    QSDVR_ERR_WORKSPACE = 3,        /* caller workspace too small                      */
    QSDVR_ERR_CUDA = 4,             /* a CUDA runtime call or launch failed            */
    QSDVR_ERR_UNSUPPORTED = 5       /* valid request this build does not implement     */
};

/* Bits of the device error word. */
enum {
    QSDVR_DEVERR_INDEX = 1u,        /* a cell / vertex index outside the grid         */
    QSDVR_DEVERR_CAPACITY = 2u,     /* a ray's samples run past the sample buffers     */
    QSDVR_DEVERR_RAY = 4u,          /* a ray record is inconsistent (count 1, overflow) */
    QSDVR_DEVERR_TIMEOUT = 8u,      /* a bounded wait on the tensor cores gave up       */
    QSDVR_DEVERR_BOUNDS = 16u       /* bounds-checked build only: an access outside its
                                       buffer was caught and redirected                 */
};

/* Shading / indexing modes.  In the fused renderer, fixed mode also computes alpha and its
 * derivatives in an overflow-free form (softplus of -k sdf) and treats an SDF sample where
 * the cell's quadric is degenerate (|grad f|^2 < 1e-30 or |sdf| > 4) as empty. */
enum {
    QSDVR_MODE_COMPAT = 0, /* the reference exactly: overlapping SH reads, sheared vertex index */
    QSDVR_MODE_FIXED = 1   /* packed SH layout, vertex index x + y(R+1) + z(R+1)^2             */
};

/* Message for the last non-OK status returned on this host thread. */
const char *qsdvr_last_error(void);
/* ABI version (major * 100 + minor). */
int qsdvr_version(void);
/* Read (and clear when clear != 0) the device error word of the current device. */
int qsdvr_device_error(uint32_t *word, int clear, cudaStream_t stream);

/* Bounds-checked build (libqsdvr_b200_debug.so, the same sources compiled with
 * -DQSDVR_DEBUG_BOUNDS; no counterpart in the reference, which checks no index).  Every global
 * access whose index a kernel derives from geometry or caller data is checked against its
 * buffer; one outside it sets QSDVR_DEVERR_BOUNDS and is redirected to an in-bounds sink, so
 * nothing faults.  qsdvr_bounds_checked returns 1 in that build and 0 in the product build.
 * qsdvr_bounds_record writes the first such access since the last clear as record[0..3] =
 * {source file (1 camera.cu, 2 surface.cu, 3 render_ops.cu, 4 fused.cu, 5 optim.cu,
 * 6 gradcheck.cu, 7 proposal.cu), source line, element index, buffer extent in elements},
 * all zeros when there is none (always in the product build). */
int qsdvr_bounds_checked(void);
int qsdvr_bounds_record(uint64_t *record, int clear, cudaStream_t stream);
/* Positive control of those checks: buffer (device memory) holds 64 floats; one thread writes
 * 1.0 to element 40 through a check that declares 32 elements.  The bounds-checked build
 * catches it (QSDVR_DEVERR_BOUNDS, a record {4, line, 40, 32}) and element 40 keeps its value;
 * the product build writes it.  In bounds either way. */
int qsdvr_check_bounds(float *buffer, cudaStream_t stream);

/* Check of the failure path of the tensor-core kernels' bounded waits (no counterpart in the
 * reference): one wait, limited to limit_ns (at most 2 s), on an mbarrier that no arrival
 * completes.  It gives up, records QSDVR_DEVERR_TIMEOUT in the device error word, writes 0 to
 * *completed (device memory) and returns; the context stays usable. */
int qsdvr_check_bounded_wait(uint64_t limit_ns, uint32_t *completed, cudaStream_t stream);

/* ---- camera (kernel/camera.cu) ----------------------------------------------------- */

/* 16-byte per-ray record; include/common.h:17-23 (RayInfo), stored as int32 [N,4]. */
typedef struct qsdvr_ray_info {
    uint32_t sdf_count;
    uint32_t sdf_offset;
    uint32_t render_count;
    uint32_t render_offset;
} qsdvr_ray_info;

/* include/camera.h:4-17 (CameraArgs): pixel (px,py) at depth z maps to
 * R * [(px+cx)/fx*z, (py+cy)/fy*z, z] + t; near/far are camera depths. */
typedef struct qsdvr_camera {
    uint32_t width;
    uint32_t height;
    float rotation[9];    /* row-major */
    float translation[3];
    float fx, fy, cx, cy;
    float near_depth, far_depth;
} qsdvr_camera;

size_t qsdvr_ray_cut_workspace_size(uint32_t pixel_count);

/* Replaces RayCut (kernel/camera.cu:98-130, include/camera.h:57).  mask: device uint8
 * [pixel_count]; rays/origin/dir: [pixel_count] records.  For masked pixels writes the
 * full record (counts < 2 zeroed, exclusive-scan offsets in pixel order); for unmasked
 * pixels only sdf_count, as the reference does.  totals (device, 2 x uint32) receives
 * the total SDF and render sample counts.  Runs entirely on the device. */
int qsdvr_ray_cut(const qsdvr_camera *camera, const uint8_t *mask, qsdvr_ray_info *rays, float *origin,
                  float *dir, float interval, uint32_t pixel_count, uint32_t *totals, void *workspace,
                  size_t workspace_bytes, cudaStream_t stream);

/* Largest pixel_count qsdvr_ray_cut_noalloc accepts (2048 x 2048). */
#define QSDVR_RAY_CUT_NOALLOC_MAX_PIXELS 4194304u

/* RayCut for callers that cannot allocate device memory (an application whose device
 * memory is all owned by its own pool, or a host that gives a plugin nothing but its input
 * and output buffers).  No counterpart in the reference.  Same arguments and results as
 * qsdvr_ray_cut minus the workspace; the scan's scratch is a fixed 128 KiB array in the
 * library's device image, held on every GPU that loads the library until the process
 * exits.  Rejects pixel_count > QSDVR_RAY_CUT_NOALLOC_MAX_PIXELS.  The first call in each
 * CUDA context (the device's primary context, a context created after a device reset, or
 * a host's own driver-API context) looks up that array's device address in the current
 * context (cudaGetSymbolAddress) and caches it under the context's ID; make that first
 * call before any stream capture.  All calls share the array: calls that overlap on the GPU
 * (other streams, other host threads) race. */
int qsdvr_ray_cut_noalloc(const qsdvr_camera *camera, const uint8_t *mask, qsdvr_ray_info *rays, float *origin,
                          float *dir, float interval, uint32_t pixel_count, uint32_t *totals, cudaStream_t stream);

/* Replaces GenerateRayPoints (kernel/camera.cu:132-147, include/camera.h:59).
 * sdf_capacity / render_capacity are the lengths of the sample lists. */
int qsdvr_generate_ray_points(const qsdvr_ray_info *rays, const float *origin, const float *dir,
                              uint32_t ray_count, float interval, uint32_t base_volume_reso,
                              float *sdf_points, int32_t *sdf_index, float *render_points,
                              int32_t *render_index, float *view_dir, uint64_t sdf_capacity,
                              uint64_t render_capacity, cudaStream_t stream);

/* ---- quadric surface grid (kernel/surface.cu) --------------------------------------- */

size_t qsdvr_layer_to_grid_workspace_size(uint32_t reso);

/* Replaces LayerToGridForward (kernel/surface.cu:148-229, include/surface.h:4).
 * Layers and offset[4] are device arrays; grid7 is [reso^3][7].  The prefix
 * recurrences run on the device. */
int qsdvr_layer_to_grid_forward(float *grid7, const float *x_layer, const float *y_layer,
                                const float *z_layer, const float *offset, uint32_t reso, void *workspace,
                                size_t workspace_bytes, cudaStream_t stream);

/* Replaces LayerToGridBackward (kernel/surface.cu:231-341, include/surface.h:6).
 * Writes (not accumulates) x/y/z layer gradients [reso] and offset gradient [4]. */
int qsdvr_layer_to_grid_backward(const float *grad7, uint32_t reso, float *x_grad, float *y_grad,
                                 float *z_grad, float *offset_grad, void *workspace, size_t workspace_bytes,
                                 cudaStream_t stream);

/* Replaces SampleSDFForward (kernel/surface.cu:343-350, include/surface.h:8).
 * grid7 [cell_count][7], points [count][3], index [count]. */
int qsdvr_sample_sdf_forward(float *out, const float *grid7, const float *points, const int32_t *index,
                             uint64_t count, float reso, uint64_t cell_count, cudaStream_t stream);

/* Replaces SampleSDFBackward (kernel/surface.cu:352-359, include/surface.h:10).
 * Accumulates into grid7_grad (caller zeroes). */
int qsdvr_sample_sdf_backward(const float *grad_out, const float *grid7, const float *points,
                              const int32_t *index, float *grid7_grad, uint64_t count, float reso,
                              uint64_t cell_count, cudaStream_t stream);

/* Replaces SampleNormalForward (kernel/surface.cu:361-367, include/surface.h:12). */
int qsdvr_sample_normal_forward(float *out, const float *grid7, const float *points, const int32_t *index,
                                uint64_t count, uint64_t cell_count, cudaStream_t stream);

/* Replaces SampleNormalBackward (kernel/surface.cu:369-375, include/surface.h:14). */
int qsdvr_sample_normal_backward(const float *grad_out, const float *grid7, const float *points,
                                 const int32_t *index, float *grid7_grad, uint64_t count, uint64_t cell_count,
                                 cudaStream_t stream);

/* ---- appearance, shading, compositing (kernel/render.cu) ---------------------------- */

/* Replaces GridInterpolationForward (kernel/render.cu:317-323, include/render.h:4).
 * data [vertex_count][32]; the corners of sample i are index[i] + {0,1} + {0,reso} +
 * {0,reso^2} (in vertices), as the reference addresses them; out [count][32]. */
int qsdvr_grid_interpolation_forward(const float *data, const float *points, const int32_t *index, float *out,
                                     uint64_t count, uint32_t reso, uint64_t vertex_count, cudaStream_t stream);

/* Replaces GridInterpolationBackward (kernel/render.cu:325-331, include/render.h:6).
 * Accumulates into data_grad [vertex_count][32] (caller zeroes). */
int qsdvr_grid_interpolation_backward(float *data_grad, const float *points, const int32_t *index,
                                      const float *grad_out, uint64_t count, uint32_t reso,
                                      uint64_t vertex_count, cudaStream_t stream);

/* Replaces ShaderForward (kernel/render.cu:333-339, include/render.h:8).  mode:
 * QSDVR_MODE_COMPAT reproduces the reference's overlapping SH read. */
int qsdvr_shader_forward(float *out, const float *normal, const float *view, const float *data,
                         float *specular, uint64_t count, int mode, cudaStream_t stream);

/* Replaces ShaderBackward (kernel/render.cu:341-347, include/render.h:10). */
int qsdvr_shader_backward(const float *grad_out, const float *normal, const float *view, const float *data,
                          const float *specular, float *normal_grad, float *data_grad, uint64_t count, int mode,
                          cudaStream_t stream);

/* Replaces RayAggregateForward (kernel/render.cu:349-355, include/render.h:12).
 * out [ray_count][3]; alpha, T [render samples]. */
int qsdvr_ray_aggregate_forward(float *out, const float *rgb, const float *sdf, const qsdvr_ray_info *rays,
                                float *alpha, float *transmittance, uint32_t ray_count, float logistic_coef,
                                uint64_t sdf_capacity, uint64_t render_capacity, cudaStream_t stream);

/* Replaces RayAggregateBackward (kernel/render.cu:357-363, include/render.h:14). */
int qsdvr_ray_aggregate_backward(const float *grad_out, const float *rgb, const float *sdf,
                                 const qsdvr_ray_info *rays, const float *alpha, const float *transmittance,
                                 float *rgb_grad, float *sdf_grad, uint32_t ray_count, float logistic_coef,
                                 uint64_t sdf_capacity, uint64_t render_capacity, cudaStream_t stream);


/* ---- fused render path (B200-native; no reference counterpart as a single kernel) ---- */

enum { QSDVR_STORAGE_F32 = 0, QSDVR_STORAGE_BF16 = 1 };
enum {
    QSDVR_TRANSMITTANCE_PRODUCT = 0, /* T_{i+1} = T_i (1 - alpha_i), as the reference        */
    QSDVR_TRANSMITTANCE_LOG = 1      /* T_i = exp(sum log(1 - alpha)), compensated summation */
};

/* One batch of rays through the whole render path.  The rays are the reference's
 * per-ray tables (RayCut output after masking: RayInfo, origin = first in-box sample,
 * unit direction); samples are generated on the fly exactly as GenerateRayPoints
 * (kernel/camera.cu:60-96) would.  Only sdf_count of each record is read.  A ray with more
 * than 8192 render samples (256 warp chunks of 32) is skipped before any access: colour 0, no
 * gradient, QSDVR_DEVERR_RAY set.  The volume's diagonal is 2 sqrt(3), so only intervals
 * below about 0.00042 can produce such a ray (the reference marches any length).
 *   sdf_grid: [R^3][8] (a0..a6 + one pad) in `storage` precision, cell x + yR + zR^2;
 *             bf16 cells are read as (a0..a5, slot 6 + slot 7), see qsdvr_sdf_cells_bf16;
 *   data:     [(R+1)^3][C] appearance rows in `storage` precision, C = 32 (SH degree 2)
 *             or 64 (degree 3);
 *   grads:    fp32, same layouts, accumulated with atomics (caller zeroes). */
typedef struct qsdvr_render_args {
    const qsdvr_ray_info *rays;
    const float *origin;      /* [ray_count][3] */
    const float *dir;         /* [ray_count][3] */
    uint32_t ray_count;
    uint32_t reso;            /* R */
    float interval;           /* sample spacing along the ray */
    float logistic_coef;      /* k of alpha = max((e^{-k s_{i+1}} - e^{-k s_i}) / (1 + e^{-k s_{i+1}}), 0) */
    int32_t mode;             /* QSDVR_MODE_* */
    int32_t storage;          /* QSDVR_STORAGE_* of sdf_grid and data */
    int32_t transmittance;    /* QSDVR_TRANSMITTANCE_* */
    int32_t sh_degree;        /* 2 (0 means 2; 32-channel rows, the reference) or 3 (fixed mode only,
                                 64-channel rows: 16x3 SH, diffuse 48..50, metallic 51, ao 52) */
    const void *sdf_grid;
    const void *data;
    float *color;             /* [ray_count][3] output of forward / train */
    const float *target;      /* [ray_count][3] train: MSE target */
    const float *grad_color;  /* [ray_count][3] backward: dL/dcolor */
    float *sdf_grad;          /* [R^3][8] accumulated */
    float *data_grad;         /* [(R+1)^3][C] accumulated */
    float *loss;              /* train: sum over rays of |color - target|^2 is added here */
    float grad_scale;         /* train: dL/dcolor = grad_scale * (color - target) */
    void *workspace;          /* optional, 256-byte aligned: enables the persistent grid with     */
    uint64_t workspace_bytes; /* dynamic ray scheduling and, in train, the per-warp row stash    */
    const float *sdf_layers;  /* optional, replaces sdf_grid: separable SDF tables [3 reso + 1][4]
                                 from qsdvr_separable_sdf_tables (fp32 whatever the storage)      */
    float *sdf_layers_grad;   /* train / backward with sdf_layers: its gradient, same layout,
                                 zeroed by the caller; qsdvr_separable_sdf_grad turns it into the
                                 layer and offset gradients                                       */
    const float *tlist;       /* optional [ray_count][33]: SDF sample positions t (from origin) of
                                 each ray, replacing the uniform march (32 render samples at the
                                 interval midpoints); rays with sdf_count < 2 stay empty          */
    float *sample_alpha;      /* optional: alpha of render sample i of ray r written at
                                 rays[r].render_offset + i (forward and train)                   */
    uint64_t sample_capacity; /* length of sample_alpha */
    const uint32_t *order;    /* optional [ray_count]: the order in which the persistent kernel
                                 takes the rays (a permutation of 0..ray_count-1, e.g. rays sorted
                                 by qsdvr_ray_order_keys); outputs stay indexed by ray          */
    int32_t data_grad_storage; /* QSDVR_STORAGE_F32 (default) or QSDVR_STORAGE_BF16: data_grad
                                  accumulated as bf16 (each contribution and each sum rounded to
                                  8 significant bits, half the gradient traffic); no reference
                                  counterpart.  The SDF gradient stays fp32.                     */
    int32_t merge_scatter;     /* nonzero: the render samples of a warp chunk (32 consecutive
                                  samples of a ray) that lie in the same cell are found with one
                                  match_any, and their appearance gradients go out as one summed
                                  RED per corner row instead of one per sample (same sums up to
                                  float reassociation); 0: one RED per sample and corner row   */
} qsdvr_render_args;

/* Sort keys that make neighbouring rays in a batch cross neighbouring cells (no counterpart
 * in the reference): the 30-bit Morton code of each ray's in-box midpoint on a 1024^3 lattice
 * of the volume, 0x7fffffff for rays with fewer than 2 SDF samples (keys sort the same signed
 * or unsigned).  Rays taken in key order
 * by qsdvr_render_* (args.order) share more gathered rows and gradient lines in L2. */
int qsdvr_ray_order_keys(const qsdvr_ray_info *rays, const float *origin, const float *dir, uint32_t ray_count,
                         float interval, uint32_t *keys, cudaStream_t stream);

/* Workspace bytes of qsdvr_ray_order for ray_count rays (a 2^15 + 1 bucket histogram and one
 * bucket per ray). */
size_t qsdvr_ray_order_workspace_size(uint32_t ray_count);

/* The ray order itself, without a library sort (no counterpart in the reference): order
 * receives a permutation of 0..ray_count-1 that lists the rays by the 15-bit Morton code of
 * their in-box midpoint (a 32^3 lattice of the volume), rays with fewer than 2 SDF samples
 * last; within one lattice cube the order is the order in which the device's atomics reach
 * the rays.  Three kernels and a memset on the stream (histogram, scan, scatter). */
int qsdvr_ray_order(const qsdvr_ray_info *rays, const float *origin, const float *dir, uint32_t ray_count,
                    float interval, uint32_t *order, void *workspace, size_t workspace_bytes, cudaStream_t stream);

/* The same counting sort for list-mode batches (no counterpart in the reference): each ray is
 * keyed on the point at its median SDF position, tlist[33 r + 16] of the [ray_count][33]
 * sample list that qsdvr_render_* takes (args.tlist), instead of its in-box midpoint.  The
 * proposal samples sit where the compositing weights are, so rays taken in this order run
 * beside the rays that hit the same patch of the surface.  Same workspace as
 * qsdvr_ray_order. */
int qsdvr_ray_order_list(const qsdvr_ray_info *rays, const float *origin, const float *dir, uint32_t ray_count,
                         const float *tlist, uint32_t *order, void *workspace, size_t workspace_bytes,
                         cudaStream_t stream);

/* Separable SDF for the fused renderer (the RenderGrid model's parametrisation,
 * models/render.py:172-207, without materialising [R^3][7]; LayerToGridForward,
 * kernel/surface.cu:148-229, computes the same cells): per-axis recurrence tables
 * [3 reso + 1][4] = (a0, a3, a6, 0) per axis index, then (offset[3], 0, 0, 0). */
int qsdvr_separable_sdf_tables(const float *x_layer, const float *y_layer, const float *z_layer,
                               const float *offset, uint32_t reso, float *tables, cudaStream_t stream);

/* Layer gradients from the table gradient the fused renderer accumulated (the reverse
 * recurrences of LayerToGridBackward, kernel/surface.cu:301-334); table_grad is consumed. */
int qsdvr_separable_sdf_grad(float *table_grad, uint32_t reso, float *x_grad, float *y_grad, float *z_grad,
                             float *offset_grad, cudaStream_t stream);

/* Workspace bytes for qsdvr_render_* with these args on the current device (mode, storage
 * and transmittance select the kernel; independent of ray_count).  One workspace must not
 * be used by launches that may overlap on the GPU. */
size_t qsdvr_render_workspace_size(const qsdvr_render_args *args);

/* Replaces RenderGrid.forward (models/render.py:225-234, i.e. the SampleSDF, SampleNormal,
 * GridInterpolation, Shader and RayAggregate forwards) fused with GenerateRayPoints
 * (kernel/camera.cu:132-147): writes color. */
int qsdvr_render_forward(const qsdvr_render_args *args, cudaStream_t stream);
/* Forward of a full frame with the appearance grid staged in shared memory by TMA, brick by
 * brick (no counterpart in the reference; a prototype beside qsdvr_render_forward).  The
 * rays should be listed tile by tile (8 x 8 pixels): each block of 64 rays marches its rays
 * one thread per ray and, in rounds, copies one 8 x 8 x 8-vertex brick of the appearance grid
 * (64 KB) into shared memory with cp.async.bulk.tensor, then renders every sample whose cell
 * lies inside it.  Fixed mode, uniform march, log transmittance and 128-byte vertex rows only
 * (bf16 SH degree 3 or fp32 degree 2); the same colours as qsdvr_render_forward up to the
 * summation order of the log-transmittance. */
int qsdvr_render_forward_bricks(const qsdvr_render_args *args, cudaStream_t stream);
/* Replaces the backward chain of RenderGrid (models/render.py:27-170: RayAggregate, Shader,
 * GridInterpolation, SampleNormal, SampleSDF backwards) for a given dL/dcolor; per-sample
 * alpha and colour are recomputed, nothing per-sample is read from memory. */
int qsdvr_render_backward(const qsdvr_render_args *args, cudaStream_t stream);
/* Forward + MSE loss gradient + backward in one launch (test.py:30-33 training step
 * without the optimizer): writes color, accumulates loss and gradients. */
int qsdvr_render_train(const qsdvr_render_args *args, cudaStream_t stream);

/* ---- fused grid optimizer ---------------------------------------------------------- */

enum {
    QSDVR_ADAM_ZERO_GRAD = 1,      /* write zeros over the gradient after using it           */
    QSDVR_ADAM_SKIP_ZERO_GRAD = 2, /* leave elements whose gradient is exactly 0 untouched    */
    QSDVR_ADAM_GRAD_BF16 = 4,      /* grad points to bf16 values (render data_grad_storage)  */
    QSDVR_ADAM_SDF_CELLS = 8,      /* param is a quadric cell grid [count/8][8] (fp32 grad): the
                                      bf16 copy is written in the cell form of qsdvr_sdf_cells_bf16 */
    QSDVR_ADAM_STATE_BF16 = 16     /* exp_avg and exp_avg_sq hold bf16 values (no reference
                                      counterpart; torch keeps fp32 moments): updated in fp32 and
                                      stochastically rounded back, 24 instead of 32 bytes of HBM
                                      traffic per parameter */
};

/* One Adam step over `count` fp32 elements.  The default (flags without SKIP_ZERO_GRAD)
 * is torch.optim.Adam's update, bias corrections included; `step` counts from 1.
 * param_bf16, when not null, receives the updated parameters rounded to bf16 (the
 * storage copy the fused render kernels read). */
typedef struct qsdvr_adam_args {
    float *param;
    float *grad;        /* fp32, or bf16 with QSDVR_ADAM_GRAD_BF16 */
    float *exp_avg;     /* fp32, or bf16 with QSDVR_ADAM_STATE_BF16 */
    float *exp_avg_sq;  /* fp32, or bf16 with QSDVR_ADAM_STATE_BF16 */
    void *param_bf16;   /* optional [count] bf16 */
    uint64_t count;
    double lr, beta1, beta2, eps; /* host precision; the kernel's float constants are derived from them */
    uint32_t step;
    int32_t flags;      /* QSDVR_ADAM_* */
} qsdvr_adam_args;

/* Replaces optimizer.step() + optimizer.zero_grad() of the reference's training loop
 * (test.py:34-35, torch.optim.Adam over renderData and the layers) for grid parameters. */
int qsdvr_adam_step(const qsdvr_adam_args *args, cudaStream_t stream);

/* BF16 storage copy of a quadric cell grid [cell_count][8] fp32 (a0..a6 + pad; no reference
 * counterpart, the reference keeps fp32 cells).  Each 16-byte bf16 cell holds a0..a5 rounded
 * to nearest and, in slots 6 and 7, a6' = a6 |bf16(a3..a5)| / |a3..a5| as hi = bf16(a6') and
 * lo = bf16(a6' - hi): the stored cell's SDF at its centre equals the master's, so rounding
 * the gradient coefficients does not rescale the cell's SDF.  The render kernels read bf16
 * cells as (a0..a5, hi + lo); a plain bf16 rounding of the fp32 layout (pad 0) is read as
 * a6 = bf16(a6). */
int qsdvr_sdf_cells_bf16(const float *cells, void *out, uint64_t cell_count, cudaStream_t stream);

/* ---- FP64 loss for finite-difference gradient checks ---------------------------------- */

/* sum_c (color_c - target_c)^2 per ray with every quantity in double (fixed mode: packed SH,
 * vertex x + y(R+1) + z(R+1)^2); grids [R^3][8] and [(R+1)^3][32] in double.  The only FP64
 * GPU code: central differences of it check qsdvr_render_backward / _train.  Restates the
 * forward of RenderGrid (models/render.py:225-234) for one loss value per ray. */
int qsdvr_render_loss_f64(const qsdvr_ray_info *rays, const float *origin, const float *dir, uint32_t ray_count,
                          uint32_t reso, float interval, double logistic_coef, const double *sdf_grid,
                          const double *data, const double *target, double *loss_per_ray, cudaStream_t stream);

/* ---- proposal network (no counterpart in the reference) ----------------------------------
 * A 32-d positional encoding -> 64 -> 64 -> 1 MLP bounding the renderer's density; BF16
 * weights (params_bf16: QSDVR_MLP_PARAMS values, layout in qsdvr_b200/csrc/proposal.cu),
 * FP32 accumulation on the tcgen05 tensor cores. */
#define QSDVR_MLP_PARAMS 6280

/* Density bound at points [count][4] (x, y, z, ignored), or, when rays is not null, at the
 * 64 coarse points t = (j + 0.5) L / 64 of every ray (L = (sdf_count - 1) interval; rays
 * with sdf_count < 2 get 0); out is [count] or [ray_count][64]. */
int qsdvr_mlp_density(const float *points, uint32_t count, const qsdvr_ray_info *rays, const float *origin,
                      const float *dir, uint32_t ray_count, float interval, const void *params_bf16, float *out,
                      cudaStream_t stream);

/* One training pass over points [count][4] (x, y, z, target density): accumulates the
 * gradient of mean_p w (log1p(bound) - log1p(target))^2 (w = under_weight where the bound is
 * below the target; points with a negative target contribute nothing) into
 * grad [QSDVR_MLP_PARAMS] fp32 and the loss into *loss. */
int qsdvr_mlp_train(const float *points, uint32_t count, const void *params_bf16, float under_weight, float *grad,
                    float *loss, cudaStream_t stream);

/* Launch shape of the persistent MLP kernels for count points (kernel 0: inference,
 * 1: training): grid size and resident CTAs per SM. */
int qsdvr_mlp_launch_shape(int kernel, uint32_t count, uint32_t *blocks, int *blocks_per_sm);

/* Fine sample positions [ray_count][33] from the coarse densities [ray_count][64]: inverse
 * CDF of the coarse compositing weights, mixed with the fraction uniform_mix (0, 1] of a
 * uniform density, at quantiles k/32. */
int qsdvr_proposal_sample(const qsdvr_ray_info *rays, uint32_t ray_count, float interval, float uniform_mix,
                          const float *coarse_density, float *tlist, cudaStream_t stream);

/* Training points for the proposal network from a uniform-march forward: render sample i
 * of ray r at rays[r].render_offset + i gets (position, -log(1 - alpha) / interval). */
int qsdvr_proposal_targets(const qsdvr_ray_info *rays, const float *origin, const float *dir, uint32_t ray_count,
                           float interval, const float *alpha, uint64_t sample_count, float *points,
                           cudaStream_t stream);

/* count training points [count][4] drawn at random (counter-based hash of seed and point
 * index) from the same alphas: a ray uniformly, then one of its render samples uniformly;
 * a point that finds no ray with samples in 16 draws gets target -1 (ignored in training). */
int qsdvr_proposal_draw(const qsdvr_ray_info *rays, const float *origin, const float *dir, uint32_t ray_count,
                        float interval, const float *alpha, uint64_t sample_count, uint32_t count, uint32_t seed,
                        float *points, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* QSDVR_B200_H */
