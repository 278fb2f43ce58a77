/*
 * rgsplat.h -- C ABI of librgsplat_b200, the B200 (sm_100a) implementation of
 * rgsplat's differentiable 3D-Gaussian-splatting training step.
 *
 * Every entry point is plain C: pointers, sizes and status codes, no CUDA or
 * torch types. Host arrays use the reference crate's own records so a Rust
 * `extern "C"` block can pass its slices straight through:
 *   Gaussian3D   59 x f32 (src/math/mod.rs:27-46): position[3], opacity_logit,
 *                rotation[4] (w, x, y, z), log_scale[3], sh_coeffs[48]
 *                (channel-major: 16 R, 16 G, 16 B).
 *   GaussianGrad 60 x f32 (src/cpu/backward.rs:33-41): d_position[3],
 *                d_rotation[4], d_log_scale[3], d_opacity_logit, d_sh[48],
 *                screen_grad_norm.
 *   Images       rendered RGB interleaved w*h*3 f32 (backward.rs:124);
 *                targets RGBA interleaved w*h*4 f32 (TargetImage, src/io/images.rs:17-22).
 *   AdamState    m1, m2 as [N][59] f32 in flatten_grad order
 *                (src/pipeline/optimizer.rs:74-84, 165-173).
 *
 * Status: every function returns RGS_OK (0) or a negative RGS_ERR_* code; the
 * message of the last failure on a context is rgs_last_error(ctx). Where the
 * reference panics (NaN depth, backward.rs:191; singular c2w,
 * src/math/mod.rs:158-159) this library returns RGS_ERR_NONFINITE /
 * RGS_ERR_SINGULAR_CAMERA instead.
 *
 * Threading: a context owns one CUDA stream and its device buffers; use one
 * context per host thread. The caller owns every host buffer.
 */
#ifndef RGSPLAT_H
#define RGSPLAT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RGS_OK 0
#define RGS_ERR_INVALID_ARG (-1)
#define RGS_ERR_OOM (-2)
#define RGS_ERR_CUDA (-3)
#define RGS_ERR_NONFINITE (-4)
#define RGS_ERR_SINGULAR_CAMERA (-5)
#define RGS_ERR_CAPACITY (-6)
#define RGS_ERR_NO_DEVICE (-7)
#define RGS_ERR_IO (-8)     /* a file could not be opened, read or written */
#define RGS_ERR_FORMAT (-9) /* a model file is not one the reader accepts */

#define RGS_GAUSSIAN_FLOATS 59
#define RGS_GRAD_FLOATS 60

typedef struct rgs_ctx rgs_ctx;

/* Camera (src/math/mod.rs:131-145); c2w row-major, OpenCV axes (+z forward). */
typedef struct rgs_camera {
    uint32_t width, height;
    float fx, fy, cx, cy;
    float c2w[16];
    float distortion[3]; /* carried, unused (as in the reference) */
} rgs_camera;

/* LossConfig (src/cpu/backward.rs:57-67). */
typedef struct rgs_loss_config {
    float lambda_dssim;
} rgs_loss_config;

/* TrainConfig (src/pipeline/optimizer.rs:22-40). */
typedef struct rgs_train_config {
    uint64_t num_iterations;
    float lr_position, lr_rotation, lr_scale, lr_opacity, lr_sh_dc, lr_sh_rest;
    float beta1, beta2, eps;
    uint64_t densify_from_iter, densify_until_iter;
    float densify_grad_threshold;
    uint64_t opacity_reset_iter;
    float prune_opacity_thresh;
    uint64_t max_gaussians;
} rgs_train_config;

/* SplatInfo2D (src/gpu/compute.rs:64-78), 40 bytes. */
typedef struct rgs_splat_info_2d {
    float sx, sy, conic_a, conic_b, conic_c, color_r, color_g, color_b, alpha, depth;
} rgs_splat_info_2d;

/* AdamState (src/pipeline/optimizer.rs:74-106) as caller-owned host arrays.
 * `len` is the number of Gaussians the arrays hold (>= n; the reference's
 * AdamState only grows). */
typedef struct rgs_adam_state {
    float* m1;            /* len * 59 */
    float* m2;            /* len * 59 */
    float* grad_accum;    /* len */
    uint32_t* grad_denom; /* len */
    size_t len;
    uint64_t t;
} rgs_adam_state;

typedef struct rgs_options {
    int device;           /* CUDA device ordinal (default 0) */
    int tile_w, tile_h;   /* CTA tile: 16x16 (default), 8x32 or 32x8 */
    int batch;            /* splats staged per shared-memory round: 128, 256 (default), 512 */
    int reference_compat; /* 1 (default): keep the reference's Adam quirks (moments are not
                             compacted on prune, optimizer.rs:97-105; "SH DC" lr applies to
                             flat indices 11..13, optimizer.rs:181). 0: moments follow their
                             Gaussians and lr_sh_dc applies to sh[0], sh[16], sh[32]. */
    int pixels_per_thread; /* forward blend: 1 or 2 (default) vertically adjacent pixels per
                              thread; the backward blend takes twice as many */
    uint64_t batch_pair_limit; /* pair budget of one batched launch: a batched step whose
                                  (Gaussian, tile) pairs outgrow the pair buffer and pass this
                                  runs as consecutive view groups within it (gradients summed
                                  across groups, one Adam step); 0 = default 2^30 (pair buffers
                                  and sort scratch take 16 bytes per pair) */
    int exact_loss;       /* 0 (default): the SSIM blurs accumulate with fused multiply-adds
                             (dL/dpixel within float rounding of the reference's); 1: the
                             reference's separate multiply and add and its divisions
                             (backward.rs:718-807), dL/dpixel bit-identical */
} rgs_options;

/* Step modes of rgs_trainer_step. */
#define RGS_STEP_PLAIN 0   /* per-view launches, host-synchronised pair counts */
#define RGS_STEP_BATCHED 1 /* all views per stage in one launch, CUDA-graph replay */

/* Projection modes of rgs_project / rgs_gpu_render. */
#define RGS_PROJECT_WGSL 0     /* the WGSL shader's arithmetic (DC colour, its J) */
#define RGS_PROJECT_CPU_MATH 1 /* the CPU path's projection (full SH, all culls) */

/* ---- context ------------------------------------------------------------- */
void rgs_options_default(rgs_options* opts);
void rgs_train_config_default(rgs_train_config* cfg); /* TrainConfig::default(), optimizer.rs:42-62 */
int rgs_create(const rgs_options* opts, rgs_ctx** out);
void rgs_destroy(rgs_ctx* ctx);
const char* rgs_last_error(const rgs_ctx* ctx);
int rgs_device_count(int* count);
int rgs_synchronize(rgs_ctx* ctx);

/* ---- drop-ins for the reference's free functions (host buffers) ---------- */

/* cpu::backward::render_and_backward (src/cpu/backward.rs:107-149).
 * grads_out: n * 60 floats (may be NULL). */
int rgs_render_and_backward(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera,
                            const float* target_rgba, const float bg[3], const rgs_loss_config* cfg,
                            float* loss_out, float* grads_out);

/* render_and_backward with a chosen blend backward, for the differentiation
 * study (no counterpart in the reference, whose backward is the recompute
 * one, src/cpu/backward.rs:391-512):
 *   RGS_BACKWARD_RECOMPUTE: the library's path -- T is rebuilt from each
 *     pixel's final T and last contributor; blend state = 8 B per pixel;
 *   RGS_BACKWARD_STORE_ALL: the forward also stores T before every
 *     contributing splat at (tile-list position, pixel in tile) and the
 *     backward reads it; blend state += 1 KiB per (tile, splat) pair (16x16
 *     tiles only).
 * report (may be NULL) receives the blend kernel times and state bytes. */
#define RGS_BACKWARD_RECOMPUTE 0
#define RGS_BACKWARD_STORE_ALL 1
typedef struct rgs_backward_report {
    float forward_ms, backward_ms; /* blend forward / backward kernels, CUDA events */
    uint64_t state_bytes;          /* device bytes of blend state kept for the backward */
    uint64_t pairs;                /* (tile, splat) pairs of the view */
} rgs_backward_report;
int rgs_render_and_backward_variant(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera,
                                    const float* target_rgba, const float bg[3], const rgs_loss_config* cfg,
                                    int variant, float* loss_out, float* grads_out, rgs_backward_report* report);

/* cpu::backward::render_color (src/cpu/backward.rs:152-166): rgb_out w*h*3. */
int rgs_render_color(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, const float bg[3],
                     float* rgb_out);

/* cpu::rasterize (src/cpu/rasterizer.rs:72-192): the forward-only preview
 * render. Same projection, depth order and 16x16 tile lists as the training
 * path, but each pixel's colour starts at bg and the splats' weighted colours
 * are added to it (bg is not scaled by the remaining transmittance,
 * rasterizer.rs:133); alpha = 1 - T; tiles no splat touches stay
 * (0, 0, 0, 0). out: w*h*4 floats (RGS_FB_RGBA_F32, Framebuffer::data) or
 * w*h*4 bytes (RGS_FB_RGBA8_SRGB, Framebuffer::to_u8_srgb, rasterizer.rs:38-48;
 * converted on the device). */
#define RGS_FB_RGBA_F32 0
#define RGS_FB_RGBA8_SRGB 1
int rgs_rasterize(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, const float bg[3], int format,
                  void* out);
/* rgs_rasterize of the trainer's device-resident Gaussians for its camera
 * `view` (a live preview during training: no parameter upload). */
int rgs_trainer_rasterize(rgs_ctx* ctx, uint32_t view, const float bg[3], int format, void* out);

/* cpu::backward::photometric_loss_grad (src/cpu/backward.rs:646-693). */
int rgs_photometric_loss_grad(rgs_ctx* ctx, const float* rendered_rgb, const float* target_rgba, uint32_t width,
                              uint32_t height, float lambda, float* loss_out, float* dl_out);

/* No counterpart in the reference. rgs_photometric_loss_grad on caller-owned
 * DEVICE buffers, for callers that must not allocate device memory: a host
 * application or framework that owns every byte of the GPU through its own
 * pool (a cudaMalloc behind its back can fail or fragment its budget), or a
 * latency-critical path where cudaMalloc's implicit device synchronisation is
 * not acceptable. It needs no context and allocates nothing; its scratch (view
 * descriptor plus two floats per 32x32 loss block) is a static device array
 * of 256 + RGS_NOALLOC_MAX_LOSS_BLOCKS * 8 bytes (128.25 KiB) that every GPU
 * loading the library holds until the process exits. Images over
 * RGS_NOALLOC_MAX_LOSS_BLOCKS loss blocks (4096x4096 pixels) return
 * RGS_ERR_CAPACITY. rendered_rgb: w*h*3, target_rgba: w*h*4, dl_out: w*h*3,
 * loss_out: 1 float, all on `device`. Work is enqueued on `cuda_stream`
 * (NULL = legacy default stream) and the call returns without synchronising.
 * The first call on a device also sets that device up (looks up the scratch
 * array's device address and sets the loss kernel's shared-memory limit), so
 * make that first call before any stream capture on the device. Every call
 * reuses the same array, which keeps the previous call's contents; calls that
 * overlap on one device race on it: serialise them. On failure a message is
 * written to err (err_len bytes, may be NULL). */
#define RGS_NOALLOC_MAX_LOSS_BLOCKS 16384
int rgs_photometric_loss_grad_noalloc(int device, const float* rendered_rgb, const float* target_rgba,
                                      uint32_t width, uint32_t height, float lambda, float* loss_out,
                                      float* dl_out, void* cuda_stream, char* err, size_t err_len);

/* pipeline::optimizer::adam_step (src/pipeline/optimizer.rs:116-163): updates
 * `gaussians` (n * 59) and `state` in place. grads: n * 60. */
int rgs_adam_step(rgs_ctx* ctx, float* gaussians, size_t n, const float* grads, rgs_adam_state* state,
                  const rgs_train_config* cfg);

/* pipeline::optimizer::densify_and_prune (src/pipeline/optimizer.rs:206-272).
 * Writes the new Gaussians to out (capacity out_cap Gaussians; 2*n always
 * suffices: every Gaussian is kept and cloned at most, or split into two)
 * and their count to *n_out. Returns RGS_ERR_CAPACITY with *n_out
 * set to the required count when out_cap is too small. As AdamState::resize
 * does, the caller grows its moment arrays to *n_out if larger (never
 * shrinking them) and zeroes grad_accum / grad_denom. */
int rgs_densify_and_prune(rgs_ctx* ctx, const float* gaussians, size_t n, const float* grad_accum,
                          const uint32_t* grad_denom, const rgs_train_config* cfg, float scene_extent,
                          float* out, size_t out_cap, size_t* n_out);

/* pipeline::optimizer::reset_opacities (src/pipeline/optimizer.rs:314-319). */
int rgs_reset_opacities(rgs_ctx* ctx, float* gaussians, size_t n);

/* gpu::GpuRenderer::project (src/gpu/compute.rs:140-207): one SplatInfo2D and one
 * depth key (~bits(depth), 0xFFFFFFFF when culled) per Gaussian. */
int rgs_project(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, int mode,
                rgs_splat_info_2d* splats_out, uint32_t* keys_out);

/* gpu::GpuRenderer::render (src/gpu/compute.rs:210-218): project, then the
 * composite of compute.rs:243-296 (depth order, per-splat 3-sigma box from the
 * conic, T < 1e-4 skip) on the GPU. rgb_out: w*h*3. */
int rgs_gpu_render(rgs_ctx* ctx, const float* gaussians, size_t n, const rgs_camera* camera, int mode,
                   const float bg[3], float* rgb_out);

/* ---- model files: io::ply (src/io/ply.rs:35-303) --------------------------
 * save_ply writes the binary little-endian 3DGS layout (62 f32 per vertex,
 * ply.rs:35-104); save_splat the lossy 32-byte display records (position,
 * exp(log_scale), RGBA bytes from the DC colour and sigmoid(opacity),
 * quaternion bytes, ply.rs:253-285); both create the parent directory.
 * load_ply accepts binary LE / BE and ASCII with properties in any order,
 * decoding each by its byte width as the reference does (ply.rs:116-252).
 * The records are packed / unpacked on the device. rgs_load_ply fills up to
 * `cap` records (n * 59 floats); with out == NULL or cap too small it sets
 * *n_out to the file's vertex count and returns RGS_ERR_CAPACITY. */
int rgs_save_ply(rgs_ctx* ctx, const float* gaussians, size_t n, const char* path);
int rgs_save_splat(rgs_ctx* ctx, const float* gaussians, size_t n, const char* path);
int rgs_load_ply(rgs_ctx* ctx, const char* path, float* out, size_t cap, size_t* n_out);
/* gaussians_from_sfm (src/pipeline/sfm.rs:365-404): n SfM points (xyz n*3
 * f64, rgb n*3 u8) -> n Gaussian3D records (out n*59 f32): the position, the
 * colour as the SH DC term of powf(u / 255, 2.2), an isotropic log scale of
 * the mean distance to the 3 nearest points of a 50-wide window of the
 * x-sorted cloud (estimate_initial_scales, :408-450), identity rotation,
 * opacity logit(0.1). A non-finite coordinate is RGS_ERR_INVALID_ARG (the
 * reference's sort panics on NaN). */
int rgs_gaussians_from_sfm(rgs_ctx* ctx, const double* xyz, const uint8_t* rgb, size_t n, float* out);
/* The same Gaussians straight into the trainer; the optimiser state restarts. */
int rgs_trainer_init_from_sfm(rgs_ctx* ctx, const double* xyz, const uint8_t* rgb, size_t n);
/* parse_points3d_bin (sfm.rs:147-183): a COLMAP points3D.bin on the host.
 * *n_out = the file's point count; xyz (n*3) and rgb (n*3) are filled when cap
 * holds them, else RGS_ERR_CAPACITY (call with null buffers to size them).
 * A file cut short is RGS_ERR_FORMAT. */
int rgs_read_points3d_bin(rgs_ctx* ctx, const char* path, double* xyz, uint8_t* rgb, size_t cap, size_t* n_out);

/* load_target's colour conversion (src/io/images.rs:67-72, srgb_to_linear
 * :76-82): 8-bit sRGB RGBA (npix * 4 bytes) -> linear RGBA f32 (npix * 4),
 * alpha linear. Decoding the file and resizing it to the camera
 * (image::open, resize_exact) stay with the caller's image library. */
int rgs_srgb8_to_linear(rgs_ctx* ctx, const uint8_t* rgba8, size_t npix, float* out);
/* Camera `index`'s target from an 8-bit sRGB RGBA image at the camera's
 * resolution (w*h*4 bytes), converted to linear on the device. */
int rgs_trainer_set_target_rgba8(rgs_ctx* ctx, size_t index, const uint8_t* rgba8);

/* The trainer's Gaussians straight from / into device memory; loading resets
 * the Adam state like rgs_trainer_set_gaussians. */
int rgs_trainer_save_ply(rgs_ctx* ctx, const char* path);
int rgs_trainer_save_splat(rgs_ctx* ctx, const char* path);
int rgs_trainer_load_ply(rgs_ctx* ctx, const char* path, size_t* n_out);

/* ---- device-resident trainer (the training loop of src/pipeline/mod.rs:203-265) */

/* Upload Gaussians (n * 59); resets the Adam state (AdamState::new). */
int rgs_trainer_set_gaussians(rgs_ctx* ctx, const float* gaussians, size_t n);
int rgs_trainer_count(rgs_ctx* ctx, size_t* n);
int rgs_trainer_get_gaussians(rgs_ctx* ctx, float* out, size_t cap, size_t* n_out);
int rgs_trainer_set_cameras(rgs_ctx* ctx, const rgs_camera* cameras, size_t count);
/* Upload camera `index`'s RGBA target (w*h*4 f32) to device memory. */
int rgs_trainer_set_target(rgs_ctx* ctx, size_t index, const float* target_rgba);

/* One training step over `nviews` camera indices: render, loss, backward,
 * gradients summed over the views, one Adam step (denominator += nviews).
 * losses_out: nviews floats (may be NULL). */
int rgs_trainer_step(rgs_ctx* ctx, const uint32_t* views, size_t nviews, const float bg[3],
                     const rgs_loss_config* loss_cfg, const rgs_train_config* train_cfg, int mode,
                     float* losses_out);

/* rgs_trainer_step (batched) with each view's RGBA target (w*h*4 f32) read
 * from caller HOST memory for this step instead of the device-resident
 * targets: the copies run on a second stream while the step projects, sorts
 * and renders, and only the loss waits for them. Page-locked host memory lets
 * the copies overlap; pageable memory works but is copied synchronously. The
 * buffers may be reused as soon as the call returns. */
int rgs_trainer_step_host_targets(rgs_ctx* ctx, const uint32_t* views, size_t nviews, const float* const* targets_rgba,
                                  const float bg[3], const rgs_loss_config* loss_cfg, const rgs_train_config* train_cfg,
                                  float* losses_out);

/* Render + backward only (mode as for rgs_trainer_step): gradients summed over
 * the views stay on the device for rgs_trainer_get_grads /
 * rgs_trainer_grad_buffer / rgs_trainer_apply_adam. */
int rgs_trainer_backward(rgs_ctx* ctx, const uint32_t* views, size_t nviews, const float bg[3],
                         const rgs_loss_config* loss_cfg, int mode, float* losses_out);
int rgs_trainer_get_grads(rgs_ctx* ctx, float* out /* n * 60 */);
/* Device gradient buffer (15 float4 planes of `plane_stride` Gaussians) for a
 * collective (e.g. an NCCL all-reduce across view-parallel ranks). */
int rgs_trainer_grad_buffer(rgs_ctx* ctx, void** device_ptr, size_t* bytes, size_t* plane_stride);
/* Adam over the device gradient buffer; grad_denom += denom_increment. */
int rgs_trainer_apply_adam(rgs_ctx* ctx, const rgs_train_config* cfg, uint32_t denom_increment);

int rgs_trainer_render(rgs_ctx* ctx, uint32_t view, const float bg[3], float* rgb_out);
int rgs_trainer_densify_and_prune(rgs_ctx* ctx, const rgs_train_config* cfg, float scene_extent, size_t* n_out);
int rgs_trainer_reset_opacities(rgs_ctx* ctx);
int rgs_trainer_get_adam_state(rgs_ctx* ctx, rgs_adam_state* state); /* fills caller arrays (len >= count) */
int rgs_trainer_set_adam_state(rgs_ctx* ctx, const rgs_adam_state* state);

/* Issue all work on `cuda_stream` (a cudaStream_t that is not the legacy
 * default stream), or on the context's own stream when NULL. */
int rgs_set_stream(rgs_ctx* ctx, void* cuda_stream);

/* Per-stage device timing of trainer steps (CUDA events between stages):
 * projection; compaction of the splats with tile pairs + depth sort; count
 * scans + (supertile, splat) entry emission; supertile sort; per-tile lists
 * (masks, scans, list writer); forward blend; loss; backward blend; geometry
 * backward + Adam. */
#define RGS_NUM_STAGES 9
#define RGS_STAGE_PROJECT 0
#define RGS_STAGE_DEPTH_SORT 1
#define RGS_STAGE_EMIT 2
#define RGS_STAGE_SUPERTILE_SORT 3
#define RGS_STAGE_TILE_LISTS 4
#define RGS_STAGE_FORWARD 5
#define RGS_STAGE_LOSS 6
#define RGS_STAGE_BACKWARD 7
#define RGS_STAGE_GEOMETRY_ADAM 8
int rgs_set_profiling(rgs_ctx* ctx, int on);
/* Milliseconds per stage accumulated since the last reset (reset != 0 clears). */
int rgs_get_stage_times(rgs_ctx* ctx, float* ms_out /* RGS_NUM_STAGES */, int reset);

/* Statistics of the last step or render. */
typedef struct rgs_stats {
    uint64_t pairs;         /* (Gaussian, tile) pairs over all views */
    uint64_t visible;       /* projected splats over all views */
    uint64_t pair_capacity; /* pair buffer capacity (batched mode) */
    uint32_t graph_captures;
    uint32_t overflow_retries;
    uint32_t view_groups;   /* groups the last batched step ran as: 1, or more
                               when its pairs passed 2^30 (each group within it) */
    uint32_t reserved;
    uint64_t supertile_entries; /* (supertile, splat) entries binned: each splat once
                                   per 4x4-tile supertile its tile rectangle meets */
} rgs_stats;
int rgs_get_stats(rgs_ctx* ctx, rgs_stats* out);

/* Device memory the context holds through its own buffers (parameters,
 * moments, targets, per-step work and pair buffers, sort scratch), and the
 * most it has held since it was created or since the last call with
 * reset_peak != 0 (which then restarts the high-water mark at the bytes held).
 * Either pointer may be NULL. The reference keeps no device state; this is
 * how the recompute and store-all backward variants report peak memory. */
int rgs_get_memory(rgs_ctx* ctx, uint64_t* held_bytes, uint64_t* peak_bytes, int reset_peak);

/* (pixel, splat) pairs the blend kernels evaluated in the trainer's most
 * recent batched pass (run as one view group): the forward walks each pixel's
 * tile list until the transmittance drops below 1e-4 (ending at the last
 * contributor) or the list ends, the backward walks from the last contributor
 * to the front (forward_pass / backward_pass, src/cpu/backward.rs:296-512).
 * The lists are the ones the pass blended (pruned to each row's reachable span
 * when the background is zero). The reference has no such counter: it is the
 * work measure of the blend kernels' FP32 roofline. RGS_ERR_INVALID_ARG when
 * no batched pass holds the pixel buffers. */
int rgs_trainer_evaluated_pairs(rgs_ctx* ctx, uint64_t* forward_pairs, uint64_t* backward_pairs);

/* ---- tiling and its autotuner ---------------------------------------------
 * Tile shape, splats staged per batch and pixels per thread change only how
 * the blend kernels are laid out, never a result (every combination is
 * bit-identical), so they may change between training steps. */
int rgs_get_options(rgs_ctx* ctx, rgs_options* out);
/* Switches the blend layout (same value sets as rgs_create); the next batched
 * step recaptures its graph. */
int rgs_set_tiling(rgs_ctx* ctx, int tile_w, int tile_h, int batch, int pixels_per_thread);

/* One autotuner measurement: device milliseconds per render + backward of the
 * tuned views (mean of `reps` batched steps without the optimiser update). */
typedef struct rgs_tune_entry {
    int tile_w, tile_h, batch, pixels_per_thread;
    float ms;
} rgs_tune_entry;
#define RGS_TUNE_CANDIDATES 18 /* {16x16, 8x32, 32x8} x {128, 256, 512} x {1, 2} */
/* Times every candidate layout on the trainer's current Gaussians and the
 * given views (render, loss and backward; parameters and Adam state are not
 * touched), keeps the fastest and returns it in *chosen. results may be NULL
 * or hold RGS_TUNE_CANDIDATES entries. */
int rgs_trainer_autotune(rgs_ctx* ctx, const uint32_t* views, size_t nviews, const float bg[3],
                         const rgs_loss_config* loss_cfg, int reps, rgs_tune_entry* results,
                         rgs_options* chosen);

#ifdef __cplusplus
}
#endif
#endif /* RGSPLAT_H */
