/*
 * msplat_cuda.h -- C-ABI of the B200 (sm_100a) backend for msplat's splatting path.
 *
 * Each entry point replaces one function of the reference's backend contract,
 * core/metal/bindings.h, cited beside it. Differences from that C++ interface:
 *  - buffers are raw pointers with explicit sizes instead of MTensor;
 *  - every call takes a context (msplat_cuda_ctx) holding the CUDA stream and the
 *    per-frame cache that the reference keeps in a process global
 *    (core/cpu/msplat_cpu.cpp:436, core/metal/msplat_metal.mm:585);
 *  - every call returns a status code; msplat_cuda_last_error() gives the message
 *    (the reference throws std::runtime_error / std::invalid_argument).
 *
 * Pointer kinds. "device" pointers must be readable by the GPU (cudaMalloc, torch
 * CUDA tensors, or msplat_cuda_alloc's managed memory). "host" pointers (the 4x4
 * matrices, camera position, background, Adam scalars) are read before the call
 * returns. Work is enqueued on the context's stream and runs asynchronously unless
 * a function says it synchronises.
 *
 * Layouts (bindings.h): means (N,3), log-scales (N,3), quats (N,4) as (w,x,y,z),
 * features_dc (N,3), features_rest (N,B-1,3), opacity logits (N,1); viewmat and
 * projmat row-major 4x4; images (H,W,3) float32; tile grid ceil(W/16) x ceil(H/16).
 */
#ifndef MSPLAT_CUDA_H
#define MSPLAT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    MSPLAT_CUDA_OK = 0,
    MSPLAT_CUDA_EINVAL = 1,       /* bad argument (reference: std::invalid_argument) */
    MSPLAT_CUDA_ECUDA = 2,        /* CUDA runtime error */
    MSPLAT_CUDA_ECAPACITY = 3,    /* capacity exceeded (reference: core/cpu/msplat_cpu.cpp:1347) */
    MSPLAT_CUDA_EOVERFLOW = 4,    /* more than 2^31 tile intersections (msplat_cpu.cpp:546-547) */
    MSPLAT_CUDA_EUNSUPPORTED = 5  /* feature outside this backend (e.g. PriorStep extras) */
};

typedef struct msplat_cuda_ctx msplat_cuda_ctx;

/* Message of the last failed call on this thread. */
const char *msplat_cuda_last_error(void);
/* Library ABI version (major * 100 + minor). */
int msplat_cuda_version(void);

/* Context: stream + frame cache. bindings.h keeps one global; see msplat_cuda_default_ctx. */
int msplat_cuda_ctx_create(msplat_cuda_ctx **out);
void msplat_cuda_ctx_destroy(msplat_cuda_ctx *ctx);
msplat_cuda_ctx *msplat_cuda_default_ctx(void);
/* Stream for all later work of this context (a cudaStream_t; NULL = legacy default). */
int msplat_cuda_ctx_set_stream(msplat_cuda_ctx *ctx, void *stream);
/* Options: "keep_grads" (1 = keep per-Gaussian gradients for msplat_cuda_frame);
 * "graph" (1 = msplat_cuda_train_batch replays a captured CUDA graph of its step);
 * "raster_variant" (0..7: the rasterizer's shared-memory staging sizes, see
 * msplat_cuda_raster_variant; results do not depend on it, speed does);
 * "raster_shape" (0..2: the pixels a block of the batched forward composites --
 * 16 x 16, 16 x 8 or 8 x 8 -- each block walking its 16 x 16 tile's whole list, so
 * results do not depend on it; the reference's Metal rasterizer runs 8 x 8 thread
 * groups in its 16 x 16 bins, core/metal/msplat_metal.mm:1187-1197; see
 * msplat_cuda_raster_shape);
 * "stage_timing" (1 = time the stages, see msplat_cuda_drain_stage_times);
 * "store_transmittance" (K > 0: the forward stores each pixel's transmittance before
 * its first K contributions and the backward reads them instead of recovering T by
 * division, which the reference does (msplat_cpu.cpp:996-997); pixels with more
 * contributions fall back to division; 0 = off, the default);
 * "chunked_raster" (depth-chunked compositing of single-view render / train_step /
 * render_backward, the Metal backend's path for small frames,
 * core/metal/msplat_metal.metal:2641-3030 with its rule at msplat_metal.mm:1101-1117:
 * each tile's list in "chunk_len"-long pieces composited in parallel from T = 1, each
 * with its own early stop, merged per pixel front to back until T <= 1e-4. 0 = off,
 * one pass per tile as core/cpu (the default); 1 = frames of fewer than 400 tiles
 * without a prior, as the Metal backend; 2 = every frame without a prior. Images
 * differ from one pass by what the per-piece stops let through, about 1e-4; the
 * batched entry points always composite in one pass);
 * "chunk_len" (the piece length, 16..2^20, 512 by default as in the Metal backend).
 * Memory: a chunked frame holds per-piece planes of 36 bytes per tile pixel (9216 B
 * per piece), for up to intersections / chunk_len + tiles pieces: about 18 B per
 * intersection at 512, 576 B at 16 -- 10 M intersections at chunk_len 16 take some
 * 6 GB. */
int msplat_cuda_ctx_set_option(msplat_cuda_ctx *ctx, const char *name, int64_t value);
/* Staging sizes of rasterizer variant v (0..7): Gaussians per forward round, per
 * backward round, and the backward reduction's sub-batch. Returns the variant count. */
int msplat_cuda_raster_variant(int v, int32_t *fwd_batch, int32_t *bwd_batch, int32_t *bwd_sub);
/* Block shape s (0..2) of the batched forward: width and height in pixels. Returns the
 * shape count. */
int msplat_cuda_raster_shape(int s, int32_t *w, int32_t *h);
/* No counterpart in the reference (measurement). The (pixel, Gaussian) pairs the
 * reference's loops evaluate over the context's last single-view frame: out[0] for the
 * forward (core/cpu/msplat_cpu.cpp:574-626: each pixel walks its tile's list up to the
 * entry that ends it, or to the end), out[1] for the backward (:959-1031: from the
 * pixel's last contributor down). Synchronises the context's stream. */
int msplat_cuda_frame_pair_counts(msplat_cuda_ctx *ctx, int64_t *out);
/* The same counts added into d_sum[0..1] (device memory, two uint64) on the
 * context's stream, without synchronising: a training loop sums its steps' pairs and
 * reads them once. */
int msplat_cuda_frame_pair_counts_device(msplat_cuda_ctx *ctx, uint64_t *d_sum);
/* No counterpart in the reference (test hook). The rasterizers' exponential -- exp(x)
 * for x in [-700, 0], Tang's table-driven method in double precision, rounded once to
 * float -- of n device inputs into out, on the context's stream. Over [-5.55, 0] it
 * runs both forms the kernels use (the forward's table of 2^(k/64) spanning the range
 * and the backward's 64-entry table with the power of two applied to the exponent)
 * and writes NaN wherever they differ. */
int msplat_cuda_rasterizer_exp(msplat_cuda_ctx *ctx, const float *x, int64_t n, float *out);
/* Bytes of device memory the context's caches hold. */
int64_t msplat_cuda_ctx_device_bytes(msplat_cuda_ctx *ctx);

/* bindings.h:8 cleanup_msplat_metal -- release the context's cached buffers. */
int msplat_cuda_cleanup(msplat_cuda_ctx *ctx);
/* bindings.h:22 msplat_commit -- work is already submitted; kept for symmetry. */
int msplat_cuda_commit(msplat_cuda_ctx *ctx);
/* bindings.h:25 msplat_gpu_sync -- wait for the context's stream. */
int msplat_cuda_sync(msplat_cuda_ctx *ctx);
/* bindings.h:18-19 gpu_zeros / gpu_empty -- managed (host- and device-visible) memory. */
int msplat_cuda_alloc(size_t bytes, int zero, void **out);
int msplat_cuda_free(void *ptr);
/* No counterpart in the reference. Plain device memory (cudaMalloc; release with
 * msplat_cuda_free), for callers that stage host data themselves with
 * msplat_cuda_copy_buffer -- the bindings.h layer keeps its per-tensor staging in it. */
int msplat_cuda_device_alloc(size_t bytes, void **out);

/* bindings.h:143 msplat_copy_buffer -- copy `bytes` from src to dst, ordered on the
 * context's stream (any mix of device, managed and host memory). */
int msplat_cuda_copy_buffer(msplat_cuda_ctx *ctx, void *dst, const void *src, size_t bytes);

/* bindings.h:81-91 msplat_render. *out_img receives a device pointer to the (H,W,3)
 * image in the frame cache, valid until the next call on this context (the
 * reference likewise returns an alias of its cache, msplat_cpu.cpp:1196). */
int msplat_cuda_render(msplat_cuda_ctx *ctx, int num_points, const float *means3d, const float *scales,
                       float glob_scale, const float *quats, const float *viewmat, const float *projmat,
                       float fx, float fy, float cx, float cy, unsigned img_height, unsigned img_width,
                       int tiles_x, int tiles_y, float clip_thresh, unsigned degree, unsigned degrees_to_use,
                       const float *cam_pos, const float *features_dc, const float *features_rest,
                       const float *opacities, const float *background, const float **out_img);

/* One view of a batched render: a scene (device parameter arrays, layouts as
 * msplat_render) seen by one camera, and the device (H,W,3) image to write. */
typedef struct msplat_cuda_view {
    int32_t num_points;
    const float *means3d, *scales, *quats, *features_dc, *features_rest, *opacities;
    float glob_scale;
    uint32_t degree, degrees_to_use;
    float viewmat[16], projmat[16]; /* row-major */
    float fx, fy, cx, cy;
    uint32_t img_height, img_width;
    float clip_thresh;
    float cam_pos[3];
    float background[3];
    float *out_img;
} msplat_cuda_view;

/* Batched msplat_render (no counterpart in the reference, whose render takes one
 * view, bindings.h:81-91): n_views views of any scenes and resolutions rendered by one
 * projection launch, one sort and one persistent rasterizer launch that pulls
 * (view, tile) work items. Each image equals what msplat_cuda_render gives for that
 * view alone, bit for bit. Synchronises once (the intersection count sizes the sort). */
int msplat_cuda_render_batch(msplat_cuda_ctx *ctx, int32_t n_views, const msplat_cuda_view *views);

/* One view of a batched training step: a camera and its device (H,W,3) target. */
typedef struct msplat_cuda_train_view {
    float viewmat[16], projmat[16]; /* row-major */
    float fx, fy, cx, cy;
    uint32_t img_height, img_width;
    float cam_pos[3];
    const float *gt;
} msplat_cuda_train_view;

/* Batched msplat_train_step (no counterpart in the reference, whose train step takes
 * one view, bindings.h:100-118): n_views views of one scene, of any resolutions,
 * trained in one step. Each view's loss is msplat's L1 + ssim_weight (1 - SSIM) with
 * its gradient scaled by 1 / (3 W H), as the single-view step scales it; the
 * gradients are summed over the views and ONE Adam step is applied (groups and
 * scalars as msplat_cuda_train_step). The densification statistics advance once per
 * view that sees a Gaussian. grads_out (NULL, or 6 device arrays in parameter layout)
 * receives the summed gradients. losses_out (host, n_views floats, or NULL) receives
 * each view's loss. A one-view batch gives msplat_cuda_train_step's update.
 * With the context option "graph" = 1, steps after the first replay a CUDA graph of
 * the whole step (projection to Adam; re-captured when a shape or buffer changes).
 * Synchronises once per call (the intersection count, or the graph's completion). */
int msplat_cuda_train_batch(msplat_cuda_ctx *ctx, int num_points, float *means3d, float *scales, float glob_scale,
                            float *quats, float *features_dc, float *features_rest, float *opacities,
                            unsigned degree, unsigned degrees_to_use, float clip_thresh, const float *background,
                            int32_t n_views, const msplat_cuda_train_view *views, float ssim_weight,
                            int num_adam_groups, float *const *adam_exp_avg, float *const *adam_exp_avg_sq,
                            const float *adam_step_sizes, const float *adam_bc2_sqrts, float adam_beta1,
                            float adam_beta2, float adam_eps, float *vis_counts, float *xys_grad_norm,
                            float *max_2d_size, float *const *grads_out, float *losses_out);
/* Graph statistics of msplat_cuda_train_batch: out4 = replays, captures, overflowed
 * steps (repeated without the graph), per-intersection capacity. */
int msplat_cuda_train_batch_stats(msplat_cuda_ctx *ctx, int64_t *out4);

/* bindings.h:100-118 msplat_train_step: forward, L1 + SSIM loss, backward, Adam on the
 * six parameter groups (means, scales, quats, features_dc, features_rest, opacities --
 * the parameter arrays themselves, which the reference's adam_params alias,
 * core/src/model.cpp:644-646), and the densification statistics. Adam runs only when
 * num_adam_groups >= 5, as in the reference (msplat_cpu.cpp:1273). *radii_out (may be
 * NULL) receives a device pointer to the int32 radii in the frame cache. When
 * loss_out is not NULL the call synchronises and writes the loss; otherwise the loss
 * stays on the device (msplat_cuda_loss_device). */
int msplat_cuda_train_step(msplat_cuda_ctx *ctx, int num_points, float *means3d, float *scales, float glob_scale,
                           float *quats, const float *viewmat, const float *projmat, float fx, float fy, float cx,
                           float cy, unsigned img_height, unsigned img_width, int tiles_x, int tiles_y,
                           float clip_thresh, unsigned degree, unsigned degrees_to_use, const float *cam_pos,
                           float *features_dc, float *features_rest, float *opacities, const float *background,
                           const float *gt, float ssim_weight, float loss_inv_n, int num_adam_groups,
                           float *const *adam_exp_avg, float *const *adam_exp_avg_sq, const float *adam_step_sizes,
                           const float *adam_bc2_sqrts, float adam_beta1, float adam_beta2, float adam_eps,
                           float *vis_counts, float *xys_grad_norm, float *max_2d_size, float inv_max_dim,
                           const int32_t **radii_out, float *loss_out);

/* bindings.h:43-77 PriorStep, the last argument of msplat_render (bindings.h:90) and
 * msplat_train_step (bindings.h:126): prior-guided extras for street captures. Device
 * pointers; the step updates in place the arrays it trains (sky texture and its
 * moments and gradient, exposure parameters and moments, exposure gradient, loss
 * terms).
 *   aux          rasterize the expected-depth numerator and a per-pixel background
 *                (required by the sky and by every prior loss)
 *   sky          learned equirect sky (sky_h, sky_w, 3) composited behind the Gaussians
 *   prior_*      per-camera depth prior (prior_h, prior_w; 0 = invalid) and aux map
 *                (prior_h, prior_w, 4 bytes: confidence, sky >= 128, keep >= 128, -)
 *                at their own resolution; loss weights; loss_terms[4] = depth, sky,
 *                fill, - (zeroed by every train step, then accumulated)
 *   exposure     affine colour transform per camera (num_cams, 12: row-major M, then
 *                b) applied to the render before the photometric loss, trained by
 *                Adam with an L2 pull towards identity; expo_grad[12] (may be NULL)
 *                is added to its gradient and zeroed
 *   log_max_scale_ratio  needle cap after the update: largest log-scale <= middle one
 *                + this (<= 0 disables). */
typedef struct msplat_cuda_prior {
    int32_t aux, sky;
    float *sky_tex, *sky_grad, *sky_exp_avg, *sky_exp_avg_sq;
    int32_t sky_w, sky_h;
    float sky_frame[9]; /* up, e1 (azimuth 0), e2 (azimuth 90 degrees) */
    float sky_step_size, sky_bc2_sqrt;
    const float *prior_depth;
    const uint8_t *prior_aux;
    int32_t prior_w, prior_h, has_depth, has_sky_mask;
    float depth_weight, sky_weight, fill_weight, huber_delta, min_alpha;
    int32_t mask_photometric;
    float *loss_terms;
    int32_t exposure, cam_index;
    float *expo_params, *expo_exp_avg, *expo_exp_avg_sq, *expo_grad;
    float expo_step_size, expo_bc2_sqrt, expo_reg;
    float log_max_scale_ratio;
    int32_t expo_num_cams; /* rows of expo_params: cam_index is checked against it (0 = unchecked) */
} msplat_cuda_prior;
/* Sets the PriorStep of this context's later msplat_cuda_render and
 * msplat_cuda_train_step calls (NULL restores the plain pipeline, the reference's
 * default). The struct is copied; the arrays it points to must stay valid while it
 * is set. Fails on inconsistent fields (a sky without its texture or moments,
 * exposure without its moments or with cam_index outside expo_num_cams, a prior_aux
 * map not 4-byte aligned). */
int msplat_cuda_set_prior(msplat_cuda_ctx *ctx, const msplat_cuda_prior *prior);
/* bindings.h:93-96 msplat_render_aux_outputs: after a render or train step with aux
 * set, device pointers to the expected-depth numerator sum_i w_i z_i (H, W) and the
 * final transmittance (H, W) in the frame cache. */
int msplat_cuda_render_aux_outputs(msplat_cuda_ctx *ctx, const float **depth, const float **final_T);

/* bindings.h:120-135 msplat_densify. The 18 buffers are capacity-sized (buf_capacity
 * rows): params[6] = means, scales, quats, features_dc, features_rest (fr_stride
 * floats per row), opacities; exp_avg[6] / exp_avg_sq[6] likewise. Requires
 * 3*N <= buf_capacity (else MSPLAT_CUDA_ECAPACITY, as the reference throws,
 * msplat_cpu.cpp:1347). Synchronises once and writes the new count to *new_count. */
int msplat_cuda_densify(msplat_cuda_ctx *ctx, int N, int buf_capacity, float grad_thresh, float size_thresh,
                        float screen_thresh, int check_screen, float cull_alpha_thresh, float cull_scale_thresh,
                        float cull_screen_size, int check_huge, const float *xys_grad_norm, const float *vis_counts,
                        const float *max_2d_size, float half_max_dim, float *const *params, int fr_stride,
                        float *const *exp_avg, float *const *exp_avg_sq, uint32_t seed, int *new_count);

/* bindings.h:139 msplat_opacity_reset -- logits clamped to <= reset_logit, the opacity
 * group's Adam moments zeroed. */
int msplat_cuda_opacity_reset(msplat_cuda_ctx *ctx, float *opacities, float *exp_avg, float *exp_avg_sq,
                              int num_points, float reset_logit);

/* bindings.h:147 msplat_radix_sort -- stable sort of (keys, vals) by the low key_bits
 * bits of the keys, in place (device pointers). */
int msplat_cuda_radix_sort(msplat_cuda_ctx *ctx, uint64_t *keys, int32_t *vals, uint32_t n, int key_bits);

/* No counterpart in the reference. The same stable radix sort as
 * msplat_cuda_radix_sort for callers that may not allocate GPU memory when they sort:
 * a serving process whose HBM is fully committed to resident scenes, a render loop
 * that cannot take the device-wide synchronisation of cudaMalloc / cudaFree, a plugin
 * host that forbids libraries to allocate. It allocates nothing and takes no context:
 * its scratch is one fixed array in device memory (MSPLAT_STATIC_SORT_BYTES, held on
 * every GPU that loads the library until the process exits), so n is limited to
 * MSPLAT_STATIC_SORT_MAX_KEYS (larger n returns MSPLAT_CUDA_ECAPACITY with a message
 * in msplat_cuda_last_error). The first call on each device looks up the array's
 * device address (cudaGetSymbolAddress) with that device current; make that first
 * call before any stream capture begins. All calls share the one array, so calls
 * whose work overlaps on the GPU (other streams, other host threads) race and must be
 * serialised by the caller. Work is enqueued on `stream` (a cudaStream_t, NULL = the
 * legacy default stream). The address is kept per device ordinal for the life of the
 * process: after cudaDeviceReset, or from a driver context other than the device's
 * primary context, the kept address is stale, so neither is supported. A CUDA error
 * already pending when the call begins is reported as such (MSPLAT_CUDA_ECUDA, "pending
 * error") and nothing is enqueued. */
#define MSPLAT_STATIC_SORT_MAX_KEYS (1u << 20)
#define MSPLAT_STATIC_SORT_BYTES (13u * 1024u * 1024u + 4096u)
int msplat_cuda_radix_sort_static(void *stream, uint64_t *keys, int32_t *vals, uint32_t n, int key_bits);

/* bindings.h:151 msplat_knn3_mean_dist -- exact mean distance from each of n points
 * (n, 3) to its 3 nearest other points. */
int msplat_cuda_knn3_mean_dist(msplat_cuda_ctx *ctx, const float *points, uint32_t n, float *mean_dist);

/* bindings.h:155 msplat_init_gaussians -- 3-NN isotropic log-scales, random rotations,
 * DC from RGB (uint8, n x 3), constant opacity logit. */
int msplat_cuda_init_gaussians(msplat_cuda_ctx *ctx, const float *means, const uint8_t *rgb, uint32_t n,
                               uint32_t seed, float opacity_logit, float *scales, float *quats, float *features_dc,
                               float *opacities);

/* Image pipeline, metrics, display (bindings.h:158-180). Image pointers are device
 * pointers unless said otherwise; results equal the reference's bit for bit. */

/* bindings.h:163 msplat_resize_area -- area (box) resample to (dh, dw, 3) float RGB;
 * src is (sh, sw, 4) RGBA8 when src_is_u8, else (sh, sw, 3) float RGB. */
int msplat_cuda_resize_area(msplat_cuda_ctx *ctx, const void *src, int src_is_u8, int sw, int sh, float *dst, int dw,
                            int dh);
/* bindings.h:167-168 msplat_undistort -- Brown-Conrady undistortion of (sh, sw, 3) into
 * the (dh, dw, 3) crop at (roi_x, roi_y); intr (host) = fx fy cx cy, dist (host) =
 * k1 k2 p1 p2 k3. */
int msplat_cuda_undistort(msplat_cuda_ctx *ctx, const float *src, int sw, int sh, const float *intr,
                          const float *dist, int roi_x, int roi_y, float *dst, int dw, int dh);
/* bindings.h:172 msplat_image_metrics -- PSNR, SSIM (11-tap Gaussian, clamp-to-edge)
 * and L1 of two (h, w, 3) images into out[3] (host). Synchronises. */
int msplat_cuda_image_metrics(msplat_cuda_ctx *ctx, const float *rendered, const float *gt, int h, int w,
                              double *out);
/* bindings.h:175 msplat_pack_rgba8 -- float RGB (n, 3) to RGBA8 (n, 4) written to out
 * (host or device). Synchronises. */
int msplat_cuda_pack_rgba8(msplat_cuda_ctx *ctx, const float *img, uint32_t n, uint8_t *out);
/* bindings.h:179-180 msplat_finalize_depth -- expected depth (depth_num / alpha *
 * inv_scale, 0 where alpha <= 1e-4) and alpha = 1 - final_T. */
int msplat_cuda_finalize_depth(msplat_cuda_ctx *ctx, const float *depth_num, const float *final_T, uint32_t n,
                               float inv_scale, float *depth_out, float *alpha_out);

/* Gradient-only backward of the last msplat_cuda_render on this context (same scene
 * and camera), for differentiable rendering (torch.autograd): given dL/d(image)
 * (H,W,3, device), writes dL/d(means, log-scales, quats, features_dc, features_rest,
 * opacity logits) to the six device arrays, zero for Gaussians the render did not
 * use. Composes rasterize_backward, reduce_isect_grads and the projection / SH VJPs
 * (core/cpu/msplat_cpu.cpp:959-1139) without the fused Adam. */
int msplat_cuda_render_backward(msplat_cuda_ctx *ctx, int num_points, const float *means3d, const float *scales,
                                float glob_scale, const float *quats, const float *viewmat, const float *projmat,
                                float fx, float fy, float cx, float cy, unsigned img_height, unsigned img_width,
                                int tiles_x, int tiles_y, float clip_thresh, unsigned degree, unsigned degrees_to_use,
                                const float *cam_pos, const float *background, const float *v_img, float *v_means,
                                float *v_scales, float *v_quats, float *v_features_dc, float *v_features_rest,
                                float *v_opacities);

/* The training loss of msplat_train_step on its own (core/cpu/msplat_cpu.cpp:669-785):
 * L1 + ssim_weight * (1 - SSIM), forward and backward in one pass. Writes
 * loss_inv_n-scaled dL/d(img) to v_img and the loss (sum / (H*W)) to the device
 * scalar *loss. All pointers are device pointers. */
int msplat_cuda_ssim_loss(msplat_cuda_ctx *ctx, const float *img, const float *gt, unsigned img_height,
                          unsigned img_width, float ssim_weight, float loss_inv_n, float *v_img, float *loss);

/* Device pointer of the last train step's loss (float, sum / (H*W)). */
int msplat_cuda_loss_device(msplat_cuda_ctx *ctx, const float **loss);

/* Per-frame intermediates of the last render / train step (test and debug hook, like
 * the reference's _gpu_* hooks, python/bindings.cpp:655-738). Names: splats (N x 12
 * floats: x y conic_a conic_b | conic_c sigmoid(opacity) r g | b depth - -), radii,
 * aabb, tile_start, tile_end, isect_gid, slots (per sorted intersection the 9 gradient
 * sums of its tile: xy conic rgb opacity-logit), out_img, final_Ts, final_idx, v_rendered and,
 * with option keep_grads, v_xy v_conic v_rgb v_opacity v_mean3d v_scale v_quat; with a
 * prior (msplat_cuda_set_prior): out_depth bg_img v_aux (dL/d depth numerator, dL/d
 * alpha per pixel) out_adj v_adj (exposure-adjusted render and its gradient) and,
 * with keep_grads, v_depth; and knn_evals (one uint64 as two int32 words: the point
 * distances the last msplat_cuda_knn3_mean_dist computed, 32 per query per candidate
 * box its bounds test kept). *count is the element count (floats or int32). Device
 * pointers. */
int msplat_cuda_frame(msplat_cuda_ctx *ctx, const char *name, const void **dev_ptr, int64_t *count);
/* Number of tile intersections of the last frame. */
int64_t msplat_cuda_num_isects(msplat_cuda_ctx *ctx);

/* bindings.h:34-39 msplat_enable_gpu_timing / msplat_drain_stage_times. With option
 * "stage_timing" set, each render / train step records CUDA events at its stage
 * boundaries (proj_sh_fwd, bin_sort, rast_fwd, loss_fwd_bwd, rast_bwd,
 * proj_sh_bwd_adam); they are read back lazily, so timing adds no synchronisation to
 * the calls. This waits for the recorded events, returns the milliseconds and call
 * counts accumulated since the last drain, and resets them. */
int msplat_cuda_drain_stage_times(msplat_cuda_ctx *ctx, double *ms, int64_t *calls, int max_stages, int *n_stages,
                                  const char **names);

#ifdef __cplusplus
}
#endif
#endif
