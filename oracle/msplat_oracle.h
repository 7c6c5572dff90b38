/*
 * msplat oracle C-ABI -- TEST INFRASTRUCTURE ONLY.
 *
 * Two shared libraries export exactly these symbols:
 *   oracle/_build/libmsplat_oracle.so  -- the CPU restatement in msplat_oracle.cpp
 *   oracle/_ref/libmsplat_ref.so       -- the reference's own core/cpu backend,
 *                                         compiled from its sources by oracle/Makefile
 * Tests load each with ctypes and compare them with each other (pinning the
 * restatement) and with the CUDA product (parity). Nothing in the product links,
 * loads or calls these libraries.
 *
 * Every pointer is a HOST pointer. Layouts follow core/metal/bindings.h:
 *   means (N,3)  scales (N,3) log-scales  quats (N,4) as (w,x,y,z), unnormalised
 *   features_dc (N,3)  features_rest (N,B-1,3)  opacities (N,1) logits
 *   viewmat / projmat row-major 4x4, images (H,W,3) float32.
 */
#ifndef MSPLAT_ORACLE_H
#define MSPLAT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Restatement only (the reference build does not export it): "reverse_sums" = 1 makes
 * the backward visit pixels and intersection slots in reverse order, i.e. the same
 * gradient sums in another float rounding order; "chunk_size" = C > 0 renders and
 * trains through depth-chunked compositing with C-long chunks (the Metal backend's
 * path for small frames), 0 through the one-pass compositing. Returns 0, or -1 if
 * unknown. */
int orc_set_option(const char *name, int value);

/* Prior-guided extras (core/metal/bindings.h:43-76, PriorStep), host pointers. The
 * prior set here applies to every later orc_render / orc_train_step until cleared with
 * NULL (the reference takes it as their last argument). Arrays the step updates
 * (sky texture, its gradient and moments, exposure parameters and moments, exposure
 * gradient, loss terms) are updated in place. */
typedef struct orc_prior {
    int aux;                    /* expected depth + per-pixel background */
    int sky;                    /* learned equirect sky behind the Gaussians */
    float *sky_tex, *sky_grad, *sky_exp_avg, *sky_exp_avg_sq;  /* (sky_h, sky_w, 3) */
    int sky_w, sky_h;
    float sky_frame[9];         /* up, e1 (azimuth 0), e2 (azimuth 90 degrees) */
    float sky_step_size, sky_bc2_sqrt;
    const float *prior_depth;   /* (prior_h, prior_w), scene units, 0 = invalid */
    const uint8_t *prior_aux;   /* (prior_h, prior_w, 4): confidence, sky, keep, - */
    int prior_w, prior_h, has_depth, has_sky_mask;
    float depth_weight, sky_weight, fill_weight, huber_delta, min_alpha;
    int mask_photometric;
    float *loss_terms;          /* [4]: depth, sky, fill, - (zeroed every step) */
    int exposure, cam_index;
    float *expo_params, *expo_exp_avg, *expo_exp_avg_sq;  /* (num_cams, 12) */
    float *expo_grad;           /* [12] or NULL, zeroed after each update */
    float expo_step_size, expo_bc2_sqrt, expo_reg;
    float log_max_scale_ratio;  /* needle cap; <= 0 disables */
} orc_prior;
int orc_set_prior(const orc_prior *prior);

/* core/metal/bindings.h:81-91 (msplat_render); writes the (H,W,3) image. */
int orc_render(int num_points, const float *means, const float *scales, float glob_scale,
               const float *quats, const float *viewmat, const float *projmat,
               float fx, float fy, float cx, float cy, unsigned img_height, unsigned img_width,
               int tiles_x, int tiles_y, float clip_thresh, unsigned degree, unsigned degrees_to_use,
               const float *cam_pos, const float *features_dc, const float *features_rest,
               const float *opacities, const float *background, float *out_img);

/* core/metal/bindings.h:100-118 (msplat_train_step). Parameters and Adam moments are
 * updated in place; group order means, scales, quats, features_dc, features_rest,
 * opacities; group_numel[g] = elements in group g. Returns the loss. */
float orc_train_step(int num_points, float *means, float *scales, float glob_scale, float *quats,
                     const float *viewmat, const float *projmat, float fx, float fy, float cx, float cy,
                     unsigned img_height, unsigned img_width, int tiles_x, int tiles_y, float clip_thresh,
                     unsigned degree, unsigned degrees_to_use, const float *cam_pos,
                     float *features_dc, float *features_rest, float *opacities, const float *background,
                     const float *gt, float ssim_weight, float loss_inv_n,
                     float **adam_exp_avg, float **adam_exp_avg_sq, const int64_t *group_numel,
                     const float *adam_step_sizes, const float *adam_bc2_sqrts,
                     float adam_beta1, float adam_beta2, float adam_eps,
                     float *vis_counts, float *xys_grad_norm, float *max_2d_size, float inv_max_dim);

/* Per-frame intermediates of the last render / train step, by name:
 *   xys depths conics colors aabb radii(i32) tile_start(i32) tile_end(i32)
 *   isect_gid(i32) out_img final_Ts final_idx(i32) v_rendered
 *   v_xy v_conic v_rgb v_opacity v_mean3d v_scale v_quat
 * and, with a prior set, out_depth bg_img v_aux (dL/d depth numerator, dL/d alpha per
 * pixel) v_depth (per Gaussian) out_adj v_adj (exposure-adjusted image, its gradient)
 * Returns the element count and sets *ptr to the library's internal storage
 * (valid until the next call), or -1 for an unknown name. */
int64_t orc_frame(const char *name, void **ptr);

/* core/metal/bindings.h:120-135 (msplat_densify); buffers are the capacity-sized
 * backing buffers (18 of them: 6 params, 6 exp_avg, 6 exp_avg_sq). Returns the new N. */
int orc_densify(int N, int buf_capacity, float grad_thresh, float size_thresh, float screen_thresh,
                int check_screen, float cull_alpha_thresh, float cull_scale_thresh, float cull_screen_size,
                int check_huge, const float *xys_grad_norm, const float *vis_counts, const float *max_2d_size,
                float half_max_dim, float *means, float *scales, float *quats, float *features_dc,
                float *features_rest, float *opacities, int fr_stride,
                float **adam_exp_avg, float **adam_exp_avg_sq, uint32_t seed);

/* core/metal/bindings.h:139 */
void orc_opacity_reset(float *opacities, float *exp_avg, float *exp_avg_sq, int num_points, float reset_logit);
/* core/metal/bindings.h:147 -- stable sort of keys by their low key_bits bits */
void orc_radix_sort(uint64_t *keys, int32_t *vals, uint32_t n, int key_bits);
/* core/metal/bindings.h:151 */
void orc_knn3_mean_dist(const float *points, uint32_t n, float *mean_dist);
/* core/metal/bindings.h:155 */
void orc_init_gaussians(const float *means, const uint8_t *rgb, uint32_t n, uint32_t seed, float opacity_logit,
                        float *scales, float *quats, float *features_dc, float *opacities);

/* core/metal/bindings.h:163-180 -- image pipeline, metrics, display */
void orc_resize_area(const void *src, int src_is_u8, int sw, int sh, float *dst, int dw, int dh);
void orc_undistort(const float *src, int sw, int sh, const float *intr, const float *dist,
                   int roi_x, int roi_y, float *dst, int dw, int dh);
void orc_image_metrics(const float *rendered, const float *gt, int h, int w, double *out3);
void orc_pack_rgba8(const float *img, uint32_t n, uint8_t *out);
void orc_finalize_depth(const float *depth_num, const float *final_T, uint32_t n, float inv_scale,
                        float *depth_out, float *alpha_out);

#ifdef __cplusplus
}
#endif
#endif
