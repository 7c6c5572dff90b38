// Internal launch interface between the C-ABI layer (capi.cu) and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace msplat {

// Records a message for msplat_cuda_last_error() and returns code (capi.cu).
int report_error(int code, const char *msg);

// One view: the scalars msplat_render / msplat_train_step take about the camera.
struct CamParams {
    float viewmat[16];  // row-major world-to-camera
    float projmat[16];  // row-major clip-from-world
    float fx, fy, cx, cy;
    float cam_pos[3];
    uint32_t width, height;
    int tiles_x, tiles_y;
    float clip;
    uint32_t degree, degrees_to_use;
};

struct ProjectArgs {
    int n;
    const float *means, *scales, *quats, *features_dc, *features_rest, *opacities;
    int rest_stride;  // floats per Gaussian in features_rest
    float glob_scale;
    CamParams cam;
    Splat *splats;
    int32_t *radii;
    float *aabb;
    int32_t *n_tiles;
};
void launch_project(const ProjectArgs &a, cudaStream_t st);

int scan_blocks(int n);
template <typename TO>
void scan_exclusive(const int32_t *in, TO *out, int n, TO *d_total, TO *partials, cudaStream_t st);

// Depth order of n Gaussians (stable) and their emission offsets in that order:
// offsets[g] = tiles of every Gaussian before g by (depth, index); *d_total = all.
struct DepthScratch {
    uint32_t *keys[2], *vals[2];  // n each
    int32_t *counts;              // n
    int64_t *off_sorted;          // n
    void *radix_scratch;          // radix_scratch_bytes(n)
};
void launch_depth_offsets(int n, const Splat *splats, const int32_t *n_tiles, DepthScratch &s, int64_t *offsets,
                          int64_t *d_total, int64_t *scan_part, cudaStream_t st);
// Emission: key = tile id (global tile id in a batch), value = emission index, or
// the Gaussian id when emit_gid is null (render only: no backward needs the map).
// cap: entries at or past it are not written (the buffers' capacity)
void launch_emit_keys(int n, const Splat *splats, const float *aabb, const int32_t *n_tiles, const int64_t *offsets,
                      int tiles_x, int tiles_y, uint32_t *keys, uint32_t *vals, int32_t *emit_gid, cudaStream_t st,
                      int64_t cap = INT64_MAX);
size_t radix_scratch_bytes(int n);
// d_n / d_T (optional): device-side counts capping the host-side capacities n / T
int radix_sort_pairs(uint64_t *k[2], uint32_t *v[2], int n, int key_bits, void *scratch, cudaStream_t st,
                     const int *d_n = nullptr);
int radix_sort_pairs32(uint32_t *k[2], uint32_t *v[2], int n, int key_bits, void *scratch, cudaStream_t st,
                       const int *d_n = nullptr);
void launch_tile_ranges(const uint32_t *keys, int n, int T, int32_t *tile_start, int32_t *tile_end, cudaStream_t st,
                        const int *d_n = nullptr, const int *d_T = nullptr);
void launch_isect_map(const uint32_t *sorted_e, int n, const int32_t *emit_gid, int32_t *isect_gid, int32_t *inv,
                      cudaStream_t st, const int *d_n = nullptr);
void launch_clamp_count(const int64_t *total, int64_t cap, int *d_n, int *overflow, cudaStream_t st);

struct RasterArgs {
    int W, H, tiles_x, tiles_y;
    const int32_t *tile_start, *tile_end, *isect_gid;
    const Splat *splats;
    float bg[3];
    float *out_img, *final_T;
    int32_t *final_idx;
    // stored-transmittance mode (null = off): T before each contribution, slot-major
    // ([tcap][W*H]), and the per-pixel count (-1 when it exceeded tcap)
    float *tstore;
    int32_t *tcount;
    int tcap;
    // prior-guided aux mode (launch_raster_fwd_aux): expected-depth numerator
    // sum_i z_i w_i per pixel, and the per-pixel background -- read from bg_img when
    // a sky pass filled it (sky_bg = 1), else bg written there
    float *out_depth, *bg_img;
    int sky_bg;
};
// Rasterizer staging variants, chosen at run time (an autotuner times them): the
// Gaussians staged in shared memory per forward round and per backward round, and
// the backward's reduction sub-batch. Every variant computes the same images and
// gradients (staging changes no arithmetic); variant 0 is the default.
struct RasterVariant {
    int fwd_batch, bwd_batch, bwd_sub;
};
constexpr int N_RASTER_VARIANTS = 8;
constexpr RasterVariant RASTER_VARIANTS[N_RASTER_VARIANTS] = {
    {128, 128, 3}, {128, 64, 3}, {128, 64, 4}, {256, 128, 3}, {64, 128, 3}, {256, 64, 4}, {128, 32, 4}, {256, 128, 4}};
inline int variant_index(int v) { return (v >= 0 && v < N_RASTER_VARIANTS) ? v : 0; }

// Block shapes of the batched forward rasterizer (pixels a block composites; every
// shape walks the 16 x 16 tile's list, so all give the same bits): 16 x 16 (the
// default), 16 x 8 and 8 x 8 (the reference's Metal thread-group shape).
struct RasterShape {
    int w, h;
};
constexpr int N_RASTER_SHAPES = 3;
constexpr RasterShape RASTER_SHAPES[N_RASTER_SHAPES] = {{16, 16}, {16, 8}, {8, 8}};
inline int shape_index(int s) { return (s >= 0 && s < N_RASTER_SHAPES) ? s : 0; }

void launch_raster_fwd(const RasterArgs &a, cudaStream_t st, int variant = 0, int shape = 0);
// (pixel, Gaussian) pairs the reference's forward / backward loops evaluate over the
// frame (out[0], out[1]; device counters, zeroed first unless accumulate)
void launch_pair_counts(const RasterArgs &a, unsigned long long *d_out, cudaStream_t st, bool accumulate = false);
// the rasterizers' exponential (exp_tab) of n device inputs
void launch_exp_tab(const float *x, int64_t n, float *out, cudaStream_t st);
void launch_raster_fwd_aux(const RasterArgs &a, cudaStream_t st, int shape = 0);

struct RasterBwdArgs;
// Depth-chunked compositing (core/metal/msplat_metal.metal:2641-3030): every tile's
// list split into chunk_len-long pieces, tile t's pieces being work items first[t] ..
// first[t + 1] - 1 (first[T] = all items). Per (item, thread of the tile block): the
// piece's own transmittance and colour composited from T = 1, its last contributor
// (-1 once the pixel's merged transmittance is spent), and for the backward the
// transmittance in front of the piece and the colour behind it. Planes are [item][256]
// (cT, clast, pre) and [item][3][256] (cC, aft).
struct ChunkArgs {
    int chunk_len;
    int32_t *first;  // [tiles + 1]
    float *cT, *cC, *pre, *aft;
    int32_t *clast;
};
// Items of each tile, their exclusive scan into first (first[T] = all); counts and
// partials are scratch of T and scan_blocks(T) + 1 entries.
void launch_chunk_items(const int32_t *tile_start, const int32_t *tile_end, int T, int chunk_len, int32_t *counts,
                        int32_t *first, int32_t *partials, cudaStream_t st);
// Pieces of at most item_cap items (a host bound on first[T]), then the per-pixel
// merge into a.out_img / final_T / final_idx.
void launch_raster_fwd_chunked(const RasterArgs &a, const ChunkArgs &c, int64_t item_cap, cudaStream_t st,
                               int variant = 0);
// Backward: prefix transmittance and suffix colour per (item, pixel), then the pieces
// back to front into a.slots.
void launch_raster_bwd_chunked(const RasterBwdArgs &a, const ChunkArgs &c, int64_t item_cap, cudaStream_t st,
                               int variant = 0);

// A batch of views rendered by one projection, one sort and one persistent raster
// launch. Instances (view, Gaussian) and tiles (view, tile) are numbered globally,
// view after view; every array lives in device memory.
struct BatchDesc {
    int n_views;
    const int *inst_off;       // [n_views + 1] first instance of each view
    const int *tile_off;       // [n_views + 1] first global tile of each view
    const int *tiles_x, *tiles_y;
    const ProjectArgs *proj;   // per view; outputs point at the batch-wide arrays
    const RasterArgs *raster;  // per view; tile ranges and lists are batch-wide
};

// The view that holds global index g: the last v with off[v] <= g (views with no
// instances share their offset with the next view and are skipped).
__device__ __forceinline__ int find_view(const int *off, int n_views, int g) {
    int lo = 0, hi = n_views - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

void launch_project_batch(const BatchDesc &d, int total, cudaStream_t st);
// ds (may be null): threads take Gaussians in ds's depth order (after
// launch_depth_offsets) instead of by index; the entries are the same.
void launch_emit_keys_batch(int n, const Splat *splats, const float *aabb, const int32_t *n_tiles,
                            const int64_t *offsets, const DepthScratch *ds, const BatchDesc &d, uint32_t *keys,
                            uint32_t *vals, int32_t *emit_gid, cudaStream_t st, int64_t cap = INT64_MAX);
void launch_raster_fwd_batch(const BatchDesc &d, int tiles_hint, int *d_counter, cudaStream_t st, int variant = 0,
                             int shape = 0);

struct RasterBwdArgs {
    int W, H, tiles_x, tiles_y;
    const int32_t *tile_start, *tile_end, *isect_gid;
    const Splat *splats;
    float bg[3];
    const float *final_T;
    const int32_t *final_idx;
    const float *v_out;
    float *slots;  // 9 floats per sorted intersection
    const float *tstore;  // stored-transmittance mode, as RasterArgs (null = divide)
    const int32_t *tcount;
    // aux mode (launch_raster_bwd_aux): per-pixel background, dL/d(depth numerator,
    // alpha) per pixel, and the depth-gradient slot of each intersection
    const float *bg_img, *v_aux;
    float *slots_depth;
};
void launch_raster_bwd(const RasterBwdArgs &a, cudaStream_t st, int variant = 0);
void launch_raster_bwd_aux(const RasterBwdArgs &a, cudaStream_t st);

struct SsimArgs {
    int W, H;
    const float *img, *gt;
    float ssim_weight, inv_n;
    float *v_out;
    double *partials;  // one per 32x32 block
    float *loss;       // device scalar: sum / (W * H)
};
int ssim_blocks(int W, int H);
void launch_ssim_loss(const SsimArgs &a, cudaStream_t st);

struct BackwardArgs {
    int n;
    const float *means, *scales, *quats;
    float glob_scale;
    CamParams cam;
    const Splat *splats;
    const int32_t *radii, *n_tiles, *inv;
    const int64_t *offsets;
    const float *slots;
    const float *slots_depth;  // aux mode: one depth-gradient value per intersection (else null)
    // optional per-Gaussian gradient outputs (null to skip)
    float *v_xy, *v_conic, *v_rgb, *v_opacity, *v_mean3d, *v_scale, *v_quat, *v_depth;
    float *g_dc, *g_rest;  // SH gradients as arrays (gradient-only mode, no Adam)
    // Adam: groups means, scales, quats, dc, rest, opacity
    int do_adam;
    float *p[6], *m1[6], *m2[6];
    float ss[6], bc2[6];
    float beta1, beta2, eps;
    int rest_stride;
    // densification statistics (null to skip)
    float *vis_counts, *xys_grad_norm, *max_2d_size;
    float inv_max_dim;
    float log_max_scale_ratio;  // needle cap after the scale update; <= 0 disables
};
void launch_backward_adam(const BackwardArgs &a, cudaStream_t st);

// Multi-view backward + Adam: instances v * n + i of Gaussian i in each view v.
struct BackwardBatchArgs {
    int n, n_views;
    const ProjectArgs *proj;   // per view (device): the camera
    const float *inv_max_dim;  // per view (device): 1 / max(W, H)
    const float *means, *scales, *quats;
    float glob_scale;
    uint32_t degrees_to_use;
    const Splat *splats;
    const int32_t *radii, *n_tiles, *inv;
    const int64_t *offsets;
    const float *slots;
    float *g[6];  // optional summed gradients (null g[0] to skip): means scales quats dc rest opacity
    int do_adam;
    float *p[6], *m1[6], *m2[6];
    const float *adam_scalars;  // device: step sizes [6], then bias-correction square roots [6]
    float beta1, beta2, eps;
    int rest_stride;
    float *vis_counts, *xys_grad_norm, *max_2d_size;  // null to skip
    const int *skip;  // device flag (capacity overflow): when set the kernel changes nothing
};
void launch_backward_adam_batch(const BackwardBatchArgs &a, cudaStream_t st);
void launch_raster_bwd_batch(const RasterBwdArgs *d_views, const int *d_tile_off, int n_views, int *d_counter,
                             cudaStream_t st, int variant = 0);
void launch_ssim_loss_batch(const SsimArgs *d_views, const int *d_boff, int n_views, int *d_counter, cudaStream_t st);

struct DensifyArgs {
    int n;
    float grad_thresh, size_thresh, screen_thresh;
    int check_screen;
    float cull_alpha, cull_scale, cull_screen;
    int check_huge;
    const float *grad_norm, *vis_counts, *max_2d;
    float half_max_dim, log_size_fac;
    uint32_t seed;
    float *buf[6], *m1[6], *m2[6];  // capacity-sized: means scales quats dc rest opacity
    int stride[6];
    int64_t cap;  // rows of every buffer: the rows after splits and clones must fit
};
struct DensifyScratch {
    int32_t *split, *dup, *split_ord, *dup_ord, *keep, *keep_ord;  // 4N rows each
    int32_t *n_split, *n_dup, *n_new, *new_count, *scan_part;
    int32_t *overflow;  // set when N + 2 splits + clones exceeds cap (nothing is written)
    int32_t *row_parent;  // 3N: the parent of each new row (split children, then clones)
    float *scratch;     // 4N x max(stride) floats
};
void launch_densify(const DensifyArgs &a, DensifyScratch &s, cudaStream_t st);
void launch_opacity_reset(float *o, float *m1, float *m2, int n, float reset_logit, cudaStream_t st);

// Image pipeline, metrics and display (image.cu).
struct MetricsScratch {
    float *hbuf;            // h * w * 15
    float *t_ssim, *t_l1;   // h * w * 3
    double *t_sq;           // h * w * 3
    double *rows;           // h * 3
};
void launch_resize_area(const void *src, int u8in, int sw, int sh, float *dst, int dw, int dh, cudaStream_t st);
void launch_undistort(const float *src, int sw, int sh, const float *intr, const float *dist, int rx, int ry,
                      float *dst, int dw, int dh, cudaStream_t st);
void launch_image_metrics(const float *a, const float *b, int h, int w, const MetricsScratch &s, double *out,
                          cudaStream_t st);
void launch_pack_rgba8(const float *img, uint32_t n, uint8_t *out, cudaStream_t st);
void launch_finalize_depth(const float *d, const float *t, uint32_t n, float inv_scale, float *od, float *oa,
                           cudaStream_t st);

// Prior-guided extras (prior.cu; core/metal/bindings.h:43-77).
struct SkyArgs {
    const float *tex;     // (tex_h, tex_w, 3), device
    int tex_w, tex_h;
    float frame[9];       // up, e1 (azimuth 0), e2 (azimuth 90 degrees)
    float fx, fy, cx, cy;
    float viewmat[16];    // row-major world-to-camera
};
struct PriorLossArgs {
    int W, H;
    const float *final_T, *out_depth;
    const float *prior_depth;     // (ph, pw) or null
    const uint8_t *prior_aux;     // (ph, pw, 4) or null
    int pw, ph, use_depth, use_sky, mask_photometric;
    float depth_weight, sky_weight, fill_weight, huber, min_alpha, inv_npix;
    float *v_photo;  // (H, W, 3): pixels outside "keep" are zeroed
    float *v_aux;    // (H, W, 2): dL/d(depth numerator), dL/d(alpha)
    float *terms;    // (3, H, W) per-pixel loss terms, null to skip them
};
struct ExposureArgs {
    float *params, *exp_avg, *exp_avg_sq;  // (num_cams, 12)
    float *grad;                           // [12] or null
    int cam;
    float step_size, bc2, reg, beta1, beta2, eps;
};
struct SkyAdamArgs {
    float *tex, *grad, *exp_avg, *exp_avg_sq;  // (tex_h, tex_w, 3)
    float step_size, bc2, beta1, beta2, eps;
};
struct SkyScratch {
    uint4 *tap_idx;      // per pixel
    float4 *tap_w, *tap_g;
    int32_t *count, *off, *scan_part, *d_total;
    uint32_t *keys[2], *vals[2];  // 4 per pixel
    void *radix_scratch;          // radix_scratch_bytes(4 * pixels)
};
void launch_sky_background(const SkyArgs &s, int W, int H, float *bg_img, cudaStream_t st);
// rows: 3 * H doubles (only with a.terms and loss_terms)
void launch_prior_loss(const PriorLossArgs &a, double *rows, float *loss_terms, cudaStream_t st);
void launch_exposure_apply(const float *img, const float *P, int64_t n, float *out, cudaStream_t st);
int exposure_blocks(int64_t n);  // partials: 12 doubles per block
void launch_exposure_backward_adam(const float *img, const float *v_adj, int64_t n, float *v_img, double *partials,
                                   const ExposureArgs &e, cudaStream_t st);
void launch_sky_backward_adam(const SkyArgs &s, int W, int H, const float *final_T, const float *v_img,
                              const SkyAdamArgs &a, SkyScratch &sc, cudaStream_t st);
void launch_needle_cap(float *scales, int n, float log_max, cudaStream_t st);

struct KnnScratch {
    unsigned int *bounds;  // 6 ordered-bit floats: min xyz, max xyz
    uint64_t *keys[2];
    uint32_t *vals[2];
    void *radix_scratch;
    float4 *sorted, *bmin, *bmax;
    unsigned long long *evals;  // (may be null) point distances the search computed
};
int knn_boxes(int n);
int launch_knn3(const float *pts, int n, float *out, KnnScratch &s, cudaStream_t st);
void launch_init_gaussians(const float *md, const uint8_t *rgb, int n, uint32_t seed, float logit, float *scales,
                           float *quats, float *dc, float *opac, cudaStream_t st);

}  // namespace msplat
