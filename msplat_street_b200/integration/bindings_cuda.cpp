// The reference's backend contract, core/metal/bindings.h, implemented over this
// library's C-ABI (include/msplat_cuda.h): what a maintainer links instead of
// core/cpu/msplat_cpu.cpp so that core/src/model.cpp, the Python module and
// tests/gradcheck.cpp run on a B200 unchanged.
//
// Compiled against the reference's own headers (core/metal/bindings.h and
// core/include/metal_tensor.hpp, found on the include path; nothing of them is copied
// here). On non-Apple hosts those MTensors are host blocks, so every call stages its
// tensors through device memory: inputs are copied in on the context's stream, and
// the arrays the call updates are copied back after the call's work, with one
// synchronisation at the end. That keeps the reference's host-side semantics (callers
// read data_ptr() after msplat_gpu_sync) at the cost of the copies; a deployment that
// keeps its tensors on the device calls the C-ABI directly. The staging buffers
// persist across calls, one per host tensor (keyed by its host address, grown when the
// tensor grows), so a training loop allocates device memory only in its first steps
// and after Model::ensureCapacity; buffers no call has used for STAGE_IDLE_CALLS calls
// are released. One context (msplat_cuda_default_ctx) stands in for the reference's
// process-global frame cache; like the reference, this layer is single-threaded.
// Errors throw std::runtime_error with the library's message, as the reference throws.
#include "bindings.h"

#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "msplat_cuda.h"

namespace {

msplat_cuda_ctx *ctx() { return msplat_cuda_default_ctx(); }

void check(int status, const char *what) {
    if (status != MSPLAT_CUDA_OK)
        throw std::runtime_error(std::string("msplat (") + what + "): " + msplat_cuda_last_error());
}

// Device staging buffers, one per host tensor address, kept across calls.
constexpr uint64_t STAGE_IDLE_CALLS = 256;

struct StageCache {
    struct Entry {
        void *dev = nullptr;
        size_t bytes = 0;
        uint64_t last_call = 0;
    };
    std::unordered_map<const void *, Entry> map;
    uint64_t calls = 0;

    void *get(const void *host, size_t bytes) {
        Entry &e = map[host];
        if (e.bytes < bytes) {
            if (e.dev) check(msplat_cuda_free(e.dev), "stage free");
            e.dev = nullptr;
            e.bytes = 0;
            check(msplat_cuda_device_alloc(bytes, &e.dev), "stage alloc");
            e.bytes = bytes;
        }
        e.last_call = calls;
        return e.dev;
    }
    // after a call's synchronisation: release what recent calls have not used
    void end_call() {
        calls++;
        if (calls % STAGE_IDLE_CALLS) return;
        for (auto it = map.begin(); it != map.end();) {
            if (calls - it->second.last_call > STAGE_IDLE_CALLS) {
                msplat_cuda_free(it->second.dev);
                it = map.erase(it);
            } else {
                ++it;
            }
        }
    }
    void clear() {
        for (auto &kv : map) msplat_cuda_free(kv.second.dev);
        map.clear();
    }
};

StageCache &cache() {
    static StageCache c;
    return c;
}

// The tensors of one call: each staged once (a tensor passed twice shares its buffer),
// inputs copied to the device when staged, updated ones copied back in finish().
struct Staging {
    struct Item {
        void *host;
        void *dev;
        size_t bytes;
        bool back;
    };
    std::vector<Item> items;

    void *stage(MTensor *t, bool back) {
        if (!t || !t->defined()) return nullptr;
        void *host = t->data_ptr();
        const size_t bytes = t->nbytes();
        for (Item &it : items)
            if (it.host == host) {
                it.back = it.back || back;
                return it.dev;
            }
        void *dev = cache().get(host, bytes ? bytes : 4);
        if (bytes) check(msplat_cuda_copy_buffer(ctx(), dev, host, bytes), "stage in");
        items.push_back({host, dev, bytes, back});
        return dev;
    }
    template <typename T = float>
    T *in(MTensor &t) {
        return static_cast<T *>(stage(&t, false));
    }
    template <typename T = float>
    T *inout(MTensor &t) {
        return static_cast<T *>(stage(&t, true));
    }
    template <typename T = float>
    T *opt(MTensor *t, bool back) {
        return static_cast<T *>(stage(t, back));
    }
    void finish() {
        for (Item &it : items)
            if (it.back && it.bytes) check(msplat_cuda_copy_buffer(ctx(), it.host, it.dev, it.bytes), "stage out");
        check(msplat_cuda_sync(ctx()), "sync");
        cache().end_call();
    }
};

// msplat_cuda_prior over staged copies of a PriorStep's tensors
msplat_cuda_prior stage_prior(const PriorStep &p, Staging &s) {
    msplat_cuda_prior c{};
    c.aux = p.aux;
    c.sky = p.sky;
    c.sky_tex = s.opt(p.sky_tex, true);
    c.sky_grad = s.opt(p.sky_grad, true);
    c.sky_exp_avg = s.opt(p.sky_exp_avg, true);
    c.sky_exp_avg_sq = s.opt(p.sky_exp_avg_sq, true);
    c.sky_w = p.sky_w;
    c.sky_h = p.sky_h;
    std::memcpy(c.sky_frame, p.sky_frame, sizeof c.sky_frame);
    c.sky_step_size = p.sky_step_size;
    c.sky_bc2_sqrt = p.sky_bc2_sqrt;
    c.prior_depth = s.opt(p.prior_depth, false);
    c.prior_aux = s.opt<uint8_t>(p.prior_aux, false);
    c.prior_w = p.prior_w;
    c.prior_h = p.prior_h;
    c.has_depth = p.has_depth;
    c.has_sky_mask = p.has_sky_mask;
    c.depth_weight = p.depth_weight;
    c.sky_weight = p.sky_weight;
    c.fill_weight = p.fill_weight;
    c.huber_delta = p.huber_delta;
    c.min_alpha = p.min_alpha;
    c.mask_photometric = p.mask_photometric;
    c.loss_terms = s.opt(p.loss_terms, true);
    c.exposure = p.exposure;
    c.cam_index = p.cam_index;
    c.expo_params = s.opt(p.expo_params, true);
    c.expo_exp_avg = s.opt(p.expo_exp_avg, true);
    c.expo_exp_avg_sq = s.opt(p.expo_exp_avg_sq, true);
    c.expo_grad = s.opt(p.expo_grad, true);
    c.expo_step_size = p.expo_step_size;
    c.expo_bc2_sqrt = p.expo_bc2_sqrt;
    c.expo_reg = p.expo_reg;
    c.log_max_scale_ratio = p.log_max_scale_ratio;
    c.expo_num_cams = p.expo_params ? (int32_t)p.expo_params->size(0) : 0;
    return c;
}

struct PriorScope {  // sets the prior for one call, clears it after
    explicit PriorScope(const msplat_cuda_prior *p) { check(msplat_cuda_set_prior(ctx(), p), "set_prior"); }
    ~PriorScope() { msplat_cuda_set_prior(ctx(), nullptr); }
};

MTensor host_tensor(std::vector<int64_t> shape, DType dt) { return MTensor(MTensor::HostDevice{}, std::move(shape), dt); }

unsigned g_last_w = 0, g_last_h = 0;

}  // namespace

void cleanup_msplat_metal() {
    check(msplat_cuda_cleanup(ctx()), "cleanup");
    cache().clear();
}
void *msplat_device() { return nullptr; }
MTensor gpu_zeros(std::vector<int64_t> shape, DType dtype) { return host_tensor(std::move(shape), dtype); }
MTensor gpu_empty(std::vector<int64_t> shape, DType dtype) { return host_tensor(std::move(shape), dtype); }
void msplat_commit() { check(msplat_cuda_commit(ctx()), "commit"); }
void msplat_gpu_sync() { check(msplat_cuda_sync(ctx()), "sync"); }
bool msplat_begin_gpu_capture(const char *) { return false; }
void msplat_end_gpu_capture() {}
void msplat_enable_gpu_timing(bool enable) {
    check(msplat_cuda_ctx_set_option(ctx(), "stage_timing", enable ? 1 : 0), "stage_timing");
}
void msplat_drain_gpu_times(std::vector<double> &out) { out.clear(); }
void msplat_drain_stage_times(std::vector<double> stage_times[], int max_stages, int &n_stages,
                              const char **stage_names) {
    std::vector<double> ms((size_t)max_stages);
    std::vector<int64_t> calls((size_t)max_stages);
    check(msplat_cuda_drain_stage_times(ctx(), ms.data(), calls.data(), max_stages, &n_stages, stage_names),
          "drain_stage_times");
    for (int i = 0; i < max_stages; i++) {
        stage_times[i].clear();
        if (i < n_stages && calls[i] > 0) stage_times[i].push_back(ms[i]);
    }
}

MTensor msplat_render(int num_points, MTensor &means3d, MTensor &scales, float glob_scale, MTensor &quats,
                      MTensor &viewmat, MTensor &projmat, float fx, float fy, float cx, float cy,
                      unsigned img_height, unsigned img_width, const std::tuple<int, int, int> tile_bounds,
                      float clip_thresh, unsigned degree, unsigned degrees_to_use, float cam_pos[3],
                      MTensor &features_dc, MTensor &features_rest, MTensor &opacities, MTensor &background,
                      const PriorStep *prior) {
    Staging s;
    msplat_cuda_prior c{};
    if (prior) c = stage_prior(*prior, s);
    PriorScope scope(prior ? &c : nullptr);
    const float *out = nullptr;
    check(msplat_cuda_render(ctx(), num_points, s.in(means3d), s.in(scales), glob_scale, s.in(quats),
                             viewmat.data<float>(), projmat.data<float>(), fx, fy, cx, cy, img_height, img_width,
                             std::get<0>(tile_bounds), std::get<1>(tile_bounds), clip_thresh, degree, degrees_to_use,
                             cam_pos, s.in(features_dc), features_rest.defined() ? s.in(features_rest) : nullptr,
                             s.in(opacities), background.data<float>(), &out),
          "render");
    MTensor img = host_tensor({(int64_t)img_height, (int64_t)img_width, 3}, DType::Float32);
    check(msplat_cuda_copy_buffer(ctx(), img.data_ptr(), out, img.nbytes()), "render copy");
    s.finish();
    g_last_w = img_width;
    g_last_h = img_height;
    return img;
}

void msplat_render_aux_outputs(MTensor &depth, MTensor &final_T) {
    const float *d = nullptr, *t = nullptr;
    check(msplat_cuda_render_aux_outputs(ctx(), &d, &t), "render_aux_outputs");
    depth = host_tensor({(int64_t)g_last_h, (int64_t)g_last_w}, DType::Float32);
    final_T = host_tensor({(int64_t)g_last_h, (int64_t)g_last_w}, DType::Float32);
    check(msplat_cuda_copy_buffer(ctx(), depth.data_ptr(), d, depth.nbytes()), "aux copy");
    check(msplat_cuda_copy_buffer(ctx(), final_T.data_ptr(), t, final_T.nbytes()), "aux copy");
    check(msplat_cuda_sync(ctx()), "sync");
}

std::tuple<MTensor, float> msplat_train_step(
    int num_points, MTensor &means3d, MTensor &scales, float glob_scale, MTensor &quats, MTensor &viewmat,
    MTensor &projmat, float fx, float fy, float cx, float cy, unsigned img_height, unsigned img_width,
    const std::tuple<int, int, int> tile_bounds, float clip_thresh, unsigned degree, unsigned degrees_to_use,
    float cam_pos[3], MTensor &features_dc, MTensor &features_rest, MTensor &opacities, MTensor &background,
    MTensor &gt, MTensor &window2d, float ssim_weight, float loss_inv_n, int features_rest_bases,
    int num_adam_groups, MTensor adam_params[], MTensor adam_exp_avg[], MTensor adam_exp_avg_sq[],
    float adam_step_sizes[], float adam_bc2_sqrts[], float adam_beta1, float adam_beta2, float adam_eps,
    MTensor &vis_counts, MTensor &xys_grad_norm, MTensor &max_2d_size, float inv_max_dim, const PriorStep *prior) {
    (void)window2d;
    (void)features_rest_bases;
    (void)adam_params;  // the parameter tensors themselves (core/src/model.cpp:644-646)
    Staging s;
    msplat_cuda_prior c{};
    if (prior) c = stage_prior(*prior, s);
    PriorScope scope(prior ? &c : nullptr);
    float *m1[6] = {}, *m2[6] = {};
    for (int g = 0; g < num_adam_groups && g < 6; g++) {
        m1[g] = adam_exp_avg[g].defined() ? s.inout(adam_exp_avg[g]) : nullptr;
        m2[g] = adam_exp_avg_sq[g].defined() ? s.inout(adam_exp_avg_sq[g]) : nullptr;
    }
    const int32_t *radii = nullptr;
    float loss = 0.f;
    check(msplat_cuda_train_step(
              ctx(), num_points, s.inout(means3d), s.inout(scales), glob_scale, s.inout(quats), viewmat.data<float>(),
              projmat.data<float>(), fx, fy, cx, cy, img_height, img_width, std::get<0>(tile_bounds),
              std::get<1>(tile_bounds), clip_thresh, degree, degrees_to_use, cam_pos, s.inout(features_dc),
              features_rest.defined() ? s.inout(features_rest) : nullptr, s.inout(opacities), background.data<float>(),
              s.in(gt), ssim_weight, loss_inv_n, num_adam_groups, m1, m2, adam_step_sizes, adam_bc2_sqrts, adam_beta1,
              adam_beta2, adam_eps, s.inout(vis_counts), s.inout(xys_grad_norm), s.inout(max_2d_size), inv_max_dim,
              &radii, &loss),
          "train_step");
    MTensor r = host_tensor({(int64_t)num_points}, DType::Int32);
    if (num_points > 0) check(msplat_cuda_copy_buffer(ctx(), r.data_ptr(), radii, r.nbytes()), "radii copy");
    s.finish();
    g_last_w = img_width;
    g_last_h = img_height;
    return std::make_tuple(r, loss);
}

int msplat_densify(int N, int buf_capacity, float grad_thresh, float size_thresh, float screen_thresh,
                   int check_screen, float cull_alpha_thresh, float cull_scale_thresh, float cull_screen_size,
                   int check_huge, MTensor &xys_grad_norm, MTensor &vis_counts, MTensor &max_2d_size,
                   float half_max_dim, MTensor &means_buf, MTensor &scales_buf, MTensor &quats_buf,
                   MTensor &featuresDc_buf, MTensor &featuresRest_buf, MTensor &opacities_buf, int fr_stride,
                   MTensor adam_exp_avg_buf[], MTensor adam_exp_avg_sq_buf[], MTensor &split_flag,
                   MTensor &dup_flag, MTensor &split_prefix, MTensor &dup_prefix, MTensor &keep_flag,
                   MTensor &keep_prefix, MTensor &block_totals, MTensor &compact_scratch, uint32_t seed) {
    (void)split_flag, (void)dup_flag, (void)split_prefix, (void)dup_prefix, (void)keep_flag, (void)keep_prefix,
        (void)block_totals, (void)compact_scratch;  // the library keeps its own scratch
    Staging s;
    float *params[6] = {s.inout(means_buf), s.inout(scales_buf), s.inout(quats_buf), s.inout(featuresDc_buf),
                        s.inout(featuresRest_buf), s.inout(opacities_buf)};
    float *m1[6], *m2[6];
    for (int g = 0; g < 6; g++) {
        m1[g] = s.inout(adam_exp_avg_buf[g]);
        m2[g] = s.inout(adam_exp_avg_sq_buf[g]);
    }
    int n = 0;
    check(msplat_cuda_densify(ctx(), N, buf_capacity, grad_thresh, size_thresh, screen_thresh, check_screen,
                              cull_alpha_thresh, cull_scale_thresh, cull_screen_size, check_huge,
                              s.in(xys_grad_norm), s.in(vis_counts), s.in(max_2d_size), half_max_dim, params,
                              fr_stride, m1, m2, seed, &n),
          "densify");
    s.finish();
    return n;
}

void msplat_opacity_reset(MTensor &opacities, MTensor &exp_avg, MTensor &exp_avg_sq, int num_points,
                          float reset_logit) {
    Staging s;
    check(msplat_cuda_opacity_reset(ctx(), s.inout(opacities), s.inout(exp_avg), s.inout(exp_avg_sq), num_points,
                                    reset_logit),
          "opacity_reset");
    s.finish();
}

void msplat_copy_buffer(MTensor &dst, const MTensor &src, size_t bytes) {
    check(msplat_cuda_copy_buffer(ctx(), dst.data_ptr(), src.data_ptr(), bytes), "copy_buffer");
    check(msplat_cuda_sync(ctx()), "sync");
}

void msplat_radix_sort(MTensor &keys, MTensor &vals, uint32_t n, int key_bits) {
    Staging s;
    check(msplat_cuda_radix_sort(ctx(), s.inout<uint64_t>(keys), s.inout<int32_t>(vals), n, key_bits),
          "radix_sort");
    s.finish();
}

void msplat_knn3_mean_dist(MTensor &points, uint32_t n, MTensor &mean_dist) {
    Staging s;
    check(msplat_cuda_knn3_mean_dist(ctx(), s.in(points), n, s.inout(mean_dist)), "knn3_mean_dist");
    s.finish();
}

void msplat_init_gaussians(MTensor &means, MTensor &rgb, uint32_t n, uint32_t seed, float opacity_logit,
                           MTensor &scales, MTensor &quats, MTensor &features_dc, MTensor &opacities) {
    Staging s;
    check(msplat_cuda_init_gaussians(ctx(), s.in(means), s.in<uint8_t>(rgb), n, seed, opacity_logit,
                                     s.inout(scales), s.inout(quats), s.inout(features_dc), s.inout(opacities)),
          "init_gaussians");
    s.finish();
}

void msplat_resize_area(const MTensor &src, bool src_is_u8, int sw, int sh, MTensor &dst, int dw, int dh) {
    Staging s;
    MTensor &in = const_cast<MTensor &>(src);
    check(msplat_cuda_resize_area(ctx(), s.in<void>(in), src_is_u8 ? 1 : 0, sw, sh, s.inout(dst), dw, dh),
          "resize_area");
    s.finish();
}

void msplat_undistort(const MTensor &src, int sw, int sh, const float intr[4], const float dist[5], int roi_x,
                      int roi_y, MTensor &dst, int dw, int dh) {
    Staging s;
    MTensor &in = const_cast<MTensor &>(src);
    check(msplat_cuda_undistort(ctx(), s.in(in), sw, sh, intr, dist, roi_x, roi_y, s.inout(dst), dw, dh),
          "undistort");
    s.finish();
}

void msplat_image_metrics(const MTensor &rendered, const MTensor &gt, int h, int w, double out[3]) {
    Staging s;
    check(msplat_cuda_image_metrics(ctx(), s.in(const_cast<MTensor &>(rendered)), s.in(const_cast<MTensor &>(gt)),
                                    h, w, out),
          "image_metrics");
    s.finish();
}

void msplat_pack_rgba8(const MTensor &img, uint32_t n, uint8_t *out) {
    Staging s;
    check(msplat_cuda_pack_rgba8(ctx(), s.in(const_cast<MTensor &>(img)), n, out), "pack_rgba8");
    s.finish();
}

void msplat_finalize_depth(const MTensor &depth_num, const MTensor &final_T, uint32_t n, float inv_scale,
                           MTensor &depth_out, MTensor &alpha_out) {
    Staging s;
    check(msplat_cuda_finalize_depth(ctx(), s.in(const_cast<MTensor &>(depth_num)),
                                     s.in(const_cast<MTensor &>(final_T)), n, inv_scale, s.inout(depth_out),
                                     s.inout(alpha_out)),
          "finalize_depth");
    s.finish();
}
