// Shim around the reference's own CPU backend -- TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles this file with the reference's core/cpu, core/include and
// core/metal directories on the include path (they are not copied into this
// repository). Including msplat_cpu.cpp puts its anonymous-namespace frame cache
// (g_frame, core/cpu/msplat_cpu.cpp:406-436) in this translation unit, so the shim
// can export the same C-ABI as the restatement (msplat_oracle.h), per-stage
// intermediates included. Host pointers are copied into and out of the reference's
// MTensor buffers around each call.

#include "msplat_cpu.cpp"

#include "msplat_oracle.h"

#include <memory>
#include <string>

namespace {

MTensor host_tensor(std::vector<int64_t> shape, DType dt, const void *src) {
    MTensor t = gpu_empty(std::move(shape), dt);
    if (src) std::memcpy(t.data_ptr(), src, t.nbytes());
    return t;
}
void copy_out(const MTensor &t, void *dst) { std::memcpy(dst, t.data_ptr(), t.nbytes()); }

struct Scene {
    MTensor means, scales, quats, vm, pm, dc, rest, opac, bg;
    Scene(int n, const float *m, const float *s, const float *q, const float *v, const float *p, unsigned degree,
          const float *d, const float *r, const float *o, const float *b) {
        const int64_t nb = (int64_t)num_sh_bases(degree);
        means = host_tensor({n, 3}, DType::Float32, m);
        scales = host_tensor({n, 3}, DType::Float32, s);
        quats = host_tensor({n, 4}, DType::Float32, q);
        vm = host_tensor({4, 4}, DType::Float32, v);
        pm = host_tensor({4, 4}, DType::Float32, p);
        dc = host_tensor({n, 3}, DType::Float32, d);
        rest = host_tensor({n, nb - 1, 3}, DType::Float32, r);
        opac = host_tensor({n, 1}, DType::Float32, o);
        bg = host_tensor({3}, DType::Float32, b);
    }
};

bool g_has_prior = false;
orc_prior g_prior;

// The reference's PriorStep over MTensor copies of the host arrays of g_prior; the
// arrays a train step updates are copied back by finish().
struct Prior {
    PriorStep ps;
    MTensor sky_tex, sky_grad, sky_m1, sky_m2, depth, aux, terms, expo, expo_m1, expo_m2, expo_grad;
    int64_t num_cams;
    explicit Prior(int64_t num_cams_) : num_cams(num_cams_) {
        const orc_prior &p = g_prior;
        ps.aux = p.aux != 0;
        ps.sky = p.sky != 0;
        const std::vector<int64_t> tex{p.sky_h, p.sky_w, 3};
        if (p.sky_tex) ps.sky_tex = &(sky_tex = host_tensor(tex, DType::Float32, p.sky_tex));
        if (p.sky_grad) ps.sky_grad = &(sky_grad = host_tensor(tex, DType::Float32, p.sky_grad));
        if (p.sky_exp_avg) ps.sky_exp_avg = &(sky_m1 = host_tensor(tex, DType::Float32, p.sky_exp_avg));
        if (p.sky_exp_avg_sq) ps.sky_exp_avg_sq = &(sky_m2 = host_tensor(tex, DType::Float32, p.sky_exp_avg_sq));
        ps.sky_w = p.sky_w;
        ps.sky_h = p.sky_h;
        std::memcpy(ps.sky_frame, p.sky_frame, sizeof ps.sky_frame);
        ps.sky_step_size = p.sky_step_size;
        ps.sky_bc2_sqrt = p.sky_bc2_sqrt;
        if (p.prior_depth) ps.prior_depth = &(depth = host_tensor({p.prior_h, p.prior_w}, DType::Float32, p.prior_depth));
        if (p.prior_aux) ps.prior_aux = &(aux = host_tensor({p.prior_h, p.prior_w, 4}, DType::UInt8, p.prior_aux));
        ps.prior_w = p.prior_w;
        ps.prior_h = p.prior_h;
        ps.has_depth = p.has_depth != 0;
        ps.has_sky_mask = p.has_sky_mask != 0;
        ps.depth_weight = p.depth_weight;
        ps.sky_weight = p.sky_weight;
        ps.fill_weight = p.fill_weight;
        ps.huber_delta = p.huber_delta;
        ps.min_alpha = p.min_alpha;
        ps.mask_photometric = p.mask_photometric != 0;
        if (p.loss_terms) ps.loss_terms = &(terms = host_tensor({4}, DType::Float32, p.loss_terms));
        ps.exposure = p.exposure != 0;
        ps.cam_index = p.cam_index;
        if (p.expo_params) ps.expo_params = &(expo = host_tensor({num_cams, 12}, DType::Float32, p.expo_params));
        if (p.expo_exp_avg) ps.expo_exp_avg = &(expo_m1 = host_tensor({num_cams, 12}, DType::Float32, p.expo_exp_avg));
        if (p.expo_exp_avg_sq)
            ps.expo_exp_avg_sq = &(expo_m2 = host_tensor({num_cams, 12}, DType::Float32, p.expo_exp_avg_sq));
        if (p.expo_grad) ps.expo_grad = &(expo_grad = host_tensor({12}, DType::Float32, p.expo_grad));
        ps.expo_step_size = p.expo_step_size;
        ps.expo_bc2_sqrt = p.expo_bc2_sqrt;
        ps.expo_reg = p.expo_reg;
        ps.log_max_scale_ratio = p.log_max_scale_ratio;
    }
    void finish() const {
        const orc_prior &p = g_prior;
        if (p.sky_tex) copy_out(sky_tex, p.sky_tex);
        if (p.sky_grad) copy_out(sky_grad, p.sky_grad);
        if (p.sky_exp_avg) copy_out(sky_m1, p.sky_exp_avg);
        if (p.sky_exp_avg_sq) copy_out(sky_m2, p.sky_exp_avg_sq);
        if (p.loss_terms) copy_out(terms, p.loss_terms);
        if (p.expo_params) copy_out(expo, p.expo_params);
        if (p.expo_exp_avg) copy_out(expo_m1, p.expo_exp_avg);
        if (p.expo_exp_avg_sq) copy_out(expo_m2, p.expo_exp_avg_sq);
        if (p.expo_grad) copy_out(expo_grad, p.expo_grad);
    }
};

}  // namespace

extern "C" {

// The shim's exposure arrays hold cam_index + 1 cameras (the rows up to the one used).
int orc_set_prior(const orc_prior *prior) {
    g_has_prior = prior != nullptr;
    if (prior) g_prior = *prior;
    return 0;
}

int orc_render(int n, const float *means, const float *scales, float gsc, const float *quats, const float *vm,
               const float *P, float fx, float fy, float cx, float cy, unsigned H, unsigned W, int tx, int ty,
               float clip, unsigned degree, unsigned dtu, const float *cam, const float *dc, const float *rest,
               const float *opac, const float *bg, float *out) {
    Scene s(n, means, scales, quats, vm, P, degree, dc, rest, opac, bg);
    float cp[3] = {cam[0], cam[1], cam[2]};
    std::unique_ptr<Prior> pr;
    if (g_has_prior) pr.reset(new Prior(std::max(0, g_prior.cam_index) + 1));
    MTensor img = msplat_render(n, s.means, s.scales, gsc, s.quats, s.vm, s.pm, fx, fy, cx, cy, H, W,
                                std::make_tuple(tx, ty, 1), clip, degree, dtu, cp, s.dc, s.rest, s.opac, s.bg,
                                pr ? &pr->ps : nullptr);
    copy_out(img, out);
    return 0;
}

float orc_train_step(int n, float *means, float *scales, float gsc, float *quats, const float *vm, const float *P,
                     float fx, float fy, float cx, float cy, unsigned H, unsigned W, int tx, int ty, float clip,
                     unsigned degree, unsigned dtu, const float *cam, float *dc, float *rest, float *opac,
                     const float *bg, const float *gt, float ssim_w, float inv_n, float **m1, float **m2,
                     const int64_t *numel, const float *ss, const float *bc2, float b1, float b2, float eps,
                     float *vis, float *gn, float *ms, float inv_max_dim) {
    Scene s(n, means, scales, quats, vm, P, degree, dc, rest, opac, bg);
    MTensor gtt = host_tensor({(int64_t)H, (int64_t)W, 3}, DType::Float32, gt);
    MTensor win = gpu_zeros({11, 11}, DType::Float32);
    MTensor params[6] = {s.means, s.scales, s.quats, s.dc, s.rest, s.opac};
    float *host_params[6] = {means, scales, quats, dc, rest, opac};
    MTensor ea[6], eas[6];
    float ssz[6], b2s[6];
    for (int g = 0; g < 6; g++) {
        ea[g] = host_tensor(params[g].shape(), DType::Float32, m1[g]);
        eas[g] = host_tensor(params[g].shape(), DType::Float32, m2[g]);
        if (params[g].numel() != numel[g]) return NAN;
        ssz[g] = ss[g];
        b2s[g] = bc2[g];
    }
    MTensor tv = host_tensor({n}, DType::Float32, vis), tg = host_tensor({n}, DType::Float32, gn),
            tm = host_tensor({n}, DType::Float32, ms);
    float cp[3] = {cam[0], cam[1], cam[2]};
    std::unique_ptr<Prior> pr;
    if (g_has_prior) pr.reset(new Prior(std::max(0, g_prior.cam_index) + 1));
    auto [radii, loss] = msplat_train_step(
        n, s.means, s.scales, gsc, s.quats, s.vm, s.pm, fx, fy, cx, cy, H, W, std::make_tuple(tx, ty, 1), clip, degree,
        dtu, cp, s.dc, s.rest, s.opac, s.bg, gtt, win, ssim_w, inv_n, (int)(num_sh_bases(degree) - 1), 6, params, ea,
        eas, ssz, b2s, b1, b2, eps, tv, tg, tm, inv_max_dim, pr ? &pr->ps : nullptr);
    (void)radii;
    if (pr) pr->finish();
    for (int g = 0; g < 6; g++) {
        copy_out(params[g], host_params[g]);
        copy_out(ea[g], m1[g]);
        copy_out(eas[g], m2[g]);
    }
    copy_out(tv, vis);
    copy_out(tg, gn);
    copy_out(tm, ms);
    return loss;
}

int64_t orc_frame(const char *name, void **ptr) {
    const std::string s(name);
    Frame &f = g_frame;
    const int n = f.num_points;
    const int T = f.tiles_x * f.tiles_y;
    const int64_t total = T ? f.tile_end[T - 1] : 0;
    const int64_t npix = (int64_t)f.W * f.H;
#define REF_V(nm, vec, cnt) \
    if (s == nm) { *ptr = (void *)vec.data(); return (int64_t)(cnt); }
#define REF_T(nm, ten, cnt) \
    if (s == nm) { *ptr = ten.defined() ? ten.data_ptr() : nullptr; return ten.defined() ? (int64_t)(cnt) : -1; }
#define REF_T0(nm, ten, cnt) \
    if (s == nm) { *ptr = ten.defined() ? ten.data_ptr() : nullptr; return ten.defined() ? (int64_t)(cnt) : 0; }
    REF_V("xys", f.xys, (int64_t)n * 2)
    REF_V("depths", f.depths, n)
    REF_V("conics", f.conics, (int64_t)n * 3)
    REF_V("colors", f.colors, (int64_t)n * 3)
    REF_V("aabb", f.aabb, (int64_t)n * 2)
    REF_T("radii", f.radii, n)
    REF_V("tile_start", f.tile_start, T)
    REF_V("tile_end", f.tile_end, T)
    REF_V("isect_gid", f.isect_gid, total)
    REF_T("out_img", f.out_img, npix * 3)
    REF_T("final_Ts", f.final_Ts, npix)
    REF_V("final_idx", f.final_idx, npix)
    REF_T("v_rendered", f.v_rendered, npix * 3)
    REF_V("v_xy", f.v_xy, (int64_t)n * 2)
    REF_V("v_conic", f.v_conic, (int64_t)n * 3)
    REF_V("v_rgb", f.v_rgb, (int64_t)n * 3)
    REF_V("v_opacity", f.v_opacity, n)
    REF_V("v_mean3d", f.v_mean3d, (int64_t)n * 3)
    REF_V("v_scale", f.v_scale, (int64_t)n * 3)
    REF_V("v_quat", f.v_quat, (int64_t)n * 4)
    REF_T0("out_depth", f.out_depth, f.aux ? npix : 0)
    REF_T0("bg_img", f.bg_img, f.aux ? npix * 3 : 0)
    REF_V("v_aux", f.v_aux, f.aux ? npix * 2 : 0)
    REF_V("v_depth", f.v_depth, std::min<int64_t>((int64_t)f.v_depth.size(), n))
    REF_T0("out_adj", f.out_adj, f.out_adj.defined() ? f.out_adj.numel() : 0)
    REF_T0("v_adj", f.v_adj, f.v_adj.defined() ? f.v_adj.numel() : 0)
#undef REF_V
#undef REF_T
#undef REF_T0
    *ptr = nullptr;
    return -1;
}

int orc_densify(int N, int cap, float grad_thresh, float size_thresh, float screen_thresh, int check_screen,
                float cull_alpha, float cull_scale, float cull_screen, int check_huge, const float *gn,
                const float *vc, const float *ms, float half_max_dim, float *means, float *scales, float *quats,
                float *fdc, float *frest, float *opac, int fr_stride, float **m1, float **m2, uint32_t seed) {
    if (3 * N > cap) return -1;
    MTensor tg = host_tensor({N}, DType::Float32, gn), tv = host_tensor({N}, DType::Float32, vc),
            tm = host_tensor({N}, DType::Float32, ms);
    const int st[6] = {3, 3, 4, 3, fr_stride, 1};
    float *hp[6] = {means, scales, quats, fdc, frest, opac};
    MTensor bufs[6], ea[6], eas[6];
    for (int g = 0; g < 6; g++) {
        bufs[g] = host_tensor({cap, st[g]}, DType::Float32, hp[g]);
        ea[g] = host_tensor({cap, st[g]}, DType::Float32, m1[g]);
        eas[g] = host_tensor({cap, st[g]}, DType::Float32, m2[g]);
    }
    MTensor dummy = gpu_zeros({1}, DType::Int32);
    int out = msplat_densify(N, cap, grad_thresh, size_thresh, screen_thresh, check_screen, cull_alpha, cull_scale,
                             cull_screen, check_huge, tg, tv, tm, half_max_dim, bufs[0], bufs[1], bufs[2], bufs[3],
                             bufs[4], bufs[5], fr_stride, ea, eas, dummy, dummy, dummy, dummy, dummy, dummy, dummy,
                             dummy, seed);
    for (int g = 0; g < 6; g++) {
        copy_out(bufs[g], hp[g]);
        copy_out(ea[g], m1[g]);
        copy_out(eas[g], m2[g]);
    }
    return out;
}

void orc_opacity_reset(float *o, float *m1, float *m2, int n, float reset_logit) {
    MTensor to = host_tensor({n}, DType::Float32, o), t1 = host_tensor({n}, DType::Float32, m1),
            t2 = host_tensor({n}, DType::Float32, m2);
    msplat_opacity_reset(to, t1, t2, n, reset_logit);
    copy_out(to, o);
    copy_out(t1, m1);
    copy_out(t2, m2);
}

void orc_radix_sort(uint64_t *keys, int32_t *vals, uint32_t n, int key_bits) {
    MTensor k = host_tensor({(int64_t)std::max<uint32_t>(n, 1)}, DType::Int64, nullptr);
    MTensor v = host_tensor({(int64_t)std::max<uint32_t>(n, 1)}, DType::Int32, nullptr);
    std::memcpy(k.data_ptr(), keys, (size_t)n * 8);
    std::memcpy(v.data_ptr(), vals, (size_t)n * 4);
    msplat_radix_sort(k, v, n, key_bits);
    std::memcpy(keys, k.data_ptr(), (size_t)n * 8);
    std::memcpy(vals, v.data_ptr(), (size_t)n * 4);
}

void orc_knn3_mean_dist(const float *pts, uint32_t n, float *out) {
    if (n == 0) return;
    MTensor p = host_tensor({(int64_t)n, 3}, DType::Float32, pts);
    MTensor d = gpu_empty({(int64_t)n}, DType::Float32);
    msplat_knn3_mean_dist(p, n, d);
    copy_out(d, out);
}

void orc_init_gaussians(const float *means, const uint8_t *rgb, uint32_t n, uint32_t seed, float ologit,
                        float *scales, float *quats, float *dc, float *opac) {
    if (n == 0) return;
    MTensor m = host_tensor({(int64_t)n, 3}, DType::Float32, means);
    MTensor c = host_tensor({(int64_t)n, 3}, DType::UInt8, rgb);
    MTensor s = gpu_empty({(int64_t)n, 3}, DType::Float32), q = gpu_empty({(int64_t)n, 4}, DType::Float32),
            d = gpu_empty({(int64_t)n, 3}, DType::Float32), o = gpu_empty({(int64_t)n, 1}, DType::Float32);
    msplat_init_gaussians(m, c, n, seed, ologit, s, q, d, o);
    copy_out(s, scales);
    copy_out(q, quats);
    copy_out(d, dc);
    copy_out(o, opac);
}

void orc_resize_area(const void *src, int u8in, int sw, int sh, float *dst, int dw, int dh) {
    MTensor s = host_tensor({sh, sw, u8in ? 4 : 3}, u8in ? DType::UInt8 : DType::Float32, src);
    MTensor d = gpu_empty({std::max(dh, 1), std::max(dw, 1), 3}, DType::Float32);
    msplat_resize_area(s, u8in != 0, sw, sh, d, dw, dh);
    if (dw > 0 && dh > 0) copy_out(d, dst);
}

void orc_undistort(const float *in, int sw, int sh, const float *intr, const float *dist, int rx, int ry, float *out,
                   int dw, int dh) {
    MTensor s = host_tensor({sh, sw, 3}, DType::Float32, in);
    MTensor d = gpu_empty({std::max(dh, 1), std::max(dw, 1), 3}, DType::Float32);
    msplat_undistort(s, sw, sh, intr, dist, rx, ry, d, dw, dh);
    if (dw > 0 && dh > 0) copy_out(d, out);
}

void orc_image_metrics(const float *a, const float *b, int h, int w, double *out) {
    MTensor ta = host_tensor({h, w, 3}, DType::Float32, a), tb = host_tensor({h, w, 3}, DType::Float32, b);
    msplat_image_metrics(ta, tb, h, w, out);
}

void orc_pack_rgba8(const float *img, uint32_t n, uint8_t *out) {
    MTensor t = host_tensor({(int64_t)n, 3}, DType::Float32, img);
    msplat_pack_rgba8(t, n, out);
}

void orc_finalize_depth(const float *d, const float *t, uint32_t n, float inv_scale, float *od, float *oa) {
    MTensor td = host_tensor({(int64_t)n}, DType::Float32, d), tt = host_tensor({(int64_t)n}, DType::Float32, t);
    MTensor a = gpu_empty({(int64_t)n}, DType::Float32), b = gpu_empty({(int64_t)n}, DType::Float32);
    msplat_finalize_depth(td, tt, n, inv_scale, a, b);
    copy_out(a, od);
    copy_out(b, oa);
}

}  // extern "C"
