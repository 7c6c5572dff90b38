// Prior-guided extras of a training step (core/metal/bindings.h:43-77, PriorStep):
// the learned equirect sky composited behind the Gaussians, the depth / sky / fill
// prior losses, the per-image affine exposure, and their backward passes with Adam.
// The needle cap is applied inside the fused backward/Adam kernel (backward.cu).
//
// Follows core/cpu/msplat_cpu.cpp:329-402 (sky sampling), 787-964 (prior_loss,
// exposure, sky backward) and 1204-1327 (their order in the step). Compiled with
// -fmad=false like the rest: per-pixel values keep the reference's operations.
// Where the reference's result depends on its host math library, the device
// evaluates in double and rounds once: log (depth residual), asin and atan2 (sky
// direction). Those agree with the host's float functions except in the last place
// for a small share of inputs, so sky and depth-prior results meet the reference
// within tolerance rather than bit for bit.
//
// Reductions are deterministic:
//  * loss terms: per-pixel float terms, summed per row in double in x order, rows
//    summed in y order (the reference's order exactly);
//  * exposure gradient: fixed-shape double partials per block, summed in block
//    order (the reference sums pixels sequentially in double; the float it keeps
//    differs at most in its last place, and only rarely);
//  * sky gradient: every (texel, pixel, tap) contribution is sorted by texel, stably,
//    so each texel sums its contributions in the reference's pixel-then-tap order.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace msplat {

namespace {

constexpr float PI_F = 3.14159265358979323846f;

// world direction of the ray through pixel (px, py) (core/cpu/msplat_cpu.cpp:353-359)
__device__ __forceinline__ V3 sky_ray(float px, float py, const SkyArgs &s) {
    const float dx = (px + 0.5f - s.cx) / s.fx;
    const float dy = (py + 0.5f - s.cy) / s.fy;
    const float *vm = s.viewmat;
    return V3{vm[0] * dx + vm[4] * dy + vm[8], vm[1] * dx + vm[5] * dy + vm[9], vm[2] * dx + vm[6] * dy + vm[10]};
}

// equirect texel coordinates of a direction (:361-372)
__device__ __forceinline__ V2 sky_uv(V3 d, const SkyArgs &s) {
    d = scl(d, 1.f / sqrtf(dot3(d, d)));
    const V3 up{s.frame[0], s.frame[1], s.frame[2]}, e1{s.frame[3], s.frame[4], s.frame[5]},
        e2{s.frame[6], s.frame[7], s.frame[8]};
    const float el = (float)asin((double)fminf(fmaxf(dot3(d, up), -1.f), 1.f));
    const float az = (float)atan2((double)dot3(d, e2), (double)dot3(d, e1));
    return V2{(az * (0.5f / PI_F) + 0.5f) * (float)s.tex_w - 0.5f, (0.5f - el / PI_F) * (float)s.tex_h - 0.5f};
}

// bilinear taps, longitude wrapping and latitude clamped (:379-395)
struct Taps {
    uint32_t idx[4];
    float w[4];
};
__device__ __forceinline__ Taps sky_taps(V2 uv, int tw, int th) {
    const float u0f = floorf(uv.x), fu = uv.x - u0f;
    int u0 = (int)u0f % tw;
    if (u0 < 0) u0 += tw;
    const int u1 = (u0 + 1) % tw;
    const float vc = fminf(fmaxf(uv.y, 0.f), (float)th - 1.f);
    const int v0 = (int)vc, v1 = min(v0 + 1, th - 1);
    const float fv = vc - (float)v0;
    Taps t;
    t.idx[0] = (uint32_t)(v0 * tw + u0);
    t.w[0] = (1.f - fu) * (1.f - fv);
    t.idx[1] = (uint32_t)(v0 * tw + u1);
    t.w[1] = fu * (1.f - fv);
    t.idx[2] = (uint32_t)(v1 * tw + u0);
    t.w[2] = (1.f - fu) * fv;
    t.idx[3] = (uint32_t)(v1 * tw + u1);
    t.w[3] = fu * fv;
    return t;
}

__device__ __forceinline__ Taps pixel_taps(int x, int y, const SkyArgs &s) {
    return sky_taps(sky_uv(sky_ray((float)x, (float)y, s), s), s.tex_w, s.tex_h);
}

// ---- sky background (rasterize_forward's per-pixel background, :607-609) ----------

__global__ void sky_background_kernel(const SkyArgs s, int W, int H, float *bg_img) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const Taps t = pixel_taps(x, y, s);
    V3 c{0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const V3 tx = ld3(s.tex, t.idx[k]);
        c = V3{tx.x * t.w[k] + c.x, tx.y * t.w[k] + c.y, tx.z * t.w[k] + c.z};
    }
    st3(bg_img, (int64_t)y * W + x, c);
}

// ---- prior losses (prior_loss, :807-901) -----------------------------------------

// bilinear prior depth unless the four samples straddle a depth edge (:788-804)
__device__ __forceinline__ float prior_depth_at(const float *d, float x, float y, int w, int h) {
    x = fminf(fmaxf(x, 0.f), (float)w - 1.f);
    y = fminf(fmaxf(y, 0.f), (float)h - 1.f);
    const int x0 = (int)x, y0 = (int)y;
    const int x1 = min(x0 + 1, w - 1), y1 = min(y0 + 1, h - 1);
    const float fx = x - (float)x0, fy = y - (float)y0;
    const float d00 = d[y0 * w + x0], d01 = d[y0 * w + x1], d10 = d[y1 * w + x0], d11 = d[y1 * w + x1];
    const float lo = fminf(fminf(d00, d01), fminf(d10, d11));
    const float hi = fmaxf(fmaxf(d00, d01), fmaxf(d10, d11));
    if (lo <= 0.f || hi > 1.05f * lo) return d[((fy < 0.5f) ? y0 : y1) * w + ((fx < 0.5f) ? x0 : x1)];
    const float top = d00 + (d01 - d00) * fx, bot = d10 + (d11 - d10) * fx;
    return top + (bot - top) * fy;
}

__device__ __forceinline__ float log_ref(float x) { return (float)log((double)x); }

__global__ void prior_loss_kernel(const PriorLossArgs a) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= a.W || gy >= a.H) return;
    const size_t pix = (size_t)gy * a.W + gx;
    const bool has = a.prior_depth && a.prior_aux && a.pw > 0 && a.ph > 0;
    const int pw = has ? a.pw : 1, ph = has ? a.ph : 1;
    const float sx = ((float)gx + 0.5f) * (float)pw / (float)a.W;
    const float sy = ((float)gy + 0.5f) * (float)ph / (float)a.H;
    const int q = min((int)sy, ph - 1) * pw + min((int)sx, pw - 1);
    // no prior: keep everything, no sky, zero confidence
    const uchar4 aux = has ? reinterpret_cast<const uchar4 *>(a.prior_aux)[q] : make_uchar4(0, 0, 255, 0);
    const bool use_depth = has && a.use_depth, use_sky = has && a.use_sky;
    const float conf = (float)aux.x * (1.f / 255.f);
    const bool sky = use_sky && aux.y >= 128;
    const bool keep = aux.z >= 128;
    float vd = 0.f, va = 0.f, ld = 0.f, ls = 0.f, lf = 0.f;
    if (!keep) {
        if (a.mask_photometric) st3(a.v_photo, (int64_t)pix, V3{0.f, 0.f, 0.f});
    } else {
        const float A = 1.f - a.final_T[pix];
        if (sky) {
            ls = a.sky_weight * A;
            va = a.sky_weight * a.inv_npix;
        } else {
            if (use_sky && a.fill_weight > 0.f) {
                lf = a.fill_weight * (1.f - A);
                va -= a.fill_weight * a.inv_npix;
            }
            const float D = a.out_depth[pix];
            if (use_depth && a.depth_weight > 0.f && conf > 0.f && A > a.min_alpha && D > 0.f) {
                const float dp = prior_depth_at(a.prior_depth, sx - 0.5f, sy - 0.5f, pw, ph);
                if (dp > 0.f) {
                    const float r = log_ref(D / A) - log_ref(dp);
                    const float ar = fabsf(r);
                    float dr;
                    if (ar < a.huber) {
                        ld = a.depth_weight * conf * 0.5f * r * r / a.huber;
                        dr = r / a.huber;
                    } else {
                        ld = a.depth_weight * conf * (ar - 0.5f * a.huber);
                        dr = r > 0.f ? 1.f : (r < 0.f ? -1.f : 0.f);
                    }
                    const float s = a.depth_weight * conf * dr * a.inv_npix;
                    vd = s / D;
                    va -= s / A;
                }
            }
        }
    }
    reinterpret_cast<float2 *>(a.v_aux)[pix] = make_float2(vd, va);
    if (a.terms) {
        a.terms[pix] = ld;
        a.terms[pix + (size_t)a.W * a.H] = ls;
        a.terms[pix + 2 * (size_t)a.W * a.H] = lf;
    }
}

// one thread per row: the row's three double sums in x order (:896)
__global__ void prior_rows_kernel(const float *terms, int W, int H, double *rows) {
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= H) return;
    const size_t plane = (size_t)W * H;
    const float *r = terms + (size_t)y * W;
    double ld = 0, ls = 0, lf = 0;
    for (int x = 0; x < W; x++) {
        ld += r[x];
        ls += r[x + plane];
        lf += r[x + 2 * plane];
    }
    rows[3 * (size_t)y] = ld;
    rows[3 * (size_t)y + 1] = ls;
    rows[3 * (size_t)y + 2] = lf;
}

// rows in y order, scaled and added to the step's loss terms (:894-900)
__global__ void prior_terms_kernel(const double *rows, int H, float inv_npix, float *loss_terms) {
    const int k = threadIdx.x;
    if (k >= 3) return;
    double t = 0.0;
    for (int y = 0; y < H; y++) t += rows[3 * (size_t)y + k];
    loss_terms[k] += (float)(t * inv_npix);
}

// ---- exposure (:904-937) ----------------------------------------------------------

__global__ void exposure_apply_kernel(const float *img, const float *P, int64_t n, float *out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3 c = ld3(img, i);
    st3(out, i, V3{dot3(V3{P[0], P[1], P[2]}, c) + P[9], dot3(V3{P[3], P[4], P[5]}, c) + P[10],
                   dot3(V3{P[6], P[7], P[8]}, c) + P[11]});
}

constexpr int EXPO_THREADS = 256, EXPO_ITEMS = 4, EXPO_PIX = EXPO_THREADS * EXPO_ITEMS;

// v_img = M^T v_adj per pixel, and per block the 12 parameter-gradient sums in double
// (each thread its EXPO_ITEMS consecutive pixels, then a fixed tree over the block)
__global__ void __launch_bounds__(EXPO_THREADS) exposure_backward_kernel(const float *img, const float *P,
                                                                          const float *v_adj, int64_t n,
                                                                          float *v_img, double *partials) {
    __shared__ double red[12][EXPO_THREADS];
    double g[12];
#pragma unroll
    for (int k = 0; k < 12; k++) g[k] = 0.0;
    const int64_t i0 = (int64_t)blockIdx.x * EXPO_PIX + (int64_t)threadIdx.x * EXPO_ITEMS;
    for (int j = 0; j < EXPO_ITEMS; j++) {
        const int64_t i = i0 + j;
        if (i >= n) break;
        const V3 c = ld3(img, i), v = ld3(v_adj, i);
        st3(v_img, i, V3{P[0] * v.x + P[3] * v.y + P[6] * v.z, P[1] * v.x + P[4] * v.y + P[7] * v.z,
                         P[2] * v.x + P[5] * v.y + P[8] * v.z});
        g[0] += v.x * c.x; g[1] += v.x * c.y; g[2] += v.x * c.z;
        g[3] += v.y * c.x; g[4] += v.y * c.y; g[5] += v.y * c.z;
        g[6] += v.z * c.x; g[7] += v.z * c.y; g[8] += v.z * c.z;
        g[9] += v.x; g[10] += v.y; g[11] += v.z;
    }
#pragma unroll
    for (int k = 0; k < 12; k++) red[k][threadIdx.x] = g[k];
    __syncthreads();
    for (int s = EXPO_THREADS / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
#pragma unroll
            for (int k = 0; k < 12; k++) red[k][threadIdx.x] += red[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 12) partials[(size_t)blockIdx.x * 12 + threadIdx.x] = red[threadIdx.x][0];
}

// the block partials in block order, then Adam towards the identity (:929-936)
__global__ void exposure_adam_kernel(const double *partials, int nblocks, ExposureArgs e) {
    const int k = threadIdx.x;
    if (k >= 12) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; b++) s += partials[(size_t)b * 12 + k];
    const int i = 12 * e.cam + k;
    const float ident = (k == 0 || k == 4 || k == 8) ? 1.f : 0.f;
    const float gk = (float)s + (e.grad ? e.grad[k] : 0.f) + e.reg * (e.params[i] - ident);
    if (e.grad) e.grad[k] = 0.f;
    adam_step(e.params[i], e.exp_avg[i], e.exp_avg_sq[i], gk, e.step_size, e.beta1, e.beta2, e.bc2, e.eps);
}

// ---- sky backward (:940-964) ------------------------------------------------------

// per pixel still seeing the sky: its taps, their weights, T * dL/dC, and how many
// taps carry weight
__global__ void sky_taps_kernel(const SkyArgs s, int W, int H, const float *final_T, const float *v_img,
                                uint4 *tap_idx, float4 *tap_w, float4 *tap_g, int32_t *count) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const size_t pix = (size_t)y * W + x;
    const float T = final_T[pix];
    if (T < 1e-4f) {
        count[pix] = 0;
        return;
    }
    const Taps t = pixel_taps(x, y, s);
    const V3 g = scl(T, ld3(v_img, (int64_t)pix));
    tap_idx[pix] = make_uint4(t.idx[0], t.idx[1], t.idx[2], t.idx[3]);
    tap_w[pix] = make_float4(t.w[0], t.w[1], t.w[2], t.w[3]);
    tap_g[pix] = make_float4(g.x, g.y, g.z, 0.f);
    count[pix] = (t.w[0] != 0.f) + (t.w[1] != 0.f) + (t.w[2] != 0.f) + (t.w[3] != 0.f);
}

// entries in pixel-then-tap order: key = texel, value = pixel * 4 + tap
__global__ void sky_emit_kernel(int64_t npix, const uint4 *tap_idx, const float4 *tap_w, const int32_t *count,
                                const int32_t *off, uint32_t *keys, uint32_t *vals) {
    const int64_t pix = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= npix || count[pix] == 0) return;
    const uint4 id = tap_idx[pix];
    const float4 w = tap_w[pix];
    const uint32_t ids[4] = {id.x, id.y, id.z, id.w};
    const float ws[4] = {w.x, w.y, w.z, w.w};
    int o = off[pix];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (ws[k] == 0.f) continue;
        keys[o] = ids[k];
        vals[o] = (uint32_t)(pix * 4 + k);
        o++;
    }
}

__device__ __forceinline__ int lower_bound_u32(const uint32_t *keys, int n, uint32_t t) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (keys[mid] < t) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// one thread per texel: its contributions in sorted (= pixel, tap) order, then Adam on
// its three channels (the reference's Adam runs over the whole texture, :959-963)
__global__ void sky_texel_adam_kernel(const uint32_t *keys, const uint32_t *vals, const int32_t *d_n, int n_texels,
                                      const float4 *tap_w, const float4 *tap_g, SkyAdamArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_texels) return;
    const int n = *d_n;
    const int lo = lower_bound_u32(keys, n, (uint32_t)t), hi = lower_bound_u32(keys, n, (uint32_t)t + 1u);
    float sx = 0.f, sy = 0.f, sz = 0.f;
    for (int e = lo; e < hi; e++) {
        const uint32_t v = vals[e];
        const uint32_t pix = v >> 2, k = v & 3u;
        const float4 w4 = tap_w[pix];
        const float w = k == 0 ? w4.x : (k == 1 ? w4.y : (k == 2 ? w4.z : w4.w));
        const float4 g = tap_g[pix];
        sx += w * g.x;
        sy += w * g.y;
        sz += w * g.z;
    }
    const float gs[3] = {sx, sy, sz};
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const size_t i = 3 * (size_t)t + c;
        a.grad[i] = gs[c];
        adam_step(a.tex[i], a.exp_avg[i], a.exp_avg_sq[i], gs[c], a.step_size, a.beta1, a.beta2, a.bc2, a.eps);
    }
}

}  // namespace

void launch_sky_background(const SkyArgs &s, int W, int H, float *bg_img, cudaStream_t st) {
    if (W <= 0 || H <= 0) return;
    const dim3 blk(16, 16), grid((W + 15) / 16, (H + 15) / 16);
    sky_background_kernel<<<grid, blk, 0, st>>>(s, W, H, bg_img);
}

void launch_prior_loss(const PriorLossArgs &a, double *rows, float *loss_terms, cudaStream_t st) {
    if (a.W <= 0 || a.H <= 0) return;
    const dim3 blk(32, 8), grid((a.W + 31) / 32, (a.H + 7) / 8);
    prior_loss_kernel<<<grid, blk, 0, st>>>(a);
    if (a.terms && loss_terms) {
        prior_rows_kernel<<<(a.H + 63) / 64, 64, 0, st>>>(a.terms, a.W, a.H, rows);
        prior_terms_kernel<<<1, 32, 0, st>>>(rows, a.H, a.inv_npix, loss_terms);
    }
}

void launch_exposure_apply(const float *img, const float *P, int64_t n, float *out, cudaStream_t st) {
    if (n <= 0) return;
    exposure_apply_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(img, P, n, out);
}

int exposure_blocks(int64_t n) { return (int)std::max<int64_t>(1, (n + EXPO_PIX - 1) / EXPO_PIX); }

void launch_exposure_backward_adam(const float *img, const float *v_adj, int64_t n, float *v_img, double *partials,
                                   const ExposureArgs &e, cudaStream_t st) {
    const int nb = exposure_blocks(n);
    const float *P = e.params + 12 * (size_t)e.cam;
    if (n > 0) exposure_backward_kernel<<<nb, EXPO_THREADS, 0, st>>>(img, P, v_adj, n, v_img, partials);
    else cudaMemsetAsync(partials, 0, 12 * sizeof(double), st);
    exposure_adam_kernel<<<1, 32, 0, st>>>(partials, nb, e);
}

void launch_sky_backward_adam(const SkyArgs &s, int W, int H, const float *final_T, const float *v_img,
                              const SkyAdamArgs &a, SkyScratch &sc, cudaStream_t st) {
    const int64_t npix = (int64_t)W * H;
    const int n_texels = s.tex_w * s.tex_h;
    if (npix > 0) {
        const dim3 blk(16, 16), grid((W + 15) / 16, (H + 15) / 16);
        sky_taps_kernel<<<grid, blk, 0, st>>>(s, W, H, final_T, v_img, sc.tap_idx, sc.tap_w, sc.tap_g, sc.count);
        scan_exclusive<int32_t>(sc.count, sc.off, (int)npix, sc.d_total, sc.scan_part, st);
        sky_emit_kernel<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(npix, sc.tap_idx, sc.tap_w, sc.count, sc.off,
                                                                       sc.keys[0], sc.vals[0]);
    } else {
        cudaMemsetAsync(sc.d_total, 0, sizeof(int32_t), st);
    }
    uint32_t *kk[2] = {sc.keys[0], sc.keys[1]};
    uint32_t *vv[2] = {sc.vals[0], sc.vals[1]};
    int bits = 0;
    while ((1 << bits) < n_texels) bits++;
    const int cur = radix_sort_pairs32(kk, vv, (int)std::max<int64_t>(4 * npix, 1), std::max(bits, 1),
                                       sc.radix_scratch, st, sc.d_total);
    sky_texel_adam_kernel<<<(n_texels + 127) / 128, 128, 0, st>>>(kk[cur], vv[cur], sc.d_total, n_texels, sc.tap_w,
                                                                   sc.tap_g, a);
}

__global__ void needle_cap_kernel(float *scales, int n, float log_max) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float *s = scales + 3 * (size_t)i;
    const float a = s[0], b = s[1], c = s[2];
    const float mx = fmaxf(a, fmaxf(b, c)), mn = fminf(a, fminf(b, c));
    const float cap = (a + b + c - mx - mn) + log_max;
    if (mx <= cap) return;
    if (a == mx) s[0] = cap;
    else if (b == mx) s[1] = cap;
    else s[2] = cap;
}

void launch_needle_cap(float *scales, int n, float log_max, cudaStream_t st) {
    if (n <= 0) return;
    needle_cap_kernel<<<(n + 255) / 256, 256, 0, st>>>(scales, n, log_max);
}

}  // namespace msplat
