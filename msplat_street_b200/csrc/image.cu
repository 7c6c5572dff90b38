// Image pipeline, evaluation metrics and display packing (the reference's
// bindings.h:158-180 group), one thread per output pixel unless said otherwise.
//
// Each kernel keeps the reference's float32 operation order (core/cpu/msplat_cpu.cpp:
// 1609-1745; -fmad=false), so resize, undistortion, packing and depth finalisation
// match it bit for bit. The metrics keep its summation order too: per-pixel terms in
// float, each row summed in double in (x, channel) order, then the rows in order.
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace msplat {

// Area (box) resample (msplat_cpu.cpp:1609-1639). src: (sh, sw, 4) RGBA8 when u8in,
// else (sh, sw, 3) float.
__global__ void resize_area_kernel(const void *src, int u8in, int sw, int sh, float *dst, int dw, int dh) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y;
    if (gx >= dw || gy >= dh) return;
    const uint8_t *u8 = u8in ? static_cast<const uint8_t *>(src) : nullptr;
    const float *fs = u8in ? nullptr : static_cast<const float *>(src);
    const float sxs = (float)sw / (float)dw, sys = (float)sh / (float)dh;
    const float y0 = (float)gy * sys, y1 = (float)(gy + 1) * sys;
    const int iy0 = (int)y0, iy1 = min((int)ceilf(y1), sh);
    const float x0 = (float)gx * sxs, x1 = (float)(gx + 1) * sxs;
    const int ix0 = (int)x0, ix1 = min((int)ceilf(x1), sw);
    float sr = 0.f, sg = 0.f, sb = 0.f, area = 0.f;
    for (int iy = iy0; iy < iy1; iy++) {
        const float wy = fminf((float)(iy + 1), y1) - fmaxf((float)iy, y0);
        for (int ix = ix0; ix < ix1; ix++) {
            const float wx = fminf((float)(ix + 1), x1) - fmaxf((float)ix, x0);
            const size_t s = (size_t)iy * sw + ix;
            float r, g, b;
            if (u8) {
                r = (float)u8[4 * s] * (1.f / 255.f);
                g = (float)u8[4 * s + 1] * (1.f / 255.f);
                b = (float)u8[4 * s + 2] * (1.f / 255.f);
            } else {
                r = fs[3 * s];
                g = fs[3 * s + 1];
                b = fs[3 * s + 2];
            }
            const float w = wx * wy;
            sr = sr + w * r;
            sg = sg + w * g;
            sb = sb + w * b;
            area += w;
        }
    }
    float *o = dst + 3 * ((size_t)gy * dw + gx);
    o[0] = sr / area;
    o[1] = sg / area;
    o[2] = sb / area;
}

// Brown-Conrady undistortion with bilinear sampling (msplat_cpu.cpp:1641-1669).
__global__ void undistort_kernel(const float *in, int sw, int sh, float fx, float fy, float cx, float cy, float k1,
                                 float k2, float p1, float p2, float k3, int rx, int ry, float *out, int dw, int dh) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y;
    if (gx >= dw || gy >= dh) return;
    const float x = ((float)(gx + rx) + 0.5f - cx) / fx;
    const float y = ((float)(gy + ry) + 0.5f - cy) / fy;
    const float r2 = x * x + y * y;
    const float rad = 1.f + k1 * r2 + k2 * r2 * r2 + k3 * r2 * r2 * r2;
    const float xd = x * rad + 2.f * p1 * x * y + p2 * (r2 + 2.f * x * x);
    const float yd = y * rad + p1 * (r2 + 2.f * y * y) + 2.f * p2 * x * y;
    const float sx = xd * fx + cx - 0.5f, sy = yd * fy + cy - 0.5f;
    const int x0 = (int)floorf(sx), y0 = (int)floorf(sy);
    const float ax = sx - floorf(sx), ay = sy - floorf(sy);
    const int xa = min(max(x0, 0), sw - 1), xb = min(max(x0 + 1, 0), sw - 1);
    const int ya = min(max(y0, 0), sh - 1), yb = min(max(y0 + 1, 0), sh - 1);
    const float *c00 = in + 3 * ((size_t)ya * sw + xa), *c10 = in + 3 * ((size_t)ya * sw + xb);
    const float *c01 = in + 3 * ((size_t)yb * sw + xa), *c11 = in + 3 * ((size_t)yb * sw + xb);
    float *o = out + 3 * ((size_t)gy * dw + gx);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float top = c00[c] * (1.f - ax) + c10[c] * ax;
        const float bot = c01[c] * (1.f - ax) + c11[c] * ax;
        o[c] = top * (1.f - ay) + bot * ay;
    }
}

__constant__ float kWinM[11] = {0.0010283801f, 0.0075987581f, 0.0360007721f, 0.1093606895f,
                                0.2130055377f, 0.2660117249f, 0.2130055377f, 0.1093606895f,
                                0.0360007721f, 0.0075987581f, 0.0010283801f};

// Metrics pass 1: horizontal 11-tap moments with clamp-to-edge columns, 15 floats per
// pixel (5 per channel) (msplat_cpu.cpp:1675-1688).
__global__ void metrics_h_kernel(const float *a, const float *b, int h, int w, float *hb) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    float *o = hb + ((size_t)y * w + x) * 15;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f, s4 = 0.f;
        for (int k = 0; k < 11; k++) {
            const int sx = min(max(x + k - 5, 0), w - 1);
            const size_t i = ((size_t)y * w + sx) * 3 + c;
            const float gk = kWinM[k], xa = a[i], yb = b[i];
            s0 += gk * xa;
            s1 += gk * yb;
            s2 += gk * xa * xa;
            s3 += gk * yb * yb;
            s4 += gk * xa * yb;
        }
        o[5 * c] = s0;
        o[5 * c + 1] = s1;
        o[5 * c + 2] = s2;
        o[5 * c + 3] = s3;
        o[5 * c + 4] = s4;
    }
}

// Metrics pass 2: vertical taps, the per-(pixel, channel) SSIM term, |d| and d^2
// (msplat_cpu.cpp:1690-1712), stored for the ordered row sums.
__global__ void metrics_v_kernel(const float *a, const float *b, int h, int w, const float *hb, float *t_ssim,
                                 float *t_l1, double *t_sq) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    const float C1 = 0.0001f, C2 = 0.0009f;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float s[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
        for (int k = 0; k < 11; k++) {
            const int sy = min(max(y + k - 5, 0), h - 1);
            const float *o = hb + ((size_t)sy * w + x) * 15 + c * 5;
#pragma unroll
            for (int q = 0; q < 5; q++) s[q] += kWinM[k] * o[q];
        }
        const float m12 = s[0] * s[1], m1 = s[0] * s[0], m2 = s[1] * s[1];
        const float num = (2.f * m12 + C1) * (2.f * (s[4] - m12) + C2);
        const float den = (m1 + m2 + C1) * ((s[2] - m1) + (s[3] - m2) + C2);
        const size_t i = ((size_t)y * w + x) * 3 + c;
        const float d = a[i] - b[i];
        t_ssim[i] = num / den;
        t_l1[i] = fabsf(d);
        t_sq[i] = (double)d * d;
    }
}

// Metrics pass 3: one thread per row sums its terms in double in (x, channel) order.
__global__ void metrics_rows_kernel(int h, int w, const float *t_ssim, const float *t_l1, const double *t_sq,
                                    double *rows) {
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= h) return;
    double rs = 0.0, rl = 0.0, rq = 0.0;
    const size_t o = (size_t)y * w * 3;
    for (int i = 0; i < w * 3; i++) {
        rs += t_ssim[o + i];
        rl += t_l1[o + i];
        rq += t_sq[o + i];
    }
    rows[3 * (size_t)y] = rs;
    rows[3 * (size_t)y + 1] = rl;
    rows[3 * (size_t)y + 2] = rq;
}

// Metrics pass 4: the rows in order, then PSNR / SSIM / L1 (msplat_cpu.cpp:1713-1720).
__global__ void metrics_final_kernel(int h, int w, const double *rows, double *out) {
    double ssim = 0.0, l1 = 0.0, sq = 0.0;
    for (int y = 0; y < h; y++) {
        ssim += rows[3 * (size_t)y];
        l1 += rows[3 * (size_t)y + 1];
        sq += rows[3 * (size_t)y + 2];
    }
    const double cnt = (double)h * w * 3, mse = sq / cnt;
    out[0] = mse > 0 ? 10.0 * log10(1.0 / mse) : INFINITY;
    out[1] = ssim / cnt;
    out[2] = l1 / cnt;
}

// Float RGB to RGBA8 (msplat_cpu.cpp:1723-1734).
__global__ void pack_rgba8_kernel(const float *img, uint32_t n, uint8_t *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uchar4 o;
    o.x = (uint8_t)(clamp01(img[3 * (size_t)i]) * 255.f);
    o.y = (uint8_t)(clamp01(img[3 * (size_t)i + 1]) * 255.f);
    o.z = (uint8_t)(clamp01(img[3 * (size_t)i + 2]) * 255.f);
    o.w = 255;
    reinterpret_cast<uchar4 *>(out)[i] = o;
}

// Expected depth and alpha from the aux render outputs (msplat_cpu.cpp:1736-1745).
__global__ void finalize_depth_kernel(const float *d, const float *t, uint32_t n, float inv_scale, float *od,
                                      float *oa) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float a = 1.f - t[i];
    oa[i] = a;
    od[i] = a > 1e-4f ? d[i] / a * inv_scale : 0.f;
}

void launch_resize_area(const void *src, int u8in, int sw, int sh, float *dst, int dw, int dh, cudaStream_t st) {
    if (dw <= 0 || dh <= 0) return;
    resize_area_kernel<<<dim3((dw + 127) / 128, dh), 128, 0, st>>>(src, u8in, sw, sh, dst, dw, dh);
}

void launch_undistort(const float *src, int sw, int sh, const float *intr, const float *dist, int rx, int ry,
                      float *dst, int dw, int dh, cudaStream_t st) {
    if (dw <= 0 || dh <= 0) return;
    undistort_kernel<<<dim3((dw + 127) / 128, dh), 128, 0, st>>>(src, sw, sh, intr[0], intr[1], intr[2], intr[3],
                                                                 dist[0], dist[1], dist[2], dist[3], dist[4], rx, ry,
                                                                 dst, dw, dh);
}

void launch_image_metrics(const float *a, const float *b, int h, int w, const MetricsScratch &s, double *out,
                          cudaStream_t st) {
    const dim3 grid((w + 127) / 128, h);
    metrics_h_kernel<<<grid, 128, 0, st>>>(a, b, h, w, s.hbuf);
    metrics_v_kernel<<<grid, 128, 0, st>>>(a, b, h, w, s.hbuf, s.t_ssim, s.t_l1, s.t_sq);
    metrics_rows_kernel<<<(h + 127) / 128, 128, 0, st>>>(h, w, s.t_ssim, s.t_l1, s.t_sq, s.rows);
    metrics_final_kernel<<<1, 1, 0, st>>>(h, w, s.rows, out);
}

void launch_pack_rgba8(const float *img, uint32_t n, uint8_t *out, cudaStream_t st) {
    if (n == 0) return;
    pack_rgba8_kernel<<<(n + 255) / 256, 256, 0, st>>>(img, n, out);
}

void launch_finalize_depth(const float *d, const float *t, uint32_t n, float inv_scale, float *od, float *oa,
                           cudaStream_t st) {
    if (n == 0) return;
    finalize_depth_kernel<<<(n + 255) / 256, 256, 0, st>>>(d, t, n, inv_scale, od, oa);
}

}  // namespace msplat
