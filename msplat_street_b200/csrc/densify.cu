// Densification: classify, split, duplicate, cull and stream compaction; opacity reset.
//
// Follows msplat_densify (core/cpu/msplat_cpu.cpp:1330-1465) step by step:
//  1. classify (:1354-1369): a Gaussian seen in at least one view with mean screen
//     gradient (gn / vc) * half_max_dim above the threshold is split when its largest
//     scale exceeds size_thresh (or its screen size split_screen_size), and cloned
//     when it is small;
//  2. ordinals by exclusive scans (the reference counts serially, :1370-1375);
//  3. split children at N + 2*ord + k, offset by a parent-rotated N(0, s) sample
//     from the PCG/Box-Muller counter RNG, scales minus log(1.6); the parent's scales
//     shrink too (:1387-1415); then clones at N + 2*n_split + ord (:1417-1430), after
//     every split (a Gaussian may be both, and the clone copies the shrunk parent).
//     These per-parent kernels write only positions and scales and record each new
//     row's parent; one row-parallel pass per parameter group then copies the
//     quaternion, colour and opacity rows and zeroes the moments, coalesced;
//  4. cull (:1432-1448) over the N_new rows and order-preserving compaction of all 18
//     buffers (6 parameters, 6 first moments, 6 second moments) through a scratch
//     buffer, one buffer at a time (:1449-1464).
// A Gaussian can be both split (large on screen) and cloned (small in the world), so
// the rows after step 3 number up to 4N, not 3N as the reference's capacity check
// assumes (its CPU port would then write past its buffers). Here every kernel from
// step 3 on first checks N + 2 splits + clones against the capacity; when it does not
// fit, nothing is written and the overflow flag is set (the host reports it).
// Child and clone moments are zeroed. Counts live on the device; the host reads the
// final count once (the reference's Metal backend also syncs there,
// core/metal/msplat_metal.mm:1998-2001).
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace msplat {

__global__ void densify_classify_kernel(DensifyArgs a, int32_t *split, int32_t *dup) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    int s = 0, d = 0;
    const float vc = a.vis_counts[i];
    if (vc > 0.0f) {
        const bool high = (a.grad_norm[i] / vc) * a.half_max_dim > a.grad_thresh;
        const float *sc = a.buf[1] + 3 * (size_t)i;
        const float mx = fmaxf(fmaxf(exp_ref(sc[0]), exp_ref(sc[1])), exp_ref(sc[2]));
        const bool large = mx > a.size_thresh;
        bool sp = large;
        if (a.check_screen && a.max_2d[i] > a.screen_thresh) sp = true;
        s = (sp && high) ? 1 : 0;
        d = (!large && high) ? 1 : 0;
    }
    split[i] = s;
    dup[i] = d;
}

// Box-Muller on the PCG counter RNG (core/cpu/msplat_cpu.cpp:315-323)
__device__ __forceinline__ V3 rand_normal3(uint32_t seed, uint32_t stream) {
    const uint32_t c = stream * 4u;
    const float u0 = rand_unif(seed, c), u1 = rand_unif(seed, c + 1u);
    const float u2 = rand_unif(seed, c + 2u), u3 = rand_unif(seed, c + 3u);
    const float r0 = sqrtf(-2.0f * (float)log((double)u0)), r1 = sqrtf(-2.0f * (float)log((double)u2));
    const float tau = 6.28318530717958647692f;
    const float t0 = tau * u1, t1 = tau * u3;
    return V3{r0 * (float)cos((double)t0), r0 * (float)sin((double)t0), r1 * (float)cos((double)t1)};
}

// rows after splits and clones, and whether they fit the buffers
__device__ __forceinline__ bool rows_fit(const DensifyArgs &a, const int32_t *n_split, const int32_t *n_dup,
                                         int64_t &total) {
    total = (int64_t)a.n + 2 * (int64_t)(*n_split) + *n_dup;
    return total <= a.cap;
}

__global__ void densify_split_kernel(DensifyArgs a, const int32_t *split, const int32_t *split_ord,
                                     const int32_t *n_split, const int32_t *n_dup, int32_t *overflow,
                                     int32_t *row_parent) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int64_t total;
    if (!rows_fit(a, n_split, n_dup, total)) {
        if (i == 0) *overflow = 1;
        return;
    }
    if (i >= a.n || !split[i]) return;
    const int ord = split_ord[i];
    float *means = a.buf[0], *scales = a.buf[1];
    const float *q = a.buf[2] + 4 * (size_t)i;
    float qw = q[0], qx = q[1], qy = q[2], qz = q[3];
    const float ql = sqrtf(qw * qw + qx * qx + qy * qy + qz * qz);
    qw /= ql;
    qx /= ql;
    qy /= ql;
    qz /= ql;
    const float sx = exp_ref(scales[3 * i]), sy = exp_ref(scales[3 * i + 1]), sz = exp_ref(scales[3 * i + 2]);
    for (int k = 0; k < 2; k++) {
        const int64_t c = (int64_t)a.n + 2 * ord + k;
        const V3 nr = rand_normal3(a.seed, (uint32_t)(ord * 2 + k));
        const float r0 = nr.x * sx, r1 = nr.y * sy, r2 = nr.z * sz;
        const float v0 = (1.f - 2.f * (qy * qy + qz * qz)) * r0 + 2.f * (qx * qy - qw * qz) * r1 +
                         2.f * (qx * qz + qw * qy) * r2;
        const float v1 = 2.f * (qx * qy + qw * qz) * r0 + (1.f - 2.f * (qx * qx + qz * qz)) * r1 +
                         2.f * (qy * qz - qw * qx) * r2;
        const float v2 = 2.f * (qx * qz - qw * qy) * r0 + 2.f * (qy * qz + qw * qx) * r1 +
                         (1.f - 2.f * (qx * qx + qy * qy)) * r2;
        means[3 * c] = means[3 * i] + v0;
        means[3 * c + 1] = means[3 * i + 1] + v1;
        means[3 * c + 2] = means[3 * i + 2] + v2;
        for (int j = 0; j < 3; j++) scales[3 * c + j] = scales[3 * i + j] - a.log_size_fac;
        row_parent[2 * ord + k] = i;  // the other groups are copied row-parallel (densify_rows_kernel)
    }
    for (int j = 0; j < 3; j++) scales[3 * i + j] -= a.log_size_fac;
}

__global__ void densify_dup_kernel(DensifyArgs a, const int32_t *dup, const int32_t *dup_ord, const int32_t *n_split,
                                   const int32_t *n_dup, int32_t *row_parent) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int64_t total;
    if (!rows_fit(a, n_split, n_dup, total)) return;
    if (i >= a.n || !dup[i]) return;
    const int64_t r = 2 * (int64_t)(*n_split) + dup_ord[i];  // new-row index; row a.n + r
    const int64_t d = (int64_t)a.n + r;
    for (int j = 0; j < 3; j++) a.buf[0][3 * d + j] = a.buf[0][3 * i + j];
    for (int j = 0; j < 3; j++) a.buf[1][3 * d + j] = a.buf[1][3 * i + j];  // a split parent's shrunk scales
    row_parent[r] = i;
}

// The new rows a.n .. total - 1 (split children, then clones), one thread per element:
// quaternion, DC, SH rest and opacity copied from the row's parent, every moment
// zeroed. Consecutive threads write consecutive floats of consecutive rows.
__global__ void densify_rows_kernel(DensifyArgs a, const int32_t *n_split, const int32_t *n_dup,
                                    const int32_t *row_parent, int g) {
    int64_t total;
    if (!rows_fit(a, n_split, n_dup, total)) return;
    const int st = a.stride[g];
    const int64_t elems = (total - a.n) * st;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < elems;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = t / st;
        const int col = (int)(t - r * st);
        const int64_t dst = ((int64_t)a.n + r) * st + col;
        if (g >= 2) a.buf[g][dst] = a.buf[g][(int64_t)row_parent[r] * st + col];
        a.m1[g][dst] = 0.f;
        a.m2[g][dst] = 0.f;
    }
}

__global__ void densify_cull_kernel(DensifyArgs a, const int32_t *split, const int32_t *n_split,
                                    const int32_t *n_dup, int32_t *keep, int32_t *n_new) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t total;
    const bool fit = rows_fit(a, n_split, n_dup, total);
    if (i == 0) *n_new = fit ? (int32_t)total : 0;  // no rows to compact when they did not fit
    if (i >= 4 * (int64_t)a.n) return;
    if (!fit || i >= total) {
        keep[i] = 0;
        return;
    }
    const float o = 1.0f / (1.0f + exp_ref(-a.buf[5][i]));
    bool cull = o < a.cull_alpha;
    if (i < a.n && split[i]) cull = true;
    if (a.check_huge) {
        const float *sc = a.buf[1] + 3 * i;
        const float mx = fmaxf(fmaxf(exp_ref(sc[0]), exp_ref(sc[1])), exp_ref(sc[2]));
        if (mx > a.cull_scale) cull = true;
        if (a.check_screen && i < a.n && a.max_2d[i] > a.cull_screen) cull = true;
    }
    keep[i] = cull ? 0 : 1;
}

// one buffer: kept rows to scratch at their ordinal, then back. Grid-stride loops with
// several elements per thread keep more loads in flight; the copy back moves float4s
// when both arrays are 16-byte aligned.
constexpr int COMPACT_ITEMS = 4;

__global__ void compact_gather_kernel(const float *src, float *scratch, int stride, const int32_t *keep,
                                      const int32_t *keep_ord, const int32_t *n_new) {
    const int64_t elems = (int64_t)(*n_new) * stride;
    const int64_t step = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; base < elems; base += step * COMPACT_ITEMS) {
#pragma unroll
        for (int u = 0; u < COMPACT_ITEMS; u++) {
            const int64_t t = base + u * step;
            if (t >= elems) break;
            const int64_t row = t / stride;
            if (!keep[row]) continue;
            const int col = (int)(t - row * stride);
            scratch[(int64_t)keep_ord[row] * stride + col] = src[t];
        }
    }
}

__global__ void compact_copy_back_kernel(float *dst, const float *scratch, int stride, const int32_t *new_count,
                                         const int32_t *overflow, int vec4) {
    if (*overflow) return;
    const int64_t elems = (int64_t)(*new_count) * stride;
    const int64_t step = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (vec4) {
        const int64_t n4 = elems / 4;
        float4 *d4 = reinterpret_cast<float4 *>(dst);
        const float4 *s4 = reinterpret_cast<const float4 *>(scratch);
        for (int64_t t = t0; t < n4; t += step) d4[t] = s4[t];
        for (int64_t t = 4 * n4 + t0; t < elems; t += step) dst[t] = scratch[t];
    } else {
        for (int64_t t = t0; t < elems; t += step) dst[t] = scratch[t];
    }
}

__global__ void opacity_reset_kernel(float *o, float *m1, float *m2, int n, float reset_logit) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    o[i] = fminf(o[i], reset_logit);
    m1[i] = 0.f;
    m2[i] = 0.f;
}

void launch_densify(const DensifyArgs &a, DensifyScratch &s, cudaStream_t st) {
    const int n = a.n;
    if (n <= 0) {
        cudaMemsetAsync(s.new_count, 0, sizeof(int32_t), st);
        return;
    }
    const int bs = 256;
    const int gb = (n + bs - 1) / bs;
    densify_classify_kernel<<<gb, bs, 0, st>>>(a, s.split, s.dup);
    scan_exclusive<int32_t>(s.split, s.split_ord, n, s.n_split, s.scan_part, st);
    scan_exclusive<int32_t>(s.dup, s.dup_ord, n, s.n_dup, s.scan_part, st);
    cudaMemsetAsync(s.overflow, 0, sizeof(int32_t), st);
    densify_split_kernel<<<gb, bs, 0, st>>>(a, s.split, s.split_ord, s.n_split, s.n_dup, s.overflow, s.row_parent);
    densify_dup_kernel<<<gb, bs, 0, st>>>(a, s.dup, s.dup_ord, s.n_split, s.n_dup, s.row_parent);
    const int64_t rows = 4 * (int64_t)n;  // at most N + 2 N splits + N clones
    for (int g = 0; g < 6; g++) {
        if (a.stride[g] <= 0) continue;
        const int64_t most = 3 * (int64_t)n * a.stride[g];  // new rows are at most 3 N
        const unsigned grid = (unsigned)std::min<int64_t>((most + bs - 1) / bs, 148 * 64);
        densify_rows_kernel<<<grid, bs, 0, st>>>(a, s.n_split, s.n_dup, s.row_parent, g);
    }
    densify_cull_kernel<<<(unsigned)((rows + bs - 1) / bs), bs, 0, st>>>(a, s.split, s.n_split, s.n_dup, s.keep,
                                                                       s.n_new);
    scan_exclusive<int32_t>(s.keep, s.keep_ord, (int)rows, s.new_count, s.scan_part, st);
    const int sms_blocks = 148 * 8;  // enough resident blocks for the grid-stride loops
    for (int b = 0; b < 18; b++) {
        const int g = b % 6;
        float *buf = b < 6 ? a.buf[g] : (b < 12 ? a.m1[g] : a.m2[g]);
        const int stride = a.stride[g];
        if (stride <= 0) continue;  // e.g. no SH rest at degree 0
        const int64_t elems = rows * stride;
        const unsigned grid =
            (unsigned)std::max<int64_t>(1, std::min<int64_t>((elems / COMPACT_ITEMS + bs - 1) / bs, sms_blocks));
        compact_gather_kernel<<<grid, bs, 0, st>>>(buf, s.scratch, stride, s.keep, s.keep_ord, s.n_new);
        const int vec4 = ((reinterpret_cast<uintptr_t>(buf) | reinterpret_cast<uintptr_t>(s.scratch)) & 15) == 0;
        compact_copy_back_kernel<<<grid, bs, 0, st>>>(buf, s.scratch, stride, s.new_count, s.overflow, vec4);
    }
}

void launch_opacity_reset(float *o, float *m1, float *m2, int n, float reset_logit, cudaStream_t st) {
    if (n <= 0) return;
    opacity_reset_kernel<<<(n + 255) / 256, 256, 0, st>>>(o, m1, m2, n, reset_logit);
}

}  // namespace msplat
