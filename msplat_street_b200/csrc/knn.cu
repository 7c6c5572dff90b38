// Exact 3-nearest-neighbour mean distance and Gaussian initialisation.
//
// msplat_knn3_mean_dist (core/cpu/msplat_cpu.cpp:1498-1580 builds a k-d tree; the
// Metal backend sorts by Morton code and culls by box distance) returns, for every
// point, the mean distance to its 3 nearest OTHER points (fewer if n < 4, 1.0 if
// none). Here points are sorted by a 30-bit Morton code with the device radix sort and
// cut into boxes of 32 consecutive points. One warp answers one box's 32 queries: its
// lanes test 32 candidate boxes at a time, nearest Morton neighbours first, against
// the query box's bounds; a box survives only if its lower-bound squared distance is
// below the warp's worst current third-best, then its 32 points are streamed through
// the warp with shuffles. The lower bound uses the same float subtractions and
// squares as the point distances, and float rounding is monotonic, so a pruned box
// can hold no point that would enter a lane's best three: the result is exact.
//
// msplat_init_gaussians (:1582-1605): isotropic log-scale log(max(d, 1e-7)), a
// uniformly random rotation from three PCG uniforms (Shoemake), DC colour from RGB
// and a constant opacity logit.
#include "common.cuh"
#include "kernels.h"

namespace msplat {

constexpr int KNN_BOX = 32;

__device__ __forceinline__ unsigned int ordered_bits(float f) {
    unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_ordered(unsigned int u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void knn_bounds_kernel(const float *pts, int n, unsigned int *bb) {
    unsigned int mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int a = 0; a < 3; a++) {
            const float v = pts[3 * (size_t)i + a];
            if (!isfinite(v)) continue;
            const unsigned int o = ordered_bits(v);
            mn[a] = min(mn[a], o);
            mx[a] = max(mx[a], o);
        }
    for (int a = 0; a < 3; a++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&bb[a], mn[a]);
            atomicMax(&bb[3 + a], mx[a]);
        }
    }
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__global__ void knn_morton_kernel(const float *pts, int n, const unsigned int *bb, uint64_t *keys, uint32_t *vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t q[3];
    for (int a = 0; a < 3; a++) {
        const float lo = from_ordered(bb[a]), hi = from_ordered(bb[3 + a]);
        const float ext = hi - lo;
        const float v = pts[3 * (size_t)i + a];
        float t = (isfinite(v) && ext > 0.f) ? (v - lo) / ext : 0.f;
        t = fminf(fmaxf(t, 0.f), 1.f);
        q[a] = (uint32_t)(t * 1023.f);
    }
    keys[i] = (uint64_t)(spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2));
    vals[i] = (uint32_t)i;
}

__global__ void knn_gather_kernel(const float *pts, int n, const uint32_t *order, float4 *sp) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t i = order[j];
    sp[j] = make_float4(pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2], __uint_as_float(i));
}

__global__ void knn_boxes_kernel(const float4 *sp, int n, int nboxes, float4 *bmin, float4 *bmax) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nboxes) return;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    const int end = min(n, (b + 1) * KNN_BOX);
    for (int j = b * KNN_BOX; j < end; j++) {
        const float4 p = sp[j];
        const float c[3] = {p.x, p.y, p.z};
        for (int a = 0; a < 3; a++)
            if (isfinite(c[a])) {
                lo[a] = fminf(lo[a], c[a]);
                hi[a] = fmaxf(hi[a], c[a]);
            }
    }
    bmin[b] = make_float4(lo[0], lo[1], lo[2], 0.f);
    bmax[b] = make_float4(hi[0], hi[1], hi[2], 0.f);
}

// best[0] <= best[1] <= best[2] (core/cpu/msplat_cpu.cpp:1522-1531)
__device__ __forceinline__ void keep3(float d, float &b0, float &b1, float &b2) {
    if (d >= b2) return;
    if (d < b1) {
        b2 = b1;
        if (d < b0) {
            b1 = b0;
            b0 = d;
        } else {
            b1 = d;
        }
    } else {
        b2 = d;
    }
}

__device__ __forceinline__ float gap(float qlo, float qhi, float blo, float bhi) {
    return fmaxf(fmaxf(blo - qhi, qlo - bhi), 0.f);
}

// evals (may be null): adds the point distances the warp computes (32 per query per
// surviving box) -- the search's work, for throughput reports.
__global__ void knn_query_kernel(const float4 *sp, int n, int nboxes, const float4 *bmin, const float4 *bmax,
                                 float *out, unsigned long long *evals) {
    const int lane = threadIdx.x & 31;
    const int own = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    if (own >= nboxes) return;  // warp-uniform
    const int j = own * KNN_BOX + lane;
    const bool valid = j < n;
    const float4 q = valid ? sp[j] : make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t self = __float_as_uint(q.w);
    const bool fin = valid && isfinite(q.x) && isfinite(q.y) && isfinite(q.z);
    // bounds of the warp's queries
    float ql[3] = {fin ? q.x : INFINITY, fin ? q.y : INFINITY, fin ? q.z : INFINITY};
    float qh[3] = {fin ? q.x : -INFINITY, fin ? q.y : -INFINITY, fin ? q.z : -INFINITY};
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ql[a] = fminf(ql[a], __shfl_xor_sync(0xffffffffu, ql[a], o));
            qh[a] = fmaxf(qh[a], __shfl_xor_sync(0xffffffffu, qh[a], o));
        }
    float b0 = INFINITY, b1 = INFINITY, b2 = INFINITY;
    const unsigned nq = __popc(__ballot_sync(0xffffffffu, fin));  // queries with a finite point
    // candidate t visits own, own+1, own-1, own+2, own-2, ...
    const int span = 2 * nboxes;
    for (int t0 = 0; t0 < span; t0 += 32) {
        const int t = t0 + lane;
        const int c = own + ((t & 1) ? (t + 1) / 2 : -(t / 2));
        float thr = fin ? b2 : -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) thr = fmaxf(thr, __shfl_xor_sync(0xffffffffu, thr, o));
        bool pass = false;
        if (t < span && c >= 0 && c < nboxes && ql[0] <= qh[0]) {
            const float4 lo = bmin[c], hi = bmax[c];
            const float gx = gap(ql[0], qh[0], lo.x, hi.x), gy = gap(ql[1], qh[1], lo.y, hi.y),
                        gz = gap(ql[2], qh[2], lo.z, hi.z);
            pass = gx * gx + gy * gy + gz * gz < thr && lo.x <= hi.x;
        }
        unsigned m = __ballot_sync(0xffffffffu, pass);
        if (evals && lane == 0 && m) atomicAdd(evals, (unsigned long long)__popc(m) * nq * KNN_BOX);
        while (m) {
            const int src = __ffs(m) - 1;
            m &= m - 1;
            const int cb = __shfl_sync(0xffffffffu, c, src);
            const int pj = cb * KNN_BOX + lane;
            const float4 p = pj < n ? sp[pj] : make_float4(INFINITY, INFINITY, INFINITY, __uint_as_float(0xffffffffu));
            for (int k = 0; k < KNN_BOX; k++) {
                const float px = __shfl_sync(0xffffffffu, p.x, k), py = __shfl_sync(0xffffffffu, p.y, k),
                            pz = __shfl_sync(0xffffffffu, p.z, k);
                const uint32_t pi = __float_as_uint(__shfl_sync(0xffffffffu, p.w, k));
                if (!fin || cb * KNN_BOX + k >= n || pi == self) continue;
                const float dx = px - q.x, dy = py - q.y, dz = pz - q.z;
                keep3(dx * dx + dy * dy + dz * dz, b0, b1, b2);
            }
        }
    }
    if (!valid) return;
    float sum = 0.f, cnt = 0.f;
    if (isfinite(b0)) { sum += sqrtf(b0); cnt += 1.f; }
    if (isfinite(b1)) { sum += sqrtf(b1); cnt += 1.f; }
    if (isfinite(b2)) { sum += sqrtf(b2); cnt += 1.f; }
    out[self] = cnt > 0.f ? sum / cnt : 1.f;
}

int knn_boxes(int n) { return (n + KNN_BOX - 1) / KNN_BOX; }

int launch_knn3(const float *pts, int n, float *out, KnnScratch &s, cudaStream_t st) {
    if (n <= 0) return 0;
    const unsigned int init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    cudaMemcpyAsync(s.bounds, init, sizeof init, cudaMemcpyHostToDevice, st);
    if (s.evals) cudaMemsetAsync(s.evals, 0, sizeof(unsigned long long), st);
    knn_bounds_kernel<<<std::min((n + 255) / 256, 1184), 256, 0, st>>>(pts, n, s.bounds);
    knn_morton_kernel<<<(n + 255) / 256, 256, 0, st>>>(pts, n, s.bounds, s.keys[0], s.vals[0]);
    const int cur = radix_sort_pairs(s.keys, s.vals, n, 30, s.radix_scratch, st);
    knn_gather_kernel<<<(n + 255) / 256, 256, 0, st>>>(pts, n, s.vals[cur], s.sorted);
    const int nb = knn_boxes(n);
    knn_boxes_kernel<<<(nb + 127) / 128, 128, 0, st>>>(s.sorted, n, nb, s.bmin, s.bmax);
    knn_query_kernel<<<(nb * 32 + 127) / 128, 128, 0, st>>>(s.sorted, n, nb, s.bmin, s.bmax, out, s.evals);
    return 0;
}

__global__ void init_gaussians_kernel(const float *md, const uint8_t *rgb, int n, uint32_t seed, float logit,
                                      float *scales, float *quats, float *dc, float *opac) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float ls = (float)log((double)fmaxf(md[i], 1e-7f));
    scales[3 * i] = scales[3 * i + 1] = scales[3 * i + 2] = ls;
    const uint32_t c = 3u * (uint32_t)i;
    const float u = rand_unif(seed, c), v = rand_unif(seed, c + 1u), w = rand_unif(seed, c + 2u);
    const float tau = 6.28318530717958647692f;
    const float a = sqrtf(1.f - u), b = sqrtf(u);
    const float tv = tau * v, tw = tau * w;
    quats[4 * i + 0] = a * (float)sin((double)tv);
    quats[4 * i + 1] = a * (float)cos((double)tv);
    quats[4 * i + 2] = b * (float)sin((double)tw);
    quats[4 * i + 3] = b * (float)cos((double)tw);
    for (int k = 0; k < 3; k++) dc[3 * i + k] = ((float)rgb[3 * i + k] * (1.f / 255.f) - 0.5f) / SH_C0;
    opac[i] = logit;
}

void launch_init_gaussians(const float *md, const uint8_t *rgb, int n, uint32_t seed, float logit, float *scales,
                           float *quats, float *dc, float *opac, cudaStream_t st) {
    if (n <= 0) return;
    init_gaussians_kernel<<<(n + 255) / 256, 256, 0, st>>>(md, rgb, n, seed, logit, scales, quats, dc, opac);
}

}  // namespace msplat
