// Fused L1 + SSIM loss, forward and backward, in one kernel.
//
// The reference runs three row passes with two (H, W, 15) float intermediates in
// memory (ssim_h_fwd, ssim_fused_v_fwd_h_bwd, ssim_v_bwd; core/cpu/msplat_cpu.cpp:
// 669-785). Here each CTA owns a 32x32 output tile and keeps every intermediate in
// shared memory: inputs with a 10-pixel halo, the horizontal moment sums, the SSIM
// derivative fields on the 5-pixel halo, and their horizontal back-convolution. HBM
// traffic is the minimum: read render + target once (plus halo), write v_rendered
// once. Channels are processed one after another to bound shared memory.
//
// Semantics kept exactly: zero-padded 11-tap Gaussian window (sigma 1.5), C1 = 1e-4,
// C2 = 9e-4; loss per pixel w * (1 - SSIM/3) + (1 - w) * L1/3 summed in double;
// v_rendered = inv_n * (-w * dSSIM + (1 - w) * sign(render - target)). Summation
// orders match the reference's loops (compiled with -fmad=false), so the derivative
// fields equal the reference's bit for bit; the loss differs only in the order of
// its double-precision sum. Per-block partial sums are reduced in a fixed order.
#include "common.cuh"
#include "kernels.h"

namespace msplat {

constexpr int ST = 32;                     // output tile edge
constexpr int SH_IN = ST + 20;             // input rows / cols with the 10-pixel halo
constexpr int SH_F = ST + 10;              // derivative-field rows / cols (5-pixel halo)
constexpr int SSIM_THREADS = 512;
constexpr int SSIM_PPT = ST * ST / SSIM_THREADS;  // output pixels per thread
__constant__ float kWin[11] = {0.0010283801f, 0.0075987581f, 0.0360007721f, 0.1093606895f,
                               0.2130055377f, 0.2660117249f, 0.2130055377f, 0.1093606895f,
                               0.0360007721f, 0.0075987581f, 0.0010283801f};

struct SsimSmem {
    float gt[SH_IN][SH_IN];
    float rd[SH_IN][SH_IN];
    float hb[SH_IN][SH_F][5];  // horizontal moments: rows y0-10.., cols x0-5..
    float f[SH_F][SH_F][3];    // derivative fields: rows y0-5.., cols x0-5..
    float dv[SH_F][ST][3];     // horizontal back-convolution: rows y0-5.., cols x0..
    float sp[ST][ST];          // per-pixel SSIM of the current channel
    double red[SSIM_THREADS / 32];
};

// One 32x32 output block (bx, by) of one image; its loss partial goes to
// a.partials[pidx]. Every thread of the block calls it.
__device__ __forceinline__ void ssim_block(const SsimArgs &a, int bx, int by, int pidx, SsimSmem &s) {
    const int W = a.W, H = a.H;
    const int x0 = bx * ST, y0 = by * ST;
    const float w = a.ssim_weight;
    // each thread owns output pixels tid, tid + SSIM_THREADS, ... of the 32x32 tile
    float ssim_acc[SSIM_PPT], l1_acc[SSIM_PPT];
#pragma unroll
    for (int u = 0; u < SSIM_PPT; u++) ssim_acc[u] = l1_acc[u] = 0.f;
    for (int c = 0; c < 3; c++) {
        // 1. inputs, zero outside the image
        for (int i = threadIdx.x; i < SH_IN * SH_IN; i += SSIM_THREADS) {
            const int r = i / SH_IN, q = i - r * SH_IN;
            const int gy = y0 - 10 + r, gx = x0 - 10 + q;
            float gv = 0.f, rv = 0.f;
            if (gy >= 0 && gy < H && gx >= 0 && gx < W) {
                const size_t idx = ((size_t)gy * W + gx) * 3 + c;
                gv = a.gt[idx];
                rv = a.img[idx];
            }
            s.gt[r][q] = gv;
            s.rd[r][q] = rv;
        }
        __syncthreads();
        // 2. horizontal moments at cols x0-5 .. x0+ST+5 (core/cpu/msplat_cpu.cpp:669-696)
        for (int i = threadIdx.x; i < SH_IN * SH_F; i += SSIM_THREADS) {
            const int r = i / SH_F, q = i - r * SH_F;  // q = column offset from x0-5
            float m0 = 0.f, m1 = 0.f, m2 = 0.f, m3 = 0.f, m4 = 0.f;
#pragma unroll
            for (int k = 0; k < 11; k++) {
                const float gv = s.gt[r][q + k], rv = s.rd[r][q + k];
                const float wk = kWin[k];
                m0 += wk * gv;
                m1 += wk * rv;
                m2 += wk * gv * gv;
                m3 += wk * rv * rv;
                m4 += wk * gv * rv;
            }
            s.hb[r][q][0] = m0;
            s.hb[r][q][1] = m1;
            s.hb[r][q][2] = m2;
            s.hb[r][q][3] = m3;
            s.hb[r][q][4] = m4;
        }
        __syncthreads();
        // 3. vertical sums, SSIM terms and derivative fields (:698-736)
        for (int i = threadIdx.x; i < SH_F * SH_F; i += SSIM_THREADS) {
            const int r = i / SH_F, q = i - r * SH_F;
            const int gy = y0 - 5 + r, gx = x0 - 5 + q;
            float f1 = 0.f, f2 = 0.f, f3 = 0.f;
            if (gy >= 0 && gy < H && gx >= 0 && gx < W) {
                float m[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int k = 0; k < 11; k++) {
                    const int yy = gy - 5 + k;
                    if (yy < 0 || yy >= H) continue;
                    const float wk = kWin[k];
#pragma unroll
                    for (int t = 0; t < 5; t++) m[t] += wk * s.hb[r + k][q][t];
                }
                const float mx = m[0], my = m[1];
                const float vx = m[2] - mx * mx, vy = m[3] - my * my, cv = m[4] - mx * my;
                const float A = 2.0f * mx * my + 0.0001f, B = 2.0f * cv + 0.0009f;
                const float Cd = mx * mx + my * my + 0.0001f, D = vx + vy + 0.0009f;
                const float iCD = 1.0f / (Cd * D);
                const float dmu = 2.0f * B * (mx * Cd - A * my) / (Cd * Cd * D);
                const float dsyq = -A * B * iCD / D, dsxy = 2.0f * A * iCD;
                f1 = dmu - 2.0f * my * dsyq - mx * dsxy;
                f2 = 2.0f * dsyq;
                f3 = dsxy;
                s.f[r][q][0] = f1;
                s.f[r][q][1] = f2;
                s.f[r][q][2] = f3;
                const int oy = r - 5, ox = q - 5;
                if (oy >= 0 && oy < ST && ox >= 0 && ox < ST) s.sp[oy][ox] = (A * B) / (Cd * D);
            } else {
                s.f[r][q][0] = 0.f;
                s.f[r][q][1] = 0.f;
                s.f[r][q][2] = 0.f;
            }
        }
        __syncthreads();
        // SSIM and L1 per owned pixel, channel by channel in order (the reference adds
        // channel 0, 1, 2 into ssim_pix / l1_pix)
#pragma unroll
        for (int u = 0; u < SSIM_PPT; u++) {
            const int p = threadIdx.x + u * SSIM_THREADS;
            const int oy = p / ST, ox = p - oy * ST;
            const int gy = y0 + oy, gx = x0 + ox;
            if (gy < H && gx < W) {
                ssim_acc[u] += s.sp[oy][ox];
                l1_acc[u] += fabsf(s.gt[oy + 10][ox + 10] - s.rd[oy + 10][ox + 10]);
            }
        }
        __syncthreads();
        // 4. horizontal back-convolution at rows y0-5 .. y0+ST+5, cols x0 .. (:737-747)
        for (int i = threadIdx.x; i < SH_F * ST; i += SSIM_THREADS) {
            const int r = i / ST, q = i - r * ST;
            float h1 = 0.f, h2 = 0.f, h3 = 0.f;
#pragma unroll
            for (int d = 0; d < 11; d++) {
                const float wk = kWin[10 - d];
                h1 += wk * s.f[r][q + d][0];
                h2 += wk * s.f[r][q + d][1];
                h3 += wk * s.f[r][q + d][2];
            }
            s.dv[r][q][0] = h1;
            s.dv[r][q][1] = h2;
            s.dv[r][q][2] = h3;
        }
        __syncthreads();
        // 5. vertical back-convolution and the pixel gradient (:760-785)
#pragma unroll
        for (int u = 0; u < SSIM_PPT; u++) {
            const int p = threadIdx.x + u * SSIM_THREADS;
            const int oy = p / ST, ox = p - oy * ST;
            const int gy = y0 + oy, gx = x0 + ox;
            if (gy >= H || gx >= W) continue;
            float a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
            for (int d = 0; d < 11; d++) {
                const int yy = gy - 5 + d;
                if (yy < 0 || yy >= H) continue;
                const float wk = kWin[10 - d];
                a1 += wk * s.dv[oy + d][ox][0];
                a2 += wk * s.dv[oy + d][ox][1];
                a3 += wk * s.dv[oy + d][ox][2];
            }
            const float rv = s.rd[oy + 10][ox + 10], gv = s.gt[oy + 10][ox + 10];
            const float vs = a1 + rv * a2 + gv * a3;
            const float vl = (gv > rv) ? -1.0f : ((gv < rv) ? 1.0f : 0.0f);
            a.v_out[((size_t)gy * W + gx) * 3 + c] = a.inv_n * (-w * vs + (1.0f - w) * vl);
        }
        __syncthreads();
    }
    // per-pixel loss in float, summed in double over the block in a fixed order
    double sum = 0.0;
#pragma unroll
    for (int u = 0; u < SSIM_PPT; u++) {
        const int p = threadIdx.x + u * SSIM_THREADS;
        const int oy = p / ST, ox = p - oy * ST;
        if (y0 + oy < H && x0 + ox < W) sum += (double)(w * (1.0f - ssim_acc[u] / 3.0f) + (1.0f - w) * l1_acc[u] / 3.0f);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) s.red[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < SSIM_THREADS / 32; i++) t += s.red[i];
        a.partials[pidx] = t;
    }
}

__global__ void __launch_bounds__(SSIM_THREADS, 2) ssim_loss_kernel(SsimArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SsimSmem &s = *reinterpret_cast<SsimSmem *>(smem_raw);
    ssim_block(a, blockIdx.x, blockIdx.y, blockIdx.y * gridDim.x + blockIdx.x, s);
}

// Persistent loss over the blocks of a batch of images (each with its own size,
// target and gradient output), pulling global block ids from a counter. Block b of
// view v writes partial boff[v] + (its index within the view), so each view's
// partials sit in the order the single-image kernel writes them.
__global__ void __launch_bounds__(SSIM_THREADS, 2) ssim_loss_batch_kernel(const SsimArgs *views, const int *boff,
                                                                       int n_views, int *counter) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SsimSmem &s = *reinterpret_cast<SsimSmem *>(smem_raw);
    __shared__ int s_blk;
    const int total = boff[n_views];
    for (;;) {
        if (threadIdx.x == 0) s_blk = atomicAdd(counter, 1);
        __syncthreads();
        const int b = s_blk;
        __syncthreads();
        if (b >= total) break;
        const int v = find_view(boff, n_views, b);
        const SsimArgs a = views[v];
        const int lb = b - boff[v], nbx = (a.W + ST - 1) / ST;
        ssim_block(a, lb % nbx, lb / nbx, b, s);
        __syncthreads();
    }
}

__device__ __forceinline__ void loss_finalize_block(const double *partials, int nb, double npix, float *loss) {
    __shared__ double red[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s += partials[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += red[i];
        *loss = (float)(t / npix);
    }
}

__global__ void loss_finalize_kernel(const double *partials, int nb, double npix, float *loss) {
    loss_finalize_block(partials, nb, npix, loss);
}

// One 1024-thread block per view: the same reduction as loss_finalize_kernel over
// that view's partials, so each view's loss equals its single-image loss.
__global__ void loss_finalize_batch_kernel(const SsimArgs *views, const int *boff) {
    const int v = blockIdx.x;
    const SsimArgs &a = views[v];
    loss_finalize_block(a.partials + boff[v], boff[v + 1] - boff[v], (double)a.W * a.H, a.loss);
}

int ssim_blocks(int W, int H) { return ((W + ST - 1) / ST) * ((H + ST - 1) / ST); }

static void ssim_set_smem_attr() {
    static const bool done = [] {
        cudaFuncSetAttribute(ssim_loss_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SsimSmem));
        cudaFuncSetAttribute(ssim_loss_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(SsimSmem));
        return true;
    }();
    (void)done;
}

// views[v].partials must all be the same batch-wide array (indexed by global block).
void launch_ssim_loss_batch(const SsimArgs *d_views, const int *d_boff, int n_views, int *d_counter, cudaStream_t st) {
    if (n_views <= 0) return;
    ssim_set_smem_attr();
    static const int grid = [] {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ssim_loss_batch_kernel, SSIM_THREADS,
                                                      sizeof(SsimSmem));
        return sms * (per_sm > 0 ? per_sm : 1);
    }();
    cudaMemsetAsync(d_counter, 0, sizeof(int), st);
    ssim_loss_batch_kernel<<<grid, SSIM_THREADS, sizeof(SsimSmem), st>>>(d_views, d_boff, n_views, d_counter);
    loss_finalize_batch_kernel<<<n_views, 1024, 0, st>>>(d_views, d_boff);
}

void launch_ssim_loss(const SsimArgs &a, cudaStream_t st) {
    if (a.W <= 0 || a.H <= 0) return;
    const size_t smem = sizeof(SsimSmem);
    ssim_set_smem_attr();
    dim3 grid((a.W + ST - 1) / ST, (a.H + ST - 1) / ST);
    ssim_loss_kernel<<<grid, SSIM_THREADS, smem, st>>>(a);
    loss_finalize_kernel<<<1, 1024, 0, st>>>(a.partials, (int)(grid.x * grid.y), (double)a.W * a.H, a.loss);
}

}  // namespace msplat
