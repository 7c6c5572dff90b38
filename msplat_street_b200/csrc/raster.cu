// 16x16-tile front-to-back alpha compositing, forward and backward.
//
// One CTA per tile (the forward may also split a tile into 16 x 8 or 8 x 8 pixel
// blocks, each walking the tile's whole list: the block shape changes no result). The
// tile's depth-sorted list is walked in batches whose splat records are staged in
// shared memory; every thread reads each record as a broadcast.
// Staging also clamps the colours once and marks which of the tile's warp blocks the
// splat can reach at all (its box and its ellipse's diagonal extents, tested on 8 x 4
// pixel blocks), so a warp passes over the splats that miss its pixels with one bit
// test and walks the rest by ballot. The forward runs one pixel per thread (256
// threads, 8 x 4 pixels per warp). The backward runs two pixels per thread (128
// threads, one column and rows y, y + 4 of the warp's 8 x 8 block): its decisions and
// sigma stay scalar, and its gradient arithmetic uses sm_100's packed FP32
// instructions (add / mul / fma .f32x2), two operations per instruction.
//
// Forward: rasterize_forward (core/cpu/msplat_cpu.cpp:574-626): sigma < 0 or >= 5.55
// skips, alpha = min(0.999, o * exp(-sigma)) with alpha < 1/255 skipped, and the pixel
// stops before the Gaussian that would take T to <= 1e-4 (last = k - 1). The block
// leaves its loop when __syncthreads_count says all 256 pixels are done.
//
// Backward: rasterize_backward (:959-1031): back to front from final_idx, T recovered
// by multiplying with 1/(1 - alpha) (the hardware reciprocal: no decision depends on
// T there), colour gradients gated on raw + 0.5 >= 0 and the
// sigma gradients only for alpha < 0.999. Each (tile, Gaussian) pair -- one sorted
// intersection -- gets one 9-float slot: xy(2) conic(3) rgb(3) opacity-logit(1),
// reduced over the tile's pixels in a fixed order (lanes through a transposed
// shared-memory buffer, then warps), so results do not depend on scheduling (the
// reference is deterministic too, :952-956). The per-Gaussian sums happen in the
// fused backward/Adam kernel.
//
// Compiled with -fmad=false: the alpha and transmittance cut-offs must fall exactly
// where the reference's do. The backward's gradient arithmetic, which no decision
// depends on, uses explicit fused multiply-adds.
//
// Staging sizes are template parameters (RASTER_VARIANTS, picked at run time by the
// autotuner); no variant changes any arithmetic or summation order, so all of them
// give the same bits. A persistent form of each pass pulls (view, tile) work items
// for batches of views.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace msplat {

// The float just below 5.55: sigma >= 5.55f is sigma > SIGMA_SKIP.
constexpr float SIGMA_SKIP = 0x1.633332p+2f;  // 5.5499997
static_assert(SIGMA_SKIP < 5.55f && SIGMA_SKIP + 0x1p-21f == 5.55f, "the float below 5.55f (ulp 2^-21 there)");

// the forward's block: one thread per pixel (8 x 4 pixels per warp); the backward's:
// 128 threads, two pixels each (8 x 8 pixels per warp)
constexpr int FWD_THREADS = TILE_PIX;
constexpr int BWD_THREADS = TILE_PIX / 2, BWD_WARPS = BWD_THREADS / 32;

// A splat's colour channel as the rasterizers use it, max(raw + 0.5, 0), computed once
// at staging. A channel clamped to zero is stored as -0.0, so its sign bit carries the
// backward's gate (the gradient passes where raw + 0.5 >= 0): -0.0 * x + y == y and
// +0.0 * x + y == y for every y the compositing sums take, so images do not change.
__device__ __forceinline__ float staged_colour(float raw) {
    const float c = raw + 0.5f;
    return c >= 0.f ? c : -0.f;
}

// Which of a tile's eight 8x4 warp blocks (warp w covers columns 8 (w % 2) .. +7 and
// rows 4 (w / 2) .. +3) a splat can reach with alpha >= 1/255: bit w set unless the
// block lies outside the splat's box (x + ex < block x0 || x - ex > x1 || y + ey < y0
// || y - ey > y1) or outside the region's extent along either diagonal, x + y and
// x - y (separating axes). Both extents come with the record, computed once per
// Gaussian by the projection in double with margins and stored rounded up, so a block
// is dropped only when no pixel in it can take part. C = record[2] (its z and w hold
// the packed box and diagonal extents).
__device__ __forceinline__ uint32_t warp_block_mask(const float4 A, const float4 C, int tx, int ty) {
    const float2 box = unpack_half2(__float_as_uint(C.z));
    const float xr = A.x + box.x, xl = A.x - box.x, yb = A.y + box.y, yt = A.y - box.y;
    uint32_t cols = 0u, mask = 0u;
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const float bx0 = (float)(tx * TILE + (c << 3)), bx1 = bx0 + 7.f;
        if (!(xr < bx0 || xl > bx1)) cols |= 1u << c;
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const float by0 = (float)(ty * TILE + (r << 2)), by1 = by0 + 3.f;
        if (!(yb < by0 || yt > by1)) mask |= cols << (2 * r);
    }
    if (!mask) return 0u;
    const float2 dg = unpack_half2(__float_as_uint(C.w));
    const float hp = dg.x, hm = dg.y;
    const float sp = A.x + A.y, sd = A.x - A.y;
#pragma unroll
    for (int w = 0; w < 8; w++) {
        const float bx0 = (float)(tx * TILE + ((w & 1) << 3)), bx1 = bx0 + 7.f;
        const float by0 = (float)(ty * TILE + ((w >> 1) << 2)), by1 = by0 + 3.f;
        if (sp + hp < bx0 + by0 || sp - hp > bx1 + by1 || sd + hm < bx0 - by1 || sd - hm > bx1 - by0)
            mask &= ~(1u << w);
    }
    return mask;
}

// The tile thread (0 .. TILE_PIX - 1, as tile_pixel maps it) that thread t of a block
// of NT threads takes in sub-block q of the tile: NT = 256, the whole tile; 128, the
// 16 x 8 half q (warps 4q .. 4q + 3); 64, the 8 x 8 quarter q = (qy, qx) (warps
// 4 qy + qx and 4 qy + 2 + qx: column half qx, rows 8 qy .. 8 qy + 7).
template <int NT>
__device__ __forceinline__ int sub_tile_thread(int t, int q) {
    if (NT == TILE_PIX) return t;
    if (NT == TILE_PIX / 2) return q * NT + t;
    return ((4 * (q >> 1) + (q & 1) + 2 * (t >> 5)) << 5) + (t & 31);
}

// One 16x16 tile: `tile` indexes tile_start / tile_end (a global tile id in a batch),
// (tx, ty) is its position in its view. Every thread of the block must call it.
// NT, q: the block runs sub-block q of the tile with NT threads (sub_tile_thread), each
// pixel walking the tile's whole list with the same decisions and sums as in a
// whole-tile block, so its results do not depend on the shape.
// FB: Gaussians staged in shared memory per round.
// AUX: also the expected-depth numerator and a per-pixel background
// (rasterize_forward_aux, core/cpu/msplat_cpu.cpp:574-626 with f.aux).
// CHUNK: composite only piece `chunk` of the list (ck->chunk_len long) from T = 1 and
// write the piece's transmittance, colour and last contributor to item `item`.
template <int FB, bool AUX = false, bool CHUNK = false, bool TS = false, int NT = FWD_THREADS>
__device__ __forceinline__ void raster_fwd_tile(const RasterArgs &a, int tile, int tx, int ty, float4 *s0,
                                                float4 *s1, float4 *s2, uint8_t *sm, const double *espan,
                                                const ChunkArgs *ck = nullptr, int item = 0, int chunk = 0,
                                                int q = 0) {
    static_assert(!CHUNK || NT == FWD_THREADS, "depth pieces are composited by whole-tile blocks");
    const int g = sub_tile_thread<NT>(threadIdx.x, q);  // this thread's place in the tile
    int lx, ly;
    tile_pixel(g, lx, ly);
    const int px = tx * TILE + lx, py = ty * TILE + ly;
    const bool inside = px < a.W && py < a.H;
    int start = a.tile_start[tile], end = a.tile_end[tile];
    if (CHUNK) {
        start += chunk * ck->chunk_len;
        end = min(end, start + ck->chunk_len);
    }
    const float fpx = (float)px, fpy = (float)py;
    const int w = g >> 5, lane = threadIdx.x & 31;  // w: the warp's block of the tile
    float T = 1.f, cr = 0.f, cg = 0.f, cb = 0.f, depth = 0.f;
    int last = start - 1;
    bool done = !inside;
    const size_t npix = (size_t)a.W * a.H;
    const size_t pid = inside ? (size_t)py * a.W + px : 0;
    int stored = 0;  // contributions seen (stored-transmittance mode)
    for (int b0 = start; b0 < end; b0 += FB) {
        if (__syncthreads_count(done) == NT) break;
        for (int si = threadIdx.x; si < FB; si += NT) {
            const int k = b0 + si;
            if (k >= end) break;
            const float4 *rec = reinterpret_cast<const float4 *>(a.splats + a.isect_gid[k]);
            const float4 A = rec[0], B = rec[1], C = rec[2];
            // the conic's diagonal halved: 0.5 (a dx dx + c dy dy) == (a/2) dx dx +
            // (c/2) dy dy bit for bit (scaling by 2^-1 commutes with each rounding)
            s0[si] = make_float4(A.x, A.y, 0.5f * A.z, A.w);
            s1[si] = make_float4(0.5f * B.x, B.y, staged_colour(B.z), staged_colour(B.w));
            // z: the sigma above which the pixel skips the splat -- the smaller of the
            // float below 5.55 (sigma >= 5.55 is sigma > that float) and the sigma above
            // which alpha = o exp(-sigma) < 1/255 for certain, ln(255 o) plus a margin
            // far above the roundings of logf, of the exponential and of the product --
            // so one compare takes both decisions the exact tests would take
            s2[si] = make_float4(staged_colour(C.x), C.y, fminf(logf(255.f * B.y) + 1e-3f, SIGMA_SKIP), C.w);
            sm[si] = (uint8_t)warp_block_mask(A, C, tx, ty);
        }
        __syncthreads();
        const int cnt = min(FB, end - b0);
        // this warp's splats in list order: 32 mask bits per ballot, then one per hit
        for (int base = 0; base < cnt; base += 32) {
            const int jl = base + lane;
            unsigned bits = __ballot_sync(0xffffffffu, jl < cnt && ((sm[jl] >> w) & 1u));
            while (bits && !done) {
                const int j = base + __ffs(bits) - 1;
                bits &= bits - 1u;
                const float4 A = s0[j], B = s1[j], C = s2[j];
                const float dx = A.x - fpx, dy = A.y - fpy;
                const float sigma = (A.z * dx * dx + B.x * dy * dy) + A.w * dx * dy;  // A.z, B.x halved
                if (sigma < 0.f || sigma > C.z) continue;
                const float alpha = fminf(0.999f, B.y * exp_span(-sigma, espan));
                if (alpha < 1.f / 255.f) continue;
                const float nT = T * (1.f - alpha);
                if (nT <= 1e-4f) {
                    last = b0 + j - 1;
                    done = true;
                    break;
                }
                if (TS) {
                    if (stored < a.tcap) a.tstore[(size_t)stored * npix + pid] = T;
                    stored++;
                }
                const float vis = alpha * T;
                cr = B.z * vis + cr;  // staged colours: max(raw + 0.5, 0)
                cg = B.w * vis + cg;
                cb = C.x * vis + cb;
                if (AUX) depth += C.y * vis;
                T = nT;
                last = b0 + j;
            }
        }
    }
    if (!inside) return;
    if (CHUNK) {
        const size_t o = (size_t)item * TILE_PIX + g, o3 = (size_t)item * 3 * TILE_PIX + g;
        ck->cT[o] = T;
        ck->cC[o3] = cr;
        ck->cC[o3 + TILE_PIX] = cg;
        ck->cC[o3 + 2 * TILE_PIX] = cb;
        ck->clast[o] = last;
        return;
    }
    if (a.final_T) a.final_T[pid] = T;
    if (a.final_idx) a.final_idx[pid] = last;
    if (TS) a.tcount[pid] = stored <= a.tcap ? stored : -1;
    float *o = a.out_img + 3 * (size_t)pid;
    if (AUX) {
        float *bp = a.bg_img + 3 * (size_t)pid;
        float br = a.bg[0], bgg = a.bg[1], bb = a.bg[2];
        if (a.sky_bg) {
            br = bp[0];
            bgg = bp[1];
            bb = bp[2];
        } else {
            bp[0] = br;
            bp[1] = bgg;
            bp[2] = bb;
        }
        a.out_depth[pid] = depth;
        o[0] = clamp01(br * T + cr);
        o[1] = clamp01(bgg * T + cg);
        o[2] = clamp01(bb * T + cb);
        return;
    }
    o[0] = clamp01(a.bg[0] * T + cr);
    o[1] = clamp01(a.bg[1] * T + cg);
    o[2] = clamp01(a.bg[2] * T + cb);
}

// One block per sub-block of a tile (NT threads: the whole 16 x 16 tile, a 16 x 8
// half or an 8 x 8 quarter; blocks SUB * t .. SUB * t + SUB - 1 share tile t's list).
template <int FB, bool AUX = false, bool TS = false, int NT = FWD_THREADS>
__global__ void __launch_bounds__(NT, 4 * FWD_THREADS / NT) raster_fwd_kernel(RasterArgs a) {
    constexpr int SUB = FWD_THREADS / NT;
    __shared__ float4 s0[FB], s1[FB], s2[FB];
    __shared__ uint8_t sm[FB];
    __shared__ double et64[EXP_TABLE], espan[EXP_SPAN];
    exp_span_init_a(et64);
    __syncthreads();
    exp_span_init_b(espan, et64);  // ready after the tile's first barrier
    const int tile = blockIdx.x / SUB;
    raster_fwd_tile<FB, AUX, false, TS, NT>(a, tile, tile % a.tiles_x, tile / a.tiles_x, s0, s1, s2, sm, espan,
                                            nullptr, 0, 0, blockIdx.x % SUB);
}

// Persistent forward over the tiles of a batch of views (each with its own scene,
// camera, resolution and output): every block pulls work items from a counter until
// none are left. An item is one of a tile's 256 / NT sub-blocks (the tile shape of the
// launch: 16 x 16, 16 x 8 or 8 x 8 pixels, each walking its tile's whole list -- the
// reference's Metal rasterizer runs 8 x 8 thread groups inside its 16 x 16 bins). A
// tile's image equals what the per-view kernel renders: the same list (the batch sort
// keeps each tile's order) and the same per-pixel code.
template <int FB, int NT>
__global__ void __launch_bounds__(NT, 4 * FWD_THREADS / NT) raster_fwd_batch_kernel(const BatchDesc d, int *counter) {
    constexpr int SUB = FWD_THREADS / NT;
    __shared__ float4 s0[FB], s1[FB], s2[FB];
    __shared__ uint8_t sm[FB];
    __shared__ int s_item, s_lt;
    __shared__ RasterArgs s_args;  // the tile's view, read from shared memory (keeps registers down)
    __shared__ double et64[EXP_TABLE], espan[EXP_SPAN];
    exp_span_init_a(et64);
    __syncthreads();
    exp_span_init_b(espan, et64);  // ready after the loop's first barrier
    const int total_items = d.tile_off[d.n_views] * SUB;  // read on the device: the launch is graph-capturable
    for (;;) {
        __syncthreads();  // the previous item's shared state is no longer read
        if (threadIdx.x == 0) {
            const int it = atomicAdd(counter, 1);
            s_item = it;
            if (it < total_items) {
                const int t = it / SUB;
                const int v = find_view(d.tile_off, d.n_views, t);
                s_args = d.raster[v];
                s_lt = t - d.tile_off[v];
            }
        }
        __syncthreads();
        const int it = s_item, lt = s_lt;
        if (it >= total_items) break;
        raster_fwd_tile<FB, false, false, false, NT>(s_args, it / SUB, lt % s_args.tiles_x, lt / s_args.tiles_x, s0,
                                                     s1, s2, sm, espan, nullptr, 0, 0, it % SUB);
    }
}

// Resident blocks of a kernel on the whole GPU.
template <typename K>
int resident_grid(K kernel, size_t smem, int threads = TILE_PIX) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    return std::max(1, sms * std::max(per_sm, 1));
}

template <int FB, int NT>
void fwd_batch_launch(const BatchDesc &d, int tiles_hint, int *d_counter, cudaStream_t st) {
    // once per variant and shape, thread-safe
    static const int grid = resident_grid(raster_fwd_batch_kernel<FB, NT>, 0, NT);
    const int items = tiles_hint * (FWD_THREADS / NT);
    const int g = tiles_hint > 0 ? std::min(grid, items) : grid;
    raster_fwd_batch_kernel<FB, NT><<<g, NT, 0, st>>>(d, d_counter);
}

template <int NT>
void fwd_batch_staging(const BatchDesc &d, int tiles_hint, int *d_counter, cudaStream_t st, int variant) {
    switch (RASTER_VARIANTS[variant_index(variant)].fwd_batch) {
        case 64: fwd_batch_launch<64, NT>(d, tiles_hint, d_counter, st); break;
        case 256: fwd_batch_launch<256, NT>(d, tiles_hint, d_counter, st); break;
        default: fwd_batch_launch<128, NT>(d, tiles_hint, d_counter, st); break;
    }
}

// tiles_hint: the batch's tile count when the host knows it (caps the grid), else 0;
// shape: RASTER_SHAPES index (16 x 16, 16 x 8 or 8 x 8 pixels a block)
void launch_raster_fwd_batch(const BatchDesc &d, int tiles_hint, int *d_counter, cudaStream_t st, int variant,
                             int shape) {
    cudaMemsetAsync(d_counter, 0, sizeof(int), st);
    switch (shape_index(shape)) {
        case 1: fwd_batch_staging<FWD_THREADS / 2>(d, tiles_hint, d_counter, st, variant); break;
        case 2: fwd_batch_staging<FWD_THREADS / 4>(d, tiles_hint, d_counter, st, variant); break;
        default: fwd_batch_staging<FWD_THREADS>(d, tiles_hint, d_counter, st, variant); break;
    }
}

// Per-warp reduction of the 9 gradient values over the warp's 32 pixels, done in
// sub-batches of SB hit Gaussians: each lane stores its contributions to a transposed
// buffer (one row of 32 lane values per output), then each lane sums a whole row with
// float4 loads as a fixed pairwise tree (15 packed adds and one add). BB Gaussians
// are staged in shared memory per round.
constexpr int PB_STRIDE = 36;  // floats per row: 32 lanes + pad, keeps float4 rows conflict-free

// NG: gradient values per intersection, 9 (xy conic rgb opacity) or 10 with the
// aux mode's depth gradient
template <int BB, int SB, int NG = 9>
constexpr size_t raster_bwd_smem() {
    return sizeof(float4) * 3 * BB + sizeof(float) * BWD_WARPS * BB * NG +
           sizeof(float) * BWD_WARPS * SB * NG * PB_STRIDE + sizeof(uint32_t) * BB + BB + 16;
}

// One warp's sums of its q (<= SB) pending splats: row o = jj * NG + c of the warp's
// row buffer holds value c of pending splat jj (the oldest first) for the warp's 32
// lanes; lane o sums it (a fixed pairwise tree) and stores the sum to
// red[warp][j][c], j the splat's staged index (pend: 8 bits per splat, the newest
// lowest). The lanes that own a splat's value 0 mark the warp in hitw[j].
template <int NG, int SB>
__device__ __forceinline__ void bwd_warp_sums(const float *mypb, float *red, uint32_t *hitw, uint32_t pend, int q,
                                              int warp, int lane, int bb) {
    __syncwarp();
    for (int o = lane; o < q * NG; o += 32) {
        const int jj = o / NG, c = o - jj * NG;
        const int j = (int)((pend >> (8 * (q - 1 - jj))) & 0xffu);
        // the row's 32 lane values summed as a fixed pairwise tree, two sums per packed add
        const float4 *row = reinterpret_cast<const float4 *>(mypb + o * PB_STRIDE);
        f32x2 p[8];
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const float4 v = row[r];
            p[r] = add2(pack2(v.x, v.y), pack2(v.z, v.w));
        }
#pragma unroll
        for (int w = 4; w >= 1; w >>= 1)
#pragma unroll
            for (int r = 0; r < w; r++) p[r] = add2(p[r], p[r + w]);
        const float2 t = unpack2(p[0]);
        red[(warp * bb + j) * NG + c] = t.x + t.y;
        if (c == 0) atomicOr(&hitw[j], 1u << warp);
    }
    __syncwarp();
}

// One tile of the backward; `tile` indexes tile_start / tile_end and the slots (a
// global tile id in a batch), (tx, ty) is its position in its view. Every thread of
// the block (BWD_THREADS) calls it; it ends with the block's shared memory free for
// reuse. Each thread owns two pixels of one column, rows y and y + 4 of its warp's
// 8 x 8 block (warp w covers columns 8 (w % 2) .. +7 and rows 8 (w / 2) .. +7), and
// evaluates both with sm_100's packed FP32 instructions: one instruction, two IEEE
// operations, each rounded as its scalar form. Per-pixel decisions (sigma range,
// alpha cut-offs, last contributor) stay per pixel; a pixel that does not take part
// in a pair carries alpha = 0 through the packed update (T * 1, fac = 0), which leaves
// its state exactly as it was.
// AUX: the per-pixel background is the pixel's own, and the expected-depth / alpha
// cotangents enter v_alpha and a tenth value per intersection (the aux branch of
// :959-1031).
// CHUNK: piece `chunk` of the list only (item `item`), each pixel starting from the
// transmittance behind the piece (prefix * piece T), the colour behind it and the
// piece's last contributor; the background term still uses the merged final T.
// TS: stored-transmittance mode (a.tstore set): T before each of a pixel's first
// a.tcap contributions is read back instead of recovered by division.
//
// Per hit the lanes keep nine sums for the slot: the colour gradients fac * v (3), the
// xy gradient vs (conic d) (2), and for vs = -alpha v_alpha its moments vs dx^2,
// vs dx dy, vs dy^2 and vs itself; the block's sum turns the moments into the
// reference's slot values once per splat (conic = vs d d^T / 2, opacity logit =
// (o - 1) vs), the reference's per-pixel arithmetic with the splat's constants
// factored out of the sums (the xy gradient stays per pixel: its two terms can cancel). The colour part of v_alpha
// needs the colour behind the pixel only through its dot product with the pixel's
// colour cotangent, so one running scalar replaces the three-channel buffer.
template <int BB, int SB, bool AUX = false, bool CHUNK = false, bool TS = false>
__device__ __forceinline__ void raster_bwd_tile(const RasterBwdArgs &a, int tile, int tx, int ty, float4 *smem4,
                                                int &kmax, const double *etab, const ChunkArgs *ck = nullptr,
                                                int item = 0, int chunk = 0) {
    constexpr int NG = AUX ? 10 : 9;
    constexpr int SUB = SB, SUB_OUT = SB * NG;
    static_assert(BB <= BWD_THREADS, "one staging thread per splat");
    float4 *s0 = smem4, *s1 = s0 + BB, *s2 = s1 + BB;
    float *red = reinterpret_cast<float *>(s2 + BB);    // [BWD_WARPS][BB][NG]
    float *pbuf = red + BWD_WARPS * BB * NG;             // [BWD_WARPS][SUB_OUT][PB_STRIDE]
    uint32_t *hitw = reinterpret_cast<uint32_t *>(pbuf + BWD_WARPS * SUB_OUT * PB_STRIDE);  // [BB] warps hit
    uint8_t *sm = reinterpret_cast<uint8_t *>(hitw + BB);  // [BB] warp masks
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int lx = ((warp & 1) << 3) + (lane & 7), ly = ((warp >> 1) << 3) + (lane >> 3);
    const int px = tx * TILE + lx, py[2] = {ty * TILE + ly, ty * TILE + ly + 4};
    const bool inside[2] = {px < a.W && py[0] < a.H, px < a.W && py[1] < a.H};
    int start = a.tile_start[tile], end = a.tile_end[tile];
    if (CHUNK) {
        start += chunk * ck->chunk_len;
        end = min(end, start + ck->chunk_len);
    }
    if (end <= start) return;  // block-uniform
    int pid[2], kf[2] = {start - 1, start - 1}, tj[2] = {-1, -1};
    float T[2] = {0.f, 0.f}, tbv[2] = {0.f, 0.f}, bv[2] = {0.f, 0.f}, vr[2] = {0.f, 0.f}, vg[2] = {0.f, 0.f},
          vb[2] = {0.f, 0.f}, vd[2] = {0.f, 0.f}, vaa[2] = {0.f, 0.f};
#pragma unroll
    for (int i = 0; i < 2; i++) {
        pid[i] = py[i] * a.W + px;
        if (!inside[i]) continue;
        const float Tf = a.final_T[pid[i]];
        T[i] = Tf;
        kf[i] = a.final_idx[pid[i]];
        const float *v = a.v_out + 3 * (size_t)pid[i];
        vr[i] = v[0];
        vg[i] = v[1];
        vb[i] = v[2];
        float bgr = a.bg[0], bgg = a.bg[1], bgb = a.bg[2];
        if (AUX) {
            const float2 va2 = reinterpret_cast<const float2 *>(a.v_aux)[pid[i]];
            vd[i] = va2.x;
            vaa[i] = va2.y;
            const float *bp = a.bg_img + 3 * (size_t)pid[i];
            bgr = bp[0];
            bgg = bp[1];
            bgb = bp[2];
        }
        // (T_final bg) . v: the background's share of every v_alpha
        tbv[i] = __fmaf_rn(Tf * bgr, vr[i], __fmaf_rn(Tf * bgg, vg[i], Tf * bgb * vb[i]));
        if (CHUNK) {  // the piece's transmittance, last contributor, and the colour behind it
            const int ti = tile_index(lx, ly + 4 * i);
            const size_t o = (size_t)item * TILE_PIX + ti, o3 = (size_t)item * 3 * TILE_PIX + ti;
            T[i] = ck->pre[o] * ck->cT[o];
            kf[i] = ck->clast[o];
            bv[i] = __fmaf_rn(ck->aft[o3], vr[i], __fmaf_rn(ck->aft[o3 + TILE_PIX], vg[i], ck->aft[o3 + 2 * TILE_PIX] * vb[i]));
        }
        if (TS) tj[i] = a.tcount[pid[i]];  // contributions left to pop, -1 = recover T by division
    }
    if (threadIdx.x == 0) kmax = start - 1;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 2; i++)
        if (inside[i]) atomicMax(&kmax, min(kf[i], end - 1));
    __syncthreads();
    const int kend = kmax + 1;  // nothing at or above kend contributes to any pixel
    // nothing above wkf contributes to this warp's pixels: the warp skips those splats
    const int wkf = __reduce_max_sync(0xffffffffu, max(inside[0] ? kf[0] : start - 1, inside[1] ? kf[1] : start - 1));
    // packed per-pixel state: (row y, row y + 4)
    f32x2 T2 = pack2(T[0], T[1]), bv2 = pack2(bv[0], bv[1]);
    const f32x2 tbv2 = pack2(tbv[0], tbv[1]), vr2 = pack2(vr[0], vr[1]), vg2 = pack2(vg[0], vg[1]),
                vb2 = pack2(vb[0], vb[1]);
    const float fpy[2] = {(float)py[0], (float)py[1]};
    f32x2 bd2 = pack2(0.f, 0.f), ba2 = pack2(0.f, 0.f);  // aux: accumulated depth and alpha behind
    const f32x2 vd2 = pack2(vd[0], vd[1]), vaa2 = pack2(vaa[0], vaa[1]);
    const float fpx = (float)px;
    float *mypb = pbuf + warp * SUB_OUT * PB_STRIDE;
    const size_t npix = (size_t)a.W * a.H;
    for (int b_end = kend; b_end > start; b_end -= BB) {
        const int b_start = max(start, b_end - BB);
        const int cnt = b_end - b_start;
        if (threadIdx.x < cnt) {
            const float4 *rec = reinterpret_cast<const float4 *>(a.splats + a.isect_gid[b_start + threadIdx.x]);
            const float4 A = rec[0], B = rec[1], C = rec[2];
            // the 8 x 4 blocks' reach bits, merged pairwise into the 8 x 8 warp blocks
            const uint32_t m8 = warp_block_mask(A, C, tx, ty);
            sm[threadIdx.x] = (uint8_t)(((m8 | (m8 >> 2)) & 3u) | ((((m8 >> 4) | (m8 >> 6)) & 3u) << 2));
            hitw[threadIdx.x] = 0u;
            // staged: (x, y, a / 2, c / 2), (conic b, opacity, colour r, g), (colour b,
            // depth, a, c) -- the halved diagonal for sigma (0.5 (a dx dx + c dy dy) ==
            // (a/2) dx dx + (c/2) dy dy bit for bit), the whole one for the gradients
            s0[threadIdx.x] = make_float4(A.x, A.y, 0.5f * A.z, 0.5f * B.x);
            s1[threadIdx.x] = make_float4(A.w, B.y, staged_colour(B.z), staged_colour(B.w));
            s2[threadIdx.x] = make_float4(staged_colour(C.x), C.y, A.z, B.x);
        }
        __syncthreads();
        // This warp's reachable splats, back to front, 32 mask bits per ballot. Splats
        // that some pixel of the warp hits are written to the warp's row buffer (one row
        // of 32 lane values, each the sum of the lane's two pixels, per gradient value);
        // every SUB of them, the warp's lanes sum whole rows (one pass of 27 sums for
        // SUB = 3) into red[warp][j], and the splat's hitw bit for this warp is set.
        // Warps that miss a splat neither store nor sum for it, and the block's sum over
        // warps (in warp order) skips them.
        int q = 0;          // splats pending in the row buffer (warp-uniform)
        uint32_t pend = 0;  // their staged indices, 8 bits each, the newest lowest
        for (int c32 = (cnt - 1) >> 5; c32 >= 0; c32--) {
            const int jl = (c32 << 5) + lane;
            uint32_t bits = __ballot_sync(0xffffffffu, jl < cnt && b_start + jl <= wkf && ((sm[jl] >> warp) & 1u));
            while (bits) {
                const int hb = 31 - __clz(bits);
                bits &= ~(1u << hb);
                const int j = (c32 << 5) + hb;
                const int k = b_start + j;
                const float4 A = s0[j], B = s1[j];
                // sigma = 0.5 (a dx^2 + c dy^2) + b dx dy per pixel, scalar and in the
                // reference's order of roundings: the decisions below must equal the
                // forward pass's, and the compiler may fuse a packed multiply into a
                // following packed add (dx is the pixels' shared column)
                const float dx = A.x - fpx;
                const float dy[2] = {A.y - fpy[0], A.y - fpy[1]};
                const float hadx2 = A.z * dx * dx, bdx = B.x * dx;  // A.z, A.w: a / 2, c / 2
                float al[2];
                bool hit[2];
#pragma unroll
                for (int i = 0; i < 2; i++) {
                    const float sigma = (hadx2 + A.w * dy[i] * dy[i]) + bdx * dy[i];
                    hit[i] = false;
                    al[i] = 0.f;
                    if (inside[i] && k <= kf[i] && sigma >= 0.f && sigma < 5.55f) {
                        // The fast exponential is within 8 ulps here; near the 1/255 and
                        // 0.999 cut-offs alpha is recomputed exactly, so every decision
                        // equals the forward pass's.
                        const float va_fast = B.y * __expf(-sigma);
                        float alpha = fminf(0.999f, va_fast);
                        if (fabsf(va_fast - 1.f / 255.f) <= 1e-5f * (1.f / 255.f) || fabsf(va_fast - 0.999f) <= 1e-5f)
                            alpha = fminf(0.999f, B.y * exp_tab(-sigma, etab));
                        if (alpha >= 1.f / 255.f) {
                            hit[i] = true;
                            al[i] = alpha;
                        }
                    }
                }
                const bool any = hit[0] || hit[1];
                if (!__ballot_sync(0xffffffffu, any)) continue;
                float g[NG];
                if (any) {
                    const float4 C = s2[j];
                    // no decision depends on T here: the hardware reciprocal (within an
                    // ulp or two) recovers it within the gradient tolerance; a pixel that
                    // takes no part keeps T (times 1) and gets fac = 0
                    float ra[2];
#pragma unroll
                    for (int i = 0; i < 2; i++) ra[i] = hit[i] ? __fdividef(1.f, 1.f - al[i]) : 1.f;
                    const f32x2 ra2 = pack2(ra[0], ra[1]);
                    if (TS && (tj[0] > 0 || tj[1] > 0)) {
                        float2 t = unpack2(T2);
#pragma unroll
                        for (int i = 0; i < 2; i++) {
                            float &Ti = i ? t.y : t.x;
                            if (!hit[i]) continue;
                            if (tj[i] > 0) {
                                tj[i]--;
                                Ti = a.tstore[(size_t)tj[i] * npix + pid[i]];  // T before this Gaussian, as stored
                            } else {
                                Ti *= ra[i];
                            }
                        }
                        T2 = pack2(t.x, t.y);
                    } else {
                        T2 = mul2(T2, ra2);  // recovered by division (core/cpu/msplat_cpu.cpp:996-997)
                    }
                    const f32x2 al2 = pack2(al[0], al[1]);
                    const f32x2 fac2 = mul2(al2, T2);
                    // gradient arithmetic (no decision depends on it) uses fused
                    // multiply-adds; the reference's values are met within the gradient
                    // tolerance, not bit for bit
                    const f32x2 cv2 = fma2(pack2(B.z, B.z), vr2, fma2(pack2(B.w, B.w), vg2, mul2(pack2(C.x, C.x), vb2)));
                    const f32x2 nra2 = pack2(-ra[0], -ra[1]);
                    f32x2 va2 = fma2(T2, cv2, mul2(nra2, add2(bv2, tbv2)));
                    if (AUX) {
                        const f32x2 z2 = pack2(C.y, C.y);
                        // (z T - bd ra) vd + (T - ba ra) vaa
                        va2 = add2(va2, fma2(fma2(bd2, nra2, mul2(z2, T2)), vd2, mul2(fma2(ba2, nra2, T2), vaa2)));
                        bd2 = fma2(z2, fac2, bd2);
                        ba2 = add2(ba2, fac2);
                        const float2 gd = unpack2(mul2(fac2, vd2));
                        g[9] = gd.x + gd.y;
                    }
                    bv2 = fma2(fac2, cv2, bv2);
                    // colour gradients; a channel whose raw + 0.5 < 0 passes none, which the
                    // block's sum applies once per splat
                    const float2 gr = unpack2(mul2(fac2, vr2)), gg = unpack2(mul2(fac2, vg2)),
                                 gb = unpack2(mul2(fac2, vb2));
                    g[5] = gr.x + gr.y;
                    g[6] = gg.x + gg.y;
                    g[7] = gb.x + gb.y;
                    // vs = -alpha v_alpha for the pixels with alpha < 0.999: the xy gradient
                    // vs (conic d) per pixel (its two terms can cancel, so the sum is not
                    // factored), and the moments vs dx^2, vs dx dy, vs dy^2 and vs
                    const f32x2 nal2 = pack2(hit[0] && al[0] < 0.999f ? -al[0] : 0.f,
                                             hit[1] && al[1] < 0.999f ? -al[1] : 0.f);
                    const f32x2 vs2 = mul2(nal2, va2), dx2 = pack2(dx, dx), dy2 = pack2(dy[0], dy[1]);
                    const float adx = C.z * dx;  // the whole conic: C.z = a, C.w = c
                    const f32x2 cdy2 = mul2(pack2(C.w, C.w), dy2);
                    const f32x2 m0 = mul2(vs2, dx2), m1 = mul2(vs2, dy2);
                    const float2 e0 = unpack2(mul2(vs2, fma2(pack2(B.x, B.x), dy2, pack2(adx, adx)))),
                                 e1 = unpack2(mul2(vs2, add2(pack2(bdx, bdx), cdy2))), e2 = unpack2(mul2(m0, dx2)),
                                 e3 = unpack2(mul2(m0, dy2)), e4 = unpack2(mul2(m1, dy2)), e8 = unpack2(vs2);
                    g[0] = e0.x + e0.y;
                    g[1] = e1.x + e1.y;
                    g[2] = e2.x + e2.y;
                    g[3] = e3.x + e3.y;
                    g[4] = e4.x + e4.y;
                    g[8] = e8.x + e8.y;
                } else {
#pragma unroll
                    for (int c = 0; c < NG; c++) g[c] = 0.f;
                }
                float *row = mypb + q * NG * PB_STRIDE + lane;
#pragma unroll
                for (int c = 0; c < NG; c++) row[c * PB_STRIDE] = g[c];
                pend = (pend << 8) | (uint32_t)j;
                if (++q == SUB) {
                    bwd_warp_sums<NG, SUB>(mypb, red, hitw, pend, q, warp, lane, BB);
                    q = 0;
                }
            }
        }
        if (q) bwd_warp_sums<NG, SUB>(mypb, red, hitw, pend, q, warp, lane, BB);
        __syncthreads();
        for (int idx = threadIdx.x; idx < cnt * NG; idx += BWD_THREADS) {
            const int j = idx / NG, c = idx - j * NG;
            const uint32_t m = hitw[j];
            float s = 0.f;
#pragma unroll
            for (int w = 0; w < BWD_WARPS; w++)
                if ((m >> w) & 1u) s += red[(w * BB + j) * NG + c];
            float out;
            if (c < 2) {
                out = s;  // v_xy
            } else if (c < 5) {
                out = 0.5f * s;  // v_conic = (vs dx dx, vs dx dy, vs dy dy) / 2
            } else if (c < 8) {  // the staged colour's sign bit: raw + 0.5 < 0 passes no gradient
                const float col = c == 5 ? s1[j].z : (c == 6 ? s1[j].w : s2[j].x);
                out = signbit(col) ? 0.f : s;
            } else if (c == 8) {
                out = __fmaf_rn(s, s1[j].y, -s);  // opacity logit: -vs (1 - o)
            } else {
                out = s;  // aux: depth
            }
            if (c < 9) a.slots[(size_t)(b_start + j) * 9 + c] = out;
            else a.slots_depth[b_start + j] = out;
        }
        __syncthreads();
    }
    // intersections above every pixel's last contributor get zero slots
    for (int k = kend + threadIdx.x; k < end; k += BWD_THREADS) {
#pragma unroll
        for (int c = 0; c < 9; c++) a.slots[(size_t)k * 9 + c] = 0.f;
        if (AUX) a.slots_depth[k] = 0.f;
    }
}

template <int BB, int SB, bool AUX = false, bool TS = false>
__global__ void __launch_bounds__(BWD_THREADS, BB <= 64 ? 6 : 5) raster_bwd_kernel(RasterBwdArgs a) {
    extern __shared__ __align__(16) float4 smem4[];
    __shared__ int kmax;
    __shared__ double etab[EXP_TABLE];
    exp_table_init(etab);  // ready after the tile's first barrier
    const int tile = blockIdx.x;
    raster_bwd_tile<BB, SB, AUX, false, TS>(a, tile, tile % a.tiles_x, tile / a.tiles_x, smem4, kmax, etab);
}

// Persistent backward over the tiles of a batch of views, pulling global tile ids
// from a counter (the forward's counterpart, raster_fwd_batch_kernel).
template <int BB, int SB>
__global__ void __launch_bounds__(BWD_THREADS, 5) raster_bwd_batch_kernel(const RasterBwdArgs *views,
                                                                        const int *tile_off, int n_views,
                                                                        int *counter) {
    extern __shared__ __align__(16) float4 smem4[];
    __shared__ int kmax, s_tile, s_lt;
    __shared__ RasterBwdArgs s_args;  // the tile's view, read from shared memory (keeps registers down)
    __shared__ double etab[EXP_TABLE];
    exp_table_init(etab);  // ready after the loop's first barrier
    const int total_tiles = tile_off[n_views];
    for (;;) {
        if (threadIdx.x == 0) {
            const int t = atomicAdd(counter, 1);
            s_tile = t;
            if (t < total_tiles) {
                const int v = find_view(tile_off, n_views, t);
                s_args = views[v];
                s_lt = t - tile_off[v];
            }
        }
        __syncthreads();
        const int t = s_tile, lt = s_lt;
        if (t >= total_tiles) break;
        raster_bwd_tile<BB, SB>(s_args, t, lt % s_args.tiles_x, lt / s_args.tiles_x, smem4, kmax, etab);
        __syncthreads();  // the tile's shared state is free before thread 0 claims the next tile
    }
}

template <int FB, bool AUX, bool TS, int NT>
void fwd_launch(const RasterArgs &a, int T, cudaStream_t st) {
    raster_fwd_kernel<FB, AUX, TS, NT><<<T * (FWD_THREADS / NT), NT, 0, st>>>(a);
}

template <int FB, bool AUX, bool TS>
void fwd_launch_shape(const RasterArgs &a, int T, cudaStream_t st, int shape) {
    switch (shape_index(shape)) {
        case 1: fwd_launch<FB, AUX, TS, FWD_THREADS / 2>(a, T, st); break;
        case 2: fwd_launch<FB, AUX, TS, FWD_THREADS / 4>(a, T, st); break;
        default: fwd_launch<FB, AUX, TS, FWD_THREADS>(a, T, st); break;
    }
}

// The aux forward runs the default staging only (the reference too forces one
// rasterizer in this mode, core/metal/bindings.h:44-46).
void launch_raster_fwd_aux(const RasterArgs &a, cudaStream_t st, int shape) {
    const int T = a.tiles_x * a.tiles_y;
    if (T <= 0) return;
    if (a.tstore) fwd_launch_shape<128, true, true>(a, T, st, shape);
    else fwd_launch_shape<128, true, false>(a, T, st, shape);
}

void launch_raster_fwd(const RasterArgs &a, cudaStream_t st, int variant, int shape) {
    const int T = a.tiles_x * a.tiles_y;
    if (T <= 0) return;
    if (a.tstore) {  // stored-transmittance mode: the default staging only
        fwd_launch_shape<128, false, true>(a, T, st, shape);
        return;
    }
    switch (RASTER_VARIANTS[variant_index(variant)].fwd_batch) {
        case 64: fwd_launch_shape<64, false, false>(a, T, st, shape); break;
        case 256: fwd_launch_shape<256, false, false>(a, T, st, shape); break;
        default: fwd_launch_shape<128, false, false>(a, T, st, shape); break;
    }
}

template <int BB, int SB, bool AUX = false, bool TS = false>
void bwd_launch(const RasterBwdArgs &a, int T, cudaStream_t st) {
    constexpr size_t smem = raster_bwd_smem<BB, SB, AUX ? 10 : 9>();
    static const bool attr = [] {  // once per instance, thread-safe
        cudaFuncSetAttribute(raster_bwd_kernel<BB, SB, AUX, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        return true;
    }();
    (void)attr;
    raster_bwd_kernel<BB, SB, AUX, TS><<<T, BWD_THREADS, smem, st>>>(a);
}

template <int BB, int SB>
void bwd_batch_launch(const RasterBwdArgs *d_views, const int *d_tile_off, int n_views, int *d_counter,
                      cudaStream_t st) {
    constexpr size_t smem = raster_bwd_smem<BB, SB>();
    static const int grid = [] {
        cudaFuncSetAttribute(raster_bwd_batch_kernel<BB, SB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        return resident_grid(raster_bwd_batch_kernel<BB, SB>, smem, BWD_THREADS);
    }();
    raster_bwd_batch_kernel<BB, SB><<<grid, BWD_THREADS, smem, st>>>(d_views, d_tile_off, n_views, d_counter);
}

// The backward variants' (staged batch, reduction sub-batch) pairs, dispatched to
// their template instances. A sub-batch of 3 gives 27 sums per warp round (9 values
// x 3 splats), one pass of the warp's lanes; 4 gives 36, two passes with 4 lanes busy.
#define MSPLAT_BWD_VARIANTS(X) X(128, 3) X(64, 3) X(64, 4) X(32, 4) X(128, 4)

void launch_raster_bwd(const RasterBwdArgs &a, cudaStream_t st, int variant) {
    const int T = a.tiles_x * a.tiles_y;
    if (T <= 0) return;
    if (a.tstore) {  // stored-transmittance mode: the default staging only
        bwd_launch<128, 3, false, true>(a, T, st);
        return;
    }
    const RasterVariant &v = RASTER_VARIANTS[variant_index(variant)];
#define X(bb, sb)                                    \
    if (v.bwd_batch == bb && v.bwd_sub == sb) {      \
        bwd_launch<bb, sb>(a, T, st);                \
        return;                                      \
    }
    MSPLAT_BWD_VARIANTS(X)
#undef X
    bwd_launch<128, 3>(a, T, st);
}

// The aux backward, default staging only (as launch_raster_fwd_aux).
void launch_raster_bwd_aux(const RasterBwdArgs &a, cudaStream_t st) {
    const int T = a.tiles_x * a.tiles_y;
    if (T <= 0) return;
    if (a.tstore) bwd_launch<64, 3, true, true>(a, T, st);
    else bwd_launch<64, 3, true, false>(a, T, st);
}

void launch_raster_bwd_batch(const RasterBwdArgs *d_views, const int *d_tile_off, int n_views, int *d_counter,
                             cudaStream_t st, int variant) {
    if (n_views <= 0) return;
    cudaMemsetAsync(d_counter, 0, sizeof(int), st);
    const RasterVariant &v = RASTER_VARIANTS[variant_index(variant)];
#define X(bb, sb)                                                      \
    if (v.bwd_batch == bb && v.bwd_sub == sb) {                        \
        bwd_batch_launch<bb, sb>(d_views, d_tile_off, n_views, d_counter, st); \
        return;                                                        \
    }
    MSPLAT_BWD_VARIANTS(X)
#undef X
    bwd_batch_launch<128, 3>(d_views, d_tile_off, n_views, d_counter, st);
}

// ---------------------------------------------------------------------------------
// Work counts of a frame (measurement): per pixel, the (pixel, Gaussian) pairs the
// reference's loops evaluate. rasterize_forward (core/cpu/msplat_cpu.cpp:574-626)
// walks the tile's list from its start until the entry that ends the pixel -- the
// first contributing entry after the pixel's last contributor, if any -- or to the
// list's end; rasterize_backward (:959-1031) walks from min(final_idx, end - 1) down
// to the start. out[0] += forward pairs, out[1] += backward pairs.
__global__ void __launch_bounds__(TILE_PIX) pair_count_kernel(RasterArgs a, unsigned long long *out) {
    __shared__ double etab[EXP_TABLE];
    exp_table_init(etab);
    __syncthreads();
    const int tile = blockIdx.x, tx = tile % a.tiles_x, ty = tile / a.tiles_x;
    int lx, ly;
    tile_pixel(threadIdx.x, lx, ly);
    const int px = tx * TILE + lx, py = ty * TILE + ly;
    unsigned long long fwd = 0, bwd = 0;
    if (px < a.W && py < a.H) {
        const int start = a.tile_start[tile], end = a.tile_end[tile];
        const size_t pid = (size_t)py * a.W + px;
        const int last = a.final_idx[pid];
        bwd = (unsigned long long)max(0, min(last, end - 1) - start + 1);
        int stop = end;  // the entry that ends the pixel, or the list's end
        for (int k = max(last + 1, start); k < end; k++) {
            const float4 *rec = reinterpret_cast<const float4 *>(a.splats + a.isect_gid[k]);
            const float4 A = rec[0], B = rec[1];
            const float dx = A.x - (float)px, dy = A.y - (float)py;
            const float sigma = 0.5f * (A.z * dx * dx + B.x * dy * dy) + A.w * dx * dy;
            if (sigma < 0.f || sigma >= 5.55f) continue;
            if (fminf(0.999f, B.y * exp_tab(-sigma, etab)) < 1.f / 255.f) continue;
            stop = k + 1;
            break;
        }
        fwd = (unsigned long long)max(0, stop - start);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        fwd += __shfl_xor_sync(0xffffffffu, fwd, o);
        bwd += __shfl_xor_sync(0xffffffffu, bwd, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, fwd);
        atomicAdd(out + 1, bwd);
    }
}

// The rasterizers' exponential over n inputs (test hook for exp_span / exp_tab
// against exp_ref).
__global__ void exp_tab_kernel(const float *x, int64_t n, float *out) {
    __shared__ double etab[EXP_TABLE], espan[EXP_SPAN];
    exp_span_init_a(etab);
    __syncthreads();
    exp_span_init_b(espan, etab);
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        // over the rasterizers' range [-5.55, 0] the forward's span-table form, NaN
        // wherever it differs from the 64-entry form the backward uses (the two are the
        // same function by construction); below it the 64-entry form
        const float xi = x[i], v = exp_tab(xi, etab);
        out[i] = xi < -5.55f ? v : (exp_span(xi, espan) == v ? v : __int_as_float(0x7fc00000));
    }
}

void launch_exp_tab(const float *x, int64_t n, float *out, cudaStream_t st) {
    if (n <= 0) return;
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 16);
    exp_tab_kernel<<<(unsigned)blocks, 256, 0, st>>>(x, n, out);
}

void launch_pair_counts(const RasterArgs &a, unsigned long long *d_out, cudaStream_t st, bool accumulate) {
    const int T = a.tiles_x * a.tiles_y;
    if (!accumulate) cudaMemsetAsync(d_out, 0, 2 * sizeof(unsigned long long), st);
    if (T > 0) pair_count_kernel<<<T, TILE_PIX, 0, st>>>(a, d_out);
}

// ---------------------------------------------------------------------------------
// Depth-chunked compositing (core/metal/msplat_metal.metal:2641-3030): for frames of
// few tiles, whose lists are long, one block per (tile, piece) instead of one per
// tile puts the whole GPU on the frame. A block finds its tile by binary search over
// the tiles' first items; blocks past the item count (the grid is a host bound)
// return at once.

__global__ void chunk_count_kernel(const int32_t *tile_start, const int32_t *tile_end, int T, int len,
                                   int32_t *counts) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < T) counts[t] = (tile_end[t] - tile_start[t] + len - 1) / len;
}

void launch_chunk_items(const int32_t *tile_start, const int32_t *tile_end, int T, int chunk_len, int32_t *counts,
                        int32_t *first, int32_t *partials, cudaStream_t st) {
    if (T <= 0) return;
    chunk_count_kernel<<<(T + 255) / 256, 256, 0, st>>>(tile_start, tile_end, T, chunk_len, counts);
    scan_exclusive<int32_t>(counts, first, T, first + T, partials, st);
}

// The tile of item i: the last t with first[t] <= i (tiles without items share their
// first with the next tile, so the search lands on one that has items).
__device__ __forceinline__ int chunk_tile(const int32_t *first, int T, int i) {
    int lo = 0, hi = T;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (first[mid] <= i) lo = mid + 1;
        else hi = mid;
    }
    return lo - 1;
}

template <int FB>
__global__ void __launch_bounds__(FWD_THREADS, 4) raster_fwd_chunk_kernel(RasterArgs a, ChunkArgs c) {
    __shared__ float4 s0[FB], s1[FB], s2[FB];
    __shared__ uint8_t sm[FB];
    const int T = a.tiles_x * a.tiles_y, item = blockIdx.x;
    if (item >= c.first[T]) return;  // block-uniform
    const int tile = chunk_tile(c.first, T, item);
    __shared__ double et64[EXP_TABLE], espan[EXP_SPAN];
    exp_span_init_a(et64);
    __syncthreads();
    exp_span_init_b(espan, et64);  // ready after the tile's first barrier
    raster_fwd_tile<FB, false, true>(a, tile, tile % a.tiles_x, tile / a.tiles_x, s0, s1, s2, sm, espan, &c, item,
                                     item - c.first[tile]);
}

// rasterize_forward_merge_kernel (.metal:2741-2808): per pixel, the tile's pieces front
// to back, C += piece C * T (fused), T *= piece T, the last contributor taken from every
// piece that has one (a piece without contributors reports its start - 1), stopping
// once T <= 1e-4; the pieces past the stop lose their contributors for the backward.
__global__ void __launch_bounds__(TILE_PIX) chunk_merge_kernel(RasterArgs a, ChunkArgs c) {
    const int tile = blockIdx.x, tx = tile % a.tiles_x, ty = tile / a.tiles_x;
    int lx, ly;
    tile_pixel(threadIdx.x, lx, ly);
    const int px = tx * TILE + lx, py = ty * TILE + ly;
    if (px >= a.W || py >= a.H) return;
    const int i0 = c.first[tile], n = c.first[tile + 1] - i0;
    float T = 1.f, cr = 0.f, cg = 0.f, cb = 0.f;
    int last = -1, cut = n;
    for (int k = 0; k < n; k++) {
        const size_t o = (size_t)(i0 + k) * TILE_PIX + threadIdx.x, o3 = (size_t)(i0 + k) * 3 * TILE_PIX + threadIdx.x;
        cr = __fmaf_rn(c.cC[o3], T, cr);
        cg = __fmaf_rn(c.cC[o3 + TILE_PIX], T, cg);
        cb = __fmaf_rn(c.cC[o3 + 2 * TILE_PIX], T, cb);
        T *= c.cT[o];
        const int cl = c.clast[o];
        if (cl >= 0) last = cl;
        if (T <= 1e-4f) {
            cut = k + 1;
            break;
        }
    }
    for (int k = cut; k < n; k++) c.clast[(size_t)(i0 + k) * TILE_PIX + threadIdx.x] = -1;
    const size_t pid = (size_t)py * a.W + px;
    a.final_T[pid] = T;
    a.final_idx[pid] = last;
    float *o = a.out_img + 3 * pid;
    o[0] = clamp01(__fmaf_rn(a.bg[0], T, cr));
    o[1] = clamp01(__fmaf_rn(a.bg[1], T, cg));
    o[2] = clamp01(__fmaf_rn(a.bg[2], T, cb));
}

template <int FB>
void fwd_chunk_launch(const RasterArgs &a, const ChunkArgs &c, int64_t items, cudaStream_t st) {
    raster_fwd_chunk_kernel<FB><<<(unsigned)items, FWD_THREADS, 0, st>>>(a, c);
}

void launch_raster_fwd_chunked(const RasterArgs &a, const ChunkArgs &c, int64_t item_cap, cudaStream_t st,
                               int variant) {
    const int T = a.tiles_x * a.tiles_y;
    if (T <= 0) return;
    if (item_cap > 0) {
        switch (RASTER_VARIANTS[variant_index(variant)].fwd_batch) {
            case 64: fwd_chunk_launch<64>(a, c, item_cap, st); break;
            case 256: fwd_chunk_launch<256>(a, c, item_cap, st); break;
            default: fwd_chunk_launch<128>(a, c, item_cap, st); break;
        }
    }
    chunk_merge_kernel<<<T, TILE_PIX, 0, st>>>(a, c);
}

// compute_chunk_prefix_suffix_kernel (.metal:2812-2848): per pixel, the product of the
// transmittances of the pieces in front of each piece and the sum over the pieces
// behind it of prefix * colour (every piece of the tile, those past the stop included).
__global__ void __launch_bounds__(TILE_PIX) chunk_prefix_kernel(int W, int H, int tiles_x, ChunkArgs c) {
    const int tile = blockIdx.x, tx = tile % tiles_x, ty = tile / tiles_x;
    int lx, ly;
    tile_pixel(threadIdx.x, lx, ly);
    if (tx * TILE + lx >= W || ty * TILE + ly >= H) return;
    const int i0 = c.first[tile], n = c.first[tile + 1] - i0;
    float p = 1.f;
    for (int k = 0; k < n; k++) {
        const size_t o = (size_t)(i0 + k) * TILE_PIX + threadIdx.x;
        c.pre[o] = p;
        p *= c.cT[o];
    }
    float ar = 0.f, ag = 0.f, ab = 0.f;
    for (int k = n - 1; k >= 0; k--) {
        const size_t o = (size_t)(i0 + k) * TILE_PIX + threadIdx.x, o3 = (size_t)(i0 + k) * 3 * TILE_PIX + threadIdx.x;
        c.aft[o3] = ar;
        c.aft[o3 + TILE_PIX] = ag;
        c.aft[o3 + 2 * TILE_PIX] = ab;
        const float pk = c.pre[o];
        ar += pk * c.cC[o3];
        ag += pk * c.cC[o3 + TILE_PIX];
        ab += pk * c.cC[o3 + 2 * TILE_PIX];
    }
}

template <int BB, int SB>
__global__ void __launch_bounds__(BWD_THREADS, 5) raster_bwd_chunk_kernel(RasterBwdArgs a, ChunkArgs c) {
    extern __shared__ __align__(16) float4 smem4[];
    __shared__ int kmax;
    const int T = a.tiles_x * a.tiles_y, item = blockIdx.x;
    if (item >= c.first[T]) return;  // block-uniform
    const int tile = chunk_tile(c.first, T, item);
    __shared__ double etab[EXP_TABLE];
    exp_table_init(etab);  // ready after the tile's first barrier
    raster_bwd_tile<BB, SB, false, true>(a, tile, tile % a.tiles_x, tile / a.tiles_x, smem4, kmax, etab, &c,
                                         item, item - c.first[tile]);
}

template <int BB, int SB>
void bwd_chunk_launch(const RasterBwdArgs &a, const ChunkArgs &c, int64_t items, cudaStream_t st) {
    constexpr size_t smem = raster_bwd_smem<BB, SB>();
    static const bool attr = [] {
        cudaFuncSetAttribute(raster_bwd_chunk_kernel<BB, SB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        return true;
    }();
    (void)attr;
    raster_bwd_chunk_kernel<BB, SB><<<(unsigned)items, BWD_THREADS, smem, st>>>(a, c);
}

void launch_raster_bwd_chunked(const RasterBwdArgs &a, const ChunkArgs &c, int64_t item_cap, cudaStream_t st,
                               int variant) {
    const int T = a.tiles_x * a.tiles_y;
    if (T <= 0) return;
    chunk_prefix_kernel<<<T, TILE_PIX, 0, st>>>(a.W, a.H, a.tiles_x, c);
    if (item_cap <= 0) return;
    const RasterVariant &v = RASTER_VARIANTS[variant_index(variant)];
#define X(bb, sb)                                   \
    if (v.bwd_batch == bb && v.bwd_sub == sb) {     \
        bwd_chunk_launch<bb, sb>(a, c, item_cap, st); \
        return;                                     \
    }
    MSPLAT_BWD_VARIANTS(X)
#undef X
    bwd_chunk_launch<128, 3>(a, c, item_cap, st);
}

}  // namespace msplat
