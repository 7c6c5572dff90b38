// Host-side state shared by the C-ABI translation units: the context (stream, frame
// cache, stage timer, batched-step state), device-buffer growth and error reporting.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/msplat_cuda.h"
#include "kernels.h"

namespace msplat {

// Records the message returned by msplat_cuda_last_error() (per thread); returns code.
int fail(int code, const char *fmt, ...);
const char *last_error_text();

#define CUDA_TRY(expr)                                                                          \
    do {                                                                                        \
        cudaError_t _e = (expr);                                                                \
        if (_e != cudaSuccess) return fail(MSPLAT_CUDA_ECUDA, "%s: %s", #expr, cudaGetErrorString(_e)); \
    } while (0)

struct Buf {
    void *ptr = nullptr;
    size_t bytes = 0;
};

}  // namespace msplat

using msplat::Buf;

// Stage timing with CUDA events on the context's stream (the reference's
// PROFILE_STAGES, core/metal/msplat_metal.mm:29-32, drained by
// msplat_drain_stage_times, core/metal/bindings.h:38).
constexpr int N_STAGES = 6;
const char *const STAGE_NAMES[N_STAGES] = {"proj_sh_fwd", "bin_sort", "rast_fwd", "loss_fwd_bwd", "rast_bwd",
                                           "proj_sh_bwd_adam"};

// Each call records its marks into one slot of a ring; a slot is read back only when
// the ring comes round to it again (long finished by then) or on drain, so timing
// adds no synchronisation to the calls themselves.
constexpr int TIMER_RING = 64;

struct StageTimer {
    bool on = false;
    int cur = 0;
    cudaEvent_t ev[TIMER_RING][N_STAGES + 1] = {};
    bool marked[TIMER_RING][N_STAGES + 1] = {};
    double acc_ms[N_STAGES] = {};
    int64_t calls[N_STAGES] = {};
    void init() {
        for (auto &slot : ev)
            for (auto &e : slot)
                if (!e) cudaEventCreate(&e);
    }
    void reset_marks() {
        for (bool &m : marked[cur]) m = false;
    }
    void mark(int i, cudaStream_t st) {
        if (!on) return;
        cudaEventRecord(ev[cur][i], st);
        marked[cur][i] = true;
    }
    // accumulate every consecutive pair of recorded marks of one slot
    void collect_slot(int s) {
        int last = -1;
        for (int i = 0; i <= N_STAGES; i++) {
            if (!marked[s][i]) continue;
            if (last >= 0) {
                cudaEventSynchronize(ev[s][i]);
                float ms = 0.f;
                if (cudaEventElapsedTime(&ms, ev[s][last], ev[s][i]) == cudaSuccess) {
                    acc_ms[last] += ms;
                    calls[last] += 1;
                }
            }
            last = i;
        }
        for (bool &m : marked[s]) m = false;
    }
    // end of a call: move to the next slot, reading back the one found there
    void collect() {
        if (!on) return;
        cur = (cur + 1) % TIMER_RING;
        collect_slot(cur);
    }
    void drain() {
        for (int s = 0; s < TIMER_RING; s++) collect_slot(s);
    }
    void destroy() {
        for (auto &slot : ev)
            for (auto &e : slot)
                if (e) cudaEventDestroy(e), e = nullptr;
    }
};

// State of the batched training step (msplat_cuda_train_batch): capacity-sized
// buffers, the per-step view descriptors, and the CUDA graph of the step.
struct TrainBatchState {
    Buf desc;                                   // device view descriptors
    unsigned char *h_stage[2] = {nullptr, nullptr};  // pinned staging, double-buffered
    size_t h_stage_bytes = 0;
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};    // upload from slot k finished
    bool stage_pending[2] = {false, false};
    int slot = 0;
    Buf pix_img, pix_T, pix_idx, pix_v, partials, losses, counters;
    int64_t isect_cap = 0;  // elements the per-intersection buffers hold
    int tile_cap = 0;       // key bits are sized for this many tiles
    void *h_out = nullptr;  // pinned readback: overflow flag, count, per-view losses
    size_t h_out_bytes = 0;
    // graph mode (option "graph"): the step from projection to Adam is captured once
    // per shape and replayed; the descriptors are uploaded before each replay
    bool graph = false;
    cudaStream_t gstream = nullptr;
    cudaEvent_t ev_in = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> key;
    int64_t replays = 0, captures = 0, overflows = 0;

    void release() {
        Buf *all[] = {&desc, &pix_img, &pix_T, &pix_idx, &pix_v, &partials, &losses, &counters};
        for (Buf *b : all) {
            if (b->ptr) cudaFree(b->ptr);
            b->ptr = nullptr;
            b->bytes = 0;
        }
        for (int k = 0; k < 2; k++) {
            if (h_stage[k]) cudaFreeHost(h_stage[k]);
            h_stage[k] = nullptr;
            if (stage_ev[k]) cudaEventDestroy(stage_ev[k]);
            stage_ev[k] = nullptr;
            stage_pending[k] = false;
        }
        h_stage_bytes = 0;
        if (h_out) cudaFreeHost(h_out);
        h_out = nullptr;
        h_out_bytes = 0;
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        key.clear();
        if (ev_in) cudaEventDestroy(ev_in);
        ev_in = nullptr;
        if (gstream) cudaStreamDestroy(gstream);
        gstream = nullptr;
        isect_cap = 0;
        tile_cap = 0;
    }
};

// Buffers of the prior-guided extras (msplat_cuda_set_prior), by index into
// msplat_cuda_ctx::pri.
enum PriBuf {
    PB_DEPTH,     // expected-depth numerator (H, W)
    PB_BG,        // per-pixel background (H, W, 3)
    PB_VAUX,      // dL/d(depth numerator, alpha) (H, W, 2)
    PB_SLOTS_D,   // depth gradient per intersection
    PB_VDEPTH,    // dL/d(view depth) per Gaussian (keep_grads)
    PB_TERMS,     // per-pixel loss terms (3, H, W)
    PB_ROWS,      // per-row loss-term sums (H, 3) double
    PB_ADJ,       // exposure-adjusted render (H, W, 3)
    PB_VADJ,      // its gradient (H, W, 3)
    PB_EXPO,      // exposure-gradient block partials (double)
    PB_SKY_IDX, PB_SKY_W, PB_SKY_G, PB_SKY_COUNT, PB_SKY_OFF, PB_SKY_PART, PB_SKY_TOTAL,  // sky backward
    PB_SKY_K0, PB_SKY_K1, PB_SKY_V0, PB_SKY_V1, PB_SKY_RS,
    PB_COUNT
};

// ChunkArgs buffers: per-tile item counts, first items, scan partials, then the
// per-(item, pixel) planes
enum ChunkBuf { CH_COUNTS, CH_FIRST, CH_PART, CH_T, CH_C, CH_LAST, CH_PRE, CH_AFT, CH_COUNT };
constexpr int CHUNK_AUTO_TILES = 400;  // core/metal/msplat_metal.mm:1103

struct msplat_cuda_ctx {
    cudaStream_t stream = nullptr;
    int raster_variant = 0;  // option "raster_variant": index into RASTER_VARIANTS
    int raster_shape = 0;    // option "raster_shape": index into RASTER_SHAPES (forward rasterizers)
    TrainBatchState tb;
    bool keep_grads = false;
    StageTimer timer;
    // frame description
    int n = 0, W = 0, H = 0, tiles_x = 0, tiles_y = 0;
    int64_t n_isect = 0;
    int sorted = 0;  // which key/value buffer pair holds the sorted result
    bool gid_in_vals = false;  // the sorted values are Gaussian ids (batched render) rather than emission indices
    // per Gaussian
    Buf splats, radii, aabb, n_tiles, offsets, scan_part, total;
    Buf v_xy, v_conic, v_rgb, v_opacity, v_mean3d, v_scale, v_quat;
    // per intersection
    Buf keys[2], vals[2], emit_gid, isect_gid, inv, slots, radix_scratch;
    // per tile / pixel
    Buf tile_start, tile_end, out_img, final_T, final_idx, v_rendered, loss_part, loss;
    // densification and primitive scratch
    Buf d_flags, d_counts, d_scratch, k_bounds, k_sorted, k_box, k_md, k_evals;
    // stored-transmittance mode (option "store_transmittance" = per-pixel capacity)
    int tstore_cap = 0;
    Buf tstore, tcount;
    Buf pairs;  // the frame's pair counts (msplat_cuda_frame_pair_counts)
    // depth-chunked compositing: option "chunked_raster" (0 off, 1 frames of fewer
    // than CHUNK_AUTO_TILES tiles, 2 every frame) and "chunk_len"; whether the last
    // single-view frame ran chunked, its item bound, and the ChunkArgs planes
    int chunk_mode = 0, chunk_len = 512;
    bool chunk_frame = false;
    int64_t chunk_cap = 0;
    Buf ch[CH_COUNT];
    // depth order of the Gaussians (or batch instances) before key emission
    Buf dkeys[2], dvals[2], dcounts, doff;
    // image pipeline scratch: metrics (moments, terms, row sums) and RGBA8 packing
    Buf img[6];
    // prior-guided extras: the prior in force, whether the last frame ran in aux
    // mode, and their buffers
    bool has_prior = false, aux_frame = false;
    msplat_cuda_prior prior{};
    Buf pri[PB_COUNT];
    int64_t *h_total = nullptr;  // pinned readback of the intersection count
    cudaEvent_t total_ev = nullptr;  // recorded after that readback
    int32_t *h_count = nullptr;  // pinned readback of the densified count
    // batched render: device view descriptors, their pinned staging copy, the
    // persistent rasterizer's work counter, and an event after the last upload
    Buf bdesc, bcounter;
    unsigned char *h_bdesc = nullptr;
    size_t h_bdesc_bytes = 0;
    cudaEvent_t bdesc_ev = nullptr;
    bool bdesc_pending = false;

    ~msplat_cuda_ctx() {
        release();
        timer.destroy();
    }
    void release() {
        Buf *all[] = {&splats, &radii, &aabb, &n_tiles, &offsets, &scan_part, &total, &v_xy, &v_conic, &v_rgb,
                      &v_opacity, &v_mean3d, &v_scale, &v_quat, &keys[0], &keys[1], &vals[0], &vals[1], &emit_gid,
                      &isect_gid, &inv, &slots, &radix_scratch, &tile_start, &tile_end, &out_img, &final_T,
                      &final_idx, &v_rendered, &loss_part, &loss, &d_flags, &d_counts, &d_scratch, &k_bounds,
                      &k_sorted, &k_box, &k_md, &k_evals, &tstore, &tcount, &pairs, &bdesc, &bcounter, &dkeys[0], &dkeys[1],
                      &dvals[0], &dvals[1], &dcounts, &doff, &img[0], &img[1], &img[2], &img[3], &img[4], &img[5]};
        for (Buf *b : all) {
            if (b->ptr) cudaFree(b->ptr);
            b->ptr = nullptr;
            b->bytes = 0;
        }
        for (Buf &b : pri) {
            if (b.ptr) cudaFree(b.ptr);
            b.ptr = nullptr;
            b.bytes = 0;
        }
        for (Buf &b : ch) {
            if (b.ptr) cudaFree(b.ptr);
            b.ptr = nullptr;
            b.bytes = 0;
        }
        aux_frame = false;
        chunk_frame = false;
        tb.release();  // its graph refers to the buffers just freed
        if (h_total) cudaFreeHost(h_total);
        h_total = nullptr;
        if (total_ev) cudaEventDestroy(total_ev);
        total_ev = nullptr;
        if (h_count) cudaFreeHost(h_count);
        h_count = nullptr;
        if (h_bdesc) cudaFreeHost(h_bdesc);
        h_bdesc = nullptr;
        h_bdesc_bytes = 0;
        if (bdesc_ev) cudaEventDestroy(bdesc_ev);
        bdesc_ev = nullptr;
        bdesc_pending = false;
    }
};

namespace msplat {

template <typename T>
inline int ensure(Buf &b, size_t count, T **out) {
    const size_t need = std::max<size_t>(count, 1) * sizeof(T);
    if (b.bytes < need) {
        if (b.ptr) {
            cudaError_t e = cudaFree(b.ptr);
            if (e != cudaSuccess) return fail(MSPLAT_CUDA_ECUDA, "cudaFree: %s", cudaGetErrorString(e));
        }
        b.ptr = nullptr;
        b.bytes = 0;
        const size_t bytes = need + need / 4;
        cudaError_t e = cudaMalloc(&b.ptr, bytes);
        if (e != cudaSuccess) {
            b.ptr = nullptr;
            return fail(MSPLAT_CUDA_ECUDA, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
        }
        b.bytes = bytes;
    }
    *out = reinterpret_cast<T *>(b.ptr);
    return MSPLAT_CUDA_OK;
}

#define ENSURE(buf, count, type, var) \
    type *var = nullptr;              \
    if (int _r = ensure<type>(buf, (size_t)(count), &var)) return _r;

inline int ceil_log2(int v) {
    int b = 0;
    while ((1 << b) < v) b++;
    return b;
}

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

int check_camera(int num_points, unsigned H, unsigned W, int tx, int ty, unsigned degree, unsigned dtu,
                 const float *viewmat, const float *projmat, const float *cam_pos, const float *bg);
CamParams make_cam(const float *viewmat, const float *projmat, float fx, float fy, float cx, float cy, unsigned H,
                   unsigned W, int tx, int ty, float clip, unsigned degree, unsigned dtu, const float *cam_pos);

// Depth-order scratch for n Gaussians (or batch instances) from the context's buffers.
inline int ensure_depth_scratch(msplat_cuda_ctx *ctx, int64_t n, DepthScratch &s) {
    ENSURE(ctx->dkeys[0], n, uint32_t, k0);
    ENSURE(ctx->dkeys[1], n, uint32_t, k1);
    ENSURE(ctx->dvals[0], n, uint32_t, v0);
    ENSURE(ctx->dvals[1], n, uint32_t, v1);
    ENSURE(ctx->dcounts, n, int32_t, counts);
    ENSURE(ctx->doff, n, int64_t, off);
    ENSURE(ctx->radix_scratch, radix_scratch_bytes((int)std::max<int64_t>(n, 1)), unsigned char, rs);
    s.keys[0] = k0;
    s.keys[1] = k1;
    s.vals[0] = v0;
    s.vals[1] = v1;
    s.counts = counts;
    s.off_sorted = off;
    s.radix_scratch = rs;
    return 0;
}

}  // namespace msplat
