// Batched training step (msplat_cuda_train_batch): several views of one scene, of
// any resolutions, trained in one step.
//
// The reference trains one view per msplat_train_step (core/metal/bindings.h:100-118,
// driven by Model::fullIteration, core/src/model.cpp:595-660). Here one step renders
// every view of the batch, takes each view's msplat loss (L1 + SSIM, its gradient
// scaled by 1 / (3 W H) as in the single-view step), sums the gradients over views and
// applies ONE Adam step; the densification statistics advance once per view that
// sees a Gaussian, as consecutive single-view steps advance them. A one-view batch is
// the single-view step.
//
// Work is numbered globally: instance v * N + i is Gaussian i seen by view v, tiles
// and pixels run view after view. Each stage is one launch over the whole batch:
// projection, scan, key emission, one stable radix sort of all (view, tile) keys,
// tile ranges, and persistent rasterizer / SSIM / raster-backward kernels that pull
// (view, tile) or (view, block) work items from counters, then the multi-view
// backward + Adam kernel.
//
// Every count the kernels need is read on the device (intersections from the scan,
// tiles and blocks from the uploaded view descriptors); the per-intersection buffers
// have a capacity. That makes the step from projection to Adam capturable as one CUDA
// graph (option "graph"): per step the host uploads the views' descriptors and
// replays the graph. A step whose intersections exceed the capacity changes nothing
// (every kernel after the count sees zero intersections and the backward skips); the
// host then grows the buffers, captures again and repeats the step.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "context.h"

using namespace msplat;

namespace {

// Offsets of the descriptor blob (device copy and pinned staging share the layout).
struct BlobLayout {
    size_t proj, ras, rbwd, ssim, inst, toff, tx, ty, boff, imd, adam, bytes;
    BlobLayout(int nv) {
        proj = 0;
        ras = align_up(proj + nv * sizeof(ProjectArgs), 256);
        rbwd = align_up(ras + nv * sizeof(RasterArgs), 256);
        ssim = align_up(rbwd + nv * sizeof(RasterBwdArgs), 256);
        inst = align_up(ssim + nv * sizeof(SsimArgs), 256);
        toff = inst + (nv + 1) * sizeof(int);
        tx = toff + (nv + 1) * sizeof(int);
        ty = tx + nv * sizeof(int);
        boff = ty + nv * sizeof(int);
        imd = boff + (nv + 1) * sizeof(int);
        adam = align_up(imd + nv * sizeof(float), 16);
        bytes = adam + 12 * sizeof(float);
    }
};

// Counters (int32) in tb.counters.
enum { C_OVERFLOW = 0, C_NISECT = 1, C_RAS = 2, C_SSIM = 3, C_RBWD = 4, N_COUNTERS = 8 };

struct StepArgs {
    int n, nv;
    float *p[6];  // means scales quats dc rest opacity
    float glob_scale, clip;
    unsigned degree, dtu;
    const float *bg;
    const msplat_cuda_train_view *views;
    float ssim_weight;
    int adam_groups;
    float *const *m1;
    float *const *m2;
    const float *ss, *bc2;
    float beta1, beta2, eps;
    float *vis, *gn, *ms;
    float *const *grads;
    int variant;  // rasterizer staging variant
    int shape;    // batched forward's block shape (RASTER_SHAPES)
};

// Device pointers of one step, derived from the context's buffers.
struct StepPtrs {
    unsigned char *desc;
    Splat *splats;
    int32_t *radii, *n_tiles;
    float *aabb;
    int64_t *offsets, *scan_part, *total;
    int32_t *tile_start, *tile_end;
    uint32_t *k[2];
    uint32_t *v[2];
    int32_t *emit_gid, *isect_gid, *inv;
    float *slots;
    void *rscratch;
    float *img, *T, *v_img;
    int32_t *idx;
    double *partials;
    float *losses;
    int *counters;
    DepthScratch depth;  // depth order of the instances
};

struct Sizes {
    int64_t inst = 0, tiles = 0, pix = 0, blocks = 0;
};

int check_step(const StepArgs &a) {
    if (a.n < 0) return fail(MSPLAT_CUDA_EINVAL, "num_points must be >= 0 (got %d)", a.n);
    if (a.nv <= 0 || !a.views) return fail(MSPLAT_CUDA_EINVAL, "need at least one view");
    if (a.degree > 4 || a.dtu > a.degree)
        return fail(MSPLAT_CUDA_EINVAL, "SH degree %u / degrees_to_use %u", a.degree, a.dtu);
    if (!a.bg) return fail(MSPLAT_CUDA_EINVAL, "null background");
    if (a.n > 0 && (!a.p[0] || !a.p[1] || !a.p[2] || !a.p[3] || !a.p[5] || (a.degree > 0 && !a.p[4])))
        return fail(MSPLAT_CUDA_EINVAL, "null Gaussian parameter pointer");
    const bool adam = a.adam_groups >= 5;
    if (adam && (!a.m1 || !a.m2 || !a.ss || !a.bc2)) return fail(MSPLAT_CUDA_EINVAL, "null Adam state");
    if (adam)
        for (int g = 0; g < std::min(a.adam_groups, 6); g++)
            if (a.n > 0 && (!a.m1[g] || !a.m2[g]) && !(g == 4 && a.degree == 0))
                return fail(MSPLAT_CUDA_EINVAL, "null Adam moment for group %d", g);
    if (a.grads && a.n > 0)
        for (int g = 0; g < 6; g++)
            if (!a.grads[g] && !(g == 4 && a.degree == 0))
                return fail(MSPLAT_CUDA_EINVAL, "null gradient output %d", g);
    if ((a.vis || a.gn || a.ms) && !(a.vis && a.gn && a.ms))
        return fail(MSPLAT_CUDA_EINVAL, "densification statistics need all three arrays");
    for (int v = 0; v < a.nv; v++) {
        const msplat_cuda_train_view &w = a.views[v];
        if (w.img_width == 0 || w.img_height == 0)
            return fail(MSPLAT_CUDA_EINVAL, "view %d: image size must be positive (%ux%u)", v, w.img_width,
                        w.img_height);
        if (!w.gt) return fail(MSPLAT_CUDA_EINVAL, "view %d: null target image", v);
    }
    return MSPLAT_CUDA_OK;
}

Sizes sizes_of(const StepArgs &a) {
    Sizes s;
    s.inst = (int64_t)a.nv * a.n;
    for (int v = 0; v < a.nv; v++) {
        const msplat_cuda_train_view &w = a.views[v];
        s.tiles += (int64_t)((w.img_width + TILE - 1) / TILE) * ((w.img_height + TILE - 1) / TILE);
        s.pix += (int64_t)w.img_width * w.img_height;
        s.blocks += ssim_blocks((int)w.img_width, (int)w.img_height);
    }
    return s;
}

// Grows every buffer the step uses to hold `sz` and `isect_cap` intersections.
int ensure_buffers(msplat_cuda_ctx *ctx, const Sizes &sz, int64_t isect_cap, int nv, StepPtrs &P) {
    TrainBatchState &tb = ctx->tb;
    const int64_t inst = sz.inst;
    ENSURE(tb.desc, BlobLayout(nv).bytes, unsigned char, desc);
    ENSURE(ctx->splats, inst, Splat, splats);
    ENSURE(ctx->radii, inst, int32_t, radii);
    ENSURE(ctx->aabb, 2 * inst, float, aabb);
    ENSURE(ctx->n_tiles, inst, int32_t, n_tiles);
    ENSURE(ctx->offsets, inst, int64_t, offsets);
    ENSURE(ctx->scan_part, scan_blocks((int)std::max<int64_t>(inst, 1)) + 1, int64_t, scan_part);
    ENSURE(ctx->total, 1, int64_t, total);
    ENSURE(ctx->tile_start, sz.tiles, int32_t, tile_start);
    ENSURE(ctx->tile_end, sz.tiles, int32_t, tile_end);
    ENSURE(ctx->keys[0], isect_cap, uint32_t, k0);
    ENSURE(ctx->keys[1], isect_cap, uint32_t, k1);
    ENSURE(ctx->vals[0], isect_cap, uint32_t, v0);
    ENSURE(ctx->vals[1], isect_cap, uint32_t, v1);
    ENSURE(ctx->emit_gid, isect_cap, int32_t, emit_gid);
    ENSURE(ctx->isect_gid, isect_cap, int32_t, isect_gid);
    ENSURE(ctx->inv, isect_cap, int32_t, inv);
    ENSURE(ctx->slots, isect_cap * 9, float, slots);
    ENSURE(ctx->radix_scratch, radix_scratch_bytes((int)isect_cap), unsigned char, rscratch);
    ENSURE(tb.pix_img, 3 * sz.pix, float, img);
    ENSURE(tb.pix_T, sz.pix, float, T);
    ENSURE(tb.pix_idx, sz.pix, int32_t, idx);
    ENSURE(tb.pix_v, 3 * sz.pix, float, v_img);
    ENSURE(tb.partials, sz.blocks, double, partials);
    ENSURE(tb.losses, nv, float, losses);
    ENSURE(tb.counters, N_COUNTERS, int, counters);
    P = StepPtrs{desc, splats, radii, n_tiles, aabb, offsets, scan_part, total, tile_start, tile_end, {k0, k1},
                 {v0, v1}, emit_gid, isect_gid, inv, slots, rscratch, img, T, v_img, idx, partials, losses, counters,
                 {}};
    // capacities as the buffers now stand (ENSURE keeps headroom)
    const int64_t cap_k = (int64_t)std::min({ctx->keys[0].bytes / 4, ctx->keys[1].bytes / 4, ctx->vals[0].bytes / 4,
                                             ctx->vals[1].bytes / 4, ctx->emit_gid.bytes / 4,
                                             ctx->isect_gid.bytes / 4, ctx->inv.bytes / 4, ctx->slots.bytes / 36});
    tb.isect_cap = std::min<int64_t>(cap_k, INT32_MAX / 2);
    // one sort scratch serves the depth sort and the tile sort, so it covers both sizes
    // (no reallocation when it already does)
    if (int r = ensure_depth_scratch(ctx, inst, P.depth)) return r;
    ENSURE(ctx->radix_scratch, radix_scratch_bytes((int)std::max<int64_t>(tb.isect_cap, inst)), unsigned char, rs2);
    P.rscratch = rs2;
    P.depth.radix_scratch = rs2;
    tb.tile_cap = (int)std::min<size_t>(std::min(ctx->tile_start.bytes, ctx->tile_end.bytes) / 4, INT32_MAX);
    return MSPLAT_CUDA_OK;
}

// Fills the descriptor blob for this step into pinned staging.
void fill_blob(unsigned char *h, const StepArgs &a, const StepPtrs &P) {
    const BlobLayout L(a.nv);
    ProjectArgs *pa = reinterpret_cast<ProjectArgs *>(h + L.proj);
    RasterArgs *ra = reinterpret_cast<RasterArgs *>(h + L.ras);
    RasterBwdArgs *rb = reinterpret_cast<RasterBwdArgs *>(h + L.rbwd);
    SsimArgs *sa = reinterpret_cast<SsimArgs *>(h + L.ssim);
    int *inst = reinterpret_cast<int *>(h + L.inst), *toff = reinterpret_cast<int *>(h + L.toff);
    int *tx = reinterpret_cast<int *>(h + L.tx), *ty = reinterpret_cast<int *>(h + L.ty);
    int *boff = reinterpret_cast<int *>(h + L.boff);
    float *imd = reinterpret_cast<float *>(h + L.imd), *adam = reinterpret_cast<float *>(h + L.adam);
    int to = 0, bo = 0;
    int64_t po = 0;
    for (int v = 0; v < a.nv; v++) {
        const msplat_cuda_train_view &w = a.views[v];
        const int W = (int)w.img_width, H = (int)w.img_height;
        const int tX = (W + TILE - 1) / TILE, tY = (H + TILE - 1) / TILE;
        ProjectArgs &p = pa[v];
        p.n = a.n;
        p.means = a.p[0];
        p.scales = a.p[1];
        p.quats = a.p[2];
        p.features_dc = a.p[3];
        p.features_rest = a.p[4];
        p.opacities = a.p[5];
        p.rest_stride = (int)(num_sh_bases(a.degree) - 1) * 3;
        p.glob_scale = a.glob_scale;
        p.cam = make_cam(w.viewmat, w.projmat, w.fx, w.fy, w.cx, w.cy, w.img_height, w.img_width, tX, tY, a.clip,
                         a.degree, a.dtu, w.cam_pos);
        p.splats = P.splats;
        p.radii = P.radii;
        p.aabb = P.aabb;
        p.n_tiles = P.n_tiles;

        RasterArgs &r = ra[v];
        r.W = W;
        r.H = H;
        r.tiles_x = tX;
        r.tiles_y = tY;
        r.tile_start = P.tile_start;
        r.tile_end = P.tile_end;
        r.isect_gid = P.isect_gid;
        r.splats = P.splats;
        for (int c = 0; c < 3; c++) r.bg[c] = a.bg[c];
        r.out_img = P.img + 3 * po;
        r.final_T = P.T + po;
        r.final_idx = P.idx + po;
        r.tstore = nullptr;
        r.tcount = nullptr;
        r.tcap = 0;

        RasterBwdArgs &b = rb[v];
        b.W = W;
        b.H = H;
        b.tiles_x = tX;
        b.tiles_y = tY;
        b.tile_start = P.tile_start;
        b.tile_end = P.tile_end;
        b.isect_gid = P.isect_gid;
        b.splats = P.splats;
        for (int c = 0; c < 3; c++) b.bg[c] = a.bg[c];
        b.final_T = P.T + po;
        b.final_idx = P.idx + po;
        b.v_out = P.v_img + 3 * po;
        b.slots = P.slots;
        b.tstore = nullptr;
        b.tcount = nullptr;

        SsimArgs &s = sa[v];
        s.W = W;
        s.H = H;
        s.img = P.img + 3 * po;
        s.gt = w.gt;
        s.ssim_weight = a.ssim_weight;
        s.inv_n = (float)(1.0 / ((double)W * H * 3));  // the single-view step's loss_inv_n
        s.v_out = P.v_img + 3 * po;
        s.partials = P.partials;
        s.loss = P.losses + v;

        inst[v] = v * a.n;
        toff[v] = to;
        tx[v] = tX;
        ty[v] = tY;
        boff[v] = bo;
        imd[v] = (float)(1.0 / (double)std::max(W, H));
        to += tX * tY;
        bo += ssim_blocks(W, H);
        po += (int64_t)W * H;
    }
    inst[a.nv] = a.nv * a.n;
    toff[a.nv] = to;
    boff[a.nv] = bo;
    for (int g = 0; g < 6; g++) {
        adam[g] = a.ss ? a.ss[g] : 0.f;
        adam[6 + g] = a.bc2 ? a.bc2[g] : 0.f;
    }
}

BatchDesc batch_desc(const StepPtrs &P, int nv) {
    const BlobLayout L(nv);
    BatchDesc d;
    d.n_views = nv;
    d.inst_off = reinterpret_cast<const int *>(P.desc + L.inst);
    d.tile_off = reinterpret_cast<const int *>(P.desc + L.toff);
    d.tiles_x = reinterpret_cast<const int *>(P.desc + L.tx);
    d.tiles_y = reinterpret_cast<const int *>(P.desc + L.ty);
    d.proj = reinterpret_cast<const ProjectArgs *>(P.desc + L.proj);
    d.raster = reinterpret_cast<const RasterArgs *>(P.desc + L.ras);
    return d;
}

// Projection, the instances' depth order and the scan of their tile counts in that
// order (emission offsets; total -> P.total).
void enqueue_count(const StepArgs &a, const StepPtrs &P, cudaStream_t st) {
    const BatchDesc d = batch_desc(P, a.nv);
    const int inst = a.nv * a.n;
    launch_project_batch(d, inst, st);
    DepthScratch ds = P.depth;
    launch_depth_offsets(inst, P.splats, P.n_tiles, ds, P.offsets, P.total, P.scan_part, st);
}

// Everything after the count: capacity check, emission, sort, ranges, forward,
// loss, backward and Adam. tiles_hint / isect_hint: host-known counts (0 = device).
// tm: stage timer (eager steps only; null while capturing).
void enqueue_rest(const StepArgs &a, const StepPtrs &P, int64_t isect_cap, int tile_cap, int tiles_hint,
                  cudaStream_t st, StageTimer *tm) {
    const BlobLayout L(a.nv);
    const BatchDesc d = batch_desc(P, a.nv);
    const int inst = a.nv * a.n;
    int *d_n = P.counters + C_NISECT, *d_over = P.counters + C_OVERFLOW;
    cudaMemsetAsync(P.counters, 0, N_COUNTERS * sizeof(int), st);
    launch_clamp_count(P.total, isect_cap, d_n, d_over, st);
    launch_emit_keys_batch(inst, P.splats, P.aabb, P.n_tiles, P.offsets, nullptr, d, P.k[0], P.v[0], P.emit_gid, st,
                           isect_cap);
    uint32_t *kk[2] = {P.k[0], P.k[1]};
    uint32_t *vv[2] = {P.v[0], P.v[1]};
    const int cap = (int)isect_cap;
    const int cur = radix_sort_pairs32(kk, vv, cap, ceil_log2(std::max(tile_cap, 1)), P.rscratch, st, d_n);
    launch_tile_ranges(kk[cur], cap, tile_cap, P.tile_start, P.tile_end, st, d_n, d.tile_off + a.nv);
    launch_isect_map(vv[cur], cap, P.emit_gid, P.isect_gid, P.inv, st, d_n);
    if (tm) tm->mark(2, st);
    launch_raster_fwd_batch(d, tiles_hint, P.counters + C_RAS, st, a.variant, a.shape);
    if (tm) tm->mark(3, st);
    launch_ssim_loss_batch(reinterpret_cast<const SsimArgs *>(P.desc + L.ssim),
                           reinterpret_cast<const int *>(P.desc + L.boff), a.nv, P.counters + C_SSIM, st);
    if (tm) tm->mark(4, st);
    launch_raster_bwd_batch(reinterpret_cast<const RasterBwdArgs *>(P.desc + L.rbwd), d.tile_off, a.nv,
                            P.counters + C_RBWD, st, a.variant);
    if (tm) tm->mark(5, st);
    BackwardBatchArgs b;
    b.n = a.n;
    b.n_views = a.nv;
    b.proj = d.proj;
    b.inv_max_dim = reinterpret_cast<const float *>(P.desc + L.imd);
    b.means = a.p[0];
    b.scales = a.p[1];
    b.quats = a.p[2];
    b.glob_scale = a.glob_scale;
    b.degrees_to_use = a.dtu;
    b.splats = P.splats;
    b.radii = P.radii;
    b.n_tiles = P.n_tiles;
    b.inv = P.inv;
    b.offsets = P.offsets;
    b.slots = P.slots;
    for (int g = 0; g < 6; g++) b.g[g] = a.grads ? a.grads[g] : nullptr;
    b.do_adam = a.adam_groups >= 5;
    for (int g = 0; g < 6; g++) {
        b.p[g] = a.p[g];
        b.m1[g] = (b.do_adam && g < a.adam_groups) ? a.m1[g] : nullptr;
        b.m2[g] = (b.do_adam && g < a.adam_groups) ? a.m2[g] : nullptr;
    }
    b.adam_scalars = reinterpret_cast<const float *>(P.desc + L.adam);
    b.beta1 = a.beta1;
    b.beta2 = a.beta2;
    b.eps = a.eps;
    b.rest_stride = (int)(num_sh_bases(a.degree) - 1) * 3;
    b.vis_counts = a.vis;
    b.xys_grad_norm = a.gn;
    b.max_2d_size = a.ms;
    b.skip = d_over;
    launch_backward_adam_batch(b, st);
    if (tm) tm->mark(6, st);
}

// Everything a captured graph depends on besides the uploaded descriptors.
std::vector<uint64_t> graph_key(const StepArgs &a, const StepPtrs &P, int64_t isect_cap, int tile_cap) {
    std::vector<uint64_t> k;
    auto u = [&](uint64_t x) { k.push_back(x); };
    auto f = [&](float x) {
        uint32_t b;
        std::memcpy(&b, &x, 4);
        k.push_back(b);
    };
    u(a.n), u(a.nv), u(a.degree), u(a.dtu), u(a.adam_groups), u(isect_cap), u(tile_cap), u(a.variant), u(a.shape);
    f(a.glob_scale), f(a.beta1), f(a.beta2), f(a.eps);
    for (int g = 0; g < 6; g++) {
        u((uintptr_t)a.p[g]);
        u(a.adam_groups >= 5 && g < a.adam_groups ? (uintptr_t)a.m1[g] : 0);
        u(a.adam_groups >= 5 && g < a.adam_groups ? (uintptr_t)a.m2[g] : 0);
        u(a.grads ? (uintptr_t)a.grads[g] : 0);
    }
    u((uintptr_t)a.vis), u((uintptr_t)a.gn), u((uintptr_t)a.ms);
    const void *ptrs[] = {P.desc, P.splats, P.radii, P.n_tiles, P.aabb, P.offsets, P.scan_part, P.total,
                          P.tile_start, P.tile_end, P.k[0], P.k[1], P.v[0], P.v[1], P.emit_gid, P.isect_gid, P.inv,
                          P.slots, P.rscratch, P.img, P.T, P.v_img, P.idx, P.partials, P.losses, P.counters,
                          P.depth.keys[0], P.depth.keys[1], P.depth.vals[0], P.depth.vals[1], P.depth.counts,
                          P.depth.off_sorted};
    for (const void *p : ptrs) u((uintptr_t)p);
    return k;
}

// Pinned staging slot for this step's descriptors (double-buffered: the slot's last
// upload must have finished before it is rewritten).
int stage_slot(TrainBatchState &tb, size_t bytes, unsigned char **out) {
    if (tb.h_stage_bytes < bytes) {
        for (int k = 0; k < 2; k++) {
            if (tb.stage_pending[k]) CUDA_TRY(cudaEventSynchronize(tb.stage_ev[k]));
            tb.stage_pending[k] = false;
            if (tb.h_stage[k]) cudaFreeHost(tb.h_stage[k]);
            tb.h_stage[k] = nullptr;
        }
        tb.h_stage_bytes = 0;
        for (int k = 0; k < 2; k++) CUDA_TRY(cudaMallocHost(&tb.h_stage[k], bytes + bytes / 4));
        tb.h_stage_bytes = bytes + bytes / 4;
    }
    for (int k = 0; k < 2; k++)
        if (!tb.stage_ev[k]) CUDA_TRY(cudaEventCreateWithFlags(&tb.stage_ev[k], cudaEventDisableTiming));
    tb.slot ^= 1;
    if (tb.stage_pending[tb.slot]) {
        CUDA_TRY(cudaEventSynchronize(tb.stage_ev[tb.slot]));
        tb.stage_pending[tb.slot] = false;
    }
    *out = tb.h_stage[tb.slot];
    return MSPLAT_CUDA_OK;
}

int upload_blob(TrainBatchState &tb, const unsigned char *h, unsigned char *d, size_t bytes, cudaStream_t st) {
    CUDA_TRY(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaEventRecord(tb.stage_ev[tb.slot], st));
    tb.stage_pending[tb.slot] = true;
    return MSPLAT_CUDA_OK;
}

int ensure_h_out(TrainBatchState &tb, int nv) {
    const size_t need = 16 + nv * sizeof(float);
    if (tb.h_out_bytes < need) {
        if (tb.h_out) cudaFreeHost(tb.h_out);
        tb.h_out = nullptr;
        tb.h_out_bytes = 0;
        CUDA_TRY(cudaMallocHost(&tb.h_out, need + 256));
        tb.h_out_bytes = need + 256;
    }
    return MSPLAT_CUDA_OK;
}

// One step without a graph: the intersection count is read back after the scan and
// sizes the buffers, so the step cannot overflow.
int step_eager(msplat_cuda_ctx *ctx, const StepArgs &a, const Sizes &sz, float *losses_out) {
    TrainBatchState &tb = ctx->tb;
    cudaStream_t st = ctx->stream;
    StepPtrs P;
    if (int r = ensure_buffers(ctx, sz, std::max<int64_t>(tb.isect_cap, 1), a.nv, P)) return r;
    if (!ctx->h_total) CUDA_TRY(cudaMallocHost(&ctx->h_total, sizeof(int64_t)));
    const BlobLayout L(a.nv);
    unsigned char *h = nullptr;
    if (int r = stage_slot(tb, L.bytes, &h)) return r;
    fill_blob(h, a, P);
    ctx->timer.reset_marks();
    ctx->timer.mark(0, st);
    if (int r = upload_blob(tb, h, P.desc, L.bytes, st)) return r;
    enqueue_count(a, P, st);
    CUDA_TRY(cudaMemcpyAsync(ctx->h_total, P.total, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t total = *ctx->h_total;
    if (total > (int64_t)INT32_MAX / 2)
        return fail(MSPLAT_CUDA_EOVERFLOW, "too many tile intersections in the batch (%lld)", (long long)total);
    ctx->n_isect = total;
    if (total > tb.isect_cap) {
        // grow (with headroom for later steps) and describe the new buffers
        if (int r = ensure_buffers(ctx, sz, total + total / 4 + 1024, a.nv, P)) return r;
        if (int r = stage_slot(tb, L.bytes, &h)) return r;
        fill_blob(h, a, P);
        if (int r = upload_blob(tb, h, P.desc, L.bytes, st)) return r;
    }
    ctx->timer.mark(1, st);
    enqueue_rest(a, P, tb.isect_cap, tb.tile_cap, (int)sz.tiles, st, &ctx->timer);
    CUDA_TRY(cudaGetLastError());
    if (losses_out) {
        CUDA_TRY(cudaMemcpyAsync(losses_out, P.losses, a.nv * sizeof(float), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
    }
    return MSPLAT_CUDA_OK;
}

// One step replayed from the captured graph (captured first when the shape changed).
// Returns 1 (no error) when the step overflowed and must be repeated eagerly.
int step_graph(msplat_cuda_ctx *ctx, const StepArgs &a, const Sizes &sz, float *losses_out, bool *overflowed) {
    TrainBatchState &tb = ctx->tb;
    *overflowed = false;
    if (!tb.gstream) CUDA_TRY(cudaStreamCreateWithFlags(&tb.gstream, cudaStreamNonBlocking));
    if (!tb.ev_in) CUDA_TRY(cudaEventCreateWithFlags(&tb.ev_in, cudaEventDisableTiming));
    cudaStream_t gs = tb.gstream;
    StepPtrs P;
    if (int r = ensure_buffers(ctx, sz, tb.isect_cap, a.nv, P)) return r;
    if (int r = ensure_h_out(tb, a.nv)) return r;
    const BlobLayout L(a.nv);
    // order after the caller's stream (targets written there)
    CUDA_TRY(cudaEventRecord(tb.ev_in, ctx->stream));
    CUDA_TRY(cudaStreamWaitEvent(gs, tb.ev_in, 0));
    unsigned char *h = nullptr;
    if (int r = stage_slot(tb, L.bytes, &h)) return r;
    fill_blob(h, a, P);
    if (int r = upload_blob(tb, h, P.desc, L.bytes, gs)) return r;
    std::vector<uint64_t> key = graph_key(a, P, tb.isect_cap, tb.tile_cap);
    if (!tb.exec || key != tb.key) {
        if (tb.exec) cudaGraphExecDestroy(tb.exec);
        tb.exec = nullptr;
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(gs, cudaStreamCaptureModeThreadLocal));
        enqueue_count(a, P, gs);
        enqueue_rest(a, P, tb.isect_cap, tb.tile_cap, 0, gs, nullptr);
        cudaError_t e = cudaStreamEndCapture(gs, &g);
        if (e != cudaSuccess) return fail(MSPLAT_CUDA_ECUDA, "graph capture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&tb.exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            tb.exec = nullptr;
            return fail(MSPLAT_CUDA_ECUDA, "graph instantiate: %s", cudaGetErrorString(e));
        }
        tb.key = key;
        tb.captures++;
    }
    CUDA_TRY(cudaGraphLaunch(tb.exec, gs));
    tb.replays++;
    int *ho = reinterpret_cast<int *>(tb.h_out);
    float *hl = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(tb.h_out) + 16);
    CUDA_TRY(cudaMemcpyAsync(ho, P.counters, 2 * sizeof(int), cudaMemcpyDeviceToHost, gs));
    CUDA_TRY(cudaMemcpyAsync(hl, P.losses, a.nv * sizeof(float), cudaMemcpyDeviceToHost, gs));
    CUDA_TRY(cudaStreamSynchronize(gs));
    if (ho[C_OVERFLOW]) {
        *overflowed = true;
        tb.overflows++;
        return MSPLAT_CUDA_OK;
    }
    ctx->n_isect = ho[C_NISECT];
    if (losses_out) std::memcpy(losses_out, hl, a.nv * sizeof(float));
    return MSPLAT_CUDA_OK;
}

}  // namespace

extern "C" int msplat_cuda_train_batch(msplat_cuda_ctx *ctx, int num_points, float *means3d, float *scales,
                                       float glob_scale, float *quats, float *features_dc, float *features_rest,
                                       float *opacities, unsigned degree, unsigned degrees_to_use, float clip_thresh,
                                       const float *background, int32_t n_views, const msplat_cuda_train_view *views,
                                       float ssim_weight, int num_adam_groups, float *const *adam_exp_avg,
                                       float *const *adam_exp_avg_sq, const float *adam_step_sizes,
                                       const float *adam_bc2_sqrts, float adam_beta1, float adam_beta2,
                                       float adam_eps, float *vis_counts, float *xys_grad_norm, float *max_2d_size,
                                       float *const *grads_out, float *losses_out) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (ctx->has_prior)
        return fail(MSPLAT_CUDA_EUNSUPPORTED, "a prior (msplat_cuda_set_prior) applies to msplat_cuda_train_step only; "
                                              "clear it before msplat_cuda_train_batch");
    StepArgs a;
    a.n = num_points;
    a.nv = n_views;
    float *p[6] = {means3d, scales, quats, features_dc, features_rest, opacities};
    for (int g = 0; g < 6; g++) a.p[g] = p[g];
    a.glob_scale = glob_scale;
    a.clip = clip_thresh;
    a.degree = degree;
    a.dtu = degrees_to_use;
    a.bg = background;
    a.views = views;
    a.ssim_weight = ssim_weight;
    a.adam_groups = num_adam_groups;
    a.m1 = adam_exp_avg;
    a.m2 = adam_exp_avg_sq;
    a.ss = adam_step_sizes;
    a.bc2 = adam_bc2_sqrts;
    a.beta1 = adam_beta1;
    a.beta2 = adam_beta2;
    a.eps = adam_eps;
    a.vis = vis_counts;
    a.gn = xys_grad_norm;
    a.ms = max_2d_size;
    a.grads = grads_out;
    a.variant = ctx->raster_variant;
    a.shape = ctx->raster_shape;
    if (int r = check_step(a)) return r;
    const Sizes sz = sizes_of(a);
    if (sz.inst >= (int64_t)INT32_MAX || sz.tiles >= (int64_t)INT32_MAX || sz.pix >= (int64_t)INT32_MAX)
        return fail(MSPLAT_CUDA_EOVERFLOW, "batch too large: %lld instances, %lld tiles, %lld pixels",
                    (long long)sz.inst, (long long)sz.tiles, (long long)sz.pix);
    ctx->n = (int)sz.inst;
    ctx->W = ctx->H = ctx->tiles_x = ctx->tiles_y = 0;  // no single-view frame to inspect
    TrainBatchState &tb = ctx->tb;
    const bool use_graph = tb.graph && tb.isect_cap > 0 && sz.tiles <= tb.tile_cap;
    if (use_graph) {
        bool over = false;
        if (int r = step_graph(ctx, a, sz, losses_out, &over)) return r;
        if (!over) return MSPLAT_CUDA_OK;
        // nothing changed; repeat the step eagerly, which grows the buffers
    }
    if (int r = step_eager(ctx, a, sz, losses_out)) return r;
    ctx->timer.collect();
    return MSPLAT_CUDA_OK;
}

extern "C" int msplat_cuda_train_batch_stats(msplat_cuda_ctx *ctx, int64_t *out4) {
    if (!ctx || !out4) return fail(MSPLAT_CUDA_EINVAL, "null argument");
    out4[0] = ctx->tb.replays;
    out4[1] = ctx->tb.captures;
    out4[2] = ctx->tb.overflows;
    out4[3] = ctx->tb.isect_cap;
    return MSPLAT_CUDA_OK;
}
