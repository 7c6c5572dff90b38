// C-ABI entry points (include/msplat_cuda.h) and the per-context frame cache.
//
// The frame cache plays the role of the reference's FusedTensorCache / Frame
// (core/metal/msplat_metal.mm:441-584, core/cpu/msplat_cpu.cpp:406-436): device
// buffers that grow on demand and are reused across frames. Growth uses cudaMalloc
// (which synchronises), so it happens only when a frame needs more room than any
// before it; buffers grow with 25% headroom.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/msplat_cuda.h"
#include "context.h"

using namespace msplat;

namespace {
thread_local std::string g_last_error;
}  // namespace

const char *msplat::last_error_text() { return g_last_error.c_str(); }

int msplat::fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

// Lets other translation units report through msplat_cuda_last_error().
int msplat::report_error(int code, const char *msg) { return fail(code, "%s", msg); }

int msplat::check_camera(int num_points, unsigned H, unsigned W, int tx, int ty, unsigned degree, unsigned dtu,
                 const float *viewmat, const float *projmat, const float *cam_pos, const float *bg) {
    if (num_points < 0) return fail(MSPLAT_CUDA_EINVAL, "num_points must be >= 0 (got %d)", num_points);
    if (W == 0 || H == 0) return fail(MSPLAT_CUDA_EINVAL, "image size must be positive (%ux%u)", W, H);
    if (tx != (int)((W + TILE - 1) / TILE) || ty != (int)((H + TILE - 1) / TILE))
        return fail(MSPLAT_CUDA_EINVAL, "tile bounds (%d, %d) do not match a %ux%u image with 16x16 tiles", tx, ty, W, H);
    if ((int64_t)tx * ty >= (1ll << 31)) return fail(MSPLAT_CUDA_EINVAL, "too many tiles");
    if (degree > 4 || dtu > degree) return fail(MSPLAT_CUDA_EINVAL, "SH degree %u / degrees_to_use %u", degree, dtu);
    if (!viewmat || !projmat || !cam_pos || !bg) return fail(MSPLAT_CUDA_EINVAL, "null camera or background pointer");
    return MSPLAT_CUDA_OK;
}

CamParams msplat::make_cam(const float *viewmat, const float *projmat, float fx, float fy, float cx, float cy,
                   unsigned H, unsigned W, int tx, int ty, float clip, unsigned degree, unsigned dtu,
                   const float *cam_pos) {
    CamParams c;
    std::memcpy(c.viewmat, viewmat, sizeof c.viewmat);
    std::memcpy(c.projmat, projmat, sizeof c.projmat);
    c.fx = fx;
    c.fy = fy;
    c.cx = cx;
    c.cy = cy;
    for (int i = 0; i < 3; i++) c.cam_pos[i] = cam_pos[i];
    c.width = W;
    c.height = H;
    c.tiles_x = tx;
    c.tiles_y = ty;
    c.clip = clip;
    c.degree = degree;
    c.degrees_to_use = dtu;
    return c;
}

namespace {

// The sky sampling parameters of a prior for one camera (make_sky_params,
// core/cpu/msplat_cpu.cpp:338-350).
SkyArgs sky_args(const msplat_cuda_prior &p, const CamParams &cam) {
    SkyArgs s;
    s.tex = p.sky_tex;
    s.tex_w = p.sky_w;
    s.tex_h = p.sky_h;
    std::memcpy(s.frame, p.sky_frame, sizeof s.frame);
    s.fx = cam.fx;
    s.fy = cam.fy;
    s.cx = cam.cx;
    s.cy = cam.cy;
    std::memcpy(s.viewmat, cam.viewmat, sizeof s.viewmat);
    return s;
}

// Projection, binning and forward rasterization: the shared forward of render and
// train (core/cpu/msplat_cpu.cpp:629-657). One host synchronisation reads the
// intersection count, which sizes the sort. With a prior whose aux flag is set, the
// aux rasterizer also writes the expected-depth numerator and the per-pixel
// background, sampled from the learned sky when one is set.
// The depth-chunked planes of the current frame (ctx->n_isect intersections over T
// tiles): at most n_isect / chunk_len + T items (each tile adds at most one partial
// piece). backward: also the prefix / suffix planes. Fills ck from the buffers.
int chunk_buffers(msplat_cuda_ctx *ctx, int T, bool backward, ChunkArgs &ck) {
    if (!backward) ctx->chunk_cap = ctx->n_isect / ctx->chunk_len + T + 1;
    const size_t cap = (size_t)ctx->chunk_cap;
    ENSURE(ctx->ch[CH_COUNTS], T, int32_t, counts);
    ENSURE(ctx->ch[CH_FIRST], (size_t)T + 1, int32_t, first);
    ENSURE(ctx->ch[CH_PART], scan_blocks(T) + 1, int32_t, part);
    ENSURE(ctx->ch[CH_T], cap * TILE_PIX, float, cT);
    ENSURE(ctx->ch[CH_C], cap * 3 * TILE_PIX, float, cC);
    ENSURE(ctx->ch[CH_LAST], cap * TILE_PIX, int32_t, clast);
    (void)counts;
    (void)part;
    ck.chunk_len = ctx->chunk_len;
    ck.first = first;
    ck.cT = cT;
    ck.cC = cC;
    ck.clast = clast;
    ck.pre = nullptr;
    ck.aft = nullptr;
    if (backward) {
        ENSURE(ctx->ch[CH_PRE], cap * TILE_PIX, float, pre);
        ENSURE(ctx->ch[CH_AFT], cap * 3 * TILE_PIX, float, aft);
        ck.pre = pre;
        ck.aft = aft;
    }
    return MSPLAT_CUDA_OK;
}

int forward(msplat_cuda_ctx *ctx, int n, const float *means, const float *scales, float glob_scale,
            const float *quats, const CamParams &cam, const float *dc, const float *rest, const float *opac,
            const float *bg) {
    cudaStream_t st = ctx->stream;
    const int T = cam.tiles_x * cam.tiles_y;
    ctx->n = n;
    ctx->W = (int)cam.width;
    ctx->H = (int)cam.height;
    ctx->tiles_x = cam.tiles_x;
    ctx->tiles_y = cam.tiles_y;
    if (n > 0 && (!means || !scales || !quats || !dc || !opac || (cam.degree > 0 && !rest)))
        return fail(MSPLAT_CUDA_EINVAL, "null Gaussian parameter pointer");
    ENSURE(ctx->splats, n, Splat, splats);
    ENSURE(ctx->radii, n, int32_t, radii);
    ENSURE(ctx->aabb, 2 * (size_t)n, float, aabb);
    ENSURE(ctx->n_tiles, n, int32_t, n_tiles);
    ENSURE(ctx->offsets, n, int64_t, offsets);
    ENSURE(ctx->scan_part, scan_blocks(std::max(n, 1)) + 1, int64_t, scan_part);
    ENSURE(ctx->total, 1, int64_t, d_total);
    ENSURE(ctx->tile_start, T, int32_t, tile_start);
    ENSURE(ctx->tile_end, T, int32_t, tile_end);
    const size_t npix = (size_t)cam.width * cam.height;
    ENSURE(ctx->out_img, npix * 3, float, out_img);
    ENSURE(ctx->final_T, npix, float, final_T);
    ENSURE(ctx->final_idx, npix, int32_t, final_idx);
    if (!ctx->h_total) CUDA_TRY(cudaMallocHost(&ctx->h_total, sizeof(int64_t)));
    const msplat_cuda_prior *pr = ctx->has_prior ? &ctx->prior : nullptr;
    const bool aux = pr && pr->aux;
    const bool sky = aux && pr->sky && pr->sky_tex;
    ctx->aux_frame = aux;
    float *out_depth = nullptr, *bg_img = nullptr;
    if (aux) {
        ENSURE(ctx->pri[PB_DEPTH], npix, float, od);
        ENSURE(ctx->pri[PB_BG], npix * 3, float, bi);
        out_depth = od;
        bg_img = bi;
    }

    ProjectArgs pa;
    pa.n = n;
    pa.means = means;
    pa.scales = scales;
    pa.quats = quats;
    pa.features_dc = dc;
    pa.features_rest = rest;
    pa.opacities = opac;
    pa.rest_stride = (int)(num_sh_bases(cam.degree) - 1) * 3;
    pa.glob_scale = glob_scale;
    pa.cam = cam;
    pa.splats = splats;
    pa.radii = radii;
    pa.aabb = aabb;
    pa.n_tiles = n_tiles;
    DepthScratch ds;
    if (int r = ensure_depth_scratch(ctx, n, ds)) return r;
    ctx->timer.reset_marks();
    ctx->timer.mark(0, st);
    launch_project(pa, st);
    launch_depth_offsets(n, splats, n_tiles, ds, offsets, d_total, scan_part, st);
    CUDA_TRY(cudaMemcpyAsync(ctx->h_total, d_total, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    if (!ctx->total_ev) CUDA_TRY(cudaEventCreateWithFlags(&ctx->total_ev, cudaEventDisableTiming));
    CUDA_TRY(cudaEventRecord(ctx->total_ev, st));
    // The key emission needs the count only for its buffers' size: it is queued before
    // the host waits for the count, into the buffers as they are (entries past their
    // capacity dropped), so the device runs it while the host reads the count and
    // queues the rest; when the buffers were too small it runs again below.
    ctx->timer.mark(1, st);
    const int64_t cap0 = (int64_t)std::min({ctx->keys[0].bytes, ctx->vals[0].bytes, ctx->emit_gid.bytes}) / 4;
    if (cap0 > 0 && n > 0)
        launch_emit_keys(n, splats, aabb, n_tiles, offsets, cam.tiles_x, cam.tiles_y,
                         reinterpret_cast<uint32_t *>(ctx->keys[0].ptr), reinterpret_cast<uint32_t *>(ctx->vals[0].ptr),
                         reinterpret_cast<int32_t *>(ctx->emit_gid.ptr), st, cap0);
    CUDA_TRY(cudaEventSynchronize(ctx->total_ev));
    const int64_t n_isect = *ctx->h_total;
    if (n_isect > (int64_t)INT32_MAX)
        return fail(MSPLAT_CUDA_EOVERFLOW, "more than 2^31 tile intersections (%lld); lower the resolution",
                    (long long)n_isect);
    ctx->n_isect = n_isect;
    const bool emitted = cap0 > 0 && n_isect <= cap0;
    if (!emitted) CUDA_TRY(cudaStreamSynchronize(st));  // the early emission is done before buffers move
    ENSURE(ctx->keys[0], n_isect, uint32_t, k0);
    ENSURE(ctx->keys[1], n_isect, uint32_t, k1);
    ENSURE(ctx->vals[0], n_isect, uint32_t, v0);
    ENSURE(ctx->vals[1], n_isect, uint32_t, v1);
    ENSURE(ctx->emit_gid, n_isect, int32_t, emit_gid);
    ENSURE(ctx->isect_gid, n_isect, int32_t, isect_gid);
    ENSURE(ctx->inv, n_isect, int32_t, inv);
    ENSURE(ctx->radix_scratch, radix_scratch_bytes((int)n_isect), unsigned char, rscratch);

    if (!emitted)
        launch_emit_keys(n, splats, aabb, n_tiles, offsets, cam.tiles_x, cam.tiles_y, k0, v0, emit_gid, st);
    uint32_t *kk[2] = {k0, k1};
    uint32_t *vv[2] = {v0, v1};
    const int cur = radix_sort_pairs32(kk, vv, (int)n_isect, ceil_log2(std::max(T, 1)), rscratch, st);
    ctx->sorted = cur;
    ctx->gid_in_vals = false;
    launch_tile_ranges(kk[cur], (int)n_isect, T, tile_start, tile_end, st);
    launch_isect_map(vv[cur], (int)n_isect, emit_gid, isect_gid, inv, st);

    RasterArgs ra{};
    ra.W = (int)cam.width;
    ra.H = (int)cam.height;
    ra.tiles_x = cam.tiles_x;
    ra.tiles_y = cam.tiles_y;
    ra.tile_start = tile_start;
    ra.tile_end = tile_end;
    ra.isect_gid = isect_gid;
    ra.splats = splats;
    for (int c = 0; c < 3; c++) ra.bg[c] = bg[c];
    ra.out_img = out_img;
    ra.final_T = final_T;
    ra.final_idx = final_idx;
    ra.tstore = nullptr;
    ra.tcount = nullptr;
    ra.tcap = 0;
    if (ctx->tstore_cap > 0) {
        ENSURE(ctx->tstore, (size_t)ctx->tstore_cap * npix, float, ts);
        ENSURE(ctx->tcount, npix, int32_t, tc);
        ra.tstore = ts;
        ra.tcount = tc;
        ra.tcap = ctx->tstore_cap;
    }
    ra.out_depth = out_depth;
    ra.bg_img = bg_img;
    ra.sky_bg = sky ? 1 : 0;
    // depth-chunked compositing for frames of few tiles (never with a prior: the aux
    // rasterizer is one-pass only, as in core/metal/msplat_metal.mm:1103-1106)
    const bool chunked =
        !aux && T > 0 && (ctx->chunk_mode == 2 || (ctx->chunk_mode == 1 && T < CHUNK_AUTO_TILES));
    ctx->chunk_frame = chunked;
    ChunkArgs ck{};
    if (chunked) {
        if (int r = chunk_buffers(ctx, T, false, ck)) return r;
        ra.tstore = nullptr;
        ra.tcount = nullptr;
        ra.tcap = 0;
    }
    ctx->timer.mark(2, st);
    if (aux) {
        if (sky) launch_sky_background(sky_args(*pr, cam), (int)cam.width, (int)cam.height, bg_img, st);
        launch_raster_fwd_aux(ra, st, ctx->raster_shape);
    } else if (chunked) {
        launch_chunk_items(tile_start, tile_end, T, ck.chunk_len, reinterpret_cast<int32_t *>(ctx->ch[CH_COUNTS].ptr),
                           ck.first, reinterpret_cast<int32_t *>(ctx->ch[CH_PART].ptr), st);
        launch_raster_fwd_chunked(ra, ck, ctx->chunk_cap, st, ctx->raster_variant);
    } else {
        launch_raster_fwd(ra, st, ctx->raster_variant, ctx->raster_shape);
    }
    ctx->timer.mark(3, st);
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

// Batched forward: the stages of forward() over every (view, Gaussian) instance and
// every (view, tile) of a batch at once. The view descriptors go to the device in
// two uploads from pinned staging: projection/emission fields first, the raster
// fields once the intersection count has sized the per-intersection buffers.
int forward_batch(msplat_cuda_ctx *ctx, int nv, const msplat_cuda_view *views) {
    cudaStream_t st = ctx->stream;
    if (nv <= 0) return fail(MSPLAT_CUDA_EINVAL, "n_views must be positive (got %d)", nv);
    if (!views) return fail(MSPLAT_CUDA_EINVAL, "null view array");
    int64_t ni = 0, nt = 0;
    for (int v = 0; v < nv; v++) {
        const msplat_cuda_view &w = views[v];
        const int tx = (int)((w.img_width + TILE - 1) / TILE), ty = (int)((w.img_height + TILE - 1) / TILE);
        if (int r = check_camera(w.num_points, w.img_height, w.img_width, tx, ty, w.degree, w.degrees_to_use,
                                 w.viewmat, w.projmat, w.cam_pos, w.background))
            return fail(r, "view %d: %s", v, last_error_text());
        if (w.num_points > 0 && (!w.means3d || !w.scales || !w.quats || !w.features_dc || !w.opacities ||
                                 (w.degree > 0 && !w.features_rest)))
            return fail(MSPLAT_CUDA_EINVAL, "view %d: null Gaussian parameter pointer", v);
        if (!w.out_img) return fail(MSPLAT_CUDA_EINVAL, "view %d: null output image", v);
        ni += w.num_points;
        nt += (int64_t)tx * ty;
    }
    if (ni >= (int64_t)INT32_MAX || nt >= (int64_t)INT32_MAX)
        return fail(MSPLAT_CUDA_EOVERFLOW, "batch too large: %lld instances, %lld tiles", (long long)ni,
                    (long long)nt);
    const int n = (int)ni, T = (int)nt;

    // staging layout: ProjectArgs[nv] | RasterArgs[nv] | inst_off, tile_off [nv+1] | tiles_x, tiles_y [nv]
    const size_t o_proj = 0;
    const size_t o_ras = align_up(o_proj + nv * sizeof(ProjectArgs), 256);
    const size_t o_inst = align_up(o_ras + nv * sizeof(RasterArgs), 256);
    const size_t o_toff = o_inst + (nv + 1) * sizeof(int);
    const size_t o_tx = o_toff + (nv + 1) * sizeof(int);
    const size_t o_ty = o_tx + nv * sizeof(int);
    const size_t bytes = o_ty + nv * sizeof(int);
    if (ctx->bdesc_pending) {  // the previous batch's raster upload still reads the staging
        CUDA_TRY(cudaEventSynchronize(ctx->bdesc_ev));
        ctx->bdesc_pending = false;
    }
    if (ctx->h_bdesc_bytes < bytes) {
        if (ctx->h_bdesc) cudaFreeHost(ctx->h_bdesc);
        ctx->h_bdesc = nullptr;
        ctx->h_bdesc_bytes = 0;
        CUDA_TRY(cudaMallocHost(&ctx->h_bdesc, bytes + bytes / 4));
        ctx->h_bdesc_bytes = bytes + bytes / 4;
    }
    if (!ctx->bdesc_ev) CUDA_TRY(cudaEventCreateWithFlags(&ctx->bdesc_ev, cudaEventDisableTiming));
    ENSURE(ctx->bdesc, bytes, unsigned char, d_desc);
    ENSURE(ctx->bcounter, 1, int, d_counter);
    ENSURE(ctx->splats, n, Splat, splats);
    ENSURE(ctx->radii, n, int32_t, radii);
    ENSURE(ctx->aabb, 2 * (size_t)n, float, aabb);
    ENSURE(ctx->n_tiles, n, int32_t, n_tiles);
    ENSURE(ctx->offsets, n, int64_t, offsets);
    ENSURE(ctx->scan_part, scan_blocks(std::max(n, 1)) + 1, int64_t, scan_part);
    ENSURE(ctx->total, 1, int64_t, d_total);
    ENSURE(ctx->tile_start, T, int32_t, tile_start);
    ENSURE(ctx->tile_end, T, int32_t, tile_end);
    if (!ctx->h_total) CUDA_TRY(cudaMallocHost(&ctx->h_total, sizeof(int64_t)));
    DepthScratch ds;
    if (int r = ensure_depth_scratch(ctx, n, ds)) return r;

    unsigned char *h = ctx->h_bdesc;
    ProjectArgs *hp = reinterpret_cast<ProjectArgs *>(h + o_proj);
    RasterArgs *hr = reinterpret_cast<RasterArgs *>(h + o_ras);
    int *h_inst = reinterpret_cast<int *>(h + o_inst), *h_toff = reinterpret_cast<int *>(h + o_toff);
    int *h_tx = reinterpret_cast<int *>(h + o_tx), *h_ty = reinterpret_cast<int *>(h + o_ty);
    int io = 0, to = 0;
    for (int v = 0; v < nv; v++) {
        const msplat_cuda_view &w = views[v];
        const int tx = (int)((w.img_width + TILE - 1) / TILE), ty = (int)((w.img_height + TILE - 1) / TILE);
        ProjectArgs &pa = hp[v];
        pa.n = w.num_points;
        pa.means = w.means3d;
        pa.scales = w.scales;
        pa.quats = w.quats;
        pa.features_dc = w.features_dc;
        pa.features_rest = w.features_rest;
        pa.opacities = w.opacities;
        pa.rest_stride = (int)(num_sh_bases(w.degree) - 1) * 3;
        pa.glob_scale = w.glob_scale;
        pa.cam = make_cam(w.viewmat, w.projmat, w.fx, w.fy, w.cx, w.cy, w.img_height, w.img_width, tx, ty,
                          w.clip_thresh, w.degree, w.degrees_to_use, w.cam_pos);
        pa.splats = splats;
        pa.radii = radii;
        pa.aabb = aabb;
        pa.n_tiles = n_tiles;
        h_inst[v] = io;
        h_toff[v] = to;
        h_tx[v] = tx;
        h_ty[v] = ty;
        io += w.num_points;
        to += tx * ty;
    }
    h_inst[nv] = io;
    h_toff[nv] = to;
    BatchDesc d;
    d.n_views = nv;
    d.inst_off = reinterpret_cast<const int *>(d_desc + o_inst);
    d.tile_off = reinterpret_cast<const int *>(d_desc + o_toff);
    d.tiles_x = reinterpret_cast<const int *>(d_desc + o_tx);
    d.tiles_y = reinterpret_cast<const int *>(d_desc + o_ty);
    d.proj = reinterpret_cast<const ProjectArgs *>(d_desc + o_proj);
    d.raster = reinterpret_cast<const RasterArgs *>(d_desc + o_ras);

    ctx->n = n;
    ctx->W = ctx->H = ctx->tiles_x = ctx->tiles_y = 0;  // no single-view frame to inspect
    ctx->timer.reset_marks();
    ctx->timer.mark(0, st);
    CUDA_TRY(cudaMemcpyAsync(d_desc, h, o_ras, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(d_desc + o_inst, h + o_inst, bytes - o_inst, cudaMemcpyHostToDevice, st));
    launch_project_batch(d, n, st);
    launch_depth_offsets(n, splats, n_tiles, ds, offsets, d_total, scan_part, st);
    CUDA_TRY(cudaMemcpyAsync(ctx->h_total, d_total, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t n_isect = *ctx->h_total;
    if (n_isect > (int64_t)INT32_MAX)
        return fail(MSPLAT_CUDA_EOVERFLOW, "more than 2^31 tile intersections in the batch (%lld)",
                    (long long)n_isect);
    ctx->n_isect = n_isect;
    ENSURE(ctx->keys[0], n_isect, uint32_t, k0);
    ENSURE(ctx->keys[1], n_isect, uint32_t, k1);
    ENSURE(ctx->vals[0], n_isect, uint32_t, v0);
    ENSURE(ctx->vals[1], n_isect, uint32_t, v1);
    ENSURE(ctx->radix_scratch, radix_scratch_bytes((int)n_isect), unsigned char, rscratch);

    ctx->timer.mark(1, st);
    // render only: the sort carries Gaussian ids, so its sorted values are the
    // per-intersection ids (no emission-index map, no inverse map)
    launch_emit_keys_batch(n, splats, aabb, n_tiles, offsets, &ds, d, k0, v0, nullptr, st);
    uint32_t *kk[2] = {k0, k1};
    uint32_t *vv[2] = {v0, v1};
    const int cur = radix_sort_pairs32(kk, vv, (int)n_isect, ceil_log2(std::max(T, 1)), rscratch, st);
    ctx->sorted = cur;
    ctx->gid_in_vals = true;
    const int32_t *isect_gid = reinterpret_cast<const int32_t *>(vv[cur]);
    launch_tile_ranges(kk[cur], (int)n_isect, T, tile_start, tile_end, st);

    for (int v = 0; v < nv; v++) {
        const msplat_cuda_view &w = views[v];
        RasterArgs &ra = hr[v];
        ra.W = (int)w.img_width;
        ra.H = (int)w.img_height;
        ra.tiles_x = h_tx[v];
        ra.tiles_y = h_ty[v];
        ra.tile_start = tile_start;
        ra.tile_end = tile_end;
        ra.isect_gid = isect_gid;
        ra.splats = splats;
        for (int c = 0; c < 3; c++) ra.bg[c] = w.background[c];
        ra.out_img = w.out_img;
        ra.final_T = nullptr;
        ra.final_idx = nullptr;
        ra.tstore = nullptr;
        ra.tcount = nullptr;
        ra.tcap = 0;
    }
    CUDA_TRY(cudaMemcpyAsync(d_desc + o_ras, h + o_ras, nv * sizeof(RasterArgs), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaEventRecord(ctx->bdesc_ev, st));
    ctx->bdesc_pending = true;
    ctx->timer.mark(2, st);
    launch_raster_fwd_batch(d, T, d_counter, st, ctx->raster_variant, ctx->raster_shape);
    ctx->timer.mark(3, st);
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

msplat_cuda_ctx *g_default = nullptr;
std::mutex g_default_mu;

}  // namespace

extern "C" {

const char *msplat_cuda_last_error(void) { return g_last_error.c_str(); }
int msplat_cuda_version(void) { return 100; }

int msplat_cuda_ctx_create(msplat_cuda_ctx **out) {
    if (!out) return fail(MSPLAT_CUDA_EINVAL, "null output pointer");
    *out = new msplat_cuda_ctx();
    return MSPLAT_CUDA_OK;
}

void msplat_cuda_ctx_destroy(msplat_cuda_ctx *ctx) {
    if (!ctx) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    else cudaDeviceSynchronize();
    delete ctx;
}

msplat_cuda_ctx *msplat_cuda_default_ctx(void) {
    std::lock_guard<std::mutex> lk(g_default_mu);
    if (!g_default) g_default = new msplat_cuda_ctx();
    return g_default;
}

int msplat_cuda_ctx_set_stream(msplat_cuda_ctx *ctx, void *stream) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    ctx->stream = reinterpret_cast<cudaStream_t>(stream);
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_ctx_set_option(msplat_cuda_ctx *ctx, const char *name, int64_t value) {
    if (!ctx || !name) return fail(MSPLAT_CUDA_EINVAL, "null context or option name");
    if (!std::strcmp(name, "keep_grads")) {
        ctx->keep_grads = value != 0;
        return MSPLAT_CUDA_OK;
    }
    if (!std::strcmp(name, "store_transmittance")) {
        if (value < 0 || value > 4096) return fail(MSPLAT_CUDA_EINVAL, "store_transmittance capacity must be 0..4096");
        ctx->tstore_cap = (int)value;
        return MSPLAT_CUDA_OK;
    }
    if (!std::strcmp(name, "stage_timing")) {
        if (value) ctx->timer.init();
        ctx->timer.on = value != 0;
        ctx->timer.reset_marks();
        return MSPLAT_CUDA_OK;
    }
    if (!std::strcmp(name, "raster_variant")) {
        if (value < 0 || value >= N_RASTER_VARIANTS)
            return fail(MSPLAT_CUDA_EINVAL, "raster_variant must be 0..%d", N_RASTER_VARIANTS - 1);
        ctx->raster_variant = (int)value;
        return MSPLAT_CUDA_OK;
    }
    if (!std::strcmp(name, "raster_shape")) {
        if (value < 0 || value >= N_RASTER_SHAPES)
            return fail(MSPLAT_CUDA_EINVAL, "raster_shape must be 0..%d", N_RASTER_SHAPES - 1);
        ctx->raster_shape = (int)value;
        return MSPLAT_CUDA_OK;
    }
    if (!std::strcmp(name, "graph")) {
        ctx->tb.graph = value != 0;
        return MSPLAT_CUDA_OK;
    }
    if (!std::strcmp(name, "chunked_raster")) {
        if (value < 0 || value > 2) return fail(MSPLAT_CUDA_EINVAL, "chunked_raster must be 0 (off), 1 (auto) or 2 (on)");
        ctx->chunk_mode = (int)value;
        return MSPLAT_CUDA_OK;
    }
    if (!std::strcmp(name, "chunk_len")) {
        // at least 16: the per-piece planes (36 bytes per pixel per piece) stay within
        // about 2.25 bytes per intersection per pixel of the tile
        if (value < 16 || value > (1 << 20)) return fail(MSPLAT_CUDA_EINVAL, "chunk_len must be 16..2^20");
        ctx->chunk_len = (int)value;
        return MSPLAT_CUDA_OK;
    }
    return fail(MSPLAT_CUDA_EINVAL, "unknown option '%s'", name);
}

int msplat_cuda_cleanup(msplat_cuda_ctx *ctx) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    CUDA_TRY(ctx->stream ? cudaStreamSynchronize(ctx->stream) : cudaDeviceSynchronize());
    ctx->release();
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_commit(msplat_cuda_ctx *ctx) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_sync(msplat_cuda_ctx *ctx) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_alloc(size_t bytes, int zero, void **out) {
    if (!out) return fail(MSPLAT_CUDA_EINVAL, "null output pointer");
    if (bytes == 0) bytes = 4;
    CUDA_TRY(cudaMallocManaged(out, bytes));
    if (zero) std::memset(*out, 0, bytes);
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_device_alloc(size_t bytes, void **out) {
    if (!out) return fail(MSPLAT_CUDA_EINVAL, "null output pointer");
    if (bytes == 0) bytes = 4;
    CUDA_TRY(cudaMalloc(out, bytes));
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_free(void *ptr) {
    if (ptr) CUDA_TRY(cudaFree(ptr));
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_copy_buffer(msplat_cuda_ctx *ctx, void *dst, const void *src, size_t bytes) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (!bytes) return MSPLAT_CUDA_OK;
    if (!dst || !src) return fail(MSPLAT_CUDA_EINVAL, "null buffer");
    CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_render(msplat_cuda_ctx *ctx, int num_points, const float *means3d, const float *scales,
                       float glob_scale, const float *quats, const float *viewmat, const float *projmat, float fx,
                       float fy, float cx, float cy, unsigned img_height, unsigned img_width, int tiles_x,
                       int tiles_y, float clip_thresh, unsigned degree, unsigned degrees_to_use,
                       const float *cam_pos, const float *features_dc, const float *features_rest,
                       const float *opacities, const float *background, const float **out_img) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (int r = check_camera(num_points, img_height, img_width, tiles_x, tiles_y, degree, degrees_to_use, viewmat,
                             projmat, cam_pos, background))
        return r;
    CamParams cam = make_cam(viewmat, projmat, fx, fy, cx, cy, img_height, img_width, tiles_x, tiles_y, clip_thresh,
                             degree, degrees_to_use, cam_pos);
    if (int r = forward(ctx, num_points, means3d, scales, glob_scale, quats, cam, features_dc, features_rest,
                        opacities, background))
        return r;
    ctx->timer.collect();
    if (out_img) *out_img = reinterpret_cast<const float *>(ctx->out_img.ptr);
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_render_batch(msplat_cuda_ctx *ctx, int32_t n_views, const msplat_cuda_view *views) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (ctx->has_prior)
        return fail(MSPLAT_CUDA_EUNSUPPORTED, "a prior (msplat_cuda_set_prior) applies to msplat_cuda_render only; "
                                              "clear it before msplat_cuda_render_batch");
    if (int r = forward_batch(ctx, n_views, views)) return r;
    ctx->timer.collect();
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_set_prior(msplat_cuda_ctx *ctx, const msplat_cuda_prior *prior) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (!prior) {
        ctx->has_prior = false;
        return MSPLAT_CUDA_OK;
    }
    const msplat_cuda_prior &p = *prior;
    if (p.aux && p.sky) {
        if (!p.sky_tex) return fail(MSPLAT_CUDA_EINVAL, "prior: sky set without sky_tex");
        if (p.sky_w < 1 || p.sky_h < 1)
            return fail(MSPLAT_CUDA_EINVAL, "prior: sky texture size %dx%d", (int)p.sky_w, (int)p.sky_h);
        if (p.sky_grad && (!p.sky_exp_avg || !p.sky_exp_avg_sq))
            return fail(MSPLAT_CUDA_EINVAL, "prior: sky_grad set without the sky's Adam moments");
    }
    if ((p.prior_depth || p.prior_aux) && (p.prior_w < 0 || p.prior_h < 0))
        return fail(MSPLAT_CUDA_EINVAL, "prior: negative prior size %dx%d", (int)p.prior_w, (int)p.prior_h);
    if (p.prior_aux && reinterpret_cast<uintptr_t>(p.prior_aux) % 4 != 0)
        return fail(MSPLAT_CUDA_EINVAL, "prior: prior_aux must be 4-byte aligned (one RGBA pixel per load)");
    if (p.exposure && p.expo_params && (!p.expo_exp_avg || !p.expo_exp_avg_sq))
        return fail(MSPLAT_CUDA_EINVAL, "prior: exposure set without its Adam moments");
    if (p.exposure && p.expo_num_cams > 0 && std::max(0, (int)p.cam_index) >= p.expo_num_cams)
        return fail(MSPLAT_CUDA_EINVAL, "prior: cam_index %d outside the %d exposure rows", (int)p.cam_index,
                    (int)p.expo_num_cams);
    ctx->prior = p;
    ctx->has_prior = true;
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_render_aux_outputs(msplat_cuda_ctx *ctx, const float **depth, const float **final_T) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (!ctx->aux_frame || !ctx->pri[PB_DEPTH].ptr)
        return fail(MSPLAT_CUDA_EINVAL, "no aux outputs: the last render / train step ran without prior->aux");
    if (depth) *depth = reinterpret_cast<const float *>(ctx->pri[PB_DEPTH].ptr);
    if (final_T) *final_T = reinterpret_cast<const float *>(ctx->final_T.ptr);
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_train_step(msplat_cuda_ctx *ctx, int num_points, float *means3d, float *scales, float glob_scale,
                           float *quats, const float *viewmat, const float *projmat, float fx, float fy, float cx,
                           float cy, unsigned img_height, unsigned img_width, int tiles_x, int tiles_y,
                           float clip_thresh, unsigned degree, unsigned degrees_to_use, const float *cam_pos,
                           float *features_dc, float *features_rest, float *opacities, const float *background,
                           const float *gt, float ssim_weight, float loss_inv_n, int num_adam_groups,
                           float *const *adam_exp_avg, float *const *adam_exp_avg_sq, const float *adam_step_sizes,
                           const float *adam_bc2_sqrts, float adam_beta1, float adam_beta2, float adam_eps,
                           float *vis_counts, float *xys_grad_norm, float *max_2d_size, float inv_max_dim,
                           const int32_t **radii_out, float *loss_out) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (int r = check_camera(num_points, img_height, img_width, tiles_x, tiles_y, degree, degrees_to_use, viewmat,
                             projmat, cam_pos, background))
        return r;
    if (!gt) return fail(MSPLAT_CUDA_EINVAL, "null target image");
    const bool adam = num_adam_groups >= 5;
    if (adam && (!adam_exp_avg || !adam_exp_avg_sq || !adam_step_sizes || !adam_bc2_sqrts))
        return fail(MSPLAT_CUDA_EINVAL, "null Adam state");
    if (adam)
        for (int g = 0; g < std::min(num_adam_groups, 6); g++)
            if (num_points > 0 && (!adam_exp_avg[g] || !adam_exp_avg_sq[g]) && !(g == 4 && degree == 0))
                return fail(MSPLAT_CUDA_EINVAL, "null Adam moment buffer for group %d", g);
    CamParams cam = make_cam(viewmat, projmat, fx, fy, cx, cy, img_height, img_width, tiles_x, tiles_y, clip_thresh,
                             degree, degrees_to_use, cam_pos);
    if (int r = forward(ctx, num_points, means3d, scales, glob_scale, quats, cam, features_dc, features_rest,
                        opacities, background))
        return r;
    cudaStream_t st = ctx->stream;
    const size_t npix = (size_t)img_width * img_height;
    const int n = num_points;
    ENSURE(ctx->v_rendered, npix * 3, float, v_rendered);
    ENSURE(ctx->loss_part, ssim_blocks((int)img_width, (int)img_height), double, loss_part);
    ENSURE(ctx->loss, 1, float, d_loss);
    ENSURE(ctx->slots, (size_t)ctx->n_isect * 9, float, slots);
    const float *out_img = reinterpret_cast<const float *>(ctx->out_img.ptr);
    const float *final_T = reinterpret_cast<const float *>(ctx->final_T.ptr);

    // prior-guided extras (core/cpu/msplat_cpu.cpp:1225-1271)
    const msplat_cuda_prior *pr = ctx->has_prior ? &ctx->prior : nullptr;
    const bool aux = pr && pr->aux;
    const bool sky = aux && pr->sky && pr->sky_tex && pr->sky_grad;
    const bool expo = pr && pr->exposure && pr->expo_params;
    if (aux && pr->loss_terms) CUDA_TRY(cudaMemsetAsync(pr->loss_terms, 0, 4 * sizeof(float), st));
    const float *loss_in = out_img;
    float *loss_grad = v_rendered;
    float *out_adj = nullptr, *v_adj = nullptr;
    if (expo) {
        ENSURE(ctx->pri[PB_ADJ], npix * 3, float, adj);
        ENSURE(ctx->pri[PB_VADJ], npix * 3, float, vadj);
        out_adj = adj;
        v_adj = vadj;
        launch_exposure_apply(out_img, pr->expo_params + 12 * (size_t)std::max(0, pr->cam_index), (int64_t)npix,
                              out_adj, st);
        loss_in = out_adj;
        loss_grad = v_adj;
    }

    SsimArgs sa;
    sa.W = (int)img_width;
    sa.H = (int)img_height;
    sa.img = loss_in;
    sa.gt = gt;
    sa.ssim_weight = ssim_weight;
    sa.inv_n = loss_inv_n;
    sa.v_out = loss_grad;
    sa.partials = loss_part;
    sa.loss = d_loss;
    launch_ssim_loss(sa, st);

    float *v_aux = nullptr, *slots_depth = nullptr;
    if (aux) {
        ENSURE(ctx->pri[PB_VAUX], npix * 2, float, va);
        ENSURE(ctx->pri[PB_SLOTS_D], ctx->n_isect, float, sd);
        v_aux = va;
        slots_depth = sd;
        PriorLossArgs pl;
        pl.W = (int)img_width;
        pl.H = (int)img_height;
        pl.final_T = final_T;
        pl.out_depth = reinterpret_cast<const float *>(ctx->pri[PB_DEPTH].ptr);
        pl.prior_depth = pr->prior_depth;
        pl.prior_aux = pr->prior_aux;
        pl.pw = pr->prior_w;
        pl.ph = pr->prior_h;
        pl.use_depth = pr->has_depth;
        pl.use_sky = pr->has_sky_mask;
        pl.mask_photometric = pr->mask_photometric;
        pl.depth_weight = pr->depth_weight;
        pl.sky_weight = pr->sky_weight;
        pl.fill_weight = pr->fill_weight;
        pl.huber = std::max(pr->huber_delta, 1e-6f);
        pl.min_alpha = pr->min_alpha;
        pl.inv_npix = 1.0f / (float)(img_width * img_height);
        pl.v_photo = loss_grad;
        pl.v_aux = v_aux;
        pl.terms = nullptr;
        double *rows = nullptr;
        if (pr->loss_terms) {
            ENSURE(ctx->pri[PB_TERMS], npix * 3, float, terms);
            ENSURE(ctx->pri[PB_ROWS], (size_t)img_height * 3, double, rw);
            pl.terms = terms;
            rows = rw;
        }
        launch_prior_loss(pl, rows, pr->loss_terms, st);
    }
    if (expo) {
        ENSURE(ctx->pri[PB_EXPO], (size_t)exposure_blocks((int64_t)npix) * 12, double, part);
        ExposureArgs e;
        e.params = pr->expo_params;
        e.exp_avg = pr->expo_exp_avg;
        e.exp_avg_sq = pr->expo_exp_avg_sq;
        e.grad = pr->expo_grad;
        e.cam = std::max(0, pr->cam_index);
        e.step_size = pr->expo_step_size;
        e.bc2 = pr->expo_bc2_sqrt;
        e.reg = pr->expo_reg;
        e.beta1 = adam_beta1;
        e.beta2 = adam_beta2;
        e.eps = adam_eps;
        launch_exposure_backward_adam(out_img, v_adj, (int64_t)npix, v_rendered, part, e, st);
    }
    if (sky) {
        if (4 * npix > (size_t)INT32_MAX)
            return fail(MSPLAT_CUDA_EINVAL, "learned sky: image too large for the sky backward (%zu pixels)", npix);
        SkyScratch sc;
        ENSURE(ctx->pri[PB_SKY_IDX], npix, uint4, tidx);
        ENSURE(ctx->pri[PB_SKY_W], npix, float4, tw);
        ENSURE(ctx->pri[PB_SKY_G], npix, float4, tg);
        ENSURE(ctx->pri[PB_SKY_COUNT], npix, int32_t, cnt);
        ENSURE(ctx->pri[PB_SKY_OFF], npix, int32_t, off);
        ENSURE(ctx->pri[PB_SKY_PART], scan_blocks((int)npix) + 1, int32_t, spart);
        ENSURE(ctx->pri[PB_SKY_TOTAL], 1, int32_t, stotal);
        ENSURE(ctx->pri[PB_SKY_K0], 4 * npix, uint32_t, k0);
        ENSURE(ctx->pri[PB_SKY_K1], 4 * npix, uint32_t, k1);
        ENSURE(ctx->pri[PB_SKY_V0], 4 * npix, uint32_t, v0);
        ENSURE(ctx->pri[PB_SKY_V1], 4 * npix, uint32_t, v1);
        ENSURE(ctx->pri[PB_SKY_RS], radix_scratch_bytes((int)(4 * npix)), unsigned char, rs);
        sc.tap_idx = tidx;
        sc.tap_w = tw;
        sc.tap_g = tg;
        sc.count = cnt;
        sc.off = off;
        sc.scan_part = spart;
        sc.d_total = stotal;
        sc.keys[0] = k0;
        sc.keys[1] = k1;
        sc.vals[0] = v0;
        sc.vals[1] = v1;
        sc.radix_scratch = rs;
        SkyAdamArgs sk;
        sk.tex = pr->sky_tex;
        sk.grad = pr->sky_grad;
        sk.exp_avg = pr->sky_exp_avg;
        sk.exp_avg_sq = pr->sky_exp_avg_sq;
        sk.step_size = pr->sky_step_size;
        sk.bc2 = pr->sky_bc2_sqrt;
        sk.beta1 = adam_beta1;
        sk.beta2 = adam_beta2;
        sk.eps = adam_eps;
        launch_sky_backward_adam(sky_args(*pr, cam), (int)img_width, (int)img_height, final_T, v_rendered, sk, sc,
                                 st);
    }
    ctx->timer.mark(4, st);

    RasterBwdArgs rb{};
    rb.W = (int)img_width;
    rb.H = (int)img_height;
    rb.tiles_x = tiles_x;
    rb.tiles_y = tiles_y;
    rb.tile_start = reinterpret_cast<const int32_t *>(ctx->tile_start.ptr);
    rb.tile_end = reinterpret_cast<const int32_t *>(ctx->tile_end.ptr);
    rb.isect_gid = reinterpret_cast<const int32_t *>(ctx->isect_gid.ptr);
    rb.splats = reinterpret_cast<const Splat *>(ctx->splats.ptr);
    for (int c = 0; c < 3; c++) rb.bg[c] = background[c];
    rb.final_T = reinterpret_cast<const float *>(ctx->final_T.ptr);
    rb.final_idx = reinterpret_cast<const int32_t *>(ctx->final_idx.ptr);
    rb.v_out = v_rendered;
    rb.slots = slots;
    rb.tstore = ctx->tstore_cap > 0 ? reinterpret_cast<const float *>(ctx->tstore.ptr) : nullptr;
    rb.tcount = ctx->tstore_cap > 0 ? reinterpret_cast<const int32_t *>(ctx->tcount.ptr) : nullptr;
    if (aux) {
        rb.bg_img = reinterpret_cast<const float *>(ctx->pri[PB_BG].ptr);
        rb.v_aux = v_aux;
        rb.slots_depth = slots_depth;
        launch_raster_bwd_aux(rb, st);
    } else if (ctx->chunk_frame) {
        ChunkArgs ck{};
        if (int r = chunk_buffers(ctx, tiles_x * tiles_y, true, ck)) return r;
        launch_raster_bwd_chunked(rb, ck, ctx->chunk_cap, st, ctx->raster_variant);
    } else {
        launch_raster_bwd(rb, st, ctx->raster_variant);
    }
    ctx->timer.mark(5, st);

    BackwardArgs ba;
    std::memset(&ba, 0, sizeof ba);
    ba.slots_depth = slots_depth;
    ba.log_max_scale_ratio = pr ? pr->log_max_scale_ratio : 0.f;
    ba.n = n;
    ba.means = means3d;
    ba.scales = scales;
    ba.quats = quats;
    ba.glob_scale = glob_scale;
    ba.cam = cam;
    ba.splats = reinterpret_cast<const Splat *>(ctx->splats.ptr);
    ba.radii = reinterpret_cast<const int32_t *>(ctx->radii.ptr);
    ba.n_tiles = reinterpret_cast<const int32_t *>(ctx->n_tiles.ptr);
    ba.inv = reinterpret_cast<const int32_t *>(ctx->inv.ptr);
    ba.offsets = reinterpret_cast<const int64_t *>(ctx->offsets.ptr);
    ba.slots = slots;
    if (ctx->keep_grads) {
        ENSURE(ctx->v_xy, 2 * (size_t)n, float, vxy);
        ENSURE(ctx->v_conic, 3 * (size_t)n, float, vcon);
        ENSURE(ctx->v_rgb, 3 * (size_t)n, float, vrgb);
        ENSURE(ctx->v_opacity, n, float, vop);
        ENSURE(ctx->v_mean3d, 3 * (size_t)n, float, vm3);
        ENSURE(ctx->v_scale, 3 * (size_t)n, float, vsc);
        ENSURE(ctx->v_quat, 4 * (size_t)n, float, vq);
        ba.v_xy = vxy;
        ba.v_conic = vcon;
        ba.v_rgb = vrgb;
        ba.v_opacity = vop;
        ba.v_mean3d = vm3;
        ba.v_scale = vsc;
        ba.v_quat = vq;
        if (aux) {
            ENSURE(ctx->pri[PB_VDEPTH], n, float, vdep);
            ba.v_depth = vdep;
        }
    }
    ba.do_adam = adam ? 1 : 0;
    float *params[6] = {means3d, scales, quats, features_dc, features_rest, opacities};
    for (int g = 0; g < 6; g++) {
        ba.p[g] = params[g];
        if (adam && g < num_adam_groups) {
            ba.m1[g] = adam_exp_avg[g];
            ba.m2[g] = adam_exp_avg_sq[g];
            ba.ss[g] = adam_step_sizes[g];
            ba.bc2[g] = adam_bc2_sqrts[g];
        }
    }
    if (adam && num_adam_groups < 6) {
        // the reference updates only groups < num_adam_groups: no opacity Adam with 5
        ba.m1[5] = ba.m2[5] = nullptr;
    }
    ba.beta1 = adam_beta1;
    ba.beta2 = adam_beta2;
    ba.eps = adam_eps;
    ba.rest_stride = (int)(num_sh_bases(degree) - 1) * 3;
    ba.vis_counts = vis_counts;
    ba.xys_grad_norm = xys_grad_norm;
    ba.max_2d_size = max_2d_size;
    ba.inv_max_dim = inv_max_dim;
    if (vis_counts && (!xys_grad_norm || !max_2d_size))
        return fail(MSPLAT_CUDA_EINVAL, "densification statistics need all three buffers");
    launch_backward_adam(ba, st);
    // without Adam the fused kernel leaves the scales alone; the cap still applies
    if (!adam && ba.log_max_scale_ratio > 0.f) launch_needle_cap(scales, n, ba.log_max_scale_ratio, st);
    ctx->timer.mark(6, st);
    CUDA_TRY(cudaGetLastError());
    ctx->timer.collect();
    if (radii_out) *radii_out = reinterpret_cast<const int32_t *>(ctx->radii.ptr);
    if (loss_out) {
        CUDA_TRY(cudaMemcpyAsync(loss_out, d_loss, sizeof(float), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
    }
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_render_backward(msplat_cuda_ctx *ctx, int num_points, const float *means3d, const float *scales,
                                float glob_scale, const float *quats, const float *viewmat, const float *projmat,
                                float fx, float fy, float cx, float cy, unsigned img_height, unsigned img_width,
                                int tiles_x, int tiles_y, float clip_thresh, unsigned degree, unsigned degrees_to_use,
                                const float *cam_pos, const float *background, const float *v_img, float *v_means,
                                float *v_scales, float *v_quats, float *v_features_dc, float *v_features_rest,
                                float *v_opacities) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (int r = check_camera(num_points, img_height, img_width, tiles_x, tiles_y, degree, degrees_to_use, viewmat,
                             projmat, cam_pos, background))
        return r;
    if (ctx->n != num_points || ctx->W != (int)img_width || ctx->H != (int)img_height || !ctx->final_T.ptr)
        return fail(MSPLAT_CUDA_EINVAL, "render_backward must follow msplat_cuda_render of the same scene and camera "
                                        "on this context");
    if (!v_img) return fail(MSPLAT_CUDA_EINVAL, "null image gradient");
    if (ctx->aux_frame)
        return fail(MSPLAT_CUDA_EUNSUPPORTED, "render_backward of a render with a prior (aux mode) is not supported; "
                                              "clear the prior with msplat_cuda_set_prior(ctx, NULL) first");
    if (num_points > 0 && (!means3d || !scales || !quats || !v_means || !v_scales || !v_quats || !v_features_dc ||
                           !v_opacities || (degree > 0 && !v_features_rest)))
        return fail(MSPLAT_CUDA_EINVAL, "null parameter or gradient pointer");
    cudaStream_t st = ctx->stream;
    const int n = num_points;
    ENSURE(ctx->slots, (size_t)ctx->n_isect * 9, float, slots);
    CamParams cam = make_cam(viewmat, projmat, fx, fy, cx, cy, img_height, img_width, tiles_x, tiles_y, clip_thresh,
                             degree, degrees_to_use, cam_pos);
    RasterBwdArgs rb;
    rb.W = (int)img_width;
    rb.H = (int)img_height;
    rb.tiles_x = tiles_x;
    rb.tiles_y = tiles_y;
    rb.tile_start = reinterpret_cast<const int32_t *>(ctx->tile_start.ptr);
    rb.tile_end = reinterpret_cast<const int32_t *>(ctx->tile_end.ptr);
    rb.isect_gid = reinterpret_cast<const int32_t *>(ctx->isect_gid.ptr);
    rb.splats = reinterpret_cast<const Splat *>(ctx->splats.ptr);
    for (int c = 0; c < 3; c++) rb.bg[c] = background[c];
    rb.final_T = reinterpret_cast<const float *>(ctx->final_T.ptr);
    rb.final_idx = reinterpret_cast<const int32_t *>(ctx->final_idx.ptr);
    rb.v_out = v_img;
    rb.slots = slots;
    rb.tstore = ctx->tstore_cap > 0 ? reinterpret_cast<const float *>(ctx->tstore.ptr) : nullptr;
    rb.tcount = ctx->tstore_cap > 0 ? reinterpret_cast<const int32_t *>(ctx->tcount.ptr) : nullptr;
    if (ctx->chunk_frame) {
        ChunkArgs ck{};
        if (int r = chunk_buffers(ctx, tiles_x * tiles_y, true, ck)) return r;
        launch_raster_bwd_chunked(rb, ck, ctx->chunk_cap, st, ctx->raster_variant);
    } else {
        launch_raster_bwd(rb, st, ctx->raster_variant);
    }
    BackwardArgs ba;
    std::memset(&ba, 0, sizeof ba);
    ba.n = n;
    ba.means = means3d;
    ba.scales = scales;
    ba.quats = quats;
    ba.glob_scale = glob_scale;
    ba.cam = cam;
    ba.splats = reinterpret_cast<const Splat *>(ctx->splats.ptr);
    ba.radii = reinterpret_cast<const int32_t *>(ctx->radii.ptr);
    ba.n_tiles = reinterpret_cast<const int32_t *>(ctx->n_tiles.ptr);
    ba.inv = reinterpret_cast<const int32_t *>(ctx->inv.ptr);
    ba.offsets = reinterpret_cast<const int64_t *>(ctx->offsets.ptr);
    ba.slots = slots;
    ba.v_mean3d = v_means;
    ba.v_scale = v_scales;
    ba.v_quat = v_quats;
    ba.v_opacity = v_opacities;
    ba.g_dc = v_features_dc;
    ba.g_rest = degree > 0 ? v_features_rest : nullptr;
    ba.rest_stride = (int)(num_sh_bases(degree) - 1) * 3;
    if (ctx->keep_grads) {  // screen-space gradients for msplat_cuda_frame
        ENSURE(ctx->v_xy, 2 * (size_t)n, float, vxy);
        ENSURE(ctx->v_conic, 3 * (size_t)n, float, vcon);
        ENSURE(ctx->v_rgb, 3 * (size_t)n, float, vrgb);
        ba.v_xy = vxy;
        ba.v_conic = vcon;
        ba.v_rgb = vrgb;
    }
    launch_backward_adam(ba, st);
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_ssim_loss(msplat_cuda_ctx *ctx, const float *img, const float *gt, unsigned img_height,
                          unsigned img_width, float ssim_weight, float loss_inv_n, float *v_img, float *loss) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (!img || !gt || !v_img || !loss) return fail(MSPLAT_CUDA_EINVAL, "null buffer");
    if (img_width == 0 || img_height == 0) return fail(MSPLAT_CUDA_EINVAL, "image size must be positive");
    ENSURE(ctx->loss_part, ssim_blocks((int)img_width, (int)img_height), double, loss_part);
    SsimArgs sa;
    sa.W = (int)img_width;
    sa.H = (int)img_height;
    sa.img = img;
    sa.gt = gt;
    sa.ssim_weight = ssim_weight;
    sa.inv_n = loss_inv_n;
    sa.v_out = v_img;
    sa.partials = loss_part;
    sa.loss = loss;
    launch_ssim_loss(sa, ctx->stream);
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_densify(msplat_cuda_ctx *ctx, int N, int buf_capacity, float grad_thresh, float size_thresh,
                        float screen_thresh, int check_screen, float cull_alpha_thresh, float cull_scale_thresh,
                        float cull_screen_size, int check_huge, const float *xys_grad_norm, const float *vis_counts,
                        const float *max_2d_size, float half_max_dim, float *const *params, int fr_stride,
                        float *const *exp_avg, float *const *exp_avg_sq, uint32_t seed, int *new_count) {
    if (!ctx || !new_count) return fail(MSPLAT_CUDA_EINVAL, "null context or output");
    if (N < 0 || fr_stride < 0) return fail(MSPLAT_CUDA_EINVAL, "negative size");
    if ((int64_t)3 * N > buf_capacity)
        return fail(MSPLAT_CUDA_ECAPACITY, "msplat_densify: 3*N (%lld) exceeds buf_capacity (%d)", 3ll * N,
                    buf_capacity);
    if (N > 0 && (!params || !exp_avg || !exp_avg_sq || !xys_grad_norm || !vis_counts || !max_2d_size))
        return fail(MSPLAT_CUDA_EINVAL, "null densify buffer");
    cudaStream_t st = ctx->stream;
    DensifyArgs a;
    std::memset(&a, 0, sizeof a);
    a.n = N;
    a.grad_thresh = grad_thresh;
    a.size_thresh = size_thresh;
    a.screen_thresh = screen_thresh;
    a.check_screen = check_screen;
    a.cull_alpha = cull_alpha_thresh;
    a.cull_scale = cull_scale_thresh;
    a.cull_screen = cull_screen_size;
    a.check_huge = check_huge;
    a.grad_norm = xys_grad_norm;
    a.vis_counts = vis_counts;
    a.max_2d = max_2d_size;
    a.half_max_dim = half_max_dim;
    a.log_size_fac = std::log(1.6f);  // the host's logf, as the reference computes it (msplat_cpu.cpp:1348)
    a.seed = seed;
    const int strides[6] = {3, 3, 4, 3, fr_stride, 1};
    int max_stride = 1;
    for (int g = 0; g < 6; g++) {
        a.stride[g] = strides[g];
        max_stride = std::max(max_stride, strides[g]);
        if (N > 0) {
            a.buf[g] = params[g];
            a.m1[g] = exp_avg[g];
            a.m2[g] = exp_avg_sq[g];
            if ((!a.buf[g] || !a.m1[g] || !a.m2[g]) && strides[g] > 0)
                return fail(MSPLAT_CUDA_EINVAL, "null buffer for group %d", g);
        }
    }
    a.cap = buf_capacity;
    const int64_t rows = 4 * (int64_t)std::max(N, 1);  // a Gaussian may be split and cloned
    if (rows > (int64_t)INT32_MAX) return fail(MSPLAT_CUDA_EINVAL, "msplat_densify: N (%d) too large", N);
    ENSURE(ctx->d_flags, 7 * rows, int32_t, flags);
    ENSURE(ctx->d_counts, 8 + scan_blocks((int)rows) + 1, int32_t, counts);
    ENSURE(ctx->d_scratch, rows * max_stride, float, scratch);
    if (!ctx->h_count) CUDA_TRY(cudaMallocHost(&ctx->h_count, sizeof(int32_t)));
    DensifyScratch s;
    s.split = flags;
    s.dup = flags + rows;
    s.split_ord = flags + 2 * rows;
    s.dup_ord = flags + 3 * rows;
    s.keep = flags + 4 * rows;
    s.keep_ord = flags + 5 * rows;
    s.row_parent = flags + 6 * rows;
    s.n_split = counts;
    s.n_dup = counts + 1;
    s.n_new = counts + 2;
    s.new_count = counts + 3;
    s.overflow = counts + 4;
    s.scan_part = counts + 8;
    s.scratch = scratch;
    launch_densify(a, s, st);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(ctx->h_count, s.new_count, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    int32_t overflow = 0;
    CUDA_TRY(cudaMemcpyAsync(&overflow, s.overflow, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (overflow)
        return fail(MSPLAT_CUDA_ECAPACITY,
                    "msplat_densify: N + 2 x splits + clones exceeds buf_capacity (%d); a Gaussian can be both "
                    "split and cloned, so up to 4 N rows are needed; the buffers are unchanged",
                    buf_capacity);
    *new_count = *ctx->h_count;
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_opacity_reset(msplat_cuda_ctx *ctx, float *opacities, float *exp_avg, float *exp_avg_sq,
                              int num_points, float reset_logit) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (num_points < 0) return fail(MSPLAT_CUDA_EINVAL, "negative count");
    if (num_points > 0 && (!opacities || !exp_avg || !exp_avg_sq)) return fail(MSPLAT_CUDA_EINVAL, "null buffer");
    launch_opacity_reset(opacities, exp_avg, exp_avg_sq, num_points, reset_logit, ctx->stream);
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_radix_sort(msplat_cuda_ctx *ctx, uint64_t *keys, int32_t *vals, uint32_t n, int key_bits) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (n == 0) return MSPLAT_CUDA_OK;
    if (!keys || !vals) return fail(MSPLAT_CUDA_EINVAL, "null keys or values");
    if (n > (uint32_t)INT32_MAX) return fail(MSPLAT_CUDA_EINVAL, "too many keys");
    if (key_bits <= 0) return MSPLAT_CUDA_OK;
    if (key_bits > 64) key_bits = 64;
    ENSURE(ctx->keys[1], n, uint64_t, k1);
    ENSURE(ctx->vals[1], n, uint32_t, v1);
    ENSURE(ctx->radix_scratch, radix_scratch_bytes((int)n), unsigned char, rs);
    uint64_t *kk[2] = {keys, k1};
    uint32_t *vv[2] = {reinterpret_cast<uint32_t *>(vals), v1};
    const int cur = radix_sort_pairs(kk, vv, (int)n, key_bits, rs, ctx->stream);
    if (cur == 1) {
        CUDA_TRY(cudaMemcpyAsync(keys, k1, (size_t)n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        CUDA_TRY(cudaMemcpyAsync(vals, v1, (size_t)n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_knn3_mean_dist(msplat_cuda_ctx *ctx, const float *points, uint32_t n, float *mean_dist) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (n == 0) return MSPLAT_CUDA_OK;
    if (!points || !mean_dist) return fail(MSPLAT_CUDA_EINVAL, "null buffer");
    if (n > (uint32_t)INT32_MAX) return fail(MSPLAT_CUDA_EINVAL, "too many points");
    const int nb = knn_boxes((int)n);
    ENSURE(ctx->k_bounds, 8, unsigned int, bounds);
    ENSURE(ctx->keys[0], n, uint64_t, k0);
    ENSURE(ctx->keys[1], n, uint64_t, k1);
    ENSURE(ctx->vals[0], n, uint32_t, v0);
    ENSURE(ctx->vals[1], n, uint32_t, v1);
    ENSURE(ctx->radix_scratch, radix_scratch_bytes((int)n), unsigned char, rs);
    ENSURE(ctx->k_sorted, n, float4, sorted);
    ENSURE(ctx->k_box, 2 * (size_t)nb, float4, boxes);
    ENSURE(ctx->k_evals, 1, unsigned long long, evals);
    KnnScratch s;
    s.evals = evals;
    s.bounds = bounds;
    s.keys[0] = k0;
    s.keys[1] = k1;
    s.vals[0] = v0;
    s.vals[1] = v1;
    s.radix_scratch = rs;
    s.sorted = sorted;
    s.bmin = boxes;
    s.bmax = boxes + nb;
    launch_knn3(points, (int)n, mean_dist, s, ctx->stream);
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_init_gaussians(msplat_cuda_ctx *ctx, const float *means, const uint8_t *rgb, uint32_t n,
                               uint32_t seed, float opacity_logit, float *scales, float *quats, float *features_dc,
                               float *opacities) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (n == 0) return MSPLAT_CUDA_OK;
    if (!means || !rgb || !scales || !quats || !features_dc || !opacities)
        return fail(MSPLAT_CUDA_EINVAL, "null buffer");
    ENSURE(ctx->k_md, n, float, md);
    if (int r = msplat_cuda_knn3_mean_dist(ctx, means, n, md)) return r;
    launch_init_gaussians(md, rgb, (int)n, seed, opacity_logit, scales, quats, features_dc, opacities, ctx->stream);
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_resize_area(msplat_cuda_ctx *ctx, const void *src, int src_is_u8, int sw, int sh, float *dst, int dw,
                            int dh) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (sw <= 0 || sh <= 0 || dw < 0 || dh < 0) return fail(MSPLAT_CUDA_EINVAL, "bad image sizes");
    if (dw == 0 || dh == 0) return MSPLAT_CUDA_OK;
    if (!src || !dst) return fail(MSPLAT_CUDA_EINVAL, "null image");
    launch_resize_area(src, src_is_u8 ? 1 : 0, sw, sh, dst, dw, dh, ctx->stream);
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_undistort(msplat_cuda_ctx *ctx, const float *src, int sw, int sh, const float *intr,
                          const float *dist, int roi_x, int roi_y, float *dst, int dw, int dh) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (sw <= 0 || sh <= 0 || dw < 0 || dh < 0) return fail(MSPLAT_CUDA_EINVAL, "bad image sizes");
    if (dw == 0 || dh == 0) return MSPLAT_CUDA_OK;
    if (!src || !dst || !intr || !dist) return fail(MSPLAT_CUDA_EINVAL, "null argument");
    launch_undistort(src, sw, sh, intr, dist, roi_x, roi_y, dst, dw, dh, ctx->stream);
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_image_metrics(msplat_cuda_ctx *ctx, const float *rendered, const float *gt, int h, int w,
                              double *out) {
    if (!ctx || !out) return fail(MSPLAT_CUDA_EINVAL, "null context or output");
    out[0] = out[1] = out[2] = 0.0;
    if (h <= 0 || w <= 0) return MSPLAT_CUDA_OK;  // the reference returns zeros too
    if (!rendered || !gt) return fail(MSPLAT_CUDA_EINVAL, "null image");
    const size_t npix = (size_t)h * w;
    MetricsScratch s;
    ENSURE(ctx->img[0], npix * 15, float, hbuf);
    ENSURE(ctx->img[1], npix * 3, float, ts);
    ENSURE(ctx->img[2], npix * 3, float, tl);
    ENSURE(ctx->img[3], npix * 3, double, tq);
    ENSURE(ctx->img[4], (size_t)h * 3 + 3, double, rows);
    s.hbuf = hbuf;
    s.t_ssim = ts;
    s.t_l1 = tl;
    s.t_sq = tq;
    s.rows = rows;
    double *dout = rows + (size_t)h * 3;
    launch_image_metrics(rendered, gt, h, w, s, dout, ctx->stream);
    CUDA_TRY(cudaMemcpyAsync(out, dout, 3 * sizeof(double), cudaMemcpyDefault, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_pack_rgba8(msplat_cuda_ctx *ctx, const float *img, uint32_t n, uint8_t *out) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (n == 0) return MSPLAT_CUDA_OK;
    if (!img || !out) return fail(MSPLAT_CUDA_EINVAL, "null image");
    ENSURE(ctx->img[5], (size_t)n * 4, uint8_t, packed);
    launch_pack_rgba8(img, n, packed, ctx->stream);
    CUDA_TRY(cudaMemcpyAsync(out, packed, (size_t)n * 4, cudaMemcpyDefault, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_finalize_depth(msplat_cuda_ctx *ctx, const float *depth_num, const float *final_T, uint32_t n,
                               float inv_scale, float *depth_out, float *alpha_out) {
    if (!ctx) return fail(MSPLAT_CUDA_EINVAL, "null context");
    if (n == 0) return MSPLAT_CUDA_OK;
    if (!depth_num || !final_T || !depth_out || !alpha_out) return fail(MSPLAT_CUDA_EINVAL, "null buffer");
    launch_finalize_depth(depth_num, final_T, n, inv_scale, depth_out, alpha_out, ctx->stream);
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_loss_device(msplat_cuda_ctx *ctx, const float **loss) {
    if (!ctx || !loss) return fail(MSPLAT_CUDA_EINVAL, "null argument");
    if (!ctx->loss.ptr) return fail(MSPLAT_CUDA_EINVAL, "no train step has run on this context");
    *loss = reinterpret_cast<const float *>(ctx->loss.ptr);
    return MSPLAT_CUDA_OK;
}

int64_t msplat_cuda_num_isects(msplat_cuda_ctx *ctx) { return ctx ? ctx->n_isect : -1; }

int msplat_cuda_rasterizer_exp(msplat_cuda_ctx *ctx, const float *x, int64_t n, float *out) {
    if (!ctx || (n > 0 && (!x || !out))) return fail(MSPLAT_CUDA_EINVAL, "null argument");
    launch_exp_tab(x, n, out, ctx->stream);
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

namespace {
// The pair counter's view of the context's last single-view frame.
RasterArgs pair_count_args(const msplat_cuda_ctx *ctx) {
    RasterArgs a{};
    a.W = ctx->W;
    a.H = ctx->H;
    a.tiles_x = ctx->tiles_x;
    a.tiles_y = ctx->tiles_y;
    a.tile_start = reinterpret_cast<const int32_t *>(ctx->tile_start.ptr);
    a.tile_end = reinterpret_cast<const int32_t *>(ctx->tile_end.ptr);
    a.isect_gid = reinterpret_cast<const int32_t *>(ctx->isect_gid.ptr);
    a.splats = reinterpret_cast<const Splat *>(ctx->splats.ptr);
    a.final_idx = reinterpret_cast<int32_t *>(ctx->final_idx.ptr);
    return a;
}
}  // namespace

int msplat_cuda_frame_pair_counts(msplat_cuda_ctx *ctx, int64_t *out) {
    if (!ctx || !out) return fail(MSPLAT_CUDA_EINVAL, "null argument");
    out[0] = out[1] = 0;
    if (ctx->tiles_x <= 0 || ctx->tiles_y <= 0 || !ctx->tile_start.ptr || !ctx->final_idx.ptr) return MSPLAT_CUDA_OK;
    if (ctx->gid_in_vals) return fail(MSPLAT_CUDA_EINVAL, "the last frame was a batched render");
    ENSURE(ctx->pairs, 2, unsigned long long, d);
    launch_pair_counts(pair_count_args(ctx), d, ctx->stream);
    unsigned long long h[2] = {0, 0};
    CUDA_TRY(cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    out[0] = (int64_t)h[0];
    out[1] = (int64_t)h[1];
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_frame_pair_counts_device(msplat_cuda_ctx *ctx, uint64_t *d_sum) {
    if (!ctx || !d_sum) return fail(MSPLAT_CUDA_EINVAL, "null argument");
    if (ctx->tiles_x <= 0 || ctx->tiles_y <= 0 || !ctx->tile_start.ptr || !ctx->final_idx.ptr) return MSPLAT_CUDA_OK;
    if (ctx->gid_in_vals) return fail(MSPLAT_CUDA_EINVAL, "the last frame was a batched render");
    launch_pair_counts(pair_count_args(ctx), reinterpret_cast<unsigned long long *>(d_sum), ctx->stream, true);
    CUDA_TRY(cudaGetLastError());
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_raster_variant(int v, int32_t *fwd_batch, int32_t *bwd_batch, int32_t *bwd_sub) {
    if (v >= 0 && v < N_RASTER_VARIANTS) {
        if (fwd_batch) *fwd_batch = RASTER_VARIANTS[v].fwd_batch;
        if (bwd_batch) *bwd_batch = RASTER_VARIANTS[v].bwd_batch;
        if (bwd_sub) *bwd_sub = RASTER_VARIANTS[v].bwd_sub;
    }
    return N_RASTER_VARIANTS;
}

int msplat_cuda_raster_shape(int s, int32_t *w, int32_t *h) {
    if (s >= 0 && s < N_RASTER_SHAPES) {
        if (w) *w = RASTER_SHAPES[s].w;
        if (h) *h = RASTER_SHAPES[s].h;
    }
    return N_RASTER_SHAPES;
}

int64_t msplat_cuda_ctx_device_bytes(msplat_cuda_ctx *ctx) {
    if (!ctx) return -1;
    const Buf *all[] = {&ctx->splats, &ctx->radii, &ctx->aabb, &ctx->n_tiles, &ctx->offsets, &ctx->scan_part,
                        &ctx->total, &ctx->v_xy, &ctx->v_conic, &ctx->v_rgb, &ctx->v_opacity, &ctx->v_mean3d,
                        &ctx->v_scale, &ctx->v_quat, &ctx->keys[0], &ctx->keys[1], &ctx->vals[0], &ctx->vals[1],
                        &ctx->emit_gid, &ctx->isect_gid, &ctx->inv, &ctx->slots, &ctx->radix_scratch,
                        &ctx->tile_start, &ctx->tile_end, &ctx->out_img, &ctx->final_T, &ctx->final_idx,
                        &ctx->v_rendered, &ctx->loss_part, &ctx->loss, &ctx->d_flags, &ctx->d_counts,
                        &ctx->d_scratch, &ctx->k_bounds, &ctx->k_sorted, &ctx->k_box, &ctx->k_md, &ctx->tstore,
                        &ctx->tcount, &ctx->bdesc, &ctx->bcounter, &ctx->tb.desc, &ctx->tb.pix_img,
                        &ctx->tb.pix_T, &ctx->tb.pix_idx, &ctx->tb.pix_v, &ctx->tb.partials, &ctx->tb.losses,
                        &ctx->tb.counters, &ctx->dkeys[0], &ctx->dkeys[1], &ctx->dvals[0], &ctx->dvals[1],
                        &ctx->dcounts, &ctx->doff, &ctx->img[0], &ctx->img[1], &ctx->img[2], &ctx->img[3],
                        &ctx->img[4], &ctx->img[5]};
    int64_t total = 0;
    for (const Buf *b : all) total += (int64_t)b->bytes;
    for (const Buf &b : ctx->pri) total += (int64_t)b.bytes;
    for (const Buf &b : ctx->ch) total += (int64_t)b.bytes;
    return total;
}

int msplat_cuda_drain_stage_times(msplat_cuda_ctx *ctx, double *ms, int64_t *calls, int max_stages, int *n_stages,
                                  const char **names) {
    if (!ctx || !n_stages) return fail(MSPLAT_CUDA_EINVAL, "null argument");
    ctx->timer.drain();
    const int n = std::min(max_stages, N_STAGES);
    for (int i = 0; i < n; i++) {
        if (ms) ms[i] = ctx->timer.acc_ms[i];
        if (calls) calls[i] = ctx->timer.calls[i];
        if (names) names[i] = STAGE_NAMES[i];
    }
    for (int i = 0; i < N_STAGES; i++) {
        ctx->timer.acc_ms[i] = 0.0;
        ctx->timer.calls[i] = 0;
    }
    *n_stages = n;
    return MSPLAT_CUDA_OK;
}

int msplat_cuda_frame(msplat_cuda_ctx *ctx, const char *name, const void **dev_ptr, int64_t *count) {
    if (!ctx || !name || !dev_ptr || !count) return fail(MSPLAT_CUDA_EINVAL, "null argument");
    const int64_t n = ctx->n, T = (int64_t)ctx->tiles_x * ctx->tiles_y, npix = (int64_t)ctx->W * ctx->H;
    struct Entry {
        const char *name;
        Buf *buf;
        int64_t count;
    } table[] = {
        {"splats", &ctx->splats, n * SPLAT_FLOATS},
        {"radii", &ctx->radii, n},
        {"aabb", &ctx->aabb, n * 2},
        {"tile_start", &ctx->tile_start, T},
        {"tile_end", &ctx->tile_end, T},
        {"isect_gid", &ctx->isect_gid, ctx->n_isect},
        {"slots", &ctx->slots, ctx->n_isect * 9},
        {"out_img", &ctx->out_img, npix * 3},
        {"final_Ts", &ctx->final_T, npix},
        {"final_idx", &ctx->final_idx, npix},
        {"v_rendered", &ctx->v_rendered, npix * 3},
        {"v_xy", &ctx->v_xy, n * 2},
        {"v_conic", &ctx->v_conic, n * 3},
        {"v_rgb", &ctx->v_rgb, n * 3},
        {"v_opacity", &ctx->v_opacity, n},
        {"v_mean3d", &ctx->v_mean3d, n * 3},
        {"v_scale", &ctx->v_scale, n * 3},
        {"v_quat", &ctx->v_quat, n * 4},
        {"out_depth", &ctx->pri[PB_DEPTH], npix},
        {"bg_img", &ctx->pri[PB_BG], npix * 3},
        {"v_aux", &ctx->pri[PB_VAUX], npix * 2},
        {"v_depth", &ctx->pri[PB_VDEPTH], n},
        {"out_adj", &ctx->pri[PB_ADJ], npix * 3},
        {"v_adj", &ctx->pri[PB_VADJ], npix * 3},
        {"chunk_first", &ctx->ch[CH_FIRST], ctx->chunk_frame ? T + 1 : 0},
        {"knn_evals", &ctx->k_evals, 2},  // one uint64: the last kNN call's point distances
    };
    if (ctx->gid_in_vals && !std::strcmp(name, "isect_gid")) {  // a batched render's ids: the sorted values
        if (!ctx->vals[ctx->sorted].ptr) return fail(MSPLAT_CUDA_EINVAL, "frame buffer 'isect_gid' has not been produced");
        *dev_ptr = ctx->vals[ctx->sorted].ptr;
        *count = ctx->n_isect;
        return MSPLAT_CUDA_OK;
    }
    for (const Entry &e : table)
        if (!std::strcmp(e.name, name)) {
            if (!e.buf->ptr) return fail(MSPLAT_CUDA_EINVAL, "frame buffer '%s' has not been produced", name);
            *dev_ptr = e.buf->ptr;
            *count = e.count;
            return MSPLAT_CUDA_OK;
        }
    return fail(MSPLAT_CUDA_EINVAL, "unknown frame buffer '%s'", name);
}

}  // extern "C"
