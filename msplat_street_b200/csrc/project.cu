// Projection with EWA 2D covariance and SH colour, one thread per Gaussian.
//
// Follows project_and_sh (core/cpu/msplat_cpu.cpp:452-500) and its helpers
// (:63-190). The output per visible Gaussian is one 48-byte Splat record (read by
// both rasterizer passes), its depth, radius, pixel AABB half-extent and the number
// of 16x16 tiles its AABB covers (the input of the key-emission scan). Compiled with
// -fmad=false: tile rectangles and depth keys must equal the reference's bit for bit.
#include "project_impl.cuh"

namespace msplat {

constexpr int PROJ_THREADS = 128;

// With SH degree 3 in use the warp stages its SH-rest rows while the geometry runs
// (issue_rest_rows); no lane leaves before the wait that every lane of the warp takes.
__global__ void __launch_bounds__(PROJ_THREADS) project_kernel(ProjectArgs a) {
    __shared__ float rest_buf[PROJ_THREADS / 32][32 * PROJ_REST3];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < a.n;
    float *buf = rest_buf[threadIdx.x >> 5];
    bool staged = false;
    if (a.rest_stride == PROJ_REST3 && a.cam.degrees_to_use >= 3)  // grid-uniform
        staged = issue_rest_rows(a.features_rest + (size_t)PROJ_REST3 * (valid ? i : 0), valid, buf);
    ProjState st;
    const bool kept = valid && project_geom(a, i, i, st);
    if (staged) rest_rows_wait();
    if (kept) project_finish(a, i, i, st, staged ? buf + PROJ_REST3 * (threadIdx.x & 31) : nullptr);
}

void launch_project(const ProjectArgs &a, cudaStream_t st) {
    if (a.n <= 0) return;
    project_kernel<<<(a.n + PROJ_THREADS - 1) / PROJ_THREADS, PROJ_THREADS, 0, st>>>(a);
}

// Every (view, Gaussian) instance of a batch: the same per-Gaussian code, reading the
// view's scene and camera and writing at the instance's global slot.
__global__ void __launch_bounds__(PROJ_THREADS) project_batch_kernel(const BatchDesc d, int total) {
    __shared__ float rest_buf[PROJ_THREADS / 32][32 * PROJ_REST3];
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = g < total;
    const int v = valid ? find_view(d.inst_off, d.n_views, g) : 0;
    const int i = valid ? g - d.inst_off[v] : 0;
    float *buf = rest_buf[threadIdx.x >> 5];
    // lanes of one warp may belong to different views: the rows must be back to back
    const bool deg3 = valid && d.proj[v].rest_stride == PROJ_REST3 && d.proj[v].cam.degrees_to_use >= 3;
    const bool staged =
        issue_rest_rows(deg3 ? d.proj[v].features_rest + (size_t)PROJ_REST3 * i : nullptr, deg3, buf);
    ProjState st;
    const bool kept = valid && project_geom(d.proj[v], i, g, st);
    if (staged) rest_rows_wait();
    if (kept) project_finish(d.proj[v], i, g, st, staged ? buf + PROJ_REST3 * (threadIdx.x & 31) : nullptr);
}

void launch_project_batch(const BatchDesc &d, int total, cudaStream_t st) {
    if (total <= 0) return;
    project_batch_kernel<<<(total + PROJ_THREADS - 1) / PROJ_THREADS, PROJ_THREADS, 0, st>>>(d, total);
}

}  // namespace msplat
