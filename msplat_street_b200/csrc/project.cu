// Projection with EWA 2D covariance and SH colour, one thread per Gaussian.
//
// Follows project_and_sh (core/cpu/msplat_cpu.cpp:452-500) and its helpers
// (:63-190). The output per visible Gaussian is one 48-byte Splat record (read by
// both rasterizer passes), its depth, radius, pixel AABB half-extent and the number
// of 16x16 tiles its AABB covers (the input of the key-emission scan). Compiled with
// -fmad=false: tile rectangles and depth keys must equal the reference's bit for bit.
#include "project_impl.cuh"

namespace msplat {

__global__ void project_kernel(ProjectArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    project_one(a, i, i);
}

void launch_project(const ProjectArgs &a, cudaStream_t st) {
    if (a.n <= 0) return;
    const int bs = 128;
    project_kernel<<<(a.n + bs - 1) / bs, bs, 0, st>>>(a);
}

// Every (view, Gaussian) instance of a batch: the same per-Gaussian code, reading the
// view's scene and camera and writing at the instance's global slot.
__global__ void project_batch_kernel(const BatchDesc d, int total) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int v = find_view(d.inst_off, d.n_views, g);
    project_one(d.proj[v], g - d.inst_off[v], g);
}

void launch_project_batch(const BatchDesc &d, int total, cudaStream_t st) {
    if (total <= 0) return;
    const int bs = 128;
    project_batch_kernel<<<(total + bs - 1) / bs, bs, 0, st>>>(d, total);
}

}  // namespace msplat
