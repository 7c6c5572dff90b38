// Shim exposing the reference's prior plumbing -- TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles this file with the reference's core/cpu, core/include,
// core/metal and core/src directories on the include path and links the reference's
// image, PLY and splat loaders (stb is vendored with the reference); nothing of it is
// copied here. Including the reference sources puts their file-local helpers
// (computeSkyFrame and initSkyTexture, core/src/model.cpp:703-809) in this
// translation unit, so the C functions below can call them. Host pointers only.

#include "msplat_cpu.cpp"
#include "priors.cpp"
#include "model.cpp"
#include "ssim.cpp"
#include "image_sizing.cpp"

#include <cstdint>
#include <cstring>

namespace {

MTensor host_copy(std::vector<int64_t> shape, DType dt, const void *src) {
    MTensor t = gpu_empty(std::move(shape), dt);
    std::memcpy(t.data_ptr(), src, t.nbytes());
    return t;
}

}  // namespace

extern "C" {

// resampleNearest (core/src/priors.cpp:152-163)
void ref_resample_nearest(const float *src, int sw, int sh, float *dst, int dw, int dh) {
    std::vector<float> s(src, src + (size_t)sw * sh);
    std::vector<float> d = resampleNearest(s, sw, sh, dw, dh);
    std::memcpy(dst, d.data(), d.size() * sizeof(float));
}

// Camera::loadPriors (core/src/priors.cpp:202-265) on the given files (empty string =
// none). First call with depth / aux NULL to get the size (*w, *h); flags[3] =
// has_depth, has_sky, has_mask. Returns 0, or -1 when the camera gets no priors.
int ref_load_priors(const char *depth, const char *conf, const char *sky, const char *mask, float depth_scale,
                    int use_mask, int *w, int *h, float *depth_out, uint8_t *aux_out, int *flags) {
    Camera cam;
    cam.priorDepthPath = depth;
    cam.priorConfidencePath = conf;
    cam.priorSkyPath = sky;
    cam.priorMaskPath = mask;
    cam.loadPriors(depth_scale, use_mask != 0);
    if (!cam.hasPriors()) return -1;
    *w = cam.priorW;
    *h = cam.priorH;
    if (flags) {
        flags[0] = cam.priorHasDepth;
        flags[1] = cam.priorHasSky;
        flags[2] = cam.priorHasMask;
    }
    if (depth_out) std::memcpy(depth_out, cam.priorDepth.data_ptr(), cam.priorDepth.nbytes());
    if (aux_out) std::memcpy(aux_out, cam.priorAux.data_ptr(), cam.priorAux.nbytes());
    return 0;
}

// computeSkyFrame (core/src/model.cpp:703-738); cam_to_world: n row-major 4x4
void ref_compute_sky_frame(int n, const float *cam_to_world, float *frame) {
    std::vector<Camera> cams((size_t)n);
    for (int i = 0; i < n; i++) std::memcpy(cams[i].camToWorld, cam_to_world + 16 * (size_t)i, 16 * sizeof(float));
    computeSkyFrame(cams, frame);
}

// initSkyTexture (core/src/model.cpp:743-809). Per camera i: cam_to_world (16),
// intr (fx, fy, cx, cy), image (ih x iw x 3 floats), aux (ph x pw x 4 bytes), and
// has_sky; sizes[4 i ..] = iw, ih, pw, ph. tex: (H, W, 3).
void ref_init_sky_texture(int n, const float *cam_to_world, const float *intr, const float *const *images,
                          const uint8_t *const *aux, const int *has_sky, const int *sizes, const float *frame, int W,
                          int H, float *tex) {
    std::vector<Camera> cams((size_t)n);
    for (int i = 0; i < n; i++) {
        Camera &c = cams[i];
        std::memcpy(c.camToWorld, cam_to_world + 16 * (size_t)i, 16 * sizeof(float));
        c.fx = intr[4 * i];
        c.fy = intr[4 * i + 1];
        c.cx = intr[4 * i + 2];
        c.cy = intr[4 * i + 3];
        const int iw = sizes[4 * i], ih = sizes[4 * i + 1], pw = sizes[4 * i + 2], ph = sizes[4 * i + 3];
        c.width = iw;
        c.height = ih;
        if (images[i]) c.image = host_copy({ih, iw, 3}, DType::Float32, images[i]);
        if (aux[i]) c.priorAux = host_copy({ph, pw, 4}, DType::UInt8, aux[i]);
        c.priorW = pw;
        c.priorH = ph;
        c.priorHasSky = has_sky[i] != 0;
    }
    initSkyTexture(cams, frame, W, H, tex);
}

}  // extern "C"
