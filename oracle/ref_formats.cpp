// Shim around the reference's own Gaussian file writers and reader -- TEST
// INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles this file with the reference's core/cpu, core/include,
// core/metal and core/src directories on the include path; nothing of the reference is
// copied here. It exports plain C entry points so the tests can compare the bytes of
// PLY / .splat files written here with the reference's (core/src/loaders/
// save_gaussians.cpp) and read files back with the reference's reader.

#include "msplat_cpu.cpp"

#include "loaders/save_gaussians.cpp"

#include <cstring>

namespace {

MTensor host_tensor(std::vector<int64_t> shape, const float *src) {
    MTensor t = gpu_empty(std::move(shape), DType::Float32);
    if (src) std::memcpy(t.data_ptr(), src, t.nbytes());
    return t;
}

}  // namespace

extern "C" {

// Writes a PLY (mode 0) or .splat (mode 1) file with the reference's writer. rest has
// n x rest_bases x 3 floats.
int ref_save_gaussians(const char *path, int mode, int n, int rest_bases, const float *means, const float *scales,
                       const float *quats, const float *dc, const float *rest, const float *opac, int step,
                       float scale, const float *translation, int keep_crs) {
    try {
        MTensor m = host_tensor({n, 3}, means), s = host_tensor({n, 3}, scales), q = host_tensor({n, 4}, quats);
        MTensor d = host_tensor({n, 3}, dc), r = host_tensor({n, rest_bases, 3}, rest), o = host_tensor({n, 1}, opac);
        GaussianParams p{m, s, q, d, r, o, scale, {translation[0], translation[1], translation[2]}, keep_crs != 0};
        if (mode == 0) saveGaussianPly(path, p, step);
        else saveGaussianSplat(path, p);
        return 0;
    } catch (...) {
        return 1;
    }
}

// Reads a PLY with the reference's reader; *n / *rest_bases receive the sizes. With
// null output arrays only the sizes are returned.
int ref_load_ply(const char *path, float scale, const float *translation, int keep_crs, int *n, int *rest_bases,
                 int *step, float *means, float *scales, float *quats, float *dc, float *rest, float *opac) {
    try {
        LoadedGaussians g = loadGaussianPly(path, scale, translation, keep_crs != 0);
        *n = (int)g.means.size(0);
        *rest_bases = (int)g.featuresRest.size(1);
        *step = g.step;
        if (means) {
            std::memcpy(means, g.means.data_ptr(), g.means.nbytes());
            std::memcpy(scales, g.scales.data_ptr(), g.scales.nbytes());
            std::memcpy(quats, g.quats.data_ptr(), g.quats.nbytes());
            std::memcpy(dc, g.featuresDc.data_ptr(), g.featuresDc.nbytes());
            std::memcpy(rest, g.featuresRest.data_ptr(), g.featuresRest.nbytes());
            std::memcpy(opac, g.opacities.data_ptr(), g.opacities.nbytes());
        }
        return 0;
    } catch (...) {
        return 1;
    }
}

}  // extern "C"
