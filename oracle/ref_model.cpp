// Shim exposing the reference's Model host logic -- TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles this file with the reference's core/cpu, core/include,
// core/metal and core/src directories on the include path; nothing of the reference
// is copied here. It drives the reference's own Model (core/src/model.cpp) with the
// step's device work replaced by recording stubs, so a test can read back, step by
// step, exactly what the reference's host code decides and passes down:
//   * prepareCam (model.cpp:498-546): level size, intrinsics, viewmat, projmat, camera
//     position, SH degrees;
//   * fullIteration's Adam scalars (model.cpp:638-651): step sizes and sqrt(bc2);
//   * schedulersStep's means learning rate (model.cpp:140-143);
//   * afterTrain's densify / opacity-reset calls and their arguments
//     (model.cpp:199-245).
// The reference's msplat_train_step / msplat_densify / msplat_opacity_reset are
// renamed while its CPU backend is included, and recording wrappers take their names
// before model.cpp is included, so model.cpp calls the wrappers. Host pointers only.

#define msplat_train_step ref_real_msplat_train_step
#define msplat_densify ref_real_msplat_densify
#define msplat_opacity_reset ref_real_msplat_opacity_reset
#include "msplat_cpu.cpp"
#undef msplat_train_step
#undef msplat_densify
#undef msplat_opacity_reset

#include <cstdint>
#include <cstring>

namespace {

// What the last iteration's stubs saw.
struct Record {
    float ss[6] = {}, bc2s[6] = {};
    int train_calls = 0;
    int densify_calls = 0;
    float densify_f[9] = {};  // grad, size, screen, cull alpha, cull scale, cull screen, half max dim
    int densify_i[5] = {};    // N, buf_capacity, check_screen, check_huge, fr_stride
    uint32_t densify_seed = 0;
    int reset_calls = 0;
    float reset_logit = 0.f;
    int reset_n = 0;
    float inv_max_dim = 0.f, loss_inv_n = 0.f;
    int img_w = 0, img_h = 0;
} g_rec;

}  // namespace

std::tuple<MTensor, float> msplat_train_step(
    int num_points, MTensor &, MTensor &, float, MTensor &, MTensor &, MTensor &, float, float, float, float,
    unsigned img_height, unsigned img_width, const std::tuple<int, int, int>, float, unsigned, unsigned, float[3],
    MTensor &, MTensor &, MTensor &, MTensor &, MTensor &, MTensor &, float, float loss_inv_n, int, int num_adam_groups,
    MTensor[], MTensor[], MTensor[], float adam_step_sizes[], float adam_bc2_sqrts[], float, float, float, MTensor &,
    MTensor &, MTensor &, float inv_max_dim, const PriorStep *) {
    for (int g = 0; g < num_adam_groups && g < 6; g++) {
        g_rec.ss[g] = adam_step_sizes[g];
        g_rec.bc2s[g] = adam_bc2_sqrts[g];
    }
    g_rec.train_calls++;
    g_rec.inv_max_dim = inv_max_dim;
    g_rec.loss_inv_n = loss_inv_n;
    g_rec.img_w = (int)img_width;
    g_rec.img_h = (int)img_height;
    return {gpu_zeros({num_points}, DType::Int32), 0.f};
}

int msplat_densify(int N, int buf_capacity, float grad_thresh, float size_thresh, float screen_thresh,
                   int check_screen, float cull_alpha_thresh, float cull_scale_thresh, float cull_screen_size,
                   int check_huge, MTensor &, MTensor &, MTensor &, float half_max_dim, MTensor &, MTensor &,
                   MTensor &, MTensor &, MTensor &, MTensor &, int fr_stride, MTensor[], MTensor[], MTensor &,
                   MTensor &, MTensor &, MTensor &, MTensor &, MTensor &, MTensor &, MTensor &, uint32_t seed) {
    g_rec.densify_calls++;
    const float f[9] = {grad_thresh, size_thresh, screen_thresh, cull_alpha_thresh, cull_scale_thresh,
                        cull_screen_size, half_max_dim, 0.f, 0.f};
    std::memcpy(g_rec.densify_f, f, sizeof(f));
    const int i[5] = {N, buf_capacity, check_screen, check_huge, fr_stride};
    std::memcpy(g_rec.densify_i, i, sizeof(i));
    g_rec.densify_seed = seed;
    return N;  // the count is unchanged: only the decision and its arguments are of interest
}

void msplat_opacity_reset(MTensor &, MTensor &, MTensor &, int num_points, float reset_logit) {
    g_rec.reset_calls++;
    g_rec.reset_logit = reset_logit;
    g_rec.reset_n = num_points;
}

#include "priors.cpp"
#include "model.cpp"
#include "ssim.cpp"
#include "image_sizing.cpp"

extern "C" {

// Model(inputData, numCameras, numDownscales, resolutionSchedule, shDegree,
// shDegreeInterval, refineEvery, warmupLength, resetAlphaEvery, densifyGradThresh,
// densifySizeThresh, stopScreenSizeAt, splitScreenSize, maxSteps, keepCrs)
// (core/src/model.cpp:37-79) over n points (xyz n x 3 floats, rgb n x 3 bytes).
void *ref_model_new(int n, const float *xyz, const uint8_t *rgb, int num_cameras, int num_downscales,
                    int resolution_schedule, int sh_degree, int sh_degree_interval, int refine_every,
                    int warmup_length, int reset_alpha_every, float densify_grad_thresh, float densify_size_thresh,
                    int stop_screen_size_at, float split_screen_size, int max_steps) {
    InputData in;
    in.points.count = n;
    in.points.xyz.assign(xyz, xyz + 3 * (size_t)n);
    in.points.rgb.assign(rgb, rgb + 3 * (size_t)n);
    return new Model(in, num_cameras, num_downscales, resolution_schedule, sh_degree, sh_degree_interval,
                     refine_every, warmup_length, reset_alpha_every, densify_grad_thresh, densify_size_thresh,
                     stop_screen_size_at, split_screen_size, max_steps, false);
}

void ref_model_free(void *m) { delete static_cast<Model *>(m); }

namespace {
Camera make_camera(const float *c2w, int width, int height, const float *intr) {
    Camera c;
    std::memcpy(c.camToWorld, c2w, 16 * sizeof(float));
    c.width = width;
    c.height = height;
    c.fx = intr[0];
    c.fy = intr[1];
    c.cx = intr[2];
    c.cy = intr[3];
    return c;
}
}  // namespace

// Model::prepareCam (model.cpp:498-546) at `step`. ints: width, height, degree,
// degreesToUse, tiles x, tiles y; floats: fx, fy, cx, cy; then viewmat (16), projmat
// (16), camera position (3).
void ref_model_prepare_cam(void *mp, const float *c2w, int width, int height, const float *intr, int step,
                           int *ints, float *floats, float *viewmat, float *projmat, float *cam_pos) {
    Model &m = *static_cast<Model *>(mp);
    Camera c = make_camera(c2w, width, height, intr);
    Model::CamSetup s = m.prepareCam(c, step);
    ints[0] = s.width;
    ints[1] = s.height;
    ints[2] = s.degree;
    ints[3] = s.degreesToUse;
    ints[4] = std::get<0>(s.tileBounds);
    ints[5] = std::get<1>(s.tileBounds);
    floats[0] = s.fx;
    floats[1] = s.fy;
    floats[2] = s.cx;
    floats[3] = s.cy;
    std::memcpy(viewmat, c.cachedViewMat.data_ptr(), 16 * sizeof(float));
    std::memcpy(projmat, c.cachedProjViewMat.data_ptr(), 16 * sizeof(float));
    std::memcpy(cam_pos, s.cam_pos, 3 * sizeof(float));
}

// Model::getDownscaleFactor (model.cpp:195-197)
int ref_model_downscale_factor(void *mp, int step) { return static_cast<Model *>(mp)->getDownscaleFactor(step); }

// One iteration's host side, in the order of GaussianTrainer::step
// (python/bindings.cpp:261-274): fullIteration, schedulersStep, afterTrain, with the
// device work stubbed. Out:
//   ss[6], bc2s[6]      Adam scalars handed to msplat_train_step
//   f[12]               means lr after schedulersStep, inv_max_dim, loss_inv_n, then the
//                       densify arguments (grad, size, screen, cull alpha, cull scale,
//                       cull screen, half max dim) and the reset logit
//   i[10]               train image w, h; densify called, N, buf_capacity, check_screen,
//                       check_huge, seed; reset called, reset N
void ref_model_iteration(void *mp, const float *c2w, int width, int height, const float *intr, int step,
                         float *ss, float *bc2s, float *f, int64_t *i) {
    Model &m = *static_cast<Model *>(mp);
    Camera c = make_camera(c2w, width, height, intr);
    g_rec = Record();
    MTensor gt;  // the stubbed step never reads it
    m.fullIteration(c, step, gt, 0.2f);
    m.schedulersStep(step);
    m.afterTrain(step);
    std::memcpy(ss, g_rec.ss, sizeof(g_rec.ss));
    std::memcpy(bc2s, g_rec.bc2s, sizeof(g_rec.bc2s));
    f[0] = m.adam_lr[0];
    f[1] = g_rec.inv_max_dim;
    f[2] = g_rec.loss_inv_n;
    for (int k = 0; k < 7; k++) f[3 + k] = g_rec.densify_f[k];
    f[10] = g_rec.reset_logit;
    f[11] = 0.f;
    i[0] = g_rec.img_w;
    i[1] = g_rec.img_h;
    i[2] = g_rec.densify_calls;
    i[3] = g_rec.densify_i[0];
    i[4] = g_rec.densify_i[1];
    i[5] = g_rec.densify_i[2];
    i[6] = g_rec.densify_i[3];
    i[7] = (int64_t)g_rec.densify_seed;
    i[8] = g_rec.reset_calls;
    i[9] = g_rec.reset_n;
}

}  // extern "C"
