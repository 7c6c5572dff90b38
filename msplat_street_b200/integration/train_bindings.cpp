// Training-step throughput through the reference's backend contract (bindings.h):
// the path core/src/model.cpp, the CLI and the Python module take when this library
// stands where core/metal sat. It trains the small plain config -- 10,000 Gaussians
// (means U[-1, 1]^3, log-scales N(-4, 0.5), normalised N(0, 1) rotations, opacity
// logits N(0, 1), SH degree 3 with DC N(0, 0.3) and the rest N(0, 0.05)), one 256 x 256
// pinhole camera (fx = fy = 300) at distance 3 looking at the origin, the target a
// render of a second scene of the same distributions -- with msplat_train_step and
// Model::fullIteration's Adam scalars, every tensor a host MTensor as the reference's
// callers hold them, and prints one JSON line: {"iters_per_s", "ms_per_step", "steps",
// "warmup", "gaussians", "width", "height"}.
//
// With the mode "c_abi" the same training runs from C++ straight through the C-ABI
// (include/msplat_cuda.h) with every tensor resident in device memory -- the form a
// C++ host that owns its device buffers takes: no per-call staging, the loss read back
// once at the end.
//
//     train_bindings [steps] [warmup] [bindings_h | c_abi]
//
// Built by msplat_street_b200.build.build_bindings_bench against the reference's
// headers (core/metal/bindings.h, core/include/metal_tensor.hpp) and
// integration/bindings_cuda.cpp; the binary runs without the reference tree.
#include "bindings.h"
#include "msplat_cuda.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

namespace {

constexpr int N = 10000, W = 256, H = 256, REST = 15;
constexpr float F = 300.f;

struct Scene {
    MTensor means, scales, quats, dc, rest, opac;
};

Scene make_scene(unsigned seed) {
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> u(-1.f, 1.f);
    std::normal_distribution<float> n01(0.f, 1.f);
    Scene s;
    s.means = gpu_empty({N, 3}, DType::Float32);
    s.scales = gpu_empty({N, 3}, DType::Float32);
    s.quats = gpu_empty({N, 4}, DType::Float32);
    s.dc = gpu_empty({N, 3}, DType::Float32);
    s.rest = gpu_empty({N, REST, 3}, DType::Float32);
    s.opac = gpu_empty({N, 1}, DType::Float32);
    float *m = s.means.data<float>(), *sc = s.scales.data<float>(), *q = s.quats.data<float>();
    float *d = s.dc.data<float>(), *r = s.rest.data<float>(), *o = s.opac.data<float>();
    for (int i = 0; i < N; i++) {
        for (int k = 0; k < 3; k++) m[3 * i + k] = u(rng);
        for (int k = 0; k < 3; k++) sc[3 * i + k] = -4.f + 0.5f * n01(rng);
        float qq[4], nn = 0.f;
        for (int k = 0; k < 4; k++) {
            qq[k] = n01(rng);
            nn += qq[k] * qq[k];
        }
        nn = std::sqrt(nn);
        for (int k = 0; k < 4; k++) q[4 * i + k] = qq[k] / nn;
        for (int k = 0; k < 3; k++) d[3 * i + k] = 0.3f * n01(rng);
        for (int k = 0; k < REST * 3; k++) r[REST * 3 * i + k] = 0.05f * n01(rng);
        o[i] = n01(rng);
    }
    return s;
}

// The camera set-up Model::prepareCam computes (core/src/model.cpp:498-546) for an
// OpenGL camera at (0, 0, 3) looking at the origin: camera-to-world = identity
// rotation, translation (0, 0, 3).
void camera(float viewmat[16], float projmat[16], float cam_pos[3]) {
    const float c2w[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 3, 0, 0, 0, 1};
    float R[3][3], T[3], Rinv[3][3], Tinv[3];
    for (int i = 0; i < 3; i++) {
        R[i][0] = c2w[i * 4];
        R[i][1] = -c2w[i * 4 + 1];
        R[i][2] = -c2w[i * 4 + 2];
        T[i] = c2w[i * 4 + 3];
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Rinv[i][j] = R[j][i];
    for (int i = 0; i < 3; i++) Tinv[i] = -(Rinv[i][0] * T[0] + Rinv[i][1] * T[1] + Rinv[i][2] * T[2]);
    const float vm[16] = {Rinv[0][0], Rinv[0][1], Rinv[0][2], Tinv[0], Rinv[1][0], Rinv[1][1], Rinv[1][2], Tinv[1],
                          Rinv[2][0], Rinv[2][1], Rinv[2][2], Tinv[2], 0, 0, 0, 1};
    const float fov_x = 2.f * std::atan((float)W / (2.f * F)), fov_y = 2.f * std::atan((float)H / (2.f * F));
    const float t_p = 0.001f * std::tan(0.5f * fov_y), r_p = 0.001f * std::tan(0.5f * fov_x);
    const float pm[16] = {0.001f / r_p, 0, 0, 0, 0, 0.001f / t_p, 0, 0,
                          0, 0, (1000.f + 0.001f) / (1000.f - 0.001f), -1000.f * 0.001f / (1000.f - 0.001f),
                          0, 0, 1, 0};
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            float acc = 0.f;
            for (int k = 0; k < 4; k++) acc += pm[i * 4 + k] * vm[k * 4 + j];
            projmat[i * 4 + j] = acc;
        }
    std::memcpy(viewmat, vm, sizeof vm);
    for (int i = 0; i < 3; i++) cam_pos[i] = T[i];
}

}  // namespace

void check(int status) {
    if (status != MSPLAT_CUDA_OK) {
        std::fprintf(stderr, "msplat_cuda: %s\n", msplat_cuda_last_error());
        std::exit(2);
    }
}

float *to_device(const MTensor &t) {
    void *d = nullptr;
    check(msplat_cuda_device_alloc(t.nbytes(), &d));
    check(msplat_cuda_copy_buffer(msplat_cuda_default_ctx(), d, t.data_ptr(), t.nbytes()));
    return static_cast<float *>(d);
}

int main(int argc, char **argv) {
    const int steps = argc > 1 ? std::atoi(argv[1]) : 200;
    const int warmup = argc > 2 ? std::atoi(argv[2]) : 10;
    const bool c_abi = argc > 3 && std::strcmp(argv[3], "c_abi") == 0;
    float vmf[16], pmf[16], cam_pos[3];
    camera(vmf, pmf, cam_pos);
    MTensor viewmat = gpu_empty({4, 4}, DType::Float32), projmat = gpu_empty({4, 4}, DType::Float32);
    std::memcpy(viewmat.data_ptr(), vmf, sizeof vmf);
    std::memcpy(projmat.data_ptr(), pmf, sizeof pmf);
    MTensor bg = gpu_empty({3}, DType::Float32);
    const float bgv[3] = {0.6130f, 0.0101f, 0.3984f};
    std::memcpy(bg.data_ptr(), bgv, sizeof bgv);
    const auto tiles = std::make_tuple((W + 15) / 16, (H + 15) / 16, 1);

    Scene target_scene = make_scene(1);
    MTensor img = msplat_render(N, target_scene.means, target_scene.scales, 1.f, target_scene.quats, viewmat,
                                projmat, F, F, W / 2.f, H / 2.f, H, W, tiles, 0.01f, 3, 3, cam_pos, target_scene.dc,
                                target_scene.rest, target_scene.opac, bg, nullptr);
    msplat_gpu_sync();
    MTensor gt = gpu_empty({H, W, 3}, DType::Float32);
    std::memcpy(gt.data_ptr(), img.data_ptr(), gt.nbytes());

    Scene s = make_scene(0);
    MTensor params[6] = {s.means, s.scales, s.quats, s.dc, s.rest, s.opac};
    MTensor m1[6], m2[6];
    for (int g = 0; g < 6; g++) {
        m1[g] = gpu_zeros(params[g].shape(), DType::Float32);
        m2[g] = gpu_zeros(params[g].shape(), DType::Float32);
    }
    MTensor vis = gpu_zeros({N}, DType::Float32), gn = gpu_zeros({N}, DType::Float32),
            ms = gpu_zeros({N}, DType::Float32);
    MTensor window = gpu_empty({11, 11}, DType::Float32);
    const float lr[6] = {0.00016f, 0.005f, 0.001f, 0.0025f, 0.000125f, 0.05f};  // model.cpp:100
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;

    // the c_abi mode's device copies of every tensor the step reads or updates
    msplat_cuda_ctx *cx = msplat_cuda_default_ctx();
    float *d_par[6] = {}, *d_m1[6] = {}, *d_m2[6] = {}, *d_gt = nullptr, *d_stat[3] = {};
    if (c_abi) {
        for (int g = 0; g < 6; g++) {
            d_par[g] = to_device(params[g]);
            d_m1[g] = to_device(m1[g]);
            d_m2[g] = to_device(m2[g]);
        }
        d_gt = to_device(gt);
        d_stat[0] = to_device(vis);
        d_stat[1] = to_device(gn);
        d_stat[2] = to_device(ms);
        check(msplat_cuda_sync(cx));
    }
    auto step = [&](int t) {
        // Model::fullIteration's bias-corrected scalars (core/src/model.cpp:638-651)
        const float bc1 = 1.0f - std::pow(beta1, t), bc2 = 1.0f - std::pow(beta2, t);
        float ss[6], b2[6];
        for (int g = 0; g < 6; g++) {
            ss[g] = lr[g] / bc1;
            b2[g] = std::sqrt(bc2);
        }
        if (c_abi) {
            check(msplat_cuda_train_step(cx, N, d_par[0], d_par[1], 1.f, d_par[2], vmf, pmf, F, F, W / 2.f, H / 2.f,
                                         H, W, std::get<0>(tiles), std::get<1>(tiles), 0.01f, 3, 3, cam_pos, d_par[3],
                                         d_par[4], d_par[5], bgv, d_gt, 0.2f, 1.f / (float)(H * W * 3), 6, d_m1, d_m2,
                                         ss, b2, beta1, beta2, eps, d_stat[0], d_stat[1], d_stat[2],
                                         1.f / (float)std::max(H, W), nullptr, nullptr));
            return 0.f;
        }
        auto r = msplat_train_step(N, s.means, s.scales, 1.f, s.quats, viewmat, projmat, F, F, W / 2.f, H / 2.f, H, W,
                                   tiles, 0.01f, 3, 3, cam_pos, s.dc, s.rest, s.opac, bg, gt, window, 0.2f,
                                   1.f / (float)(H * W * 3), REST, 6, params, m1, m2, ss, b2, beta1, beta2, eps, vis,
                                   gn, ms, 1.f / (float)std::max(H, W), nullptr);
        return std::get<1>(r);
    };
    int t = 0;
    for (int i = 0; i < warmup; i++) step(++t);
    msplat_gpu_sync();
    const auto t0 = std::chrono::steady_clock::now();
    float loss = 0.f;
    for (int i = 0; i < steps; i++) loss = step(++t);
    if (c_abi) {  // the last step's loss, read once after the timed loop
        const float *dl = nullptr;
        check(msplat_cuda_loss_device(cx, &dl));
        check(msplat_cuda_copy_buffer(cx, &loss, dl, sizeof(float)));
    }
    msplat_gpu_sync();
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("{\"mode\": \"%s\", \"iters_per_s\": %.3f, \"ms_per_step\": %.4f, \"steps\": %d, \"warmup\": %d, "
                "\"gaussians\": %d, \"width\": %d, \"height\": %d, \"final_loss\": %.6f}\n",
                c_abi ? "c_abi" : "bindings_h", steps / sec, 1e3 * sec / steps, steps, warmup, N, W, H, loss);
    for (int g = 0; g < 6; g++) {
        msplat_cuda_free(d_par[g]);
        msplat_cuda_free(d_m1[g]);
        msplat_cuda_free(d_m2[g]);
    }
    msplat_cuda_free(d_gt);
    for (float *p : d_stat) msplat_cuda_free(p);
    cleanup_msplat_metal();
    return std::isfinite(loss) ? 0 : 1;
}
