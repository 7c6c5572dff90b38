// Fused per-Gaussian backward + Adam + densification statistics.
//
// One thread per Gaussian replaces four reference passes:
//  1. reduce_isect_grads (core/cpu/msplat_cpu.cpp:1034-1064): the Gaussian's
//     intersection slots, found through the inverse sort permutation, are summed in
//     sorted (= tile) order;
//  2. project_and_sh_backward_adam (:1068-1139): projection, EWA and covariance VJPs
//     (:197-291) for visible Gaussians, SH gradients fused into Adam for DC and rest;
//  3. adam_dense (:1142-1147) over ALL N for means, scales, quats and opacity
//     (invisible Gaussians see a zero gradient, their moments decay);
//  4. the densification statistics (:1312-1324).
// The SH-rest Adam is warp-cooperative: each lane computes its Gaussian's basis and
// colour gradient, then the warp walks the 32 x (B-1) x 3 rest block of its 32
// Gaussians in memory order, so those loads and stores coalesce.
// Compiled with -fmad=false; expressions keep the reference's operation order.
#include "common.cuh"
#include "kernels.h"

namespace msplat {

namespace {

// pixel-centre VJP through the perspective divide (:197-205)
__device__ __forceinline__ V3 center_vjp(const float *P, V3 p, uint32_t w, uint32_t h, float gx, float gy) {
    float hx = P[0] * p.x + P[1] * p.y + P[2] * p.z + P[3];
    float hy = P[4] * p.x + P[5] * p.y + P[6] * p.z + P[7];
    float hw = P[12] * p.x + P[13] * p.y + P[14] * p.z + P[15];
    float rw = 1.f / (hw + 1e-6f);
    float nx = 0.5f * (float)w * gx, ny = 0.5f * (float)h * gy;
    float px = nx * rw, py = ny * rw, pz = 0.f, pw = -(nx * hx + ny * hy) * rw * rw;
    return V3{P[0] * px + P[4] * py + P[8] * pz + P[12] * pw, P[1] * px + P[5] * py + P[9] * pz + P[13] * pw,
              P[2] * px + P[6] * py + P[10] * pz + P[14] * pw};
}

// conic VJP, -X G X with 2x2 column-major products (:207-214)
__device__ __forceinline__ void conic_vjp(V3 cn, V3 g, float *out) {
    const float X00 = cn.x, X01 = cn.y, X10 = cn.y, X11 = cn.z;  // X[col][row]
    const float G00 = g.x, G01 = g.y, G10 = g.y, G11 = g.z;
    // P = X * G
    const float P00 = X00 * G00 + X10 * G01, P01 = X01 * G00 + X11 * G01;
    const float P10 = X00 * G10 + X10 * G11, P11 = X01 * G10 + X11 * G11;
    // Q = P * X
    const float Q00 = P00 * X00 + P10 * X01, Q01 = P01 * X00 + P11 * X01;
    const float Q10 = P00 * X10 + P10 * X11, Q11 = P01 * X10 + P11 * X11;
    const float S00 = Q00 * -1.f, S01 = Q01 * -1.f, S10 = Q10 * -1.f, S11 = Q11 * -1.f;
    out[0] = S00;
    out[1] = S10 + S01;
    out[2] = S11;
}

// EWA VJP (:216-255); adds the mean gradient into gm
__device__ __forceinline__ void ewa_vjp(const float *cov, const float *vm, float fx, float fy, float tfx, float tfy,
                                        V3 gc2, float *gm, float *gc3, V3 pv) {
    float lx = 1.3f * tfx, ly = 1.3f * tfy;
    pv.x = pv.z * fminf(lx, fmaxf(-lx, pv.x / pv.z));
    pv.y = pv.z * fminf(ly, fmaxf(-ly, pv.y / pv.z));
    float rz = 1.f / pv.z, rz2 = rz * rz;
    M3 W = m3(vm[0], vm[4], vm[8], vm[1], vm[5], vm[9], vm[2], vm[6], vm[10]);
    M3 J = m3(fx * rz, 0.f, 0.f, 0.f, fy * rz, 0.f, -fx * pv.x * rz2, -fy * pv.y * rz2, 0.f);
    M3 V = m3(cov[0], cov[1], cov[2], cov[1], cov[3], cov[4], cov[2], cov[4], cov[5]);
    M3 G = m3(gc2.x, 0.5f * gc2.y, 0.f, 0.5f * gc2.y, gc2.z, 0.f, 0.f, 0.f, 0.f);
    M3 T = mul(J, W);
    M3 gV = mul(mul(tr(T), G), T);
    M3 gT = plus(mul(mul(G, T), tr(V)), mul(mul(tr(G), T), V));
    gc3[0] = gV.c[0].x;
    gc3[1] = gV.c[0].y + gV.c[1].x;
    gc3[2] = gV.c[0].z + gV.c[2].x;
    gc3[3] = gV.c[1].y;
    gc3[4] = gV.c[1].z + gV.c[2].y;
    gc3[5] = gV.c[2].z;
    M3 gJ = mul(gT, tr(W));
    float fxr2 = fx * rz2, fyr2 = fy * rz2, rz3 = rz2 * rz;
    V3 gt{-fxr2 * gJ.c[2].x, -fyr2 * gJ.c[2].y,
          -fxr2 * gJ.c[0].x + 2.f * fx * pv.x * rz3 * gJ.c[2].x - fyr2 * gJ.c[1].y + 2.f * fy * pv.y * rz3 * gJ.c[2].y};
    gm[0] += dot3(gt, W.c[0]);
    gm[1] += dot3(gt, W.c[1]);
    gm[2] += dot3(gt, W.c[2]);
}

// rotation VJP, tangent to the unit sphere (:259-274). G(col, row) of the column-major v_R.
__device__ __forceinline__ Q4 rotmat_vjp(Q4 q, const M3 &g) {
    float s = 1.f / sqrtf(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    float w = q.x * s, x = q.y * s, y = q.z * s, z = q.w * s;
#define G(col, row) el(g.c[col], row)
    Q4 r;
    r.x = 2.f * (x * (G(1, 2) - G(2, 1)) + y * (G(2, 0) - G(0, 2)) + z * (G(0, 1) - G(1, 0)));
    r.y = 2.f * (-2.f * x * (G(1, 1) + G(2, 2)) + y * (G(0, 1) + G(1, 0)) + z * (G(0, 2) + G(2, 0)) +
                 w * (G(1, 2) - G(2, 1)));
    r.z = 2.f * (x * (G(0, 1) + G(1, 0)) - 2.f * y * (G(0, 0) + G(2, 2)) + z * (G(1, 2) + G(2, 1)) +
                 w * (G(2, 0) - G(0, 2)));
    r.w = 2.f * (x * (G(0, 2) + G(2, 0)) + y * (G(1, 2) + G(2, 1)) - 2.f * z * (G(0, 0) + G(1, 1)) +
                 w * (G(0, 1) - G(1, 0)));
#undef G
    float radial = r.x * w + r.y * x + r.z * y + r.w * z;
    return Q4{(r.x - radial * w) * s, (r.y - radial * x) * s, (r.z - radial * y) * s, (r.w - radial * z) * s};
}

// covariance VJP to scale and quaternion (:276-291)
__device__ __forceinline__ void cov3d_vjp(V3 sc, float gs, Q4 q, const float *gc, float *gsv, float *gq) {
    M3 gV = m3(gc[0], 0.5f * gc[1], 0.5f * gc[2], 0.5f * gc[1], gc[3], 0.5f * gc[4], 0.5f * gc[2], 0.5f * gc[4], gc[5]);
    M3 R = rotmat(q);
    M3 S = diag_scale(sc, gs);
    M3 M = mul(R, S);
    M3 gM = smul(2.f, mul(gV, M));
    gsv[0] = dot3(R.c[0], gM.c[0]);
    gsv[1] = dot3(R.c[1], gM.c[1]);
    gsv[2] = dot3(R.c[2], gM.c[2]);
    Q4 r = rotmat_vjp(q, mul(gM, S));
    gq[0] = r.x;
    gq[1] = r.y;
    gq[2] = r.z;
    gq[3] = r.w;
}


// Sums of the 9 raster-backward values over each visible Gaussian's intersection
// slots, in sorted (tile) order. Most Gaussians cover a few tiles: each lane sums its
// own Gaussian's slots one after another, so the lanes' independent loads overlap.
// A Gaussian covering more than SLOT_LANE_MAX tiles (near the camera: hundreds) is
// summed by the whole warp afterwards: lane l takes its intersections l, l+32, ... and
// a fixed butterfly combines the lanes. Both orders are fixed, so the sums do not
// depend on scheduling. g0 = index of the warp's first Gaussian in offsets / n_tiles;
// s9 is zero for invisible Gaussians. With slots_depth (aux mode) the depth slots are
// summed the same way into *sd.
constexpr int SLOT_LANE_MAX = 64;

__device__ __forceinline__ void warp_slot_sums(bool vis, int64_t g0, const int64_t *offsets, const int32_t *n_tiles,
                                               const int32_t *inv, const float *slots, float s9[9],
                                               const float *slots_depth = nullptr, float *sd = nullptr) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int c = 0; c < 9; c++) s9[c] = 0.f;
    if (sd) *sd = 0.f;
    long long my_e0 = 0;
    int my_cnt = 0;
    if (vis) {
        my_e0 = offsets[g0 + lane];
        my_cnt = n_tiles[g0 + lane];
    }
    if (vis && my_cnt <= SLOT_LANE_MAX) {
        for (int j = 0; j < my_cnt; j++) {
            const int32_t k = inv[my_e0 + j];
            const float *sl = slots + (size_t)k * 9;
#pragma unroll
            for (int c = 0; c < 9; c++) s9[c] += sl[c];
            if (slots_depth) *sd += slots_depth[k];
        }
    }
    const unsigned big = __ballot_sync(0xffffffffu, vis && my_cnt > SLOT_LANE_MAX);
    for (unsigned bits = big; bits; bits &= bits - 1u) {  // warp-uniform
        const int gl = __ffs(bits) - 1;
        const long long e0 = __shfl_sync(0xffffffffu, my_e0, gl);
        const int cnt = __shfl_sync(0xffffffffu, my_cnt, gl);
        float p[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, pd = 0.f;
        for (int j = lane; j < cnt; j += 32) {
            const int32_t k = inv[e0 + j];
            const float *sl = slots + (size_t)k * 9;
#pragma unroll
            for (int c = 0; c < 9; c++) p[c] += sl[c];
            if (slots_depth) pd += slots_depth[k];
        }
#pragma unroll
        for (int c = 0; c < 9; c++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) p[c] += __shfl_xor_sync(0xffffffffu, p[c], o);
            if (lane == gl) s9[c] = p[c];
        }
        if (slots_depth) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) pd += __shfl_xor_sync(0xffffffffu, pd, o);
            if (lane == gl) *sd = pd;
        }
    }
}

// Projection, EWA and covariance VJPs of one visible Gaussian i seen by camera cam
// (core/cpu/msplat_cpu.cpp:1068-1110): mean, scale and quaternion gradients from its
// summed xy / conic gradients, and its unit view direction for the SH gradients.
// v_depth: dL/d(view-space depth), from the aux mode's expected-depth loss (else 0).
__device__ __forceinline__ void projection_vjp(const CamParams &cam, const float *means, const float *scales,
                                               const float *quats, float glob_scale, const Splat *sp, int i,
                                               const float s9[9], float gm[3], float gsv[3], float gq[4], V3 &dir,
                                               float v_depth = 0.f) {
    const float *vm = cam.viewmat;
    V3 pw = ld3(means, i);
    V3 vmn = center_vjp(cam.projmat, pw, cam.width, cam.height, s9[0], s9[1]);
    vmn = add(vmn, scl(V3{vm[8], vm[9], vm[10]}, v_depth));
    gm[0] = vmn.x;
    gm[1] = vmn.y;
    gm[2] = vmn.z;
    const float4 sp0 = reinterpret_cast<const float4 *>(sp)[0];
    const float4 sp1 = reinterpret_cast<const float4 *>(sp)[1];
    float gc2[3];
    conic_vjp(V3{sp0.z, sp0.w, sp1.x}, V3{s9[2], s9[3], s9[4]}, gc2);
    V3 ls = ld3(scales, i);
    // gradient arithmetic: single-precision exp (within 2 ulps) is enough here
    V3 es{expf(ls.x), expf(ls.y), expf(ls.z)};
    const float4 qq = reinterpret_cast<const float4 *>(quats)[i];
    Q4 q{qq.x, qq.y, qq.z, qq.w};
    float cov[6];
    cov3d_of(es, glob_scale, q, cov);
    const float tfx = 0.5f * (float)cam.width / cam.fx, tfy = 0.5f * (float)cam.height / cam.fy;
    V3 pv{vm[0] * pw.x + vm[1] * pw.y + vm[2] * pw.z + vm[3], vm[4] * pw.x + vm[5] * pw.y + vm[6] * pw.z + vm[7],
          vm[8] * pw.x + vm[9] * pw.y + vm[10] * pw.z + vm[11]};
    float gc3[6];
    ewa_vjp(cov, vm, cam.fx, cam.fy, tfx, tfy, V3{gc2[0], gc2[1], gc2[2]}, gm, gc3, pv);
    cov3d_vjp(es, glob_scale, q, gc3, gsv, gq);
    gsv[0] *= es.x;
    gsv[1] *= es.y;
    gsv[2] *= es.z;
    dir = unit(sub(pw, V3{cam.cam_pos[0], cam.cam_pos[1], cam.cam_pos[2]}));
}

// The 15 SH basis values beyond DC for unit direction (x, y, z)
// (core/cpu/msplat_cpu.cpp:101-130).
__device__ __forceinline__ void sh_rest_basis(V3 d, float *bs) {
    float x = d.x, y = d.y, z = d.z;
    float xx = x * x, xy = x * y, xz = x * z, yy = y * y, yz = y * z, zz = z * z;
    bs[0] = -SH_C1 * y;
    bs[1] = SH_C1 * z;
    bs[2] = -SH_C1 * x;
    bs[3] = SH_C2_0 * xy;
    bs[4] = SH_C2_1 * yz;
    bs[5] = SH_C2_2 * (2.f * zz - xx - yy);
    bs[6] = SH_C2_3 * xz;
    bs[7] = SH_C2_4 * (xx - yy);
    bs[8] = SH_C3_0 * y * (3.f * xx - yy);
    bs[9] = SH_C3_1 * xy * z;
    bs[10] = SH_C3_2 * y * (4.f * zz - xx - yy);
    bs[11] = SH_C3_3 * z * (2.f * zz - 3.f * xx - 3.f * yy);
    bs[12] = SH_C3_4 * x * (4.f * zz - xx - yy);
    bs[13] = SH_C3_5 * z * (xx - yy);
    bs[14] = SH_C3_6 * x * (xx - 3.f * yy);
}

// Adam over the SH-rest rows of a warp's Gaussians (rows of `stride` floats starting at
// p, m1, m2), walked as one flat range of rows x stride floats: every access of the
// warp covers 32 consecutive floats, and each lane loads its U elements before it
// updates any, so the loads of a row block overlap instead of following one row at a
// time. grad(r, e) is the gradient of float e of row r; rows with vis[r] == 0 and
// floats e >= used keep their values. Each element gets the same adam_step as in the
// row-by-row walk.
template <int U, typename Grad>
__device__ __forceinline__ void warp_rest_adam(float *__restrict__ p, float *__restrict__ m1,
                                               float *__restrict__ m2, int rows, int stride, int used,
                                               const int *vis, Grad grad, float ss, float b1, float b2, float bc2,
                                               float eps) {
    if (stride <= 0 || rows <= 0) return;
    const int lane = threadIdx.x & 31;
    const int total = rows * stride;
    int r = 0, e = lane;  // row and float of this lane's next element
    while (e >= stride) {
        e -= stride;
        r++;
    }
    for (int j0 = 0; j0 < total; j0 += 32 * U) {
        float pv[U], v1[U], v2[U];
        int rr[U], ee[U];
        bool up[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int j = j0 + u * 32 + lane;
            rr[u] = r;
            ee[u] = e;
            up[u] = j < total && e < used && vis[r] != 0;  // vis[r] read only for j < total
            if (up[u]) {
                pv[u] = p[j];
                v1[u] = m1[j];
                v2[u] = m2[j];
            }
            e += 32;
            while (e >= stride) {
                e -= stride;
                r++;
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (up[u]) {
                const int j = j0 + u * 32 + lane;
                adam_step(pv[u], v1[u], v2[u], grad(rr[u], ee[u]), ss, b1, b2, bc2, eps);
                p[j] = pv[u];
                m1[j] = v1[u];
                m2[j] = v2[u];
            }
        }
    }
}

// Writes a warp's SH-rest gradient rows (gradient-only mode) as one flat range:
// grad(r, e) where e < used and row r is visible (every row when vis is null), else 0.
template <typename Grad>
__device__ __forceinline__ void warp_rest_grad(float *__restrict__ out, int rows, int stride, int used,
                                               const int *vis, Grad grad) {
    if (stride <= 0 || rows <= 0) return;
    const int lane = threadIdx.x & 31;
    const int total = rows * stride;
    int r = 0, e = lane;
    while (e >= stride) {
        e -= stride;
        r++;
    }
    for (int j = lane; j < total; j += 32) {
        out[j] = (e < used && (vis == nullptr || vis[r] != 0)) ? grad(r, e) : 0.f;
        e += 32;
        while (e >= stride) {
            e -= stride;
            r++;
        }
    }
}

constexpr int REST_UNROLL = 4;

}  // namespace

constexpr int BWD_THREADS = 256;
constexpr int MAX_REST = 15;  // SH bases beyond DC that the backward updates (degree <= 3)

__global__ void __launch_bounds__(BWD_THREADS, 4) backward_adam_kernel(BackwardArgs a) {
    __shared__ float s_basis[BWD_THREADS][MAX_REST + 1];
    __shared__ float s_vrgb[BWD_THREADS][3];
    __shared__ int s_vis[BWD_THREADS];
    const int i = blockIdx.x * BWD_THREADS + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool valid = i < a.n;
    const bool vis = valid && a.radii[i] > 0;
    const float b1 = a.beta1, b2 = a.beta2, eps = a.eps;

    // 1. per-Gaussian sums of the intersection slots
    float s9[9], sd = 0.f;
    warp_slot_sums(vis, (int64_t)blockIdx.x * BWD_THREADS + (threadIdx.x - lane), a.offsets, a.n_tiles, a.inv,
                   a.slots, s9, a.slots_depth, a.slots_depth ? &sd : nullptr);
    if (valid) {  // s9 is zero for invisible Gaussians
        if (a.v_xy) {
            a.v_xy[2 * i] = s9[0];
            a.v_xy[2 * i + 1] = s9[1];
        }
        if (a.v_conic) {
            a.v_conic[3 * i] = s9[2];
            a.v_conic[3 * i + 1] = s9[3];
            a.v_conic[3 * i + 2] = s9[4];
        }
        if (a.v_rgb) {
            a.v_rgb[3 * i] = s9[5];
            a.v_rgb[3 * i + 1] = s9[6];
            a.v_rgb[3 * i + 2] = s9[7];
        }
        if (a.v_opacity) a.v_opacity[i] = s9[8];
        if (a.v_depth) a.v_depth[i] = sd;
    }

    // 2. projection VJPs
    float gm[3] = {0.f, 0.f, 0.f}, gsv[3] = {0.f, 0.f, 0.f}, gq[4] = {0.f, 0.f, 0.f, 0.f};
    V3 dir{0.f, 0.f, 1.f};
    if (vis)
        projection_vjp(a.cam, a.means, a.scales, a.quats, a.glob_scale, a.splats + i, i, s9, gm, gsv, gq, dir, sd);
    if (valid && a.v_mean3d) {
        for (int c = 0; c < 3; c++) {
            a.v_mean3d[3 * i + c] = gm[c];
            a.v_scale[3 * i + c] = gsv[c];
        }
        for (int c = 0; c < 4; c++) a.v_quat[4 * i + c] = gq[c];
    }

    // 3. dense Adam: means, scales, quats, opacity (all N)
    if (valid && a.do_adam) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const size_t k = 3 * (size_t)i + c;
            adam_step(a.p[0][k], a.m1[0][k], a.m2[0][k], gm[c], a.ss[0], b1, b2, a.bc2[0], eps);
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const size_t k = 3 * (size_t)i + c;
            adam_step(a.p[1][k], a.m1[1][k], a.m2[1][k], gsv[c], a.ss[1], b1, b2, a.bc2[1], eps);
        }
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const size_t k = 4 * (size_t)i + c;
            adam_step(a.p[2][k], a.m1[2][k], a.m2[2][k], gq[c], a.ss[2], b1, b2, a.bc2[2], eps);
        }
        if (a.m1[5]) adam_step(a.p[5][i], a.m1[5][i], a.m2[5][i], s9[8], a.ss[5], b1, b2, a.bc2[5], eps);
        // needle cap after the scale update (scale_ratio_cap, core/cpu/msplat_cpu.cpp:1295-1309)
        if (a.log_max_scale_ratio > 0.f) {
            float *sc = a.p[1] + 3 * (size_t)i;
            const float x = sc[0], y = sc[1], z = sc[2];
            const float mx = fmaxf(x, fmaxf(y, z)), mn = fminf(x, fminf(y, z));
            const float cap = (x + y + z - mx - mn) + a.log_max_scale_ratio;
            if (mx > cap) {
                if (x == mx) sc[0] = cap;
                else if (y == mx) sc[1] = cap;
                else sc[2] = cap;
            }
        }
        // DC for visible Gaussians
        if (vis) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const size_t k = 3 * (size_t)i + c;
                adam_step(a.p[3][k], a.m1[3][k], a.m2[3][k], SH_C0 * s9[5 + c], a.ss[3], b1, b2, a.bc2[3], eps);
            }
        }
    }

    // 4. densification statistics
    if (vis && a.vis_counts) {
        a.vis_counts[i] += 1.0f;
        const float gx = s9[0], gy = s9[1];
        a.xys_grad_norm[i] += sqrtf(gx * gx + gy * gy);
        a.max_2d_size[i] = fmaxf(a.max_2d_size[i], (float)a.radii[i] * a.inv_max_dim);
    }

    // gradient-only mode (autograd): the SH colour gradients as arrays
    if (valid && a.g_dc) {
#pragma unroll
        for (int c = 0; c < 3; c++) a.g_dc[3 * (size_t)i + c] = vis ? SH_C0 * s9[5 + c] : 0.f;
    }

    // 5. SH rest Adam (or its gradient), warp-cooperative over the warp's 32 Gaussians
    if ((!a.do_adam && !a.g_rest) || a.rest_stride <= 0) return;
    const uint32_t dtu = a.cam.degrees_to_use;
    const int active = dtu < 1 ? 0 : dtu < 2 ? 3 : dtu < 3 ? 8 : 15;  // bases updated
    if (active == 0 && !a.g_rest) return;
    {
        sh_rest_basis(dir, s_basis[threadIdx.x]);
        s_vrgb[threadIdx.x][0] = s9[5];
        s_vrgb[threadIdx.x][1] = s9[6];
        s_vrgb[threadIdx.x][2] = s9[7];
        s_vis[threadIdx.x] = vis ? 1 : 0;
    }
    __syncwarp();
    const int wbase_t = threadIdx.x - lane;                          // first thread of this warp
    const int64_t g0 = (int64_t)blockIdx.x * BWD_THREADS + wbase_t;  // its Gaussian
    const int stride = a.rest_stride;
    const int used = 3 * active;  // floats of each row that get a gradient
    const int rows = (int)min((int64_t)32, (int64_t)a.n - g0);
    const size_t off = (size_t)g0 * stride;
    auto grad = [&](int r, int e) {
        const int base = e / 3;
        return s_basis[wbase_t + r][base] * s_vrgb[wbase_t + r][e - 3 * base];
    };
    if (a.g_rest) {  // gradient-only mode: every row, zero where invisible or inactive
        warp_rest_grad(a.g_rest + off, rows, stride, used, s_vis + wbase_t, grad);
        return;
    }
    warp_rest_adam<REST_UNROLL>(a.p[4] + off, a.m1[4] + off, a.m2[4] + off, rows, stride, used, s_vis + wbase_t, grad,
                                a.ss[4], b1, b2, a.bc2[4], eps);
}

void launch_backward_adam(const BackwardArgs &a, cudaStream_t st) {
    if (a.n <= 0) return;
    backward_adam_kernel<<<(a.n + BWD_THREADS - 1) / BWD_THREADS, BWD_THREADS, 0, st>>>(a);
}

// The multi-view form: one thread per Gaussian walks the batch's views in order,
// sums each view's slots (instance v * n + i), runs that view's projection VJPs and
// accumulates the gradients, then applies one Adam step. The densification
// statistics advance once per view that sees the Gaussian, as consecutive
// single-view steps would advance them. A one-view batch reproduces
// backward_adam_kernel's update.
__global__ void __launch_bounds__(BWD_THREADS) backward_adam_batch_kernel(BackwardBatchArgs a) {
    __shared__ float s_grest[BWD_THREADS][3 * MAX_REST];
    __shared__ int s_vis[BWD_THREADS];
    if (a.skip && *a.skip) return;  // block-uniform: the step overflowed its capacity
    const int i = blockIdx.x * BWD_THREADS + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool valid = i < a.n;
    const float b1 = a.beta1, b2 = a.beta2, eps = a.eps;
    const uint32_t dtu = a.degrees_to_use;
    const int active = dtu < 1 ? 0 : dtu < 2 ? 3 : dtu < 3 ? 8 : 15;  // SH bases beyond DC with gradients
    const int used = 3 * active;
    float *grest = s_grest[threadIdx.x];
    for (int j = 0; j < 3 * MAX_REST; j++) grest[j] = 0.f;
    float gm[3] = {0.f, 0.f, 0.f}, gsv[3] = {0.f, 0.f, 0.f}, gq[4] = {0.f, 0.f, 0.f, 0.f};
    float gop = 0.f, gdc[3] = {0.f, 0.f, 0.f};
    float st_vis = 0.f, st_gn = 0.f, st_ms = 0.f;
    if (valid && a.vis_counts) {
        st_vis = a.vis_counts[i];
        st_gn = a.xys_grad_norm[i];
        st_ms = a.max_2d_size[i];
    }
    bool any = false;
    for (int v = 0; v < a.n_views; v++) {
        const int64_t g = (int64_t)v * a.n + i;
        const bool vis = valid && a.radii[g] > 0;
        float s9[9];
        warp_slot_sums(vis, (int64_t)v * a.n + (int64_t)blockIdx.x * BWD_THREADS + (threadIdx.x - lane), a.offsets,
                       a.n_tiles, a.inv, a.slots, s9);
        if (!vis) continue;
        any = true;
        const CamParams &cam = a.proj[v].cam;
        float vm[3] = {0.f, 0.f, 0.f}, vs[3] = {0.f, 0.f, 0.f}, vq[4] = {0.f, 0.f, 0.f, 0.f};
        V3 dir;
        projection_vjp(cam, a.means, a.scales, a.quats, a.glob_scale, a.splats + g, i, s9, vm, vs, vq, dir);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            gm[c] += vm[c];
            gsv[c] += vs[c];
            gdc[c] += SH_C0 * s9[5 + c];
        }
#pragma unroll
        for (int c = 0; c < 4; c++) gq[c] += vq[c];
        gop += s9[8];
        if (active > 0) {
            float bs[MAX_REST];
            sh_rest_basis(dir, bs);
#pragma unroll
            for (int k = 0; k < MAX_REST; k++) {
                if (k >= active) break;
#pragma unroll
                for (int c = 0; c < 3; c++) grest[3 * k + c] += bs[k] * s9[5 + c];
            }
        }
        st_vis += 1.0f;
        st_gn += sqrtf(s9[0] * s9[0] + s9[1] * s9[1]);
        st_ms = fmaxf(st_ms, (float)a.radii[g] * a.inv_max_dim[v]);
    }
    s_vis[threadIdx.x] = any ? 1 : 0;
    if (valid && a.vis_counts && any) {
        a.vis_counts[i] = st_vis;
        a.xys_grad_norm[i] = st_gn;
        a.max_2d_size[i] = st_ms;
    }
    if (valid && a.g[0]) {  // summed gradients (zero for Gaussians no view sees)
        for (int c = 0; c < 3; c++) {
            a.g[0][3 * (size_t)i + c] = gm[c];
            a.g[1][3 * (size_t)i + c] = gsv[c];
            a.g[3][3 * (size_t)i + c] = gdc[c];
        }
        for (int c = 0; c < 4; c++) a.g[2][4 * (size_t)i + c] = gq[c];
        a.g[5][i] = gop;
    }
    const float *ss = a.adam_scalars, *bc2 = a.adam_scalars + 6;
    if (valid && a.do_adam) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const size_t k = 3 * (size_t)i + c;
            adam_step(a.p[0][k], a.m1[0][k], a.m2[0][k], gm[c], ss[0], b1, b2, bc2[0], eps);
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const size_t k = 3 * (size_t)i + c;
            adam_step(a.p[1][k], a.m1[1][k], a.m2[1][k], gsv[c], ss[1], b1, b2, bc2[1], eps);
        }
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const size_t k = 4 * (size_t)i + c;
            adam_step(a.p[2][k], a.m1[2][k], a.m2[2][k], gq[c], ss[2], b1, b2, bc2[2], eps);
        }
        if (a.m1[5]) adam_step(a.p[5][i], a.m1[5][i], a.m2[5][i], gop, ss[5], b1, b2, bc2[5], eps);
        if (any) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const size_t k = 3 * (size_t)i + c;
                adam_step(a.p[3][k], a.m1[3][k], a.m2[3][k], gdc[c], ss[3], b1, b2, bc2[3], eps);
            }
        }
    }
    // SH rest: Adam (or the gradient) warp-cooperatively over the warp's 32 Gaussians
    if ((!a.do_adam && !a.g[4]) || a.rest_stride <= 0) return;
    __syncwarp();
    const int wbase_t = threadIdx.x - lane;
    const int64_t g0 = (int64_t)blockIdx.x * BWD_THREADS + wbase_t;
    const int stride = a.rest_stride;
    const int rows = (int)min((int64_t)32, (int64_t)a.n - g0);
    const size_t off = (size_t)g0 * stride;
    auto grad = [&](int r, int e) { return s_grest[wbase_t + r][e]; };
    if (a.g[4]) {  // every row: the summed gradient where used (zero where no view saw it)
        warp_rest_grad(a.g[4] + off, rows, stride, used, nullptr, grad);
    }
    if (!a.do_adam || active == 0) return;
    warp_rest_adam<REST_UNROLL>(a.p[4] + off, a.m1[4] + off, a.m2[4] + off, rows, stride, used, s_vis + wbase_t, grad,
                                ss[4], b1, b2, bc2[4], eps);
}

void launch_backward_adam_batch(const BackwardBatchArgs &a, cudaStream_t st) {
    if (a.n <= 0) return;
    backward_adam_batch_kernel<<<(a.n + BWD_THREADS - 1) / BWD_THREADS, BWD_THREADS, 0, st>>>(a);
}

}  // namespace msplat
