// CPU restatement of msplat's core/cpu backend -- TEST INFRASTRUCTURE ONLY.
//
// This file is the parity oracle for the CUDA product: tests run it on the same
// seeded inputs as the GPU path and compare. It restates, in code of its own, the
// algorithm of core/cpu/msplat_cpu.cpp (itself a kernel-by-kernel port of
// core/metal/msplat_metal.metal). Each function names the reference lines it
// follows. Floating-point expressions keep the reference's operation order, and the
// file is compiled with -ffp-contract=off, so it reproduces the reference's float
// results bit for bit; the test suite checks that against the reference's own
// backend (oracle/_ref) and against committed golden vectors.
//
// Matrices are column-major (M.c[col][row]) because the reference's math uses MSL
// semantics (core/cpu/cpu_math.hpp:1-4).

#include "msplat_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

// core/cpu/msplat_cpu.cpp:27 -- tile size
constexpr int TILE = 16;

// core/cpu/msplat_cpu.cpp:29-38 -- real SH basis constants
const float kC0 = 0.28209479177387814f;
const float kC1 = 0.4886025119029199f;
const float kC2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f, -1.0925484305920792f,
                      0.5462742152960396f};
const float kC3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f, 0.3731763325901154f,
                      -0.4570457994644658f, 1.445305721320277f, -0.5900435899266435f};
const float kC4[9] = {2.5033429417967046f, -1.7701307697799304f, 0.9461746957575601f, -0.6690465435572892f,
                      0.10578554691520431f, -0.6690465435572892f, 0.47308734787878004f, -1.7701307697799304f,
                      0.6258357354491761f};

// core/cpu/msplat_cpu.cpp:40-45 -- 11-tap Gaussian window, sigma 1.5
const float kWin[11] = {0.0010283801f, 0.0075987581f, 0.0360007721f, 0.1093606895f, 0.2130055377f, 0.2660117249f,
                        0.2130055377f, 0.1093606895f, 0.0360007721f, 0.0075987581f, 0.0010283801f};
const float kSsimC1 = 0.0001f, kSsimC2 = 0.0009f;

struct V2 { float x, y; };
struct V3 { float x, y, z; };
struct Q4 { float x, y, z, w; };  // memory order (w, x, y, z) lands in x, y, z, w

inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 scl(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 scl(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 ld3(const float *p, int64_t i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
inline V2 ld2(const float *p, int64_t i) { return {p[2 * i], p[2 * i + 1]}; }
inline void st3(float *p, int64_t i, V3 v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }
inline float clamp01(float v) { return std::min(std::max(v, 0.f), 1.f); }

struct M3 {
    V3 c[3];
};
inline M3 m3(float a0, float a1, float a2, float b0, float b1, float b2, float d0, float d1, float d2) {
    return M3{{{a0, a1, a2}, {b0, b1, b2}, {d0, d1, d2}}};
}
inline float &at(M3 &m, int col, int row) { return row == 0 ? m.c[col].x : (row == 1 ? m.c[col].y : m.c[col].z); }
inline float at(const M3 &m, int col, int row) { return row == 0 ? m.c[col].x : (row == 1 ? m.c[col].y : m.c[col].z); }
// Column-major product, summed over k in order 0,1,2 (core/cpu/cpu_math.hpp:112-118)
inline M3 mul(const M3 &A, const M3 &B) {
    M3 R;
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < 3; i++)
            at(R, j, i) = at(A, 0, i) * at(B, j, 0) + at(A, 1, i) * at(B, j, 1) + at(A, 2, i) * at(B, j, 2);
    return R;
}
inline M3 tr(const M3 &A) {
    return m3(A.c[0].x, A.c[1].x, A.c[2].x, A.c[0].y, A.c[1].y, A.c[2].y, A.c[0].z, A.c[1].z, A.c[2].z);
}
inline M3 plus(const M3 &A, const M3 &B) { return M3{{add(A.c[0], B.c[0]), add(A.c[1], B.c[1]), add(A.c[2], B.c[2])}}; }
inline M3 smul(float s, const M3 &A) { return M3{{scl(A.c[0], s), scl(A.c[1], s), scl(A.c[2], s)}}; }

uint32_t sh_bases(uint32_t degree) { return degree == 0 ? 1 : degree == 1 ? 4 : degree == 2 ? 9 : degree == 3 ? 16 : 25; }

// core/cpu/msplat_cpu.cpp:63-74 -- rows of a row-major 4x4 applied to (p, 1)
inline V3 xform43(const float *m, V3 p) {
    return {m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
            m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]};
}
struct V4 { float x, y, z, w; };
inline V4 xform44(const float *m, V3 p) {
    return {m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
            m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11], m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15]};
}

// core/cpu/msplat_cpu.cpp:77-84 -- rotation from the (w,x,y,z) quaternion, normalised
inline M3 rotmat(Q4 q) {
    float s = 1.f / std::sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    float w = q.x * s, x = q.y * s, y = q.z * s, z = q.w * s;
    return m3(1.f - 2.f * (y * y + z * z), 2.f * (x * y + w * z), 2.f * (x * z - w * y),
              2.f * (x * y - w * z), 1.f - 2.f * (x * x + z * z), 2.f * (y * z + w * x),
              2.f * (x * z + w * y), 2.f * (y * z - w * x), 1.f - 2.f * (x * x + y * y));
}
inline M3 diag_scale(V3 s, float g) {
    M3 S = m3(1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f);
    S.c[0].x = g * s.x;
    S.c[1].y = g * s.y;
    S.c[2].z = g * s.z;
    return S;
}
// core/cpu/msplat_cpu.cpp:94-100
inline void cov3d_of(V3 scale, float g, Q4 q, float *cov) {
    M3 M = mul(rotmat(q), diag_scale(scale, g));
    M3 t = mul(M, tr(M));
    cov[0] = t.c[0].x; cov[1] = t.c[0].y; cov[2] = t.c[0].z;
    cov[3] = t.c[1].y; cov[4] = t.c[1].z; cov[5] = t.c[2].z;
}

// core/cpu/msplat_cpu.cpp:103-125 -- EWA with the 1.3x FOV clamp and 0.3 px dilation
inline V3 ewa_cov2d(const float *cov, const float *vm, float fx, float fy, float tfx, float tfy, V3 pv) {
    float lx = 1.3f * tfx, ly = 1.3f * tfy;
    pv.x = pv.z * std::min(lx, std::max(-lx, pv.x / pv.z));
    pv.y = pv.z * std::min(ly, std::max(-ly, pv.y / pv.z));
    float rz = 1.f / pv.z, rz2 = rz * rz;
    float j00 = fx * rz, j11 = fy * rz;
    float j20 = -fx * pv.x * rz2, j21 = -fy * pv.y * rz2;
    V3 r0{vm[0], vm[1], vm[2]}, r1{vm[4], vm[5], vm[6]}, r2{vm[8], vm[9], vm[10]};
    V3 t0 = add(scl(j00, r0), scl(j20, r2));
    V3 t1 = add(scl(j11, r1), scl(j21, r2));
    V3 a{t0.x * cov[0] + t0.y * cov[1] + t0.z * cov[2], t0.x * cov[1] + t0.y * cov[3] + t0.z * cov[4],
         t0.x * cov[2] + t0.y * cov[4] + t0.z * cov[5]};
    V3 b{t1.x * cov[0] + t1.y * cov[1] + t1.z * cov[2], t1.x * cov[1] + t1.y * cov[3] + t1.z * cov[4],
         t1.x * cov[2] + t1.y * cov[4] + t1.z * cov[5]};
    return {dot3(a, t0) + 0.3f, dot3(a, t1), dot3(b, t1) + 0.3f};
}

// core/cpu/msplat_cpu.cpp:127-138
inline bool conic_radius(V3 cov2d, V3 &conic, float &radius) {
    float det = cov2d.x * cov2d.z - cov2d.y * cov2d.y;
    if (det == 0.f) return false;
    float inv = 1.f / det;
    conic = {cov2d.z * inv, -cov2d.y * inv, cov2d.x * inv};
    float b = 0.5f * (cov2d.x + cov2d.z);
    float disc = std::sqrt(std::max(0.1f, b * b - det));
    radius = std::ceil(3.f * std::sqrt(b + disc));
    return true;
}

// core/cpu/msplat_cpu.cpp:140-146
inline float to_pix(float x, float W, float c) { return 0.5f * W * x + c - 0.5f; }
inline V2 project_center(const float *P, V3 p, uint32_t w, uint32_t h, float cx, float cy) {
    V4 ph = xform44(P, p);
    float rw = 1.f / (ph.w + 1e-6f);
    return {to_pix(ph.x * rw, (float)(int)w, cx), to_pix(ph.y * rw, (float)(int)h, cy)};
}

// core/cpu/msplat_cpu.cpp:149-157 -- [x0,x1) x [y0,y1) in tiles, clamped
inline void tile_rect(V2 c, V2 r, int tx, int ty, int &x0, int &y0, int &x1, int &y1) {
    V2 cc{c.x / (float)TILE, c.y / (float)TILE};
    V2 rr{r.x / (float)TILE, r.y / (float)TILE};
    x0 = std::min(std::max(0, (int)(cc.x - rr.x)), tx);
    x1 = std::min(std::max(0, (int)(cc.x + rr.x + 1)), tx);
    y0 = std::min(std::max(0, (int)(cc.y - rr.y)), ty);
    y1 = std::min(std::max(0, (int)(cc.y + rr.y + 1)), ty);
}

// core/cpu/msplat_cpu.cpp:160-190 -- raw SH colour, no +0.5
void sh_color(uint32_t degree, V3 d, const float *dc, const float *rest, float *out) {
    for (int c = 0; c < 3; ++c) out[c] = kC0 * dc[c];
    if (degree < 1) return;
    float x = d.x, y = d.y, z = d.z;
    float xx = x * x, xy = x * y, xz = x * z, yy = y * y, yz = y * z, zz = z * z;
    for (int c = 0; c < 3; ++c) {
        const float *r = rest + c;
        out[c] += kC1 * (-y * r[0] + z * r[3] - x * r[6]);
        if (degree < 2) continue;
        out[c] += (kC2[0] * xy * r[9] + kC2[1] * yz * r[12] + kC2[2] * (2.f * zz - xx - yy) * r[15] +
                   kC2[3] * xz * r[18] + kC2[4] * (xx - yy) * r[21]);
        if (degree < 3) continue;
        out[c] += (kC3[0] * y * (3.f * xx - yy) * r[24] + kC3[1] * xy * z * r[27] +
                   kC3[2] * y * (4.f * zz - xx - yy) * r[30] + kC3[3] * z * (2.f * zz - 3.f * xx - 3.f * yy) * r[33] +
                   kC3[4] * x * (4.f * zz - xx - yy) * r[36] + kC3[5] * z * (xx - yy) * r[39] +
                   kC3[6] * x * (xx - 3.f * yy) * r[42]);
        if (degree < 4) continue;
        out[c] += (kC4[0] * xy * (xx - yy) * r[45] + kC4[1] * yz * (3.f * xx - yy) * r[48] +
                   kC4[2] * xy * (7.f * zz - 1.f) * r[51] + kC4[3] * yz * (7.f * zz - 3.f) * r[54] +
                   kC4[4] * (zz * (35.f * zz - 30.f) + 3.f) * r[57] + kC4[5] * xz * (7.f * zz - 3.f) * r[60] +
                   kC4[6] * (xx - yy) * (7.f * zz - 1.f) * r[63] + kC4[7] * xz * (xx - 3.f * yy) * r[66] +
                   kC4[8] * (xx * (xx - 3.f * yy) - yy * (3.f * xx - yy)) * r[69]);
    }
}

inline V3 unit(V3 a) { return scl(a, 1.f / std::sqrt(dot3(a, a))); }

// ---- backward helpers ---------------------------------------------------------

// core/cpu/msplat_cpu.cpp:197-205 -- through the perspective divide, with the w row
inline V3 center_vjp(const float *P, V3 p, uint32_t w, uint32_t h, V2 g) {
    V4 ph = xform44(P, p);
    float rw = 1.f / (ph.w + 1e-6f);
    V2 gn{0.5f * (float)w * g.x, 0.5f * (float)h * g.y};
    V4 gp{gn.x * rw, gn.y * rw, 0.f, -(gn.x * ph.x + gn.y * ph.y) * rw * rw};
    return {P[0] * gp.x + P[4] * gp.y + P[8] * gp.z + P[12] * gp.w, P[1] * gp.x + P[5] * gp.y + P[9] * gp.z + P[13] * gp.w,
            P[2] * gp.x + P[6] * gp.y + P[10] * gp.z + P[14] * gp.w};
}

// core/cpu/msplat_cpu.cpp:207-214 -- d(conic)/d(cov2d) = -X G X, 2x2 column-major
inline void conic_vjp(V3 conic, V3 g, float *out) {
    // X = [[a b][b d]], G likewise; P = X*G, Q = P*X, entries summed k=0,1 in order
    float X[2][2] = {{conic.x, conic.y}, {conic.y, conic.z}};
    float Gm[2][2] = {{g.x, g.y}, {g.y, g.z}};
    float P[2][2], Qm[2][2];
    for (int j = 0; j < 2; j++)
        for (int i = 0; i < 2; i++) P[j][i] = X[0][i] * Gm[j][0] + X[1][i] * Gm[j][1];
    for (int j = 0; j < 2; j++)
        for (int i = 0; i < 2; i++) Qm[j][i] = P[0][i] * X[j][0] + P[1][i] * X[j][1];
    float S[2][2];
    for (int j = 0; j < 2; j++)
        for (int i = 0; i < 2; i++) S[j][i] = Qm[j][i] * -1.f;
    out[0] = S[0][0];
    out[1] = S[1][0] + S[0][1];
    out[2] = S[1][1];
}

// core/cpu/msplat_cpu.cpp:216-255
inline void ewa_vjp(const float *cov, const float *vm, float fx, float fy, float tfx, float tfy, V3 gc2,
                    float *g_mean, float *g_cov3, V3 pv) {
    float lx = 1.3f * tfx, ly = 1.3f * tfy;
    pv.x = pv.z * std::min(lx, std::max(-lx, pv.x / pv.z));
    pv.y = pv.z * std::min(ly, std::max(-ly, pv.y / pv.z));
    float rz = 1.f / pv.z, rz2 = rz * rz;
    M3 W = m3(vm[0], vm[4], vm[8], vm[1], vm[5], vm[9], vm[2], vm[6], vm[10]);
    M3 J = m3(fx * rz, 0.f, 0.f, 0.f, fy * rz, 0.f, -fx * pv.x * rz2, -fy * pv.y * rz2, 0.f);
    M3 V = m3(cov[0], cov[1], cov[2], cov[1], cov[3], cov[4], cov[2], cov[4], cov[5]);
    M3 G = m3(gc2.x, 0.5f * gc2.y, 0.f, 0.5f * gc2.y, gc2.z, 0.f, 0.f, 0.f, 0.f);
    M3 T = mul(J, W);
    M3 gV = mul(mul(tr(T), G), T);
    M3 gT = plus(mul(mul(G, T), tr(V)), mul(mul(tr(G), T), V));
    g_cov3[0] = gV.c[0].x;
    g_cov3[1] = gV.c[0].y + gV.c[1].x;
    g_cov3[2] = gV.c[0].z + gV.c[2].x;
    g_cov3[3] = gV.c[1].y;
    g_cov3[4] = gV.c[1].z + gV.c[2].y;
    g_cov3[5] = gV.c[2].z;
    M3 gJ = mul(gT, tr(W));
    float fxr2 = fx * rz2, fyr2 = fy * rz2, rz3 = rz2 * rz;
    V3 gt{-fxr2 * gJ.c[2].x, -fyr2 * gJ.c[2].y,
          -fxr2 * gJ.c[0].x + 2.f * fx * pv.x * rz3 * gJ.c[2].x - fyr2 * gJ.c[1].y + 2.f * fy * pv.y * rz3 * gJ.c[2].y};
    g_mean[0] += dot3(gt, W.c[0]);
    g_mean[1] += dot3(gt, W.c[1]);
    g_mean[2] += dot3(gt, W.c[2]);
}

// core/cpu/msplat_cpu.cpp:259-274 -- tangent to the unit sphere
inline Q4 rotmat_vjp(Q4 q, const M3 &g) {
    float s = 1.f / std::sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    float w = q.x * s, x = q.y * s, y = q.z * s, z = q.w * s;
    auto G = [&](int col, int row) { return at(g, col, row); };
    Q4 r;
    r.x = 2.f * (x * (G(1, 2) - G(2, 1)) + y * (G(2, 0) - G(0, 2)) + z * (G(0, 1) - G(1, 0)));
    r.y = 2.f * (-2.f * x * (G(1, 1) + G(2, 2)) + y * (G(0, 1) + G(1, 0)) + z * (G(0, 2) + G(2, 0)) +
                 w * (G(1, 2) - G(2, 1)));
    r.z = 2.f * (x * (G(0, 1) + G(1, 0)) - 2.f * y * (G(0, 0) + G(2, 2)) + z * (G(1, 2) + G(2, 1)) +
                 w * (G(2, 0) - G(0, 2)));
    r.w = 2.f * (x * (G(0, 2) + G(2, 0)) + y * (G(1, 2) + G(2, 1)) - 2.f * z * (G(0, 0) + G(1, 1)) +
                 w * (G(0, 1) - G(1, 0)));
    float radial = r.x * w + r.y * x + r.z * y + r.w * z;
    return {(r.x - radial * w) * s, (r.y - radial * x) * s, (r.z - radial * y) * s, (r.w - radial * z) * s};
}

// core/cpu/msplat_cpu.cpp:276-291
inline void cov3d_vjp(V3 scale, float gs, Q4 q, const float *gc, float *g_scale, float *g_quat) {
    M3 gV = m3(gc[0], 0.5f * gc[1], 0.5f * gc[2], 0.5f * gc[1], gc[3], 0.5f * gc[4], 0.5f * gc[2], 0.5f * gc[4], gc[5]);
    M3 R = rotmat(q);
    M3 S = diag_scale(scale, gs);
    M3 M = mul(R, S);
    M3 gM = smul(2.f, mul(gV, M));
    g_scale[0] = dot3(R.c[0], gM.c[0]);
    g_scale[1] = dot3(R.c[1], gM.c[1]);
    g_scale[2] = dot3(R.c[2], gM.c[2]);
    Q4 r = rotmat_vjp(q, mul(gM, S));
    g_quat[0] = r.x; g_quat[1] = r.y; g_quat[2] = r.z; g_quat[3] = r.w;
}

// core/cpu/msplat_cpu.cpp:293-300
inline void adam(float &p, float &m1, float &m2, float g, float ss, float b1, float b2, float bc2, float eps) {
    float m = b1 * m1 + (1.0f - b1) * g;
    float v = b2 * m2 + (1.0f - b2) * g * g;
    p -= ss * m / (std::sqrt(v) / bc2 + eps);
    m1 = m;
    m2 = v;
}

// core/cpu/msplat_cpu.cpp:304-323 -- counter-based PCG hash RNG, Box-Muller normals
inline uint32_t pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
inline float unif(uint32_t seed, uint32_t ctr) {
    uint32_t h = pcg(seed ^ pcg(ctr));
    return ((float)(h >> 8) + 0.5f) * (1.0f / 16777216.0f);
}
inline V3 normal3(uint32_t seed, uint32_t stream) {
    uint32_t c = stream * 4u;
    float u0 = unif(seed, c), u1 = unif(seed, c + 1u), u2 = unif(seed, c + 2u), u3 = unif(seed, c + 3u);
    float r0 = std::sqrt(-2.0f * std::log(u0)), r1 = std::sqrt(-2.0f * std::log(u2));
    const float tau = 6.28318530717958647692f;
    float t0 = tau * u1, t1 = tau * u3;
    return {r0 * std::cos(t0), r0 * std::sin(t0), r1 * std::cos(t1)};
}

// ---- per-frame state (core/cpu/msplat_cpu.cpp:406-436) -------------------------

struct State {
    int n = 0;
    uint32_t W = 0, H = 0;
    int tx = 0, ty = 0;
    std::vector<float> xys, depths, conics, colors, aabb;
    std::vector<int32_t> radii;
    std::vector<int32_t> tile_start, tile_end, isect_gid;
    std::vector<float> pk_xyo, pk_conic, pk_rgb;
    std::vector<float> out_img, final_Ts;
    std::vector<int32_t> final_idx;
    std::vector<float> v_rendered, isect_grad;
    std::vector<float> v_xy, v_conic, v_rgb, v_opacity, v_mean3d, v_scale, v_quat;
    // prior-guided extras: expected-depth numerator, per-pixel background, dL/d(depth,
    // alpha) per pixel, per-Gaussian depth gradient, exposure-adjusted image and its
    // gradient
    bool aux = false;
    std::vector<float> out_depth, bg_img, v_aux, v_depth, out_adj, v_adj;
    // depth-chunked frames: tile t's chunks are items ch_first[t] .. ch_first[t + 1] - 1;
    // per (item, tile pixel q = row * 16 + column): the chunk's own transmittance,
    // colour and last contributor (-1 past the pixel's cut-off)
    bool chunked = false;
    std::vector<int32_t> ch_first, ch_last;
    std::vector<float> ch_T, ch_C;
};
State g;
bool g_has_prior = false;
orc_prior g_prior;

// ---- learned sky (core/cpu/msplat_cpu.cpp:329-402) --------------------------------

struct Sky {
    V3 up{0.f, 0.f, 0.f}, e1{0.f, 0.f, 0.f}, e2{0.f, 0.f, 0.f};
    float fx = 1.f, fy = 1.f, cx = 0.f, cy = 0.f;
    uint32_t w = 1, h = 1;
    bool on = false;
};

Sky make_sky(const orc_prior *p, float fx, float fy, float cx, float cy) {
    Sky s;
    s.fx = fx;
    s.fy = fy;
    s.cx = cx;
    s.cy = cy;
    if (p && p->aux && p->sky && p->sky_tex) {
        s.up = V3{p->sky_frame[0], p->sky_frame[1], p->sky_frame[2]};
        s.e1 = V3{p->sky_frame[3], p->sky_frame[4], p->sky_frame[5]};
        s.e2 = V3{p->sky_frame[6], p->sky_frame[7], p->sky_frame[8]};
        s.w = (uint32_t)p->sky_w;
        s.h = (uint32_t)p->sky_h;
        s.on = true;
    }
    return s;
}

// world direction of the ray through pixel (px, py); vm is world-to-camera
inline V3 ray_dir(float px, float py, const float *vm, const Sky &s) {
    const float dx = (px + 0.5f - s.cx) / s.fx, dy = (py + 0.5f - s.cy) / s.fy;
    return V3{vm[0] * dx + vm[4] * dy + vm[8], vm[1] * dx + vm[5] * dy + vm[9], vm[2] * dx + vm[6] * dy + vm[10]};
}

inline V2 sky_uv(V3 d, const Sky &s) {
    const float pi = 3.14159265358979323846f;
    d = scl(d, 1.f / std::sqrt(dot3(d, d)));
    const float el = std::asin(std::min(std::max(dot3(d, s.up), -1.f), 1.f));
    const float az = std::atan2(dot3(d, s.e2), dot3(d, s.e1));
    return V2{(az * (0.5f / pi) + 0.5f) * (float)s.w - 0.5f, (0.5f - el / pi) * (float)s.h - 0.5f};
}

// bilinear taps: longitude wraps, latitude clamps
struct Taps {
    uint32_t idx[4];
    float w[4];
};
inline Taps sky_taps(V2 uv, uint32_t w, uint32_t h) {
    const float u0f = std::floor(uv.x), fu = uv.x - u0f;
    int u0 = (int)u0f % (int)w;
    if (u0 < 0) u0 += (int)w;
    const int u1 = (u0 + 1) % (int)w;
    const float vc = std::min(std::max(uv.y, 0.f), (float)h - 1.f);
    const int v0 = (int)vc, v1 = std::min(v0 + 1, (int)h - 1);
    const float fv = vc - (float)v0;
    Taps t;
    t.idx[0] = (uint32_t)(v0 * (int)w + u0); t.w[0] = (1.f - fu) * (1.f - fv);
    t.idx[1] = (uint32_t)(v0 * (int)w + u1); t.w[1] = fu * (1.f - fv);
    t.idx[2] = (uint32_t)(v1 * (int)w + u0); t.w[2] = (1.f - fu) * fv;
    t.idx[3] = (uint32_t)(v1 * (int)w + u1); t.w[3] = fu * fv;
    return t;
}
inline V3 sky_sample(const float *tex, V2 uv, uint32_t w, uint32_t h) {
    const Taps t = sky_taps(uv, w, h);
    V3 c{0.f, 0.f, 0.f};
    for (int k = 0; k < 4; k++) c = add(scl(ld3(tex, t.idx[k]), t.w[k]), c);
    return c;
}

// core/cpu/msplat_cpu.cpp:452-500
void project(State &f, int N, const float *means, const float *scales, float gsc, const float *quats,
             const float *vm, const float *P, float fx, float fy, float cx, float cy, float clip,
             uint32_t degree, uint32_t dtu, const float *cam, const float *dc, const float *rest) {
    f.xys.resize((size_t)N * 2);
    f.depths.resize(N);
    f.conics.resize((size_t)N * 3);
    f.colors.resize((size_t)N * 3);
    f.aabb.resize((size_t)N * 2);
    f.radii.assign(std::max(N, 1), 0);
    const V3 cp{cam[0], cam[1], cam[2]};
    const uint32_t nb = sh_bases(degree);
    const uint32_t W = f.W, H = f.H;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        V3 pw = ld3(means, i);
        V3 pv = xform43(vm, pw);
        if (pv.z <= clip) continue;
        V3 ls = ld3(scales, i);
        V3 s{std::exp(ls.x), std::exp(ls.y), std::exp(ls.z)};
        Q4 q{quats[4 * i], quats[4 * i + 1], quats[4 * i + 2], quats[4 * i + 3]};
        float cov[6];
        cov3d_of(s, gsc, q, cov);
        float tfx = 0.5f * (float)W / fx, tfy = 0.5f * (float)H / fy;
        V3 c2 = ewa_cov2d(cov, vm, fx, fy, tfx, tfy, pv);
        V3 conic;
        float rad;
        if (!conic_radius(c2, conic, rad)) continue;
        st3(f.conics.data(), i, conic);
        V2 ctr = project_center(P, pw, W, H, cx, cy);
        float ax = std::ceil(3.0f * std::sqrt(c2.x));
        float ay = std::ceil(3.0f * std::sqrt(c2.z));
        int x0, y0, x1, y1;
        tile_rect(ctr, {ax, ay}, f.tx, f.ty, x0, y0, x1, y1);
        if ((x1 - x0) * (y1 - y0) <= 0) continue;
        f.depths[i] = pv.z;
        f.radii[i] = (int)rad;
        f.xys[2 * i] = ctr.x;
        f.xys[2 * i + 1] = ctr.y;
        f.aabb[2 * i] = ax;
        f.aabb[2 * i + 1] = ay;
        V3 dir = unit(sub(pw, cp));
        sh_color(dtu, dir, dc + 3 * (size_t)i, rest + (size_t)(nb - 1) * 3 * i, f.colors.data() + 3 * (size_t)i);
    }
}

// core/cpu/msplat_cpu.cpp:505-567 -- per-tile lists ordered by (depth bits, index),
// packed [x, y, sigmoid(opacity)], conic, rgb
void bin_sort(State &f, int N, const float *opac) {
    const int T = f.tx * f.ty;
    std::vector<int64_t> cnt(T + 1, 0);
    auto rect = [&](int i, int &x0, int &y0, int &x1, int &y1) {
        tile_rect(ld2(f.xys.data(), i), ld2(f.aabb.data(), i), f.tx, f.ty, x0, y0, x1, y1);
    };
    for (int i = 0; i < N; i++) {
        if (f.radii[i] <= 0) continue;
        int x0, y0, x1, y1;
        rect(i, x0, y0, x1, y1);
        for (int y = y0; y < y1; y++)
            for (int x = x0; x < x1; x++) cnt[y * f.tx + x + 1]++;
    }
    for (int t = 0; t < T; t++) cnt[t + 1] += cnt[t];
    const int64_t total = cnt[T];
    if (total > std::numeric_limits<int32_t>::max())
        throw std::runtime_error("more than 2^31 tile intersections");
    std::vector<uint64_t> bins(std::max<int64_t>(total, 1));
    std::vector<int64_t> cur(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < N; i++) {
        if (f.radii[i] <= 0) continue;
        int x0, y0, x1, y1;
        rect(i, x0, y0, x1, y1);
        uint32_t db;
        std::memcpy(&db, &f.depths[i], 4);
        uint64_t key = ((uint64_t)db << 32) | (uint32_t)i;
        for (int y = y0; y < y1; y++)
            for (int x = x0; x < x1; x++) bins[cur[y * f.tx + x]++] = key;
    }
    f.tile_start.assign(T, 0);
    f.tile_end.assign(T, 0);
    for (int t = 0; t < T; t++) {
        f.tile_start[t] = (int32_t)cnt[t];
        f.tile_end[t] = (int32_t)cnt[t + 1];
    }
    f.isect_gid.resize(std::max<int64_t>(total, 1));
    f.pk_xyo.resize(std::max<int64_t>(total, 1) * 3);
    f.pk_conic.resize(std::max<int64_t>(total, 1) * 3);
    f.pk_rgb.resize(std::max<int64_t>(total, 1) * 3);
#pragma omp parallel for schedule(dynamic, 8)
    for (int t = 0; t < T; t++) {
        std::sort(bins.begin() + cnt[t], bins.begin() + cnt[t + 1]);
        for (int64_t k = cnt[t]; k < cnt[t + 1]; k++) {
            int32_t gi = (int32_t)(bins[k] & 0xFFFFFFFFull);
            f.isect_gid[k] = gi;
            float o = 1.f / (1.f + std::exp(-opac[gi]));
            f.pk_xyo[3 * k] = f.xys[2 * (size_t)gi];
            f.pk_xyo[3 * k + 1] = f.xys[2 * (size_t)gi + 1];
            f.pk_xyo[3 * k + 2] = o;
            st3(f.pk_conic.data(), k, ld3(f.conics.data(), gi));
            st3(f.pk_rgb.data(), k, ld3(f.colors.data(), gi));
        }
    }
}

// core/cpu/msplat_cpu.cpp:569-571
inline float sigma_of(V3 conic, V2 d) {
    return 0.5f * (conic.x * d.x * d.x + conic.z * d.y * d.y) + conic.y * d.x * d.y;
}

// core/cpu/msplat_cpu.cpp:574-626; with f.aux also the expected-depth numerator
// sum_i z_i w_i and the per-pixel background (the learned sky when on)
void raster_fwd(State &f, const float *bg, const float *sky_tex = nullptr, const Sky *sky = nullptr,
                const float *vm = nullptr) {
    const int W = (int)f.W, H = (int)f.H, T = f.tx * f.ty;
    f.out_img.assign((size_t)W * H * 3, 0.f);
    f.final_Ts.assign((size_t)W * H, 0.f);
    f.final_idx.assign((size_t)W * H, 0);
    if (f.aux) {
        f.out_depth.assign((size_t)W * H, 0.f);
        f.bg_img.assign((size_t)W * H * 3, 0.f);
    }
    const bool use_sky = f.aux && sky && sky->on && sky_tex;
    const V3 b{bg[0], bg[1], bg[2]};
#pragma omp parallel for schedule(dynamic, 1)
    for (int t = 0; t < T; t++) {
        const int tx = t % f.tx, ty = t / f.tx;
        const int s = f.tile_start[t], e = f.tile_end[t];
        for (int i = ty * TILE; i < std::min(H, (ty + 1) * TILE); i++)
            for (int j = tx * TILE; j < std::min(W, (tx + 1) * TILE); j++) {
                const float px = (float)j, py = (float)i;
                float Tr = 1.f;
                V3 acc{0.f, 0.f, 0.f};
                float depth = 0.f;
                int last = s - 1;
                for (int k = s; k < e; k++) {
                    V3 xyo = ld3(f.pk_xyo.data(), k);
                    float sg = sigma_of(ld3(f.pk_conic.data(), k), {xyo.x - px, xyo.y - py});
                    if (sg < 0.f || sg >= 5.55f) continue;
                    float a = std::min(0.999f, xyo.z * std::exp(-sg));
                    if (a < 1.f / 255.f) continue;
                    float nT = Tr * (1.f - a);
                    if (nT <= 1e-4f) {
                        last = k - 1;
                        break;
                    }
                    float vis = a * Tr;
                    V3 rgb = ld3(f.pk_rgb.data(), k);
                    V3 c{std::max(rgb.x + 0.5f, 0.f), std::max(rgb.y + 0.5f, 0.f), std::max(rgb.z + 0.5f, 0.f)};
                    acc = add(scl(c, vis), acc);
                    if (f.aux) depth += f.depths[f.isect_gid[k]] * vis;
                    Tr = nT;
                    last = k;
                }
                const size_t pid = (size_t)i * W + j;
                f.final_Ts[pid] = Tr;
                f.final_idx[pid] = last;
                V3 bp = b;
                if (use_sky) bp = sky_sample(sky_tex, sky_uv(ray_dir(px, py, vm, *sky), *sky), sky->w, sky->h);
                if (f.aux) {
                    f.out_depth[pid] = depth;
                    st3(f.bg_img.data(), (int64_t)pid, bp);
                }
                V3 o = add(scl(bp, Tr), acc);
                f.out_img[3 * pid] = clamp01(o.x);
                f.out_img[3 * pid + 1] = clamp01(o.y);
                f.out_img[3 * pid + 2] = clamp01(o.z);
            }
    }
}

// ---- depth-chunked compositing (core/metal/msplat_metal.metal:2641-3030) -------------
//
// Test-visible switch (orc_set_option "chunk_size"): 0 composites each tile's list in
// one pass (the CPU backend); C > 0 splits every tile's list into C-long depth chunks
// (the Metal backend's path for frames of fewer than 400 tiles, chunk length 512,
// core/metal/msplat_metal.mm:1101-1117), each composited from T = 1 with its own
// early stop, then merged per pixel front to back. Within a chunk the arithmetic is
// the one-pass loop's; the merge, prefix and suffix use the Metal kernels' formulas
// (fma where they write fma). Every chunk of a tile is kept: the Metal path sizes its
// chunk count from six times the mean list length and drops entries past it; here a
// tile has ceil(len / C) chunks.
int g_chunk = 0;

// Chunk k of a tile whose list is [s, e): [s + k C, min(s + (k + 1) C, e)).
void raster_fwd_chunked(State &f, const float *bg) {
    const int W = (int)f.W, H = (int)f.H, T = f.tx * f.ty, C = g_chunk;
    f.out_img.assign((size_t)W * H * 3, 0.f);
    f.final_Ts.assign((size_t)W * H, 0.f);
    f.final_idx.assign((size_t)W * H, 0);
    f.ch_first.assign((size_t)T + 1, 0);
    for (int t = 0; t < T; t++) f.ch_first[t + 1] = f.ch_first[t] + (f.tile_end[t] - f.tile_start[t] + C - 1) / C;
    const size_t items = (size_t)f.ch_first[T];
    f.ch_T.assign(items * 256, 1.f);
    f.ch_C.assign(items * 256 * 3, 0.f);
    f.ch_last.assign(items * 256, -1);
    const V3 b{bg[0], bg[1], bg[2]};
#pragma omp parallel for schedule(dynamic, 1)
    for (int t = 0; t < T; t++) {
        const int tx = t % f.tx, ty = t / f.tx;
        const int s = f.tile_start[t], e = f.tile_end[t], i0 = f.ch_first[t], nch = f.ch_first[t + 1] - i0;
        for (int i = ty * TILE; i < std::min(H, (ty + 1) * TILE); i++)
            for (int j = tx * TILE; j < std::min(W, (tx + 1) * TILE); j++) {
                const float px = (float)j, py = (float)i;
                const size_t q = (size_t)(i - ty * TILE) * TILE + (j - tx * TILE);
                // rasterize_forward_chunked_kernel (.metal:2641-2736): each chunk alone
                for (int k = 0; k < nch; k++) {
                    const int cs = s + k * C, ce = std::min(cs + C, e);
                    float Tr = 1.f;
                    V3 acc{0.f, 0.f, 0.f};
                    int last = cs - 1;
                    for (int kk = cs; kk < ce; kk++) {
                        V3 xyo = ld3(f.pk_xyo.data(), kk);
                        float sg = sigma_of(ld3(f.pk_conic.data(), kk), {xyo.x - px, xyo.y - py});
                        if (sg < 0.f || sg >= 5.55f) continue;
                        float a = std::min(0.999f, xyo.z * std::exp(-sg));
                        if (a < 1.f / 255.f) continue;
                        float nT = Tr * (1.f - a);
                        if (nT <= 1e-4f) {
                            last = kk - 1;
                            break;
                        }
                        float vis = a * Tr;
                        V3 rgb = ld3(f.pk_rgb.data(), kk);
                        V3 c{std::max(rgb.x + 0.5f, 0.f), std::max(rgb.y + 0.5f, 0.f), std::max(rgb.z + 0.5f, 0.f)};
                        acc = add(scl(c, vis), acc);
                        Tr = nT;
                        last = kk;
                    }
                    const size_t it = (size_t)(i0 + k) * 256 + q;
                    f.ch_T[it] = Tr;
                    f.ch_C[3 * it] = acc.x;
                    f.ch_C[3 * it + 1] = acc.y;
                    f.ch_C[3 * it + 2] = acc.z;
                    f.ch_last[it] = last;
                }
                // rasterize_forward_merge_kernel (.metal:2741-2808): front to back, stop
                // once T <= 1e-4; the chunks past the stop lose their contributors
                float Tr = 1.f;
                V3 acc{0.f, 0.f, 0.f};
                int last = -1, cut = nch;
                for (int k = 0; k < nch; k++) {
                    const size_t it = (size_t)(i0 + k) * 256 + q;
                    acc.x = std::fma(f.ch_C[3 * it], Tr, acc.x);
                    acc.y = std::fma(f.ch_C[3 * it + 1], Tr, acc.y);
                    acc.z = std::fma(f.ch_C[3 * it + 2], Tr, acc.z);
                    Tr *= f.ch_T[it];
                    if (f.ch_last[it] >= 0) last = f.ch_last[it];
                    if (Tr <= 1e-4f) {
                        cut = k + 1;
                        break;
                    }
                }
                for (int k = cut; k < nch; k++) f.ch_last[(size_t)(i0 + k) * 256 + q] = -1;
                const size_t pid = (size_t)i * W + j;
                f.final_Ts[pid] = Tr;
                f.final_idx[pid] = last;
                f.out_img[3 * pid] = clamp01(std::fma(b.x, Tr, acc.x));
                f.out_img[3 * pid + 1] = clamp01(std::fma(b.y, Tr, acc.y));
                f.out_img[3 * pid + 2] = clamp01(std::fma(b.z, Tr, acc.z));
            }
    }
}

// core/cpu/msplat_cpu.cpp:629-657
void forward(State &f, int N, const float *means, const float *scales, float gsc, const float *quats,
             const float *vm, const float *P, float fx, float fy, float cx, float cy, unsigned H, unsigned W,
             int tx, int ty, float clip, unsigned degree, unsigned dtu, const float *cam, const float *dc,
             const float *rest, const float *opac, const float *bg) {
    f.n = N;
    f.W = W;
    f.H = H;
    f.tx = tx;
    f.ty = ty;
    const orc_prior *pr = g_has_prior ? &g_prior : nullptr;
    f.aux = pr && pr->aux;
    project(f, N, means, scales, gsc, quats, vm, P, fx, fy, cx, cy, clip, degree, dtu, cam, dc, rest);
    bin_sort(f, N, opac);
    const Sky sky = make_sky(pr, fx, fy, cx, cy);
    f.chunked = g_chunk > 0 && !f.aux;  // the aux rasterizer is one-pass only (as in Metal)
    if (f.chunked)
        raster_fwd_chunked(f, bg);
    else
        raster_fwd(f, bg, sky.on ? pr->sky_tex : nullptr, &sky, vm);
}

// core/cpu/msplat_cpu.cpp:669-785 -- zero-padded separable SSIM + L1, forward and
// backward in three row passes. Returns the summed per-pixel loss (double).
double ssim_loss(const float *r, const float *gt, uint32_t W, uint32_t H, float w, float inv_n, float *v_out) {
    std::vector<float> hb((size_t)W * H * 15), dv((size_t)W * H * 15);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < (int)H; y++)
        for (uint32_t x = 0; x < W; x++)
            for (int c = 0; c < 3; c++) {
                float m[5] = {0, 0, 0, 0, 0};
                for (int k = 0; k < 11; k++) {
                    int gx = (int)x - 5 + k;
                    float gv = 0.f, rv = 0.f;
                    if (gx >= 0 && gx < (int)W) {
                        size_t idx = ((size_t)y * W + gx) * 3 + c;
                        gv = gt[idx];
                        rv = r[idx];
                    }
                    float wk = kWin[k];
                    m[0] += wk * gv;
                    m[1] += wk * rv;
                    m[2] += wk * gv * gv;
                    m[3] += wk * rv * rv;
                    m[4] += wk * gv * rv;
                }
                std::memcpy(&hb[((size_t)y * W + x) * 15 + c * 5], m, sizeof m);
            }
    std::vector<double> rows(H, 0.0);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < (int)H; y++) {
        const int ext = (int)W + 10;
        std::vector<float> f1(ext), f2(ext), f3(ext), sp(W, 0.f), lp(W, 0.f);
        for (int c = 0; c < 3; c++) {
            for (int xe = 0; xe < ext; xe++) {
                const int xp = xe - 5;
                if (xp < 0 || xp >= (int)W) {
                    f1[xe] = f2[xe] = f3[xe] = 0.f;
                    continue;
                }
                float s[5] = {0, 0, 0, 0, 0};
                for (int k = 0; k < 11; k++) {
                    int gy = y - 5 + k;
                    if (gy < 0 || gy >= (int)H) continue;
                    const float *h = &hb[((size_t)gy * W + xp) * 15 + c * 5];
                    for (int q = 0; q < 5; q++) s[q] += kWin[k] * h[q];
                }
                float mx = s[0], my = s[1], sxx = s[2], syy = s[3], sxy = s[4];
                float vx = sxx - mx * mx, vy = syy - my * my, cv = sxy - mx * my;
                float A = 2.0f * mx * my + kSsimC1, B = 2.0f * cv + kSsimC2;
                float Cd = mx * mx + my * my + kSsimC1, D = vx + vy + kSsimC2;
                float iCD = 1.0f / (Cd * D);
                float dmu = 2.0f * B * (mx * Cd - A * my) / (Cd * Cd * D);
                float dsyq = -A * B * iCD / D, dsxy = 2.0f * A * iCD;
                f1[xe] = dmu - 2.0f * my * dsyq - mx * dsxy;
                f2[xe] = 2.0f * dsyq;
                f3[xe] = dsxy;
                size_t i = ((size_t)y * W + xp) * 3 + c;
                sp[xp] += (A * B) / (Cd * D);
                lp[xp] += std::fabs(gt[i] - r[i]);
            }
            for (uint32_t x = 0; x < W; x++) {
                float h1 = 0, h2 = 0, h3 = 0;
                for (int d = 0; d < 11; d++) {
                    float wk = kWin[10 - d];
                    h1 += wk * f1[x + d];
                    h2 += wk * f2[x + d];
                    h3 += wk * f3[x + d];
                }
                float *o = &dv[((size_t)y * W + x) * 15 + c * 5];
                o[0] = h1; o[1] = h2; o[2] = h3;
            }
        }
        double sum = 0.0;
        for (uint32_t x = 0; x < W; x++) sum += w * (1.0f - sp[x] / 3.0f) + (1.0f - w) * lp[x] / 3.0f;
        rows[y] = sum;
    }
    double total = 0.0;
    for (double v : rows) total += v;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < (int)H; y++)
        for (uint32_t x = 0; x < W; x++)
            for (int c = 0; c < 3; c++) {
                float a1 = 0, a2 = 0, a3 = 0;
                for (int d = 0; d < 11; d++) {
                    int gy = y - 5 + d;
                    if (gy < 0 || gy >= (int)H) continue;
                    const float *dd = &dv[((size_t)gy * W + x) * 15 + c * 5];
                    float wk = kWin[10 - d];
                    a1 += wk * dd[0];
                    a2 += wk * dd[1];
                    a3 += wk * dd[2];
                }
                size_t i = ((size_t)y * W + x) * 3 + c;
                float rv = r[i], gv = gt[i];
                float vs = a1 + rv * a2 + gv * a3;
                float vl = (gv > rv) ? -1.0f : ((gv < rv) ? 1.0f : 0.0f);
                v_out[i] = inv_n * (-w * vs + (1.0f - w) * vl);
            }
    return total;
}

constexpr int GS = 10;  // per-intersection slot: xy(2) conic(3) rgb(3) opacity depth

// Test-only switch: visit a tile's pixels (and a Gaussian's slots) in reverse order
// in the backward pass. The result is the same sum in another float rounding order,
// which measures how far summation order alone moves the reference's gradients.
bool g_reverse_sums = false;

// core/cpu/msplat_cpu.cpp:959-1031 -- back to front, T recovered by division;
// per-intersection slots accumulated over the tile's pixels. With f.aux the pixel's
// background is its own (bg_img) and the expected depth / alpha gradients (v_aux)
// enter v_alpha and slot 9.
void raster_bwd(State &f, const float *bg, const float *v_img) {
    const int W = (int)f.W, H = (int)f.H, T = f.tx * f.ty;
    const int64_t total = T ? f.tile_end[T - 1] : 0;
    f.isect_grad.assign((size_t)std::max<int64_t>(total, 1) * GS, 0.f);
    const V3 b{bg[0], bg[1], bg[2]};
#pragma omp parallel for schedule(dynamic, 1)
    for (int t = 0; t < T; t++) {
        const int s = f.tile_start[t], e = f.tile_end[t];
        if (e == s) continue;
        float *lv = f.isect_grad.data() + (size_t)s * GS;
        const int tx = t % f.tx, ty = t / f.tx;
        const int i0 = ty * TILE, i1 = std::min(H, (ty + 1) * TILE), j0 = tx * TILE, j1 = std::min(W, (tx + 1) * TILE);
        const int npx = (i1 - i0) * (j1 - j0);
        for (int pi = 0; pi < npx; pi++) {
                const int q = g_reverse_sums ? npx - 1 - pi : pi;
                const int i = i0 + q / (j1 - j0), j = j0 + q % (j1 - j0);
                const size_t pid = (size_t)i * W + j;
                const float px = (float)j, py = (float)i;
                const float Tf = f.final_Ts[pid];
                float Tr = Tf;
                V3 buf{0.f, 0.f, 0.f};
                float buf_d = 0.f, buf_a = 0.f;
                const int kf = f.final_idx[pid];
                const V3 vo = ld3(v_img, pid);
                const float vd = f.aux ? f.v_aux[2 * pid] : 0.f, vaa = f.aux ? f.v_aux[2 * pid + 1] : 0.f;
                const V3 Tbg = scl(Tf, f.aux ? ld3(f.bg_img.data(), (int64_t)pid) : b);
                for (int k = std::min(kf, e - 1); k >= s; k--) {
                    V3 xyo = ld3(f.pk_xyo.data(), k);
                    V3 cn = ld3(f.pk_conic.data(), k);
                    V2 d{xyo.x - px, xyo.y - py};
                    float sg = sigma_of(cn, d);
                    if (sg < 0.f || sg >= 5.55f) continue;
                    float a = std::min(0.999f, xyo.z * std::exp(-sg));
                    if (a < 1.f / 255.f) continue;
                    float ra = 1.f / (1.f - a);
                    Tr *= ra;
                    const float fac = a * Tr;
                    const V3 raw = ld3(f.pk_rgb.data(), k);
                    const V3 rgb{std::max(raw.x + 0.5f, 0.f), std::max(raw.y + 0.5f, 0.f), std::max(raw.z + 0.5f, 0.f)};
                    // fma3(rgb, T, fma3(-buffer, ra, -ra * T_final_bg))
                    V3 nb{-buf.x, -buf.y, -buf.z};
                    V3 inner = add(scl(nb, ra), scl(-ra, Tbg));
                    V3 outer = add(scl(rgb, Tr), inner);
                    float va = dot3(outer, vo);
                    float z = 0.f;
                    if (f.aux) {
                        z = f.depths[f.isect_gid[k]];
                        va += (z * Tr - buf_d * ra) * vd + (Tr - buf_a * ra) * vaa;
                    }
                    buf = add(scl(rgb, fac), buf);
                    float *gg = lv + (size_t)(k - s) * GS;
                    if (raw.x + 0.5f >= 0.f) gg[5] += fac * vo.x;
                    if (raw.y + 0.5f >= 0.f) gg[6] += fac * vo.y;
                    if (raw.z + 0.5f >= 0.f) gg[7] += fac * vo.z;
                    if (f.aux) {
                        buf_d += z * fac;
                        buf_a += fac;
                        gg[9] += fac * vd;
                    }
                    if (a < 0.999f) {
                        const float vs = -a * va;
                        gg[2] += 0.5f * vs * d.x * d.x;
                        gg[3] += 0.5f * vs * d.x * d.y;
                        gg[4] += 0.5f * vs * d.y * d.y;
                        gg[0] += vs * (cn.x * d.x + cn.y * d.y);
                        gg[1] += vs * (cn.y * d.x + cn.z * d.y);
                        gg[8] += -vs * (1.f - xyo.z);
                    }
                }
            }
    }
}

// Backward of a depth-chunked frame: compute_chunk_prefix_suffix_kernel
// (.metal:2812-2848) gives each chunk the transmittance in front of it and the colour
// behind it (every later chunk of the tile, those past the cut-off included, as
// there), and rasterize_backward_chunked_kernel (:2852-3030) walks the chunk back to
// front from its own last contributor, starting from T = prefix * chunk T and that
// colour. The per-Gaussian arithmetic is the one-pass backward's.
void raster_bwd_chunked(State &f, const float *bg, const float *v_img) {
    const int W = (int)f.W, H = (int)f.H, T = f.tx * f.ty, C = g_chunk;
    const int64_t total = T ? f.tile_end[T - 1] : 0;
    f.isect_grad.assign((size_t)std::max<int64_t>(total, 1) * GS, 0.f);
    const V3 b{bg[0], bg[1], bg[2]};
#pragma omp parallel for schedule(dynamic, 1)
    for (int t = 0; t < T; t++) {
        const int s = f.tile_start[t], e = f.tile_end[t], i0 = f.ch_first[t], nch = f.ch_first[t + 1] - i0;
        if (e == s) continue;
        const int tx = t % f.tx, ty = t / f.tx;
        const int r0 = ty * TILE, r1 = std::min(H, (ty + 1) * TILE), c0 = tx * TILE, c1 = std::min(W, (tx + 1) * TILE);
        const int npx = (r1 - r0) * (c1 - c0);
        std::vector<float> pre(nch), aft(3 * (size_t)nch);
        for (int k = 0; k < nch; k++) {
            const int cs = s + k * C, ce = std::min(cs + C, e);
            float *lv = f.isect_grad.data() + (size_t)cs * GS;
            for (int pi = 0; pi < npx; pi++) {
                const int qq = g_reverse_sums ? npx - 1 - pi : pi;
                const int i = r0 + qq / (c1 - c0), j = c0 + qq % (c1 - c0);
                const size_t q = (size_t)(i - r0) * TILE + (j - c0);
                // prefix and suffix of this pixel's chunks
                float pT = 1.f;
                for (int m = 0; m < nch; m++) {
                    pre[m] = pT;
                    pT *= f.ch_T[(size_t)(i0 + m) * 256 + q];
                }
                V3 aC{0.f, 0.f, 0.f};
                for (int m = nch - 1; m >= 0; m--) {
                    aft[3 * m] = aC.x;
                    aft[3 * m + 1] = aC.y;
                    aft[3 * m + 2] = aC.z;
                    const size_t it = (size_t)(i0 + m) * 256 + q;
                    aC.x += pre[m] * f.ch_C[3 * it];
                    aC.y += pre[m] * f.ch_C[3 * it + 1];
                    aC.z += pre[m] * f.ch_C[3 * it + 2];
                }
                const size_t it = (size_t)(i0 + k) * 256 + q;
                const int kf = f.ch_last[it];
                if (kf < cs) continue;  // no contributor in this chunk (or past the cut-off)
                const size_t pid = (size_t)i * W + j;
                const float px = (float)j, py = (float)i;
                const float Tf = f.final_Ts[pid];
                float Tr = pre[k] * f.ch_T[it];
                V3 buf{aft[3 * k], aft[3 * k + 1], aft[3 * k + 2]};
                const V3 vo = ld3(v_img, pid);
                const V3 Tbg = scl(Tf, b);
                for (int kk = std::min(kf, ce - 1); kk >= cs; kk--) {
                    V3 xyo = ld3(f.pk_xyo.data(), kk);
                    V3 cn = ld3(f.pk_conic.data(), kk);
                    V2 d{xyo.x - px, xyo.y - py};
                    float sg = sigma_of(cn, d);
                    if (sg < 0.f || sg >= 5.55f) continue;
                    float a = std::min(0.999f, xyo.z * std::exp(-sg));
                    if (a < 1.f / 255.f) continue;
                    float ra = 1.f / (1.f - a);
                    Tr *= ra;
                    const float fac = a * Tr;
                    const V3 raw = ld3(f.pk_rgb.data(), kk);
                    const V3 rgb{std::max(raw.x + 0.5f, 0.f), std::max(raw.y + 0.5f, 0.f), std::max(raw.z + 0.5f, 0.f)};
                    V3 nb{-buf.x, -buf.y, -buf.z};
                    V3 inner = add(scl(nb, ra), scl(-ra, Tbg));
                    V3 outer = add(scl(rgb, Tr), inner);
                    float va = dot3(outer, vo);
                    buf = add(scl(rgb, fac), buf);
                    float *gg = lv + (size_t)(kk - cs) * GS;
                    if (raw.x + 0.5f >= 0.f) gg[5] += fac * vo.x;
                    if (raw.y + 0.5f >= 0.f) gg[6] += fac * vo.y;
                    if (raw.z + 0.5f >= 0.f) gg[7] += fac * vo.z;
                    if (a < 0.999f) {
                        const float vs = -a * va;
                        gg[2] += 0.5f * vs * d.x * d.x;
                        gg[3] += 0.5f * vs * d.x * d.y;
                        gg[4] += 0.5f * vs * d.y * d.y;
                        gg[0] += vs * (cn.x * d.x + cn.y * d.y);
                        gg[1] += vs * (cn.y * d.x + cn.z * d.y);
                        gg[8] += -vs * (1.f - xyo.z);
                    }
                }
            }
        }
    }
}

// core/cpu/msplat_cpu.cpp:1034-1064 -- sums of the slots per Gaussian in k order
void reduce_slots(State &f, int N) {
    const int T = f.tx * f.ty;
    const int64_t total = T ? f.tile_end[T - 1] : 0;
    std::vector<int32_t> off((size_t)N + 1, 0), lst(std::max<int64_t>(total, 1));
    for (int64_t k = 0; k < total; k++) off[f.isect_gid[k] + 1]++;
    for (int i = 0; i < N; i++) off[i + 1] += off[i];
    {
        std::vector<int32_t> cur(off.begin(), off.end() - 1);
        for (int64_t k = 0; k < total; k++) lst[cur[f.isect_gid[k]]++] = (int32_t)k;
    }
    f.v_xy.assign((size_t)N * 2, 0.f);
    f.v_conic.assign((size_t)N * 3, 0.f);
    f.v_rgb.assign((size_t)N * 3, 0.f);
    f.v_opacity.assign(N, 0.f);
    f.v_depth.assign(N, 0.f);
#pragma omp parallel for schedule(static)
    for (int gi = 0; gi < N; gi++) {
        float s[GS] = {0};
        for (int32_t qq = off[gi]; qq < off[gi + 1]; qq++) {
            const int32_t q = g_reverse_sums ? off[gi + 1] - 1 - (qq - off[gi]) : qq;
            const float *v = f.isect_grad.data() + (size_t)lst[q] * GS;
            for (int c = 0; c < GS; c++) s[c] += v[c];
        }
        f.v_xy[2 * gi] = s[0]; f.v_xy[2 * gi + 1] = s[1];
        f.v_conic[3 * gi] = s[2]; f.v_conic[3 * gi + 1] = s[3]; f.v_conic[3 * gi + 2] = s[4];
        f.v_rgb[3 * gi] = s[5]; f.v_rgb[3 * gi + 1] = s[6]; f.v_rgb[3 * gi + 2] = s[7];
        f.v_opacity[gi] = s[8];
        f.v_depth[gi] = s[9];
    }
}

// core/cpu/msplat_cpu.cpp:1068-1139 -- projection VJPs; SH backward fused into Adam
void proj_bwd_adam(State &f, int N, const float *means, const float *scales, float gsc, const float *quats,
                   const float *vm, const float *P, float fx, float fy, uint32_t degree, uint32_t dtu,
                   const float *cam, float *dc, float *rest, float *dc1, float *dc2, float *re1, float *re2,
                   float dss, float dbc, float rss, float rbc, float b1, float b2, float eps) {
    f.v_mean3d.assign((size_t)N * 3, 0.f);
    f.v_scale.assign((size_t)N * 3, 0.f);
    f.v_quat.assign((size_t)N * 4, 0.f);
    const uint32_t W = f.W, H = f.H;
    const V3 cp{cam[0], cam[1], cam[2]};
    const uint32_t nb = sh_bases(degree);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        float *gm = f.v_mean3d.data() + 3 * (size_t)i;
        float *gsv = f.v_scale.data() + 3 * (size_t)i;
        float *gq = f.v_quat.data() + 4 * (size_t)i;
        if (f.radii[i] <= 0) continue;
        V3 pw = ld3(means, i);
        V3 vmn = center_vjp(P, pw, W, H, ld2(f.v_xy.data(), i));
        vmn = add(vmn, scl(V3{vm[8], vm[9], vm[10]}, f.v_depth[i]));  // zero without priors
        gm[0] = vmn.x; gm[1] = vmn.y; gm[2] = vmn.z;
        float gc2[3];
        conic_vjp(ld3(f.conics.data(), i), ld3(f.v_conic.data(), i), gc2);
        V3 ls = ld3(scales, i);
        V3 es{std::exp(ls.x), std::exp(ls.y), std::exp(ls.z)};
        Q4 q{quats[4 * i], quats[4 * i + 1], quats[4 * i + 2], quats[4 * i + 3]};
        float cov[6];
        cov3d_of(es, gsc, q, cov);
        float tfx = 0.5f * (float)W / fx, tfy = 0.5f * (float)H / fy;
        V3 pv = xform43(vm, pw);
        float gc3[6];
        ewa_vjp(cov, vm, fx, fy, tfx, tfy, {gc2[0], gc2[1], gc2[2]}, gm, gc3, pv);
        cov3d_vjp(es, gsc, q, gc3, gsv, gq);
        gsv[0] *= es.x; gsv[1] *= es.y; gsv[2] *= es.z;

        V3 d = unit(sub(pw, cp));
        const size_t di = 3 * (size_t)i, ri = (size_t)(nb - 1) * 3 * i;
        const float vc[3] = {f.v_rgb[3 * i], f.v_rgb[3 * i + 1], f.v_rgb[3 * i + 2]};
        for (int c = 0; c < 3; c++) adam(dc[di + c], dc1[di + c], dc2[di + c], kC0 * vc[c], dss, b1, b2, dbc, eps);
        if (dtu < 1) continue;
        float x = d.x, y = d.y, z = d.z;
        float xx = x * x, xy = x * y, xz = x * z, yy = y * y, yz = y * z, zz = z * z;
        auto up = [&](int base, float sh) {
            for (int c = 0; c < 3; c++) {
                size_t k = ri + (size_t)base * 3 + c;
                adam(rest[k], re1[k], re2[k], sh * vc[c], rss, b1, b2, rbc, eps);
            }
        };
        up(0, -kC1 * y); up(1, kC1 * z); up(2, -kC1 * x);
        if (dtu < 2) continue;
        up(3, kC2[0] * xy); up(4, kC2[1] * yz); up(5, kC2[2] * (2.f * zz - xx - yy));
        up(6, kC2[3] * xz); up(7, kC2[4] * (xx - yy));
        if (dtu < 3) continue;
        up(8, kC3[0] * y * (3.f * xx - yy)); up(9, kC3[1] * xy * z);
        up(10, kC3[2] * y * (4.f * zz - xx - yy)); up(11, kC3[3] * z * (2.f * zz - 3.f * xx - 3.f * yy));
        up(12, kC3[4] * x * (4.f * zz - xx - yy)); up(13, kC3[5] * z * (xx - yy));
        up(14, kC3[6] * x * (xx - 3.f * yy));
    }
}

// core/cpu/msplat_cpu.cpp:1142-1147
void adam_dense(float *p, const float *gr, float *m1, float *m2, size_t n, float ss, float b1, float b2, float bc2,
                float eps) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) adam(p[i], m1[i], m2[i], gr[i], ss, b1, b2, bc2, eps);
}

// ---- prior-guided extras (core/cpu/msplat_cpu.cpp:787-950, :1295-1309) ------------

// prior depth, bilinear unless the four samples straddle a depth edge (then nearest)
float prior_depth_at(const float *d, float x, float y, uint32_t w, uint32_t h) {
    x = std::min(std::max(x, 0.f), (float)w - 1.f);
    y = std::min(std::max(y, 0.f), (float)h - 1.f);
    const uint32_t x0 = (uint32_t)x, y0 = (uint32_t)y;
    const uint32_t x1 = std::min(x0 + 1, w - 1), y1 = std::min(y0 + 1, h - 1);
    const float fx = x - (float)x0, fy = y - (float)y0;
    const float d00 = d[y0 * w + x0], d01 = d[y0 * w + x1], d10 = d[y1 * w + x0], d11 = d[y1 * w + x1];
    const float lo = std::min(std::min(d00, d01), std::min(d10, d11));
    const float hi = std::max(std::max(d00, d01), std::max(d10, d11));
    if (lo <= 0.f || hi > 1.05f * lo) return d[((fy < 0.5f) ? y0 : y1) * w + ((fx < 0.5f) ? x0 : x1)];
    const float top = d00 + (d01 - d00) * fx, bot = d10 + (d11 - d10) * fx;
    return top + (bot - top) * fy;
}

// Depth / sky / fill prior losses: per-pixel dL/d(depth numerator, alpha) into
// f.v_aux, pixels outside `keep` removed from the photometric gradient, loss terms
// summed per row in double and accumulated into p.loss_terms (:807-901).
void prior_loss(State &f, const orc_prior &p, float *v_photo) {
    const uint32_t W = f.W, H = f.H;
    const bool has = p.prior_depth && p.prior_aux && p.prior_w > 0 && p.prior_h > 0;
    const uint32_t pw = has ? (uint32_t)p.prior_w : 1u, ph = has ? (uint32_t)p.prior_h : 1u;
    static const uint8_t dflt_aux[4] = {0, 0, 255, 0};  // keep everything, no sky, zero confidence
    static const float dflt_depth[1] = {0.f};
    const uint8_t *aux = has ? p.prior_aux : dflt_aux;
    const float *pd = has ? p.prior_depth : dflt_depth;
    const bool use_depth = has && p.has_depth, use_sky = has && p.has_sky_mask;
    const float huber = std::max(p.huber_delta, 1e-6f);
    const float inv_npix = 1.0f / (float)(W * H);
    f.v_aux.assign((size_t)W * H * 2, 0.f);
    std::vector<double> terms((size_t)H * 3, 0.0);
#pragma omp parallel for schedule(static)
    for (int gy = 0; gy < (int)H; gy++) {
        double ld = 0, ls = 0, lf = 0;
        for (uint32_t gx = 0; gx < W; gx++) {
            const size_t pix = (size_t)gy * W + gx;
            const float sx = ((float)gx + 0.5f) * (float)pw / (float)W;
            const float sy = ((float)gy + 0.5f) * (float)ph / (float)H;
            const uint32_t q = std::min((uint32_t)sy, ph - 1) * pw + std::min((uint32_t)sx, pw - 1);
            const float conf = (float)aux[4 * q] * (1.f / 255.f);
            const bool sky = use_sky && aux[4 * q + 1] >= 128;
            const bool keep = aux[4 * q + 2] >= 128;
            float vd = 0.f, va = 0.f;
            if (!keep) {
                if (p.mask_photometric) st3(v_photo, (int64_t)pix, V3{0.f, 0.f, 0.f});
            } else {
                const float A = 1.f - f.final_Ts[pix];
                if (sky) {
                    ls += p.sky_weight * A;
                    va = p.sky_weight * inv_npix;
                } else {
                    if (use_sky && p.fill_weight > 0.f) {
                        lf += p.fill_weight * (1.f - A);
                        va -= p.fill_weight * inv_npix;
                    }
                    const float D = f.out_depth[pix];
                    if (use_depth && p.depth_weight > 0.f && conf > 0.f && A > p.min_alpha && D > 0.f) {
                        const float dp = prior_depth_at(pd, sx - 0.5f, sy - 0.5f, pw, ph);
                        if (dp > 0.f) {
                            const float r = std::log(D / A) - std::log(dp);
                            const float ar = std::fabs(r);
                            float dr;
                            if (ar < huber) {
                                ld += p.depth_weight * conf * 0.5f * r * r / huber;
                                dr = r / huber;
                            } else {
                                ld += p.depth_weight * conf * (ar - 0.5f * huber);
                                dr = r > 0.f ? 1.f : (r < 0.f ? -1.f : 0.f);
                            }
                            const float s = p.depth_weight * conf * dr * inv_npix;
                            vd = s / D;
                            va -= s / A;
                        }
                    }
                }
            }
            f.v_aux[2 * pix] = vd;
            f.v_aux[2 * pix + 1] = va;
        }
        terms[3 * (size_t)gy] = ld;
        terms[3 * (size_t)gy + 1] = ls;
        terms[3 * (size_t)gy + 2] = lf;
    }
    if (p.loss_terms) {
        double t[3] = {0, 0, 0};
        for (uint32_t y = 0; y < H; y++)
            for (int k = 0; k < 3; k++) t[k] += terms[3 * y + k];
        for (int k = 0; k < 3; k++) p.loss_terms[k] += (float)(t[k] * inv_npix);
    }
}

// per-image affine exposure: out = M c + t, M = P[0..8] row-major, t = P[9..11] (:904-913)
void exposure_apply(const float *img, const float *P, size_t n, float *out) {
    for (size_t i = 0; i < n; i++) {
        const V3 c = ld3(img, (int64_t)i);
        st3(out, (int64_t)i, V3{dot3(V3{P[0], P[1], P[2]}, c) + P[9], dot3(V3{P[3], P[4], P[5]}, c) + P[10],
                                dot3(V3{P[6], P[7], P[8]}, c) + P[11]});
    }
}

// exposure backward (gradient to the render, the 12 parameters' gradient summed in
// double in pixel order) and Adam towards the identity-regularised parameters (:916-937)
void exposure_backward_adam(const float *img, const orc_prior &p, size_t n, const float *v_adj, float *v_img,
                            float b1, float b2, float eps) {
    const uint32_t cam = (uint32_t)std::max(0, p.cam_index);
    float *params = p.expo_params;
    const float *P = params + 12 * cam;
    double gg[12] = {0};
    for (size_t i = 0; i < n; i++) {
        const V3 c = ld3(img, (int64_t)i), v = ld3(v_adj, (int64_t)i);
        st3(v_img, (int64_t)i, V3{P[0] * v.x + P[3] * v.y + P[6] * v.z, P[1] * v.x + P[4] * v.y + P[7] * v.z,
                                  P[2] * v.x + P[5] * v.y + P[8] * v.z});
        gg[0] += v.x * c.x; gg[1] += v.x * c.y; gg[2] += v.x * c.z;
        gg[3] += v.y * c.x; gg[4] += v.y * c.y; gg[5] += v.y * c.z;
        gg[6] += v.z * c.x; gg[7] += v.z * c.y; gg[8] += v.z * c.z;
        gg[9] += v.x; gg[10] += v.y; gg[11] += v.z;
    }
    for (int k = 0; k < 12; k++) {
        const uint32_t i = 12 * cam + k;
        const float ident = (k == 0 || k == 4 || k == 8) ? 1.f : 0.f;
        const float gk = (float)gg[k] + (p.expo_grad ? p.expo_grad[k] : 0.f) + p.expo_reg * (params[i] - ident);
        if (p.expo_grad) p.expo_grad[k] = 0.f;
        adam(params[i], p.expo_exp_avg[i], p.expo_exp_avg_sq[i], gk, p.expo_step_size, b1, b2, p.expo_bc2_sqrt, eps);
    }
}

// sky texture gradient (each pixel still seeing the sky adds T dL/dC to its four
// taps, in pixel order) and Adam over the texture (:940-964)
void sky_backward_adam(State &f, const orc_prior &p, const Sky &sky, const float *vm, const float *v_img, float b1,
                       float b2, float eps) {
    float *grad = p.sky_grad;
    for (uint32_t y = 0; y < f.H; y++)
        for (uint32_t x = 0; x < f.W; x++) {
            const size_t pix = (size_t)y * f.W + x;
            const float T = f.final_Ts[pix];
            if (T < 1e-4f) continue;
            const V3 gv = scl(T, ld3(v_img, (int64_t)pix));
            const Taps taps = sky_taps(sky_uv(ray_dir((float)x, (float)y, vm, sky), sky), sky.w, sky.h);
            for (int k = 0; k < 4; k++) {
                if (taps.w[k] == 0.f) continue;
                float *t = grad + 3 * (size_t)taps.idx[k];
                t[0] += taps.w[k] * gv.x;
                t[1] += taps.w[k] * gv.y;
                t[2] += taps.w[k] * gv.z;
            }
        }
    const size_t n = (size_t)p.sky_w * p.sky_h * 3;
    for (size_t i = 0; i < n; i++)
        adam(p.sky_tex[i], p.sky_exp_avg[i], p.sky_exp_avg_sq[i], grad[i], p.sky_step_size, b1, b2, p.sky_bc2_sqrt,
             eps);
}

// needle cap: the largest log-scale at most log_max above the middle one (:1295-1309)
void needle_cap(float *s, int n, float log_max) {
    for (int i = 0; i < n; i++) {
        const float a = s[3 * i], b = s[3 * i + 1], c = s[3 * i + 2];
        const float mx = std::max(a, std::max(b, c)), mn = std::min(a, std::min(b, c));
        const float cap = (a + b + c - mx - mn) + log_max;
        if (mx <= cap) continue;
        if (a == mx) s[3 * i] = cap;
        else if (b == mx) s[3 * i + 1] = cap;
        else s[3 * i + 2] = cap;
    }
}

// k-d tree with median splits for exact 3-NN (core/cpu/msplat_cpu.cpp:1498-1580)
struct Kd {
    const float *p = nullptr;
    std::vector<uint32_t> id;
    std::vector<uint8_t> ax;
    void build(uint32_t lo, uint32_t hi) {
        if (hi - lo <= 8) return;
        float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t i = lo; i < hi; i++)
            for (int a = 0; a < 3; a++) {
                mn[a] = std::min(mn[a], p[3 * id[i] + a]);
                mx[a] = std::max(mx[a], p[3 * id[i] + a]);
            }
        int a = 0;
        for (int b = 1; b < 3; b++)
            if (mx[b] - mn[b] > mx[a] - mn[a]) a = b;
        uint32_t mid = (lo + hi) / 2;
        std::nth_element(id.begin() + lo, id.begin() + mid, id.begin() + hi,
                         [&](uint32_t u, uint32_t v) { return p[3 * u + a] < p[3 * v + a]; });
        ax[mid] = (uint8_t)a;
        build(lo, mid);
        build(mid + 1, hi);
    }
    static void keep3(float d, float b[3]) {
        if (d >= b[2]) return;
        if (d < b[1]) {
            b[2] = b[1];
            if (d < b[0]) { b[1] = b[0]; b[0] = d; } else b[1] = d;
        } else b[2] = d;
    }
    void query(uint32_t lo, uint32_t hi, uint32_t self, const float *q, float b[3]) const {
        if (hi - lo <= 8) {
            for (uint32_t i = lo; i < hi; i++) {
                uint32_t u = id[i];
                if (u == self) continue;
                float dx = p[3 * u] - q[0], dy = p[3 * u + 1] - q[1], dz = p[3 * u + 2] - q[2];
                keep3(dx * dx + dy * dy + dz * dz, b);
            }
            return;
        }
        uint32_t mid = (lo + hi) / 2, u = id[mid];
        int a = ax[mid];
        if (u != self) {
            float dx = p[3 * u] - q[0], dy = p[3 * u + 1] - q[1], dz = p[3 * u + 2] - q[2];
            keep3(dx * dx + dy * dy + dz * dz, b);
        }
        float diff = q[a] - p[3 * u + a];
        if (diff < 0) {
            query(lo, mid, self, q, b);
            if (diff * diff < b[2]) query(mid + 1, hi, self, q, b);
        } else {
            query(mid + 1, hi, self, q, b);
            if (diff * diff < b[2]) query(lo, mid, self, q, b);
        }
    }
};

}  // namespace

extern "C" {

// "reverse_sums": see g_reverse_sums. Returns 0, or -1 for an unknown option.
int orc_set_option(const char *name, int value) {
    if (std::string(name) == "reverse_sums") {
        g_reverse_sums = value != 0;
        return 0;
    }
    if (std::string(name) == "chunk_size") {
        if (value < 0) return -1;
        g_chunk = value;
        return 0;
    }
    return -1;
}

int orc_render(int n, const float *means, const float *scales, float gsc, const float *quats, const float *vm,
               const float *P, float fx, float fy, float cx, float cy, unsigned H, unsigned W, int tx, int ty,
               float clip, unsigned degree, unsigned dtu, const float *cam, const float *dc, const float *rest,
               const float *opac, const float *bg, float *out) {
    forward(g, n, means, scales, gsc, quats, vm, P, fx, fy, cx, cy, H, W, tx, ty, clip, degree, dtu, cam, dc, rest,
            opac, bg);
    std::memcpy(out, g.out_img.data(), g.out_img.size() * sizeof(float));
    return 0;
}

// Copies the prior (its pointers stay the caller's); NULL clears it.
int orc_set_prior(const orc_prior *prior) {
    g_has_prior = prior != nullptr;
    if (prior) g_prior = *prior;
    return 0;
}

// core/cpu/msplat_cpu.cpp:1204-1327, with the prior set by orc_set_prior
float orc_train_step(int n, float *means, float *scales, float gsc, float *quats, const float *vm, const float *P,
                     float fx, float fy, float cx, float cy, unsigned H, unsigned W, int tx, int ty, float clip,
                     unsigned degree, unsigned dtu, const float *cam, float *dc, float *rest, float *opac,
                     const float *bg, const float *gt, float ssim_w, float inv_n, float **m1, float **m2,
                     const int64_t *numel, const float *ss, const float *bc2, float b1, float b2, float eps,
                     float *vis, float *gn, float *ms, float inv_max_dim) {
    State &f = g;
    const orc_prior *pr = g_has_prior ? &g_prior : nullptr;
    const bool aux = pr && pr->aux;
    const bool sky_on = aux && pr->sky && pr->sky_tex && pr->sky_grad;
    const bool expo = pr && pr->exposure && pr->expo_params;
    const size_t npix = (size_t)W * H;
    forward(f, n, means, scales, gsc, quats, vm, P, fx, fy, cx, cy, H, W, tx, ty, clip, degree, dtu, cam, dc, rest,
            opac, bg);
    if (aux && pr->loss_terms) std::fill(pr->loss_terms, pr->loss_terms + 4, 0.f);
    if (sky_on) std::fill(pr->sky_grad, pr->sky_grad + (size_t)pr->sky_w * pr->sky_h * 3, 0.f);
    f.v_rendered.assign(npix * 3, 0.f);
    const float *loss_in = f.out_img.data();
    float *loss_grad = f.v_rendered.data();
    if (expo) {
        f.out_adj.assign(npix * 3, 0.f);
        f.v_adj.assign(npix * 3, 0.f);
        exposure_apply(f.out_img.data(), pr->expo_params + 12 * std::max(0, pr->cam_index), npix, f.out_adj.data());
        loss_in = f.out_adj.data();
        loss_grad = f.v_adj.data();
    }
    double loss = ssim_loss(loss_in, gt, W, H, ssim_w, inv_n, loss_grad);
    if (aux) prior_loss(f, *pr, loss_grad);
    if (expo) exposure_backward_adam(f.out_img.data(), *pr, npix, f.v_adj.data(), f.v_rendered.data(), b1, b2, eps);
    if (sky_on) sky_backward_adam(f, *pr, make_sky(pr, fx, fy, cx, cy), vm, f.v_rendered.data(), b1, b2, eps);
    if (f.chunked)
        raster_bwd_chunked(f, bg, f.v_rendered.data());
    else
        raster_bwd(f, bg, f.v_rendered.data());
    reduce_slots(f, n);
    proj_bwd_adam(f, n, means, scales, gsc, quats, vm, P, fx, fy, degree, dtu, cam, dc, rest, m1[3], m2[3], m1[4],
                  m2[4], ss[3], bc2[3], ss[4], bc2[4], b1, b2, eps);
    float *params[6] = {means, scales, quats, dc, rest, opac};
    const float *grads[6] = {f.v_mean3d.data(), f.v_scale.data(), f.v_quat.data(), nullptr, nullptr,
                             f.v_opacity.data()};
    for (int gi = 0; gi < 6; gi++) {
        if (gi == 3 || gi == 4 || numel[gi] == 0) continue;
        adam_dense(params[gi], grads[gi], m1[gi], m2[gi], (size_t)numel[gi], ss[gi], b1, b2, bc2[gi], eps);
    }
    if (pr && pr->log_max_scale_ratio > 0.f) needle_cap(scales, n, pr->log_max_scale_ratio);
    for (int i = 0; i < n; i++) {
        if (f.radii[i] <= 0) continue;
        vis[i] += 1.0f;
        float gx = f.v_xy[2 * i], gy = f.v_xy[2 * i + 1];
        gn[i] += std::sqrt(gx * gx + gy * gy);
        ms[i] = std::max(ms[i], (float)f.radii[i] * inv_max_dim);
    }
    return (float)(loss / (double)((size_t)W * H));
}

int64_t orc_frame(const char *name, void **ptr) {
    const std::string s(name);
    const int T = g.tx * g.ty;
    const int64_t total = T ? g.tile_end[T - 1] : 0;
#define ORC_F(nm, vec, cnt) \
    if (s == nm) { *ptr = (void *)vec.data(); return (int64_t)(cnt); }
    ORC_F("xys", g.xys, (int64_t)g.n * 2)
    ORC_F("depths", g.depths, g.n)
    ORC_F("conics", g.conics, (int64_t)g.n * 3)
    ORC_F("colors", g.colors, (int64_t)g.n * 3)
    ORC_F("aabb", g.aabb, (int64_t)g.n * 2)
    ORC_F("radii", g.radii, g.n)
    ORC_F("tile_start", g.tile_start, T)
    ORC_F("tile_end", g.tile_end, T)
    ORC_F("isect_gid", g.isect_gid, total)
    ORC_F("out_img", g.out_img, (int64_t)g.W * g.H * 3)
    ORC_F("final_Ts", g.final_Ts, (int64_t)g.W * g.H)
    ORC_F("final_idx", g.final_idx, (int64_t)g.W * g.H)
    ORC_F("v_rendered", g.v_rendered, (int64_t)g.W * g.H * 3)
    ORC_F("v_xy", g.v_xy, (int64_t)g.n * 2)
    ORC_F("v_conic", g.v_conic, (int64_t)g.n * 3)
    ORC_F("v_rgb", g.v_rgb, (int64_t)g.n * 3)
    ORC_F("v_opacity", g.v_opacity, g.n)
    ORC_F("v_mean3d", g.v_mean3d, (int64_t)g.n * 3)
    ORC_F("v_scale", g.v_scale, (int64_t)g.n * 3)
    ORC_F("v_quat", g.v_quat, (int64_t)g.n * 4)
    ORC_F("out_depth", g.out_depth, g.aux ? (int64_t)g.W * g.H : 0)
    ORC_F("bg_img", g.bg_img, g.aux ? (int64_t)g.W * g.H * 3 : 0)
    ORC_F("v_aux", g.v_aux, g.aux ? (int64_t)g.W * g.H * 2 : 0)
    ORC_F("v_depth", g.v_depth, (int64_t)g.v_depth.size())
    ORC_F("out_adj", g.out_adj, (int64_t)g.out_adj.size())
    ORC_F("v_adj", g.v_adj, (int64_t)g.v_adj.size())
    ORC_F("chunk_first", g.ch_first, g.chunked ? (int64_t)g.ch_first.size() : 0)
#undef ORC_F
    *ptr = nullptr;
    return -1;
}

// core/cpu/msplat_cpu.cpp:1330-1465
int orc_densify(int N, int cap, float grad_thresh, float size_thresh, float screen_thresh, int check_screen,
                float cull_alpha, float cull_scale, float cull_screen, int check_huge, const float *gn,
                const float *vc, const float *ms, float half_max_dim, float *means, float *scales, float *quats,
                float *fdc, float *frest, float *opac, int fr_stride, float **m1, float **m2, uint32_t seed) {
    if (3 * N > cap) return -1;
    const float lsf = std::log(1.6f);
    std::vector<uint8_t> split(N), dup(N);
    for (int i = 0; i < N; i++) {
        split[i] = dup[i] = 0;
        if (vc[i] <= 0.0f) continue;
        bool hg = (gn[i] / vc[i]) * half_max_dim > grad_thresh;
        float mx = std::max(std::max(std::exp(scales[3 * i]), std::exp(scales[3 * i + 1])), std::exp(scales[3 * i + 2]));
        bool large = mx > size_thresh;
        bool sp = large;
        if (check_screen && ms[i] > screen_thresh) sp = true;
        split[i] = (sp && hg) ? 1 : 0;
        dup[i] = (!large && hg) ? 1 : 0;
    }
    std::vector<int32_t> so(N), dor(N);
    int ns = 0, nd = 0;
    for (int i = 0; i < N; i++) {
        so[i] = split[i] ? ns++ : -1;
        dor[i] = dup[i] ? nd++ : -1;
    }
    const int st[6] = {3, 3, 4, 3, fr_stride, 1};
    auto zero_moments = [&](int c) {
        for (int gi = 0; gi < 6; gi++) {
            std::fill(m1[gi] + (size_t)c * st[gi], m1[gi] + (size_t)(c + 1) * st[gi], 0.f);
            std::fill(m2[gi] + (size_t)c * st[gi], m2[gi] + (size_t)(c + 1) * st[gi], 0.f);
        }
    };
    for (int i = 0; i < N; i++) {
        if (!split[i]) continue;
        const int o = so[i];
        float qw = quats[4 * i], qx = quats[4 * i + 1], qy = quats[4 * i + 2], qz = quats[4 * i + 3];
        float ql = std::sqrt(qw * qw + qx * qx + qy * qy + qz * qz);
        qw /= ql; qx /= ql; qy /= ql; qz /= ql;
        float sx = std::exp(scales[3 * i]), sy = std::exp(scales[3 * i + 1]), sz = std::exp(scales[3 * i + 2]);
        for (int k = 0; k < 2; k++) {
            const int c = N + 2 * o + k;
            V3 nr = normal3(seed, (uint32_t)(o * 2 + k));
            float r0 = nr.x * sx, r1 = nr.y * sy, r2 = nr.z * sz;
            float v0 = (1 - 2 * (qy * qy + qz * qz)) * r0 + 2 * (qx * qy - qw * qz) * r1 + 2 * (qx * qz + qw * qy) * r2;
            float v1 = 2 * (qx * qy + qw * qz) * r0 + (1 - 2 * (qx * qx + qz * qz)) * r1 + 2 * (qy * qz - qw * qx) * r2;
            float v2 = 2 * (qx * qz - qw * qy) * r0 + 2 * (qy * qz + qw * qx) * r1 + (1 - 2 * (qx * qx + qy * qy)) * r2;
            means[3 * c] = means[3 * i] + v0;
            means[3 * c + 1] = means[3 * i + 1] + v1;
            means[3 * c + 2] = means[3 * i + 2] + v2;
            for (int j = 0; j < 3; j++) scales[3 * c + j] = scales[3 * i + j] - lsf;
            for (int j = 0; j < 4; j++) quats[4 * c + j] = quats[4 * i + j];
            for (int j = 0; j < 3; j++) fdc[3 * c + j] = fdc[3 * i + j];
            for (int j = 0; j < fr_stride; j++) frest[(size_t)c * fr_stride + j] = frest[(size_t)i * fr_stride + j];
            opac[c] = opac[i];
            zero_moments(c);
        }
        for (int j = 0; j < 3; j++) scales[3 * i + j] -= lsf;
    }
    for (int i = 0; i < N; i++) {
        if (!dup[i]) continue;
        const int d = N + 2 * ns + dor[i];
        for (int j = 0; j < 3; j++) means[3 * d + j] = means[3 * i + j];
        for (int j = 0; j < 3; j++) scales[3 * d + j] = scales[3 * i + j];
        for (int j = 0; j < 4; j++) quats[4 * d + j] = quats[4 * i + j];
        for (int j = 0; j < 3; j++) fdc[3 * d + j] = fdc[3 * i + j];
        for (int j = 0; j < fr_stride; j++) frest[(size_t)d * fr_stride + j] = frest[(size_t)i * fr_stride + j];
        opac[d] = opac[i];
        zero_moments(d);
    }
    const int Nn = N + 2 * ns + nd;
    std::vector<uint8_t> keep(Nn);
    for (int i = 0; i < Nn; i++) {
        float o = 1.0f / (1.0f + std::exp(-opac[i]));
        bool cull = o < cull_alpha;
        if (i < N && split[i]) cull = true;
        if (check_huge) {
            float mx = std::max(std::max(std::exp(scales[3 * i]), std::exp(scales[3 * i + 1])), std::exp(scales[3 * i + 2]));
            if (mx > cull_scale) cull = true;
            if (check_screen && i < N && ms[i] > cull_screen) cull = true;
        }
        keep[i] = cull ? 0 : 1;
    }
    float *bufs[18] = {means, scales, quats, fdc, frest, opac};
    for (int gi = 0; gi < 6; gi++) {
        bufs[6 + gi] = m1[gi];
        bufs[12 + gi] = m2[gi];
    }
    int out = 0;
    for (int i = 0; i < Nn; i++) {
        if (!keep[i]) continue;
        if (out != i)
            for (int b = 0; b < 18; b++) {
                const int s = st[b % 6];
                std::memmove(bufs[b] + (size_t)out * s, bufs[b] + (size_t)i * s, sizeof(float) * s);
            }
        out++;
    }
    return out;
}

// core/cpu/msplat_cpu.cpp:1467-1475
void orc_opacity_reset(float *o, float *m1, float *m2, int n, float reset_logit) {
    for (int i = 0; i < n; i++) {
        o[i] = std::min(o[i], reset_logit);
        m1[i] = 0.f;
        m2[i] = 0.f;
    }
}

// core/cpu/msplat_cpu.cpp:1481-1494
void orc_radix_sort(uint64_t *keys, int32_t *vals, uint32_t n, int key_bits) {
    if (n == 0) return;
    const uint64_t mask = key_bits >= 64 ? ~0ull : ((1ull << key_bits) - 1ull);
    std::vector<uint32_t> ord(n);
    std::iota(ord.begin(), ord.end(), 0u);
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return (keys[a] & mask) < (keys[b] & mask); });
    std::vector<uint64_t> k2(n);
    std::vector<int32_t> v2(n);
    for (uint32_t i = 0; i < n; i++) {
        k2[i] = keys[ord[i]];
        v2[i] = vals[ord[i]];
    }
    std::memcpy(keys, k2.data(), n * sizeof(uint64_t));
    std::memcpy(vals, v2.data(), n * sizeof(int32_t));
}

// core/cpu/msplat_cpu.cpp:1561-1580
void orc_knn3_mean_dist(const float *pts, uint32_t n, float *out) {
    if (n == 0) return;
    Kd t;
    t.p = pts;
    t.id.resize(n);
    t.ax.assign(n, 0);
    std::iota(t.id.begin(), t.id.end(), 0u);
    t.build(0, n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        float b[3] = {INFINITY, INFINITY, INFINITY};
        t.query(0, n, (uint32_t)i, pts + 3 * i, b);
        float sum = 0.f, cnt = 0.f;
        for (int k = 0; k < 3; k++)
            if (std::isfinite(b[k])) {
                sum += std::sqrt(b[k]);
                cnt += 1.f;
            }
        out[i] = cnt > 0.f ? sum / cnt : 1.f;
    }
}

// core/cpu/msplat_cpu.cpp:1582-1605
void orc_init_gaussians(const float *means, const uint8_t *rgb, uint32_t n, uint32_t seed, float ologit,
                        float *scales, float *quats, float *dc, float *opac) {
    if (n == 0) return;
    std::vector<float> md(n);
    orc_knn3_mean_dist(means, n, md.data());
    const float tau = 6.28318530717958647692f;
    for (uint32_t i = 0; i < n; i++) {
        float ls = std::log(std::max(md[i], 1e-7f));
        scales[3 * i] = scales[3 * i + 1] = scales[3 * i + 2] = ls;
        float u = unif(seed, 3u * i), v = unif(seed, 3u * i + 1u), w = unif(seed, 3u * i + 2u);
        quats[4 * i + 0] = std::sqrt(1.f - u) * std::sin(tau * v);
        quats[4 * i + 1] = std::sqrt(1.f - u) * std::cos(tau * v);
        quats[4 * i + 2] = std::sqrt(u) * std::sin(tau * w);
        quats[4 * i + 3] = std::sqrt(u) * std::cos(tau * w);
        for (int k = 0; k < 3; k++) dc[3 * i + k] = ((float)rgb[3 * i + k] * (1.f / 255.f) - 0.5f) / kC0;
        opac[i] = ologit;
    }
}

// core/cpu/msplat_cpu.cpp:1609-1639 -- area resample
void orc_resize_area(const void *src, int u8in, int sw, int sh, float *dst, int dw, int dh) {
    if (dw <= 0 || dh <= 0) return;
    const uint8_t *u8 = u8in ? (const uint8_t *)src : nullptr;
    const float *fs = u8in ? nullptr : (const float *)src;
    const float sxs = (float)sw / (float)dw, sys = (float)sh / (float)dh;
    for (int gy = 0; gy < dh; gy++) {
        const float y0 = (float)gy * sys, y1 = (float)(gy + 1) * sys;
        const int iy0 = (int)y0, iy1 = std::min((int)std::ceil(y1), sh);
        for (int gx = 0; gx < dw; gx++) {
            const float x0 = (float)gx * sxs, x1 = (float)(gx + 1) * sxs;
            const int ix0 = (int)x0, ix1 = std::min((int)std::ceil(x1), sw);
            V3 sum{0.f, 0.f, 0.f};
            float area = 0.f;
            for (int iy = iy0; iy < iy1; iy++) {
                float wy = std::min((float)(iy + 1), y1) - std::max((float)iy, y0);
                for (int ix = ix0; ix < ix1; ix++) {
                    float wx = std::min((float)(ix + 1), x1) - std::max((float)ix, x0);
                    size_t s = (size_t)iy * sw + ix;
                    V3 c = u8 ? scl(V3{(float)u8[4 * s], (float)u8[4 * s + 1], (float)u8[4 * s + 2]}, 1.f / 255.f)
                              : ld3(fs, s);
                    sum = add(sum, scl(wx * wy, c));
                    area += wx * wy;
                }
            }
            st3(dst, (size_t)gy * dw + gx, V3{sum.x / area, sum.y / area, sum.z / area});
        }
    }
}

// core/cpu/msplat_cpu.cpp:1641-1669 -- Brown-Conrady undistortion, bilinear
void orc_undistort(const float *in, int sw, int sh, const float *intr, const float *dist, int rx, int ry, float *out,
                   int dw, int dh) {
    if (dw <= 0 || dh <= 0) return;
    const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
    const float k1 = dist[0], k2 = dist[1], p1 = dist[2], p2 = dist[3], k3 = dist[4];
    for (int gy = 0; gy < dh; gy++)
        for (int gx = 0; gx < dw; gx++) {
            float x = ((float)(gx + rx) + 0.5f - cx) / fx;
            float y = ((float)(gy + ry) + 0.5f - cy) / fy;
            float r2 = x * x + y * y;
            float rad = 1.f + k1 * r2 + k2 * r2 * r2 + k3 * r2 * r2 * r2;
            float xd = x * rad + 2.f * p1 * x * y + p2 * (r2 + 2.f * x * x);
            float yd = y * rad + p1 * (r2 + 2.f * y * y) + 2.f * p2 * x * y;
            float sx = xd * fx + cx - 0.5f, sy = yd * fy + cy - 0.5f;
            int x0 = (int)std::floor(sx), y0 = (int)std::floor(sy);
            float ax = sx - std::floor(sx), ay = sy - std::floor(sy);
            int xa = std::clamp(x0, 0, sw - 1), xb = std::clamp(x0 + 1, 0, sw - 1);
            int ya = std::clamp(y0, 0, sh - 1), yb = std::clamp(y0 + 1, 0, sh - 1);
            V3 c00 = ld3(in, (size_t)ya * sw + xa), c10 = ld3(in, (size_t)ya * sw + xb);
            V3 c01 = ld3(in, (size_t)yb * sw + xa), c11 = ld3(in, (size_t)yb * sw + xb);
            V3 top = add(scl(c00, 1.f - ax), scl(c10, ax)), bot = add(scl(c01, 1.f - ax), scl(c11, ax));
            st3(out, (size_t)gy * dw + gx, add(scl(top, 1.f - ay), scl(bot, ay)));
        }
}

// core/cpu/msplat_cpu.cpp:1671-1721 -- PSNR, SSIM with clamp-to-edge borders, L1
void orc_image_metrics(const float *a, const float *b, int h, int w, double *out) {
    out[0] = out[1] = out[2] = 0.0;
    if (h <= 0 || w <= 0) return;
    std::vector<float> hb((size_t)h * w * 15);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++)
            for (int c = 0; c < 3; c++) {
                float s[5] = {0, 0, 0, 0, 0};
                for (int k = 0; k < 11; k++) {
                    int sx = std::clamp(x + k - 5, 0, w - 1);
                    size_t i = ((size_t)y * w + sx) * 3 + c;
                    float gk = kWin[k], xa = a[i], yb = b[i];
                    s[0] += gk * xa; s[1] += gk * yb; s[2] += gk * xa * xa; s[3] += gk * yb * yb; s[4] += gk * xa * yb;
                }
                std::memcpy(&hb[((size_t)y * w + x) * 15 + c * 5], s, sizeof s);
            }
    double ssim = 0, l1 = 0, sq = 0;
    for (int y = 0; y < h; y++) {
        double rs = 0, rl = 0, rq = 0;
        for (int x = 0; x < w; x++)
            for (int c = 0; c < 3; c++) {
                float s[5] = {0, 0, 0, 0, 0};
                for (int k = 0; k < 11; k++) {
                    int sy = std::clamp(y + k - 5, 0, h - 1);
                    const float *o = &hb[((size_t)sy * w + x) * 15 + c * 5];
                    for (int q = 0; q < 5; q++) s[q] += kWin[k] * o[q];
                }
                float m12 = s[0] * s[1], m1 = s[0] * s[0], m2 = s[1] * s[1];
                float num = (2.f * m12 + kSsimC1) * (2.f * (s[4] - m12) + kSsimC2);
                float den = (m1 + m2 + kSsimC1) * ((s[2] - m1) + (s[3] - m2) + kSsimC2);
                rs += num / den;
                size_t i = ((size_t)y * w + x) * 3 + c;
                float d = a[i] - b[i];
                rl += std::fabs(d);
                rq += (double)d * d;
            }
        ssim += rs; l1 += rl; sq += rq;
    }
    double cnt = (double)h * w * 3, mse = sq / cnt;
    out[0] = mse > 0 ? 10.0 * std::log10(1.0 / mse) : INFINITY;
    out[1] = ssim / cnt;
    out[2] = l1 / cnt;
}

// core/cpu/msplat_cpu.cpp:1723-1734
void orc_pack_rgba8(const float *img, uint32_t n, uint8_t *out) {
    for (uint32_t i = 0; i < n; i++) {
        V3 c = scl(V3{clamp01(img[3 * i]), clamp01(img[3 * i + 1]), clamp01(img[3 * i + 2])}, 255.f);
        out[4 * i] = (uint8_t)c.x;
        out[4 * i + 1] = (uint8_t)c.y;
        out[4 * i + 2] = (uint8_t)c.z;
        out[4 * i + 3] = 255;
    }
}

// core/cpu/msplat_cpu.cpp:1736-1745
void orc_finalize_depth(const float *d, const float *t, uint32_t n, float inv_scale, float *od, float *oa) {
    for (uint32_t i = 0; i < n; i++) {
        float a = 1.f - t[i];
        oa[i] = a;
        od[i] = a > 1e-4f ? d[i] / a * inv_scale : 0.f;
    }
}

}  // extern "C"
