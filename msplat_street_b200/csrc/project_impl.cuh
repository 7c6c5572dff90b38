// Per-Gaussian projection shared by the single-view and batched kernels, in two steps
// (project_geom, then project_finish) so that a warp's SH-rest rows can be copied into
// shared memory while the geometry runs.
//
// Follows project_and_sh (core/cpu/msplat_cpu.cpp:452-500) and its helpers
// (:63-190): cull at the clip depth, 3D covariance, EWA 2D covariance with the 1.3x
// FOV clamp and 0.3 px dilation, conic and radius, pixel centre through the full
// projection, 3-sigma tile rectangle, raw SH colour. Writes Gaussian i's 48-byte Splat
// record, radius, AABB half-extents and tile count at output slot o. The including
// translation unit must be compiled with -fmad=false: tile rectangles and depth keys
// must equal the reference's bit for bit.
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace msplat {
namespace proj_detail {

__device__ __forceinline__ V3 xform43(const float *m, V3 p) {
    return V3{m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
              m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]};
}

}  // namespace proj_detail
using proj_detail::xform43;

// SH-rest staging for degree 3 (45 floats a Gaussian). A lane reading its own 180-byte
// row makes every load instruction of the warp touch 32 sectors; when the warp's 32
// lanes project Gaussians whose rows lie back to back in one array (row0, row0 + 45,
// ...), the warp instead copies the 32 rows (1440 contiguous floats) into shared
// memory with asynchronous 4-byte copies whose addresses are consecutive across the
// lanes (4 sectors an instruction), which complete while the geometry runs. Every
// lane of the warp must call issue_rest_rows; it returns whether the copies were
// issued (warp-uniform). The caller then has every lane call rest_rows_wait before
// any lane reads its row at buf + 45 * lane (stride 45 words: no bank conflicts).
constexpr int PROJ_REST3 = 45;

__device__ __forceinline__ bool issue_rest_rows(const float *row, bool use, float *buf) {
    const int lane = threadIdx.x & 31;
    const float *row0 = reinterpret_cast<const float *>(
        __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(row), 0));
    if (!__all_sync(0xffffffffu, use && row == row0 + PROJ_REST3 * lane)) return false;
    const unsigned dst = (unsigned)__cvta_generic_to_shared(buf);
#pragma unroll 9
    for (int k = 0; k < PROJ_REST3; k++) {
        const int e = k * 32 + lane;  // < 1440: inside the 32 rows
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst + 4u * (unsigned)e), "l"(row0 + e)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    return true;
}

__device__ __forceinline__ void rest_rows_wait() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncwarp();
}

__device__ __forceinline__ void tile_rect(float cx, float cy, float rx, float ry, int tx, int ty, int &x0, int &y0,
                                          int &x1, int &y1) {
    float ccx = cx / (float)TILE, ccy = cy / (float)TILE;
    float rrx = rx / (float)TILE, rry = ry / (float)TILE;
    x0 = min(max(0, (int)(ccx - rrx)), tx);
    x1 = min(max(0, (int)(ccx + rrx + 1)), tx);
    y0 = min(max(0, (int)(ccy - rry)), ty);
    y1 = min(max(0, (int)(ccy + rry + 1)), ty);
}

// What the colour and record step needs from the geometry step.
struct ProjState {
    V3 pw;
    float depth;
    V3 conic;
    float ctx, cty, op, ex, ey, hp, hm;
};

// Geometry of Gaussian i (output slot o): cull, covariance, EWA, conic, radius, tile
// rectangle, opacity and the pixel-reach extents. Returns false where the Gaussian
// is culled (its radius and tile count left at zero).
__device__ __forceinline__ bool project_geom(const ProjectArgs &a, int i, int64_t o, ProjState &st) {
    a.radii[o] = 0;
    a.n_tiles[o] = 0;
    const float *vm = a.cam.viewmat;
    V3 pw = ld3(a.means, i);
    V3 pv = xform43(vm, pw);
    if (pv.z <= a.cam.clip) return false;
    V3 ls = ld3(a.scales, i);
    V3 s{exp_ref(ls.x), exp_ref(ls.y), exp_ref(ls.z)};
    const float4 qq = reinterpret_cast<const float4 *>(a.quats)[i];
    Q4 q{qq.x, qq.y, qq.z, qq.w};
    float cov[6];
    cov3d_of(s, a.glob_scale, q, cov);
    const float fx = a.cam.fx, fy = a.cam.fy;
    const float tfx = 0.5f * (float)a.cam.width / fx, tfy = 0.5f * (float)a.cam.height / fy;
    // EWA (core/cpu/msplat_cpu.cpp:103-125)
    V3 c2;
    {
        V3 p = pv;
        float lx = 1.3f * tfx, ly = 1.3f * tfy;
        p.x = p.z * fminf(lx, fmaxf(-lx, p.x / p.z));
        p.y = p.z * fminf(ly, fmaxf(-ly, p.y / p.z));
        float rz = 1.f / p.z, rz2 = rz * rz;
        float j00 = fx * rz, j11 = fy * rz;
        float j20 = -fx * p.x * rz2, j21 = -fy * p.y * rz2;
        V3 r0{vm[0], vm[1], vm[2]}, r1{vm[4], vm[5], vm[6]}, r2{vm[8], vm[9], vm[10]};
        V3 t0 = add(scl(j00, r0), scl(j20, r2));
        V3 t1 = add(scl(j11, r1), scl(j21, r2));
        V3 u{t0.x * cov[0] + t0.y * cov[1] + t0.z * cov[2], t0.x * cov[1] + t0.y * cov[3] + t0.z * cov[4],
             t0.x * cov[2] + t0.y * cov[4] + t0.z * cov[5]};
        V3 w{t1.x * cov[0] + t1.y * cov[1] + t1.z * cov[2], t1.x * cov[1] + t1.y * cov[3] + t1.z * cov[4],
             t1.x * cov[2] + t1.y * cov[4] + t1.z * cov[5]};
        c2 = V3{dot3(u, t0) + 0.3f, dot3(u, t1), dot3(w, t1) + 0.3f};
    }
    // conic and radius (core/cpu/msplat_cpu.cpp:127-138)
    float det = c2.x * c2.z - c2.y * c2.y;
    if (det == 0.f) return false;
    float inv = 1.f / det;
    V3 conic{c2.z * inv, -c2.y * inv, c2.x * inv};
    float bb = 0.5f * (c2.x + c2.z);
    float disc = sqrtf(fmaxf(0.1f, bb * bb - det));
    float radius = ceilf(3.f * sqrtf(bb + disc));
    // pixel centre (core/cpu/msplat_cpu.cpp:140-146)
    const float *P = a.cam.projmat;
    float hx = P[0] * pw.x + P[1] * pw.y + P[2] * pw.z + P[3];
    float hy = P[4] * pw.x + P[5] * pw.y + P[6] * pw.z + P[7];
    float hw = P[12] * pw.x + P[13] * pw.y + P[14] * pw.z + P[15];
    float rw = 1.f / (hw + 1e-6f);
    float ctx = 0.5f * (float)(int)a.cam.width * (hx * rw) + a.cam.cx - 0.5f;
    float cty = 0.5f * (float)(int)a.cam.height * (hy * rw) + a.cam.cy - 0.5f;
    float ax = ceilf(3.0f * sqrtf(c2.x));
    float ay = ceilf(3.0f * sqrtf(c2.z));
    int x0, y0, x1, y1;
    tile_rect(ctx, cty, ax, ay, a.cam.tiles_x, a.cam.tiles_y, x0, y0, x1, y1);
    const int area = (x1 - x0) * (y1 - y0);
    if (area <= 0) return false;
    a.radii[o] = (int)radius;
    a.n_tiles[o] = area;
    a.aabb[2 * o] = ax;
    a.aabb[2 * o + 1] = ay;

    // sigmoid opacity as the pack step computes it (core/cpu/msplat_cpu.cpp:560)
    const float op = 1.f / (1.f + exp_ref(-a.opacities[i]));
    // Half-extents of the region a pixel can be composited in: sigma < 5.55 and
    // op * exp(-sigma) >= 1/255, i.e. 0.5 d^T conic d <= L. Its bounding box has
    // half-widths sqrt(2 L conic_c / det) and sqrt(2 L conic_a / det), evaluated in
    // double with margins, so the rasterizers may skip pixel blocks outside it without
    // changing any result. An empty box marks a Gaussian that never reaches 1/255.
    float ex = -1e30f, ey = -1e30f;
    const double lg = log(255.0 * (double)op);
    const double L = fmin(5.55, lg + 1e-4);
    if (L > 0.0) {
        const double ca = conic.x, cb = conic.y, cc = conic.z;
        const double cdet = ca * cc - cb * cb;
        if (cdet > 0.0 && ca > 0.0 && cc > 0.0) {
            ex = (float)(sqrt(2.0 * L * cc / cdet) * 1.001 + 0.5);
            ey = (float)(sqrt(2.0 * L * ca / cdet) * 1.001 + 0.5);
        } else {
            ex = ey = 1e30f;  // not positive definite: never skip
        }
    }
    // The same region's half-extents along the diagonals, sqrt(2 L u^T C^-1 u) for
    // u = (1, 1) and (1, -1), with a wider margin on L: the rasterizers test each
    // warp's 8x4 pixel block against them (separating axes; rotated, elongated splats
    // have boxes much larger than themselves). Infinite: the box test alone.
    float hp = __int_as_float(0x7f800000), hm = hp;
    {
        const double ca = conic.x, cb = conic.y, cc = conic.z;
        const double det2 = ca * cc - cb * cb;
        const double Ld = fmin(5.55, lg) + 1e-2;
        if (det2 > 0.0 && ca > 0.0 && cc > 0.0 && Ld > 0.0) {
            hp = (float)(sqrt(2.0 * Ld * fmax(ca + cc - 2.0 * cb, 0.0) / det2) * 1.001 + 0.5);
            hm = (float)(sqrt(2.0 * Ld * fmax(ca + cc + 2.0 * cb, 0.0) / det2) * 1.001 + 0.5);
        }
    }
    if (ex < -1e29f) ex = ey = -__int_as_float(0x7f800000);  // never reaches 1/255
    st.pw = pw;
    st.depth = pv.z;
    st.conic = conic;
    st.ctx = ctx;
    st.cty = cty;
    st.op = op;
    st.ex = ex;
    st.ey = ey;
    st.hp = hp;
    st.hm = hm;
    return true;
}

// The raw SH colour of a Gaussian the geometry step kept, and its 48-byte record.
// rest_row (may be null): its SH-rest row where the caller staged it (shared memory),
// else the row is read from features_rest.
__device__ __forceinline__ void project_finish(const ProjectArgs &a, int i, int64_t o, const ProjState &st,
                                               const float *rest_row) {
    const V3 pw = st.pw;
    // SH colour, raw (core/cpu/msplat_cpu.cpp:160-190)
    V3 cp{a.cam.cam_pos[0], a.cam.cam_pos[1], a.cam.cam_pos[2]};
    V3 d = unit(sub(pw, cp));
    const float *dc = a.features_dc + 3 * (size_t)i;
    const float *rest = rest_row ? rest_row : a.features_rest + (size_t)a.rest_stride * i;
    float col[3];
    const uint32_t deg = a.cam.degrees_to_use;
#pragma unroll
    for (int c = 0; c < 3; ++c) col[c] = SH_C0 * dc[c];
    if (deg >= 1) {
        float x = d.x, y = d.y, z = d.z;
        float xx = x * x, xy = x * y, xz = x * z, yy = y * y, yz = y * z, zz = z * z;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float *r = rest + c;
            col[c] += SH_C1 * (-y * r[0] + z * r[3] - x * r[6]);
            if (deg < 2) continue;
            col[c] += (SH_C2_0 * xy * r[9] + SH_C2_1 * yz * r[12] + SH_C2_2 * (2.f * zz - xx - yy) * r[15] +
                       SH_C2_3 * xz * r[18] + SH_C2_4 * (xx - yy) * r[21]);
            if (deg < 3) continue;
            col[c] += (SH_C3_0 * y * (3.f * xx - yy) * r[24] + SH_C3_1 * xy * z * r[27] +
                       SH_C3_2 * y * (4.f * zz - xx - yy) * r[30] +
                       SH_C3_3 * z * (2.f * zz - 3.f * xx - 3.f * yy) * r[33] +
                       SH_C3_4 * x * (4.f * zz - xx - yy) * r[36] + SH_C3_5 * z * (xx - yy) * r[39] +
                       SH_C3_6 * x * (xx - 3.f * yy) * r[42]);
            if (deg < 4) continue;
            col[c] += (SH_C4_0 * xy * (xx - yy) * r[45] + SH_C4_1 * yz * (3.f * xx - yy) * r[48] +
                       SH_C4_2 * xy * (7.f * zz - 1.f) * r[51] + SH_C4_3 * yz * (7.f * zz - 3.f) * r[54] +
                       SH_C4_4 * (zz * (35.f * zz - 30.f) + 3.f) * r[57] + SH_C4_5 * xz * (7.f * zz - 3.f) * r[60] +
                       SH_C4_6 * (xx - yy) * (7.f * zz - 1.f) * r[63] + SH_C4_7 * xz * (xx - 3.f * yy) * r[66] +
                       SH_C4_8 * (xx * (xx - 3.f * yy) - yy * (3.f * xx - yy)) * r[69]);
        }
    }
    float4 *rec = reinterpret_cast<float4 *>(a.splats + o);
    rec[0] = make_float4(st.ctx, st.cty, st.conic.x, st.conic.y);
    rec[1] = make_float4(st.conic.z, st.op, col[0], col[1]);
    rec[2] = make_float4(col[2], st.depth, __uint_as_float(pack_half2_up(st.ex, st.ey)),
                         __uint_as_float(pack_half2_up(st.hp, st.hm)));
}


}  // namespace msplat
