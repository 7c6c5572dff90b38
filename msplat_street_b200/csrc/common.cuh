// Shared device helpers for the msplat B200 kernels.
//
// Parity contract. The splatting kernels reproduce the reference backend's float32
// results (core/cpu/msplat_cpu.cpp, itself a port of core/metal/msplat_metal.metal)
// bit for bit wherever an integer decision depends on them: tile rectangles, radii,
// depth keys and the alpha / transmittance cut-offs. To that end
//  * the translation units that compute them are compiled with -fmad=false, so every
//    a*b+c stays two rounded operations, in the reference's order;
//  * exponentials use exp_ref(): exp evaluated in double and rounded once to float,
//    which agrees with a correctly rounded expf except in rare near-halfway cases;
//  * division and square root are IEEE (nvcc's default -prec-div / -prec-sqrt).
// Matrices are column-major (c[col] is a column) because the reference's helper
// types follow MSL conventions (core/cpu/cpu_math.hpp:1-4).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace msplat {

constexpr int TILE = 16;            // core/cpu/msplat_cpu.cpp:27
constexpr int TILE_PIX = TILE * TILE;

// Real SH basis constants (core/cpu/msplat_cpu.cpp:29-38).
constexpr float SH_C0 = 0.28209479177387814f;
constexpr float SH_C1 = 0.4886025119029199f;
constexpr float SH_C2_0 = 1.0925484305920792f, SH_C2_1 = -1.0925484305920792f, SH_C2_2 = 0.31539156525252005f,
                SH_C2_3 = -1.0925484305920792f, SH_C2_4 = 0.5462742152960396f;
constexpr float SH_C3_0 = -0.5900435899266435f, SH_C3_1 = 2.890611442640554f, SH_C3_2 = -0.4570457994644658f,
                SH_C3_3 = 0.3731763325901154f, SH_C3_4 = -0.4570457994644658f, SH_C3_5 = 1.445305721320277f,
                SH_C3_6 = -0.5900435899266435f;
constexpr float SH_C4_0 = 2.5033429417967046f, SH_C4_1 = -1.7701307697799304f, SH_C4_2 = 0.9461746957575601f,
                SH_C4_3 = -0.6690465435572892f, SH_C4_4 = 0.10578554691520431f, SH_C4_5 = -0.6690465435572892f,
                SH_C4_6 = 0.47308734787878004f, SH_C4_7 = -1.7701307697799304f, SH_C4_8 = 0.6258357354491761f;

__host__ __device__ inline uint32_t num_sh_bases(uint32_t degree) {
    return degree == 0 ? 1 : degree == 1 ? 4 : degree == 2 ? 9 : degree == 3 ? 16 : 25;
}

// exp in double, rounded once to float
__device__ __forceinline__ float exp_ref(float x) { return (float)exp((double)x); }

// The rasterizers' exponential, exp(x) rounded once to float for x = -sigma in
// [-5.55, 0]: Tang's table-driven method (P. T. P. Tang, ACM TOMS 15(2), 1989) in
// double precision. x = (64 m + j) ln2 / 64 + r with |r| <= ln2 / 128, so
// exp(x) = 2^m 2^(j/64) exp(r); exp(r) is its Taylor polynomial of degree 5 (truncation
// below 3.5e-17 on the interval) and 2^(j/64) comes from a 64-entry table that the
// block fills once (exp_table_init). The double result is within a few ulps of exp(x),
// so the float it rounds to equals exp_ref's unless exp(x) lies within about 1e-15 of
// a float rounding boundary. Valid for x in [-700, 0].
constexpr double EXP_INV_LN2_64 = 92.33248261689366;    // 64 / ln 2
constexpr double EXP_LN2_64_HI = 0x1.62e42fefa2000p-7;  // ln 2 / 64 to 40 bits: k * HI is exact
constexpr double EXP_LN2_64_LO = 0x1.9ef35793c7673p-47; // ln 2 / 64 - HI
constexpr int EXP_TABLE = 64;

// Every thread of the block calls it; the table is ready after the next barrier.
__device__ __forceinline__ void exp_table_init(double *t) {
    for (int j = threadIdx.x; j < EXP_TABLE; j += blockDim.x) t[j] = exp2((double)j * (1.0 / EXP_TABLE));
}

__device__ __forceinline__ float exp_tab(float xf, const double *t) {
    const double x = (double)xf;
    // k = round(x 64 / ln 2): adding 1.5 * 2^52 leaves the rounded integer in the low
    // word of the sum (exact for |k| < 2^31)
    const double shifted = fma(x, EXP_INV_LN2_64, 0x1.8p52);
    const int ki = __double2loint(shifted);
    const double k = shifted - 0x1.8p52;
    double r = fma(-k, EXP_LN2_64_HI, x);
    r = fma(-k, EXP_LN2_64_LO, r);
    double p = fma(r, 1.0 / 120.0, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    const double v = t[ki & (EXP_TABLE - 1)] * p;
    const int m = ki >> 6;  // floor(ki / 64): the power of two, added to the exponent field
    return (float)__hiloint2double(__double2hiint(v) + m * (1 << 20), __double2loint(v));
}

// The same exponential with the power of two folded into the table, for x in
// [-5.55, 0] (-sigma over the rasterizers' range): entry i = 2^m 2^(j/64) for
// ki = -i = 64 m + j, the old table's entry scaled exactly, so v = entry * p is the
// old t[j] * p scaled by 2^m -- the same double, rounded to the same float -- with the
// exponent-field arithmetic gone. Indices past the span are clamped (not reached for
// x >= -5.55). The block fills the table in two steps with one barrier between
// (exp_span_init_a, __syncthreads, exp_span_init_b).
constexpr int EXP_SPAN = 520;  // covers ki = round(x 64 / ln 2) down to -519 (x >= -5.62)

__device__ __forceinline__ void exp_span_init_a(double *t64) { exp_table_init(t64); }
__device__ __forceinline__ void exp_span_init_b(double *span, const double *t64) {
    for (int i = threadIdx.x; i < EXP_SPAN; i += blockDim.x) {
        const int ki = -i;
        span[i] = scalbn(t64[ki & (EXP_TABLE - 1)], ki >> 6);
    }
}

__device__ __forceinline__ float exp_span(float xf, const double *span) {
    const double x = (double)xf;
    const double shifted = fma(x, EXP_INV_LN2_64, 0x1.8p52);
    const int ki = __double2loint(shifted);
    const double k = shifted - 0x1.8p52;
    double r = fma(-k, EXP_LN2_64_HI, x);
    r = fma(-k, EXP_LN2_64_LO, r);
    double p = fma(r, 1.0 / 120.0, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    return (float)(span[min(-ki, EXP_SPAN - 1)] * p);
}

// Two float32 values in one 64-bit register pair, for sm_100's packed FP32
// instructions (PTX add / mul / fma .rn.f32x2): one instruction issues two IEEE
// single-precision operations, each rounded exactly as its scalar form, so packing
// changes no result -- only the instruction count of an issue-bound kernel.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pack2(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 unpack2(f32x2 v) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

struct V2 { float x, y; };
struct V3 { float x, y, z; };
struct Q4 { float x, y, z, w; };  // quaternion stored (w, x, y, z) lands in x, y, z, w

__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 scl(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 scl(float s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 ld3(const float *p, int64_t i) { return V3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ void st3(float *p, int64_t i, V3 v) {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}
__device__ __forceinline__ float clamp01(float v) { return fminf(fmaxf(v, 0.f), 1.f); }
__device__ __forceinline__ V3 unit(V3 a) { return scl(a, 1.f / sqrtf(dot3(a, a))); }

struct M3 {
    V3 c[3];
};
__device__ __forceinline__ M3 m3(float a0, float a1, float a2, float b0, float b1, float b2, float d0, float d1,
                                 float d2) {
    M3 m;
    m.c[0] = V3{a0, a1, a2};
    m.c[1] = V3{b0, b1, b2};
    m.c[2] = V3{d0, d1, d2};
    return m;
}
__device__ __forceinline__ float el(const V3 &v, int r) { return r == 0 ? v.x : (r == 1 ? v.y : v.z); }
// Column-major product R[j][i] = sum_k A[k][i] * B[j][k], k in order 0,1,2
__device__ __forceinline__ M3 mul(const M3 &A, const M3 &B) {
    M3 R;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        float r0 = A.c[0].x * el(B.c[j], 0) + A.c[1].x * el(B.c[j], 1) + A.c[2].x * el(B.c[j], 2);
        float r1 = A.c[0].y * el(B.c[j], 0) + A.c[1].y * el(B.c[j], 1) + A.c[2].y * el(B.c[j], 2);
        float r2 = A.c[0].z * el(B.c[j], 0) + A.c[1].z * el(B.c[j], 1) + A.c[2].z * el(B.c[j], 2);
        R.c[j] = V3{r0, r1, r2};
    }
    return R;
}
__device__ __forceinline__ M3 tr(const M3 &A) {
    return m3(A.c[0].x, A.c[1].x, A.c[2].x, A.c[0].y, A.c[1].y, A.c[2].y, A.c[0].z, A.c[1].z, A.c[2].z);
}
__device__ __forceinline__ M3 plus(const M3 &A, const M3 &B) {
    M3 R;
    R.c[0] = add(A.c[0], B.c[0]);
    R.c[1] = add(A.c[1], B.c[1]);
    R.c[2] = add(A.c[2], B.c[2]);
    return R;
}
__device__ __forceinline__ M3 smul(float s, const M3 &A) {
    M3 R;
    R.c[0] = scl(A.c[0], s);
    R.c[1] = scl(A.c[1], s);
    R.c[2] = scl(A.c[2], s);
    return R;
}

// Rotation from the (w,x,y,z) quaternion, normalised (core/cpu/msplat_cpu.cpp:77-84)
__device__ __forceinline__ M3 rotmat(Q4 q) {
    float s = 1.f / sqrtf(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    float w = q.x * s, x = q.y * s, y = q.z * s, z = q.w * s;
    return m3(1.f - 2.f * (y * y + z * z), 2.f * (x * y + w * z), 2.f * (x * z - w * y), 2.f * (x * y - w * z),
              1.f - 2.f * (x * x + z * z), 2.f * (y * z + w * x), 2.f * (x * z + w * y), 2.f * (y * z - w * x),
              1.f - 2.f * (x * x + y * y));
}

__device__ __forceinline__ M3 diag_scale(V3 s, float g) {
    M3 S = m3(1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f);
    S.c[0].x = g * s.x;
    S.c[1].y = g * s.y;
    S.c[2].z = g * s.z;
    return S;
}

// 3D covariance R S S^T R^T, upper triangle (core/cpu/msplat_cpu.cpp:94-100)
__device__ __forceinline__ void cov3d_of(V3 s, float g, Q4 q, float *cov) {
    M3 M = mul(rotmat(q), diag_scale(s, g));
    M3 t = mul(M, tr(M));
    cov[0] = t.c[0].x;
    cov[1] = t.c[0].y;
    cov[2] = t.c[0].z;
    cov[3] = t.c[1].y;
    cov[4] = t.c[1].z;
    cov[5] = t.c[2].z;
}

// Two floats as a half2 (low half first), each rounded toward +infinity (values
// beyond the half range become +inf, or -65504 from below).
__device__ __forceinline__ uint32_t pack_half2_up(float lo, float hi) {
    const __half l = __float2half_ru(lo), h = __float2half_ru(hi);
    return (uint32_t)__half_as_ushort(l) | ((uint32_t)__half_as_ushort(h) << 16);
}
__device__ __forceinline__ float2 unpack_half2(uint32_t v) {
    return make_float2(__half2float(__ushort_as_half((unsigned short)(v & 0xffffu))),
                       __half2float(__ushort_as_half((unsigned short)(v >> 16))));
}

// One splat record per Gaussian, read by the rasterizer: centre, conic, sigmoid
// opacity, raw SH colour, depth, and the extents of the region where it can be
// composited (alpha >= 1/255): the half-widths of its box and its half-extents along
// the diagonals x + y and x - y, each a half-precision float rounded up (a region
// never shrinks; -inf marks a splat that never reaches 1/255, +inf an extent with no
// bound). 48 bytes, loaded as three float4.
struct __align__(16) Splat {
    float x, y, cx, cy;   // pixel centre, conic (a, b)
    float cz, op, r, g;   // conic c, sigmoid(opacity), raw colour r g
    float b, depth;       // raw colour b, view depth
    uint32_t box, diag;   // half2 (ex, ey) and half2 (hp, hm)
};
constexpr int SPLAT_FLOATS = sizeof(Splat) / sizeof(float);

// Pixels of a 16x16 tile owned by one warp: an 8x4 block (warp w covers columns
// 8 * (w % 2) .. +7 and rows 4 * (w / 2) .. +3), compact so that per-warp culling
// against a Gaussian's box skips as much as possible.
__device__ __forceinline__ void tile_pixel(int t, int &lx, int &ly) {
    const int w = t >> 5, l = t & 31;
    lx = ((w & 1) << 3) + (l & 7);
    ly = ((w >> 1) << 2) + (l >> 3);
}
// The thread index tile_pixel maps to pixel (lx, ly) of the tile (its inverse).
__device__ __forceinline__ int tile_index(int lx, int ly) {
    return ((((ly >> 2) << 1) + (lx >> 3)) << 5) + ((ly & 3) << 3) + (lx & 7);
}

// Counter-based RNG: PCG hash + Box-Muller (core/cpu/msplat_cpu.cpp:304-323)
__host__ __device__ __forceinline__ uint32_t pcg_hash(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
__host__ __device__ __forceinline__ float rand_unif(uint32_t seed, uint32_t ctr) {
    uint32_t h = pcg_hash(seed ^ pcg_hash(ctr));
    return ((float)(h >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

// Adam with precomputed step_size = lr / bc1 (core/cpu/msplat_cpu.cpp:293-300)
__device__ __forceinline__ void adam_step(float &p, float &m1, float &m2, float g, float ss, float b1, float b2,
                                          float bc2, float eps) {
    float m = b1 * m1 + (1.0f - b1) * g;
    float v = b2 * m2 + (1.0f - b2) * g * g;
    p -= ss * m / (sqrtf(v) / bc2 + eps);
    m1 = m;
    m2 = v;
}

}  // namespace msplat
