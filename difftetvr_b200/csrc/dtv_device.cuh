// Device-side helpers shared by the sm_100a kernels of the tetrahedral
// volume-rendering path.  The discrete parts (projection to 1/256-pixel fixed
// point, the edge-function coverage rule, the FP32 depth key) use explicitly
// rounded FP32 intrinsics so they are bit-reproducible; the continuous parts
// (barycentrics, colours, segment integrals, adjoints) use ordinary FP32 with
// the fast reciprocal (__fdividef) where a quotient feeds only them, on
// screen positions kept as snapped fixed point plus an FP32 residual.  No
// FP64 arithmetic runs on the device.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "dtv_types.h"

namespace dtv {

// Two-wide FP32 arithmetic of sm_100: one FFMA2 / FMUL2 / FADD2 issues two
// FP32 operations, each rounded as its scalar form.
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, bc2(-1.0f), a); }  // a - b
__device__ __forceinline__ float hsum2(float2 a) { return a.x + a.y; }

// Projected vertex: screen position, 1/ze and ze (view depth).
__device__ __forceinline__ float4 project_vertex(const CamDev& c, float x, float y, float z, int2& fix) {
    const float* V = c.V;
    float xv = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(V[0], x), __fmul_rn(V[4], y)), __fmul_rn(V[8], z)), V[12]);
    float yv = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(V[1], x), __fmul_rn(V[5], y)), __fmul_rn(V[9], z)), V[13]);
    float zv = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(V[2], x), __fmul_rn(V[6], y)), __fmul_rn(V[10], z)), V[14]);
    float ze = -zv;
    float iz = __fdiv_rn(1.0f, ze);
    float sx = __fadd_rn(c.cx, __fmul_rn(c.f, __fmul_rn(xv, iz)));
    float sy = __fsub_rn(c.cy, __fmul_rn(c.f, __fmul_rn(yv, iz)));
    bool valid = (ze >= c.znear) && (ze <= c.zfar) && (fabsf(sx) <= kGuardPx) && (fabsf(sy) <= kGuardPx);
    if (valid) {
        fix.x = __float2int_rn(__fmul_rn(sx, 256.0f));
        fix.y = __float2int_rn(__fmul_rn(sy, 256.0f));
    } else {
        fix.x = kInvalidFix;
        fix.y = kInvalidFix;
    }
    return make_float4(sx, sy, iz, ze);
}

// Float-float arithmetic (an unevaluated sum hi + lo of two FP32 values) for
// the continuous path's projection: error-free sum and product (Knuth's
// TwoSum, the FMA product error), so a screen position is carried to about
// 2^-44 relative without FP64.
struct F2 {
    float hi, lo;
};

__device__ __forceinline__ F2 two_sum(float a, float b) {
    const float s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    return F2{s, __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb))};
}

__device__ __forceinline__ F2 fast_two_sum(float a, float b) {  // |a| >= |b|
    const float s = __fadd_rn(a, b);
    return F2{s, __fsub_rn(b, __fsub_rn(s, a))};
}

__device__ __forceinline__ F2 two_prod(float a, float b) {
    const float p = __fmul_rn(a, b);
    return F2{p, __fmaf_rn(a, b, -p)};
}

// m0 x + m1 y + m2 z + m3 (one row of the view matrix applied to a point).
__device__ __forceinline__ F2 row_dot_ff(float m0, float m1, float m2, float m3, float x, float y, float z) {
    const F2 p0 = two_prod(m0, x), p1 = two_prod(m1, y), p2 = two_prod(m2, z);
    F2 s = two_sum(p0.hi, p1.hi);
    float lo = __fadd_rn(__fadd_rn(p0.lo, p1.lo), s.lo);
    s = two_sum(s.hi, p2.hi);
    lo = __fadd_rn(lo, __fadd_rn(p2.lo, s.lo));
    s = two_sum(s.hi, m3);
    lo = __fadd_rn(lo, s.lo);
    return fast_two_sum(s.hi, lo);
}

// a / b: the remainder a.hi - q b.hi of the correctly rounded quotient is
// exact in FP32 (one FMA), the rest of the remainder is added before the
// correction term is divided out.
__device__ __forceinline__ F2 div_ff(const F2& a, const F2& b) {
    const float q = __fdiv_rn(a.hi, b.hi);
    float r = __fmaf_rn(-q, b.hi, a.hi);
    r = __fadd_rn(r, __fmaf_rn(-q, b.lo, a.lo));
    return fast_two_sum(q, __fdiv_rn(r, b.hi));
}

// Continuous-path projection of the vertex whose coverage-rule fixed point is
// `fix`: x = cx + f xv / ze, y = cy - f yv / ze in float-float, stored as the
// snapped position fix / 256 plus the residual (VGeo).  The oracle's FP64
// projection and this one agree to ~1e-11 px.
__device__ __forceinline__ VGeo project_vertex_geo(const CamDev& c, float x, float y, float z, int2 fix) {
    const float* V = c.V;
    const F2 xv = row_dot_ff(V[0], V[4], V[8], V[12], x, y, z);
    const F2 yv = row_dot_ff(V[1], V[5], V[9], V[13], x, y, z);
    const F2 zv = row_dot_ff(V[2], V[6], V[10], V[14], x, y, z);
    const F2 ze{-zv.hi, -zv.lo};
    const F2 qx = div_ff(xv, ze), qy = div_ff(yv, ze);
    // f q in float-float (f = c.f + c.f_lo), then cx + f qx and cy - f qy.
    const F2 mx = two_prod(c.f, qx.hi), my = two_prod(c.f, qy.hi);
    const float mxl = __fadd_rn(mx.lo, __fmaf_rn(c.f, qx.lo, __fmul_rn(c.f_lo, qx.hi)));
    const float myl = __fadd_rn(my.lo, __fmaf_rn(c.f, qy.lo, __fmul_rn(c.f_lo, qy.hi)));
    const F2 sx = two_sum(c.cx, mx.hi), sy = two_sum(c.cy, -my.hi);
    const float sxl = __fadd_rn(sx.lo, mxl), syl = __fsub_rn(sy.lo, myl);
    VGeo g;
    const bool valid = fix.x != kInvalidFix;
    g.sx = valid ? __fmul_rn(float(fix.x), 0.00390625f) : sx.hi;
    g.sy = valid ? __fmul_rn(float(fix.y), 0.00390625f) : sy.hi;
    g.rx = __fadd_rn(__fsub_rn(sx.hi, g.sx), sxl);  // the difference is exact (Sterbenz)
    g.ry = __fadd_rn(__fsub_rn(sy.hi, g.sy), syl);
    // 1 / ze with one Newton correction on the float-float depth.
    const float i0 = __frcp_rn(ze.hi);
    const float e = __fmaf_rn(-i0, ze.lo, __fmaf_rn(-i0, ze.hi, 1.0f));
    g.iz = __fmaf_rn(i0, e, i0);
    g.ze = ze.hi;
    g.xv = xv.hi;
    g.yv = yv.hi;
    return g;
}

__device__ __forceinline__ long long floor_div256(long long a) { return a >> 8; }  // arithmetic shift = floor
__device__ __forceinline__ long long ceil_div256(long long a) { return -((-a) >> 8); }

// Coverage tie rule for a sample exactly on edge a->b of a triangle whose
// interior has E > 0: the sample belongs to the triangle iff the point nudged
// by (eps, eps^2) is inside.  Shared edges are owned by exactly one face.
__device__ __forceinline__ bool edge_inside(long long E, long long dx, long long dy) {
    return (E > 0) || (E == 0 && ((dy < 0) || (dy == 0 && dx > 0)));
}

// FP32 depth key: perspective-correct view depth at the pixel centre.  The
// operation order matches the CPU oracle exactly.
__device__ __forceinline__ float depth_key(const float4& a, const float4& b, const float4& c, float qx, float qy) {
    float d0x = __fsub_rn(a.x, qx), d0y = __fsub_rn(a.y, qy);
    float d1x = __fsub_rn(b.x, qx), d1y = __fsub_rn(b.y, qy);
    float d2x = __fsub_rn(c.x, qx), d2y = __fsub_rn(c.y, qy);
    float E0 = __fsub_rn(__fmul_rn(d1x, d2y), __fmul_rn(d1y, d2x));
    float E1 = __fsub_rn(__fmul_rn(d2x, d0y), __fmul_rn(d2y, d0x));
    float E2 = __fsub_rn(__fmul_rn(d0x, d1y), __fmul_rn(d0y, d1x));
    float num = __fadd_rn(__fadd_rn(__fmul_rn(E0, a.z), __fmul_rn(E1, b.z)), __fmul_rn(E2, c.z));
    float den = __fadd_rn(__fadd_rn(E0, E1), E2);
    float z = __fdiv_rn(den, num);  // z = 1 / sum(lam_j / ze_j)
    float zmin = fminf(fminf(a.w, b.w), c.w);
    float zmax = fmaxf(fmaxf(a.w, b.w), c.w);
    return fminf(fmaxf(z, zmin), zmax);
}

// Continuous fragment values: perspective-correct barycentrics of the pixel
// centre on the face.  Signed weights (a pixel centre the fixed-point
// coverage rule places just outside the exact projection extrapolates
// linearly, which keeps the values smooth in the vertex positions for a fixed
// list); the depth is clamped to the face's vertex depth range.  Depth and
// colour of a fragment come from the same weights.
struct FaceInterp {
    float lam[3];   // screen-space weights E_j / sum(E)
    float A;        // sum(E)
    float dx[3], dy[3];
    float zb;       // 1 / sum(lam_j iz_j)
    float z;        // zb clamped to the vertex depth range
    bool clamped;
    float bary[3];  // perspective-correct weights
};

// Cross product (a + ar) x (b + br) of two vertex-to-pixel vectors, each the
// exact difference of a snapped position and the pixel centre (a, b) plus its
// residual (ar, br).  ax by - ay bx is formed with one rounding (the FMA
// product error w - ay bx is exact), the residual terms are a few 2^-9 px of
// the vertex distance and go through one FMA chain.  For a face w px wide and
// L px long the edge function is kept to about 2^-24 (L / 256 + |E|), where
// plain FP32 screen coordinates lose 2^-24 |x| L (|x| ~ 1000 px).
__device__ __forceinline__ float cross_res(float ax, float ay, float arx, float ary, float bx, float by, float brx,
                                           float bry) {
    const float w = __fmul_rn(ay, bx);
    const float e = __fmaf_rn(-ay, bx, w);
    const float f = __fmaf_rn(ax, by, -w);
    float t = __fmul_rn(arx, bry);
    t = __fmaf_rn(-ary, brx, t);
    t = __fmaf_rn(ax, bry, t);
    t = __fmaf_rn(arx, by, t);
    t = __fmaf_rn(-ay, brx, t);
    t = __fmaf_rn(-ary, bx, t);
    return __fadd_rn(f, __fadd_rn(e, t));
}

__device__ __forceinline__ void face_interp(const VGeo& a, const VGeo& b, const VGeo& c, float qx, float qy,
                                            FaceInterp& fi) {
    // Snapped differences: multiples of 1/256 px below 2^16 px, exact (x and
    // y as one FP32 pair).
    const float2 nq = make_float2(-qx, -qy);
    const float2 d0 = add2(make_float2(a.sx, a.sy), nq), d1 = add2(make_float2(b.sx, b.sy), nq),
                 d2 = add2(make_float2(c.sx, c.sy), nq);
    const float d0x = d0.x, d0y = d0.y, d1x = d1.x, d1y = d1.y, d2x = d2.x, d2y = d2.y;
    const float E0 = cross_res(d1x, d1y, b.rx, b.ry, d2x, d2y, c.rx, c.ry);
    const float E1 = cross_res(d2x, d2y, c.rx, c.ry, d0x, d0y, a.rx, a.ry);
    const float E2 = cross_res(d0x, d0y, a.rx, a.ry, d1x, d1y, b.rx, b.ry);
    fi.A = E0 + E1 + E2;
    const float iA = __fdividef(1.0f, fi.A);
    fi.lam[0] = E0 * iA;
    fi.lam[1] = E1 * iA;
    fi.lam[2] = E2 * iA;
    const float2 e0 = add2(d0, make_float2(a.rx, a.ry)), e1 = add2(d1, make_float2(b.rx, b.ry)),
                 e2 = add2(d2, make_float2(c.rx, c.ry));
    fi.dx[0] = e0.x; fi.dx[1] = e1.x; fi.dx[2] = e2.x;
    fi.dy[0] = e0.y; fi.dy[1] = e1.y; fi.dy[2] = e2.y;
    const float u0 = fi.lam[0] * a.iz, u1 = fi.lam[1] * b.iz, u2 = fi.lam[2] * c.iz;
    fi.zb = __fdividef(1.0f, u0 + u1 + u2);
    fi.bary[0] = u0 * fi.zb;
    fi.bary[1] = u1 * fi.zb;
    fi.bary[2] = u2 * fi.zb;
    const float zmin = fminf(fminf(a.ze, b.ze), c.ze), zmax = fmaxf(fmaxf(a.ze, b.ze), c.ze);
    fi.clamped = !(fi.zb >= zmin && fi.zb <= zmax);
    fi.z = fminf(fmaxf(fi.zb, zmin), zmax);
}

// Forward-only variant (depth and weights).
__device__ __forceinline__ void face_bary(const VGeo& a, const VGeo& b, const VGeo& c, float qx, float qy,
                                          float bary[3], float& z) {
    FaceInterp fi;
    face_interp(a, b, c, qx, qy, fi);
    bary[0] = fi.bary[0];
    bary[1] = fi.bary[1];
    bary[2] = fi.bary[2];
    z = fi.z;
}

__device__ __forceinline__ bool skip_pair(uint32_t bits0, uint32_t bits1) {
    // Forward.glsl:183-185: back-facing boundary followed by front-facing boundary.
    return ((bits0 & 3u) == 2u) && ((bits1 & 3u) == 3u);
}

}  // namespace dtv
