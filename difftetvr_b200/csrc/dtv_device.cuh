// Device-side helpers shared by the sm_100a kernels of the tetrahedral
// volume-rendering path.  The discrete parts (projection to 1/256-pixel fixed
// point, the edge-function coverage rule, the FP32 depth key) use explicitly
// rounded FP32 intrinsics so they are bit-reproducible; the continuous parts
// (barycentrics, colours, segment integrals, adjoints) use ordinary FP32 with
// the fast reciprocal (__fdividef) where a quotient feeds only them.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "dtv_types.h"

namespace dtv {

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

// FP64 projection of the same vertex (continuous path).
__device__ __forceinline__ VGeo project_vertex_geo(const CamDev& c, float x, float y, float z) {
    const float* V = c.V;
    const double X = x, Y = y, Z = z;
    const double xv = ((double(V[0]) * X + double(V[4]) * Y) + double(V[8]) * Z) + double(V[12]);
    const double yv = ((double(V[1]) * X + double(V[5]) * Y) + double(V[9]) * Z) + double(V[13]);
    const double zv = ((double(V[2]) * X + double(V[6]) * Y) + double(V[10]) * Z) + double(V[14]);
    const double ze = -zv;
    const double iz = 1.0 / ze;
    VGeo g;
    g.sx = double(c.cx) + c.fd * (xv * iz);
    g.sy = double(c.cy) - c.fd * (yv * iz);
    g.iz = float(iz);
    g.ze = float(ze);
    g.xv = float(xv);
    g.yv = float(yv);
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
// centre on the face, from the FP64 screen positions (edge functions in FP64,
// so thin, nearly edge-on faces keep accurate weights).  Signed weights (a
// pixel centre the fixed-point coverage rule places just outside the exact
// projection extrapolates linearly); the depth is clamped to the face's vertex
// depth range.  Depth and colour of a fragment come from the same weights.
struct FaceInterp {
    float lam[3];   // screen-space weights E_j / sum(E)
    float A;        // sum(E)
    float dx[3], dy[3];
    float zb;       // 1 / sum(lam_j iz_j)
    float z;        // zb clamped to the vertex depth range
    bool clamped;
    float bary[3];  // perspective-correct weights
};

__device__ __forceinline__ void face_interp(const VGeo& a, const VGeo& b, const VGeo& c, float qx, float qy,
                                            FaceInterp& fi) {
    const double d0x = a.sx - double(qx), d0y = a.sy - double(qy);
    const double d1x = b.sx - double(qx), d1y = b.sy - double(qy);
    const double d2x = c.sx - double(qx), d2y = c.sy - double(qy);
    const double E0 = d1x * d2y - d1y * d2x;
    const double E1 = d2x * d0y - d2y * d0x;
    const double E2 = d0x * d1y - d0y * d1x;
    const double A = E0 + E1 + E2;
    fi.A = float(A);
    const float iA = __fdividef(1.0f, fi.A);
    fi.lam[0] = float(E0) * iA;
    fi.lam[1] = float(E1) * iA;
    fi.lam[2] = float(E2) * iA;
    fi.dx[0] = float(d0x); fi.dx[1] = float(d1x); fi.dx[2] = float(d2x);
    fi.dy[0] = float(d0y); fi.dy[1] = float(d1y); fi.dy[2] = float(d2y);
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

__device__ __forceinline__ float4 lerp4(const float4& a, const float4& b, float t) {
    return make_float4(a.x + (b.x - a.x) * t, a.y + (b.y - a.y) * t, a.z + (b.z - a.z) * t, a.w + (b.w - a.w) * t);
}

__device__ __forceinline__ float4 f4add(float4 a, float4 b) {
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

__device__ __forceinline__ float4 f4scale(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }

}  // namespace dtv
