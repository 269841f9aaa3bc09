// Plain structs and constants shared by host code and the sm_100a kernels.
#pragma once
#include <cstdint>
#include <climits>

namespace dtv {

constexpr int kNumSubdivs = 4;             // Data/Shaders/Common/RayCommon.glsl:1-2
constexpr float kGuardPx = 1048576.0f;     // |screen coord| limit (2^20 px) for int64 edge functions
constexpr int32_t kInvalidFix = INT32_MIN; // marks a vertex outside [znear, zfar] or the guard band

// Camera constants, computed once on the host (see dtv_camera_constants).
struct CamDev {
    float V[16];    // view matrix, column-major
    float f;        // 0.5 * H / tan(fovy/2), rounded to FP32 (discrete path)
    float f_lo;     // its rounding error: f + f_lo carries the constant to ~2^-48 (continuous path)
    float cx, cy;   // 0.5 * W, 0.5 * H
    float znear, zfar;
    int W, H;
};

// Projection of a vertex for the continuous path (barycentrics, depth,
// adjoint), all FP32.  The screen position is split into the vertex's
// 1/256-pixel fixed-point position of the coverage rule (sx, sy: exact
// multiples of 1/256 px) and the residual of the exact projection against it
// (rx, ry, |r| <= ~1/512 px, from a compensated float-float projection).
// Pixel-centre differences of the snapped part are exact in FP32, so the
// edge functions of thin, nearly edge-on faces are formed from exact products
// plus small correction terms (face_interp).  1/ze, ze and the view-space
// x, y for the depth and the world-space adjoint.  32 bytes.
struct alignas(16) VGeo {
    float sx, sy;   // snapped position (px)
    float rx, ry;   // exact projected position - snapped position (px)
    float iz, ze, xv, yv;
};

// Per-render settings that the kernels read.
struct ShadeDev {
    float atten;
    float ert_thresh;   // terminate before a segment once T < ert_thresh
    int use_ert;
    int use_abs_grad;
    float clear[4];
};

}  // namespace dtv
