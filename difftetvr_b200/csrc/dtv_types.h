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
    double fd;      // the same in FP64 (continuous path)
    float cx, cy;   // 0.5 * W, 0.5 * H
    float znear, zfar;
    int W, H;
};

// FP64 projection of a vertex for the continuous path (barycentrics, depth,
// adjoint): screen position in FP64 so that thin, nearly edge-on faces keep
// accurate weights; 1/ze, ze and the view-space x, y in FP32.  32 bytes.
struct alignas(16) VGeo {
    double sx, sy;
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
