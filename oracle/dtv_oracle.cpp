// CPU oracle for the differentiable tetrahedral volume-rendering hot path.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product (difftetvr_b200/) links,
// loads or calls this file; only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py use it, always as the
// checker or as the timed CPU baseline, never as the thing shipped.
//
// It is a plain C++ restatement of the reference's algorithm (GLSL shaders and
// C++ host code of DiffTetVR), instantiated in double (the FP64 oracle) and in
// float (the timed CPU port).  Every function cites the reference file:line it
// follows.  Discrete decisions (which pixel a face covers, the per-pixel depth
// order) are computed with integer / explicitly-ordered FP32 arithmetic that
// the CUDA path reproduces bit for bit; everything continuous (depth used for
// segment lengths, barycentrics, colours, the segment integral, the adjoint)
// runs in the template precision R.
//
// Parity status: the reference cannot run here (Vulkan only), and it ships no
// golden vectors.  This oracle is pinned by closed-form known answers
// (single-tet optical depth, empty pixels, a->0 limit of the segment
// integral), by FP64 central differences of its own forward, and by the mesh
// fixtures of TetMesh::loadTestData; see tests/test_oracle_*.py.

#include <cstdint>
#include <cstring>
#include <cmath>
#include <vector>
#include <algorithm>
#include <atomic>
#include <type_traits>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Face table, src/Tet/TetMesh.cpp:1175-1181 (also Data/Shaders/Common/TetFaceTable.glsl:29-34):
// consistent outward winding for each of the four faces of a tet.
const int kTetFace[4][4] = {
    {0, 1, 2, 3}, {1, 0, 3, 2}, {0, 2, 3, 1}, {2, 1, 3, 0},
};

constexpr int kNumSubdivs = 4;             // Data/Shaders/Common/RayCommon.glsl:1-2
constexpr float kGuardPx = 1048576.0f;     // |screen coord| limit (2^20 px) for the int64 edge functions

struct Camera {
    float view[16];   // column-major, as Renderer.set_view_matrix (src/Module/Module.cpp:904-911)
    float fovy;       // radians
    float znear, zfar;
    int32_t width, height;
};

struct Params {
    float attenuation;        // TetMeshVolumeRenderer::attenuationCoefficient
    int32_t use_ert;          // USE_TERMINATION_INDEX (TetMeshVolumeRenderer.cpp:417-419)
    float ert_thresh;         // earlyRayOutThresh = 1 - earlyRayTerminationAlpha
    float clear_color[4];     // blended under the premultiplied result (BACK_TO_FRONT_PREMUL_ALPHA)
    int32_t use_abs_grad;     // Backward.glsl:449-468
    int32_t row_begin, row_end;  // pixel rows to process (bounded CPU samples); row_end<=0 means all
};

// Camera constants.  Perspective RH, depth [0,1], y flipped for a top-left
// origin (TetMeshRendererPPLL.cpp:675-681 shows the same perspectiveRH_ZO with
// [1][1] negated).  Screen x = cx + f * xv/ze, y = cy - f * yv/ze, ze = -zv.
struct CamConst {
    float V[16];
    float f, cx, cy, znear, zfar;
    double fd, cxd, cyd;
    int W, H;
};

CamConst make_cam(const Camera& c) {
    CamConst k;
    std::memcpy(k.V, c.view, sizeof(k.V));
    const double tanh = std::tan(0.5 * double(c.fovy));
    k.fd = 0.5 * double(c.height) / tanh;
    k.f = float(k.fd);
    k.cx = 0.5f * float(c.width);
    k.cy = 0.5f * float(c.height);
    k.cxd = k.cx;
    k.cyd = k.cy;
    k.znear = c.znear;
    k.zfar = c.zfar;
    k.W = c.width;
    k.H = c.height;
    return k;
}

// FP32 projection with a fixed operation order (the CUDA path uses the same
// sequence with __fmul_rn/__fadd_rn, so the snapped coordinates, the coverage
// and the sort keys agree bit for bit).  LinkedListGather.glsl:55-68 projects
// with viewProjectionMatrix; here the projection is split into view transform
// and perspective divide.
struct ProjF {
    float sx, sy, iz, ze;
    int32_t X, Y;     // 1/256-pixel fixed point
    bool valid;
};

ProjF project_f(const CamConst& c, float x, float y, float z) {
    ProjF p;
    const float* V = c.V;
    float xv = ((V[0] * x + V[4] * y) + V[8] * z) + V[12];
    float yv = ((V[1] * x + V[5] * y) + V[9] * z) + V[13];
    float zv = ((V[2] * x + V[6] * y) + V[10] * z) + V[14];
    p.ze = -zv;
    p.iz = 1.0f / p.ze;
    p.sx = c.cx + c.f * (xv * p.iz);
    p.sy = c.cy - c.f * (yv * p.iz);
    p.valid = (p.ze >= c.znear) && (p.ze <= c.zfar) && std::fabs(p.sx) <= kGuardPx &&
              std::fabs(p.sy) <= kGuardPx;
    if (p.valid) {
        p.X = int32_t(std::nearbyint(p.sx * 256.0f));
        p.Y = int32_t(std::nearbyint(p.sy * 256.0f));
    } else {
        p.X = p.Y = 0;
    }
    return p;
}

template <class R>
struct ProjR {
    R sx, sy, iz, ze, xv, yv;
};

template <class R>
ProjR<R> project_r(const CamConst& c, R x, R y, R z) {
    ProjR<R> p;
    const float* V = c.V;
    p.xv = ((R(V[0]) * x + R(V[4]) * y) + R(V[8]) * z) + R(V[12]);
    p.yv = ((R(V[1]) * x + R(V[5]) * y) + R(V[9]) * z) + R(V[13]);
    R zv = ((R(V[2]) * x + R(V[6]) * y) + R(V[10]) * z) + R(V[14]);
    p.ze = -zv;
    p.iz = R(1) / p.ze;
    const R f = std::is_same<R, float>::value ? R(c.f) : R(c.fd);
    p.sx = R(c.cx) + f * (p.xv * p.iz);
    p.sy = R(c.cy) - f * (p.yv * p.iz);
    return p;
}

inline int64_t floor_div(int64_t a, int64_t b) {  // b > 0
    int64_t q = a / b;
    if ((a % b) != 0 && (a < 0)) --q;
    return q;
}
inline int64_t ceil_div(int64_t a, int64_t b) { return -floor_div(-a, b); }

// Top-left style tie rule: a sample exactly on an edge a->b (of a triangle
// oriented so that the interior has E > 0) belongs to the triangle iff the
// sample point nudged by (eps, eps^2) lies inside.  Shared edges are then
// owned by exactly one of the two triangles, so interior faces tile the screen
// without gaps or double hits (the rule of a hardware rasteriser, written out
// so the CPU and the GPU agree exactly).
inline bool edge_inside(int64_t E, int64_t dx, int64_t dy) {
    if (E > 0) return true;
    if (E < 0) return false;
    return (dy < 0) || (dy == 0 && dx > 0);
}

// FP32 depth key of a fragment: perspective-correct view depth at the pixel
// centre from the face's projected vertices.  Fixed operation order; the CUDA
// kernel computes the same bits.  (The reference stores gl_FragCoord.z,
// LinkedListGather.glsl:97; view depth is used here so the segment length
// keeps full FP32 precision.)
inline float depth_key_f(const ProjF& a, const ProjF& b, const ProjF& c, float qx, float qy) {
    float d0x = a.sx - qx, d0y = a.sy - qy;
    float d1x = b.sx - qx, d1y = b.sy - qy;
    float d2x = c.sx - qx, d2y = c.sy - qy;
    float E0 = d1x * d2y - d1y * d2x;
    float E1 = d2x * d0y - d2y * d0x;
    float E2 = d0x * d1y - d0y * d1x;
    float z = ((E0 + E1) + E2) / ((E0 * a.iz + E1 * b.iz) + E2 * c.iz);  // 1 / sum(lam_j / ze_j)
    float zmin = std::fmin(std::fmin(a.ze, b.ze), c.ze);
    float zmax = std::fmax(std::fmax(a.ze, b.ze), c.ze);
    return std::fmin(std::fmax(z, zmin), zmax);
}

inline uint32_t f2u(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline float u2f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// Exact fixed-point coverage of pixel (px, py) by face f (the rule of
// build_fragments); *area2 receives the signed doubled area in the stored winding.
inline bool face_covers(const std::vector<ProjF>& proj, const uint32_t* tri, uint32_t f, int64_t px, int64_t py,
                        int64_t* area2_out) {
    const ProjF& p0 = proj[tri[3 * f]];
    const ProjF& p1 = proj[tri[3 * f + 1]];
    const ProjF& p2 = proj[tri[3 * f + 2]];
    *area2_out = 0;
    if (!(p0.valid && p1.valid && p2.valid)) return false;
    int64_t ax[3] = {p0.X, p1.X, p2.X}, ay[3] = {p0.Y, p1.Y, p2.Y};
    const int64_t area2 = (ax[1] - ax[0]) * (ay[2] - ay[0]) - (ay[1] - ay[0]) * (ax[2] - ax[0]);
    *area2_out = area2;
    if (area2 == 0) return false;
    if (area2 < 0) {
        std::swap(ax[1], ax[2]);
        std::swap(ay[1], ay[2]);
    }
    const int64_t Xc = 256 * px + 128, Yc = 256 * py + 128;
    for (int e = 0; e < 3; ++e) {
        const int a = (e + 1) % 3, b = (e + 2) % 3;
        const int64_t dx = ax[b] - ax[a], dy = ay[b] - ay[a];
        if (!edge_inside(dx * (Yc - ay[a]) - dy * (Xc - ax[a]), dx, dy)) return false;
    }
    return true;
}

struct FragLists {
    std::vector<int64_t> offsets;   // P+1
    std::vector<uint64_t> records;  // (depth bits << 32) | (face << 2) | (boundary << 1) | front
};

// Rasterise every face into per-pixel fragment lists and sort each list.
// LinkedListGather.glsl:84-121 (one node per covered pixel per face, faceBits =
// faceIndex<<2 | boundary<<1 | frontFacing) and LinkedListSort.glsl:189-216 /
// Forward.glsl:107-114 (front-to-back order).  The order here is total: depth
// key, then face index.  Only rows [row_begin, row_end) are emitted.
FragLists build_fragments(const uint32_t* tri, const uint32_t* face_boundary, int64_t F,
                          const std::vector<ProjF>& proj, const CamConst& cam, int row_begin,
                          int row_end) {
    const int W = cam.W, H = cam.H;
    const int64_t P = int64_t(W) * H;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    std::vector<std::vector<std::pair<uint32_t, uint64_t>>> per_thread(nthreads);
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        auto& out = per_thread[tid];
#pragma omp for schedule(dynamic, 256)
        for (int64_t f = 0; f < F; ++f) {
            const ProjF& p0 = proj[tri[3 * f + 0]];
            const ProjF& p1 = proj[tri[3 * f + 1]];
            const ProjF& p2 = proj[tri[3 * f + 2]];
            if (!(p0.valid && p1.valid && p2.valid)) continue;
            int64_t X0 = p0.X, Y0 = p0.Y, X1 = p1.X, Y1 = p1.Y, X2 = p2.X, Y2 = p2.Y;
            int64_t area2 = (X1 - X0) * (Y2 - Y0) - (Y1 - Y0) * (X2 - X0);
            if (area2 == 0) continue;
            const uint32_t front = area2 < 0 ? 1u : 0u;
            const uint32_t bits = (uint32_t(f) << 2) | ((face_boundary[f] & 1u) << 1) | front;
            // Orient so the interior has positive edge functions.
            int64_t ax[3] = {X0, X1, X2}, ay[3] = {Y0, Y1, Y2};
            if (area2 < 0) {
                std::swap(ax[1], ax[2]);
                std::swap(ay[1], ay[2]);
            }
            int64_t minX = std::min({X0, X1, X2}), maxX = std::max({X0, X1, X2});
            int64_t minY = std::min({Y0, Y1, Y2}), maxY = std::max({Y0, Y1, Y2});
            int64_t px0 = std::max<int64_t>(0, ceil_div(minX - 128, 256));
            int64_t px1 = std::min<int64_t>(W - 1, floor_div(maxX - 128, 256));
            int64_t py0 = std::max<int64_t>(std::max(0, row_begin), ceil_div(minY - 128, 256));
            int64_t py1 = std::min<int64_t>(std::min(H, row_end) - 1, floor_div(maxY - 128, 256));
            for (int64_t py = py0; py <= py1; ++py) {
                const int64_t Yc = 256 * py + 128;
                for (int64_t px = px0; px <= px1; ++px) {
                    const int64_t Xc = 256 * px + 128;
                    bool in = true;
                    for (int e = 0; e < 3 && in; ++e) {
                        int a = (e + 1) % 3, b = (e + 2) % 3;
                        int64_t dx = ax[b] - ax[a], dy = ay[b] - ay[a];
                        int64_t E = dx * (Yc - ay[a]) - dy * (Xc - ax[a]);
                        in = edge_inside(E, dx, dy);
                    }
                    if (!in) continue;
                    float qx = float(px) + 0.5f, qy = float(py) + 0.5f;
                    float z = depth_key_f(p0, p1, p2, qx, qy);
                    uint64_t rec = (uint64_t(f2u(z)) << 32) | bits;
                    out.emplace_back(uint32_t(py * W + px), rec);
                }
            }
        }
    }
    FragLists fl;
    fl.offsets.assign(P + 1, 0);
    for (auto& v : per_thread)
        for (auto& pr : v) fl.offsets[pr.first + 1]++;
    for (int64_t i = 0; i < P; ++i) fl.offsets[i + 1] += fl.offsets[i];
    fl.records.resize(fl.offsets[P]);
    std::vector<int64_t> cursor(fl.offsets.begin(), fl.offsets.end() - 1);
    for (auto& v : per_thread)
        for (auto& pr : v) fl.records[cursor[pr.first]++] = pr.second;
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t p = 0; p < P; ++p)
        std::sort(fl.records.begin() + fl.offsets[p], fl.records.begin() + fl.offsets[p + 1]);
    return fl;
}

// ---------------------------------------------------------------------------
// Continuous per-fragment values in precision R.
template <class R>
struct Frag {
    R z;
    R col[4];
    uint32_t face;
    bool boundary, front;
};

template <class R>
struct MeshR {
    const uint32_t* tri;
    const R* pos;
    const R* col;
    std::vector<ProjR<R>> proj;
};

// Perspective-correct barycentrics of the pixel centre on the face (screen
// space), which equal the world-space barycentrics of the point where the pixel
// ray meets the face plane.  Forward.glsl:80-103 computes the same point by
// unprojecting gl_FragCoord.z and takes unsigned cross-product ratios; here
// the signed ratios are used (equal inside the face; linear just outside it,
// where the fixed-point coverage rule can place a pixel centre).  The depth
// is clamped to the face's vertex depth range; the fragment's depth and
// colour come from the same weights.
template <class R>
void face_bary(const ProjR<R>& a, const ProjR<R>& b, const ProjR<R>& c, R qx, R qy, R lam[3], R bary[3],
               R& z, bool* z_clamped = nullptr) {
    R d0x = a.sx - qx, d0y = a.sy - qy;
    R d1x = b.sx - qx, d1y = b.sy - qy;
    R d2x = c.sx - qx, d2y = c.sy - qy;
    R E0 = d1x * d2y - d1y * d2x;
    R E1 = d2x * d0y - d2y * d0x;
    R E2 = d0x * d1y - d0y * d1x;
    R A = (E0 + E1) + E2;
    lam[0] = E0 / A;
    lam[1] = E1 / A;
    lam[2] = E2 / A;
    R u0 = lam[0] * a.iz, u1 = lam[1] * b.iz, u2 = lam[2] * c.iz;
    R w = (u0 + u1) + u2;
    R zb = R(1) / w;
    bary[0] = u0 * zb;
    bary[1] = u1 * zb;
    bary[2] = u2 * zb;
    R zmin = std::min(std::min(a.ze, b.ze), c.ze), zmax = std::max(std::max(a.ze, b.ze), c.ze);
    z = std::min(std::max(zb, zmin), zmax);
    if (z_clamped) *z_clamped = !(zb >= zmin && zb <= zmax);
}

template <class R>
Frag<R> eval_frag(const MeshR<R>& m, uint64_t rec, int px, int py) {
    Frag<R> fr;
    uint32_t bits = uint32_t(rec & 0xffffffffu);
    fr.face = bits >> 2;
    fr.boundary = (bits >> 1) & 1u;
    fr.front = bits & 1u;
    uint32_t i0 = m.tri[3 * fr.face], i1 = m.tri[3 * fr.face + 1], i2 = m.tri[3 * fr.face + 2];
    R lam[3], b[3];
    face_bary(m.proj[i0], m.proj[i1], m.proj[i2], R(px) + R(0.5), R(py) + R(0.5), lam, b, fr.z);
    for (int k = 0; k < 4; ++k)
        fr.col[k] = b[0] * m.col[4 * i0 + k] + b[1] * m.col[4 * i1 + k] + b[2] * m.col[4 * i2 + k];
    return fr;
}

// Series of phi1(x) = (1 - e^-x)/x, psi(x) = (phi1(x) - e^-x)/x and
// chi(x) = (1 - e^-x (1 + x + x^2))/x^2 (coefficients from the exponential
// series), used for small optical depth x where the direct forms cancel.
template <class R>
inline R poly(const double* c, int n, R x) {
    R p = R(c[n - 1]);
    for (int i = n - 2; i >= 0; --i) p = p * x + R(c[i]);
    return p;
}
const double kPhi1[10] = {1.0, -1.0 / 2, 1.0 / 6, -1.0 / 24, 1.0 / 120, -1.0 / 720, 1.0 / 5040, -1.0 / 40320,
                          1.0 / 362880, -1.0 / 3628800};
const double kPsi[10] = {1.0 / 2, -2.0 / 6, 3.0 / 24, -4.0 / 120, 5.0 / 720, -6.0 / 5040, 7.0 / 40320, -8.0 / 362880,
                         9.0 / 3628800, -10.0 / 39916800};
const double kChi[10] = {-1.0 / 2, 4.0 / 6, -9.0 / 24, 16.0 / 120, -25.0 / 720, 36.0 / 5040, -49.0 / 40320,
                         64.0 / 362880, -81.0 / 3628800, 100.0 / 39916800};
template <class R>
inline R series_cut() { return std::is_same<R, float>::value ? R(0.5) : R(1e-3); }

// accumulateLinearConst, Data/Shaders/Common/ForwardCommon.glsl:42-49:
//   A = exp(-a t),  C = (1 - A) c0 + ((t + 1/a) A - 1/a) (c0 - c1),  alpha = 1 - A,
// written as 1 - A = x phi1(x), (t + 1/a) A - 1/a = -t x psi(x) with x = a t.
// The reference drops the term for a < 1e-6; here only a <= 0 is dropped and
// 0 < a < 1e-6 keeps the (continuous) value, which differs by at most a t.
template <class R>
inline bool seg_integral(R t, const R c0[3], const R c1[3], R a, R cacc[3], R& A) {
    if (!(a > R(0))) {
        A = R(1);
        cacc[0] = cacc[1] = cacc[2] = R(0);
        return false;
    }
    const R x = a * t;
    A = std::exp(-x);
    R omA, K;
    if (std::fabs(x) < series_cut<R>()) {
        omA = x * poly(kPhi1, 10, x);
        K = -t * x * poly(kPsi, 10, x);
    } else {
        omA = R(1) - A;
        K = (t + R(1) / a) * A - R(1) / a;
    }
    for (int k = 0; k < 3; ++k) cacc[k] = omA * c0[k] + K * (c0[k] - c1[k]);
    return true;
}
template <class R>
inline bool skip_pair(const Frag<R>& f0, const Frag<R>& f1) {
    // Forward.glsl:183-185: gap between a back-facing and a front-facing boundary face.
    return (f0.boundary && !f0.front) && (f1.boundary && f1.front);
}

template <class R>
void sub_inputs(const Frag<R>& f0, const Frag<R>& f1, int s, R atten, R c0[3], R c1[3], R& a) {
    const R inv = R(1) / R(kNumSubdivs);
    R fb = R(s) * inv, fm = (R(s) + R(0.5)) * inv, fe = (R(s) + R(1)) * inv;
    for (int k = 0; k < 3; ++k) {
        c0[k] = f0.col[k] + (f1.col[k] - f0.col[k]) * fb;
        c1[k] = f0.col[k] + (f1.col[k] - f0.col[k]) * fe;
    }
    a = (f0.col[3] + (f1.col[3] - f0.col[3]) * fm) * atten;
}

// Front-to-back compositing of one pixel, Forward.glsl:159-211 and :250-261.
// State is (premultiplied colour C, transmittance T); alpha = 1 - T.  Early ray
// termination (Forward.glsl:169-173) stops before segment i once T < thresh.
template <class R>
void composite_pixel(const MeshR<R>& m, const Params& prm, const uint64_t* recs, int64_t n, int px, int py,
                     R out[4], R& Tfinal, uint32_t& term) {
    R C[3] = {0, 0, 0};
    R T = 1;
    uint32_t i = 1;
    if (n >= 2) {
        Frag<R> f1 = eval_frag(m, recs[0], px, py), f0;
        for (i = 1; i < uint32_t(n); ++i) {
            if (prm.use_ert && T < R(prm.ert_thresh)) break;
            f0 = f1;
            f1 = eval_frag(m, recs[i], px, py);
            if (skip_pair(f0, f1)) continue;
            R t = f1.z - f0.z;
            R tSeg = t / R(kNumSubdivs);
            for (int s = 0; s < kNumSubdivs; ++s) {
                R c0[3], c1[3], a, cacc[3], A;
                sub_inputs(f0, f1, s, R(prm.attenuation), c0, c1, a);
                if (!seg_integral(tSeg, c0, c1, a, cacc, A)) continue;
                for (int k = 0; k < 3; ++k) C[k] += T * cacc[k];
                T *= A;
            }
        }
    } else {
        i = uint32_t(n);
    }
    term = (n >= 2) ? i : uint32_t(n);
    Tfinal = T;
    for (int k = 0; k < 3; ++k) out[k] = C[k] + T * R(prm.clear_color[k]);
    out[3] = (R(1) - T) + T * R(prm.clear_color[3]);
}

// Adjoint of seg_integral w.r.t. (tSeg, a, c0, c1); BackwardCommon.glsl:116-133
// (accumulateLinearConstAdjoint), with dK/da = t^2 chi(x).  For a <= 0 the
// forward drops the term; its gradient is the a -> 0+ limit (the reference's
// small-a branch), so a density clamped to zero can grow again.
template <class R>
void seg_integral_adjoint(R tSeg, const R c0[3], const R c1[3], R a, R A, const R gc[3], R gA, R& g_t,
                          R& g_a, R g_c0[3], R g_c1[3]) {
    if (!(a > R(0))) {
        g_t = 0;
        g_a = R(0);
        for (int k = 0; k < 3; ++k) {
            g_a += gc[k] * (tSeg * c0[k] + R(0.5) * tSeg * tSeg * (c1[k] - c0[k]));
            g_c0[k] = g_c1[k] = R(0);
        }
        g_a += -gA * tSeg;  // alpha_acc = 1 - A ~ a t  =>  d alpha/da = t, gA = -g_alpha
        return;
    }
    const R x = a * tSeg;
    R omA, K, chi;
    if (std::fabs(x) < series_cut<R>()) {
        omA = x * poly(kPhi1, 10, x);
        K = -tSeg * x * poly(kPsi, 10, x);
        chi = poly(kChi, 10, x);
    } else {
        omA = R(1) - A;
        K = (tSeg + R(1) / a) * A - R(1) / a;
        chi = (omA - x * A * (R(1) + x)) / (x * x);
    }
    const R dK = tSeg * tSeg * chi;
    R dot_t = 0, dot_a = 0;
    for (int k = 0; k < 3; ++k) {
        dot_t += gc[k] * (a * A * (c0[k] + tSeg * (c1[k] - c0[k])));
        dot_a += gc[k] * (tSeg * A * c0[k] + dK * (c0[k] - c1[k]));
        g_c0[k] = (omA + K) * gc[k];
        g_c1[k] = -K * gc[k];
    }
    g_t = dot_t + gA * (-a * A);
    g_a = dot_a + gA * (-tSeg * A);
}

// Back-propagate (dL/dz, dL/dcolour) of one fragment to its face's three
// vertex positions and colours (exact derivative of face_bary + projection).
template <class R>
void frag_vertex_grads(const MeshR<R>& m, const CamConst& cam, uint32_t face, int px, int py, R gz,
                       const R gcol[4], bool use_abs, R* grad_pos, R* grad_col) {
    const uint32_t vi[3] = {m.tri[3 * face], m.tri[3 * face + 1], m.tri[3 * face + 2]};
    const ProjR<R>* P[3] = {&m.proj[vi[0]], &m.proj[vi[1]], &m.proj[vi[2]]};
    const R qx = R(px) + R(0.5), qy = R(py) + R(0.5);
    R dx[3], dy[3];
    for (int j = 0; j < 3; ++j) {
        dx[j] = P[j]->sx - qx;
        dy[j] = P[j]->sy - qy;
    }
    R E[3] = {dx[1] * dy[2] - dy[1] * dx[2], dx[2] * dy[0] - dy[2] * dx[0], dx[0] * dy[1] - dy[0] * dx[1]};
    R A = (E[0] + E[1]) + E[2];
    R lam[3], u[3], w = 0;
    for (int j = 0; j < 3; ++j) {
        lam[j] = E[j] / A;
        u[j] = lam[j] * P[j]->iz;
        w += u[j];
    }
    const R zb = R(1) / w;  // weights use the unclamped 1/w; the depth is clamped
    const R zmin = std::min(std::min(P[0]->ze, P[1]->ze), P[2]->ze);
    const R zmax = std::max(std::max(P[0]->ze, P[1]->ze), P[2]->ze);
    const bool clamped = !(zb >= zmin && zb <= zmax);
    R b[3], gb[3], sb = 0;
    for (int j = 0; j < 3; ++j) {
        b[j] = u[j] * zb;
        gb[j] = 0;
        if (m.col)
            for (int k = 0; k < 4; ++k) gb[j] += gcol[k] * m.col[4 * vi[j] + k];
        sb += gb[j] * b[j];
    }
    R glam[3], giz[3], sl = 0;
    for (int j = 0; j < 3; ++j) {
        R gu = zb * (gb[j] - sb) - (clamped ? R(0) : gz * zb * zb);
        glam[j] = gu * P[j]->iz;
        giz[j] = gu * lam[j];
        sl += glam[j] * lam[j];
    }
    R gE[3];
    for (int j = 0; j < 3; ++j) gE[j] = (glam[j] - sl) / A;
    // dE0/d(d1) = (d2y, -d2x), dE0/d(d2) = (-d1y, d1x); cyclic for E1, E2.
    R gsx[3], gsy[3];
    gsx[0] = gE[1] * (-dy[2]) + gE[2] * dy[1];
    gsy[0] = gE[1] * dx[2] + gE[2] * (-dx[1]);
    gsx[1] = gE[0] * dy[2] + gE[2] * (-dy[0]);
    gsy[1] = gE[0] * (-dx[2]) + gE[2] * dx[0];
    gsx[2] = gE[0] * (-dy[1]) + gE[1] * dy[0];
    gsy[2] = gE[0] * dx[1] + gE[1] * (-dx[0]);
    const R f = std::is_same<R, float>::value ? R(cam.f) : R(cam.fd);
    const float* V = cam.V;
    for (int j = 0; j < 3; ++j) {
        const ProjR<R>& p = *P[j];
        R gxv = gsx[j] * f * p.iz;
        R gyv = -gsy[j] * f * p.iz;
        R giz_t = giz[j] + gsx[j] * f * p.xv - gsy[j] * f * p.yv;
        R gzv = giz_t * p.iz * p.iz;  // iz = -1/zv  =>  d iz/d zv = iz^2
        R gp[3] = {R(V[0]) * gxv + R(V[1]) * gyv + R(V[2]) * gzv, R(V[4]) * gxv + R(V[5]) * gyv + R(V[6]) * gzv,
                   R(V[8]) * gxv + R(V[9]) * gyv + R(V[10]) * gzv};
        R gc[4];
        for (int k = 0; k < 4; ++k) gc[k] = b[j] * gcol[k];
        if (use_abs) {
            for (int k = 0; k < 3; ++k) gp[k] = std::fabs(gp[k]);
            for (int k = 0; k < 4; ++k) gc[k] = std::fabs(gc[k]);
        }
        for (int k = 0; k < 3; ++k) grad_pos[3 * vi[j] + k] += gp[k];
        if (grad_col)
            for (int k = 0; k < 4; ++k) grad_col[4 * vi[j] + k] += gc[k];
    }
}

// Adjoint of one pixel, back to front from the termination index.
// Backward.glsl:107-512 restated as the exact derivative of composite_pixel:
// transmittance is rebuilt from the final value by T_in = T_out / A (the
// inversion of Weiss et al. that Backward.glsl:231-246 applies to alpha), all
// four sub-segments are differentiated, and segment length / barycentric
// adjoints follow the screen-space construction of face_bary.
template <class R>
void adjoint_pixel(const MeshR<R>& m, const CamConst& cam, const Params& prm, const uint64_t* recs, int64_t n,
                   int px, int py, R Tfinal, uint32_t term, const R g[4], R* grad_pos, R* grad_col) {
    if (n < 2) return;
    const R atten = R(prm.attenuation);
    R gC[3] = {g[0], g[1], g[2]};
    R gT = g[0] * R(prm.clear_color[0]) + g[1] * R(prm.clear_color[1]) + g[2] * R(prm.clear_color[2]) +
           g[3] * (R(prm.clear_color[3]) - R(1));
    R T = Tfinal;
    int64_t last = prm.use_ert ? int64_t(term) - 1 : n - 1;  // last composited segment index
    if (last < 1) return;
    // Fragment accumulators: fragment i (back of segment i) and i-1 (front).
    Frag<R> fb = eval_frag(m, recs[last], px, py);
    R gz_b = 0, gcol_b[4] = {0, 0, 0, 0};
    for (int64_t i = last; i >= 1; --i) {
        Frag<R> ff = eval_frag(m, recs[i - 1], px, py);
        R gz_f = 0, gcol_f[4] = {0, 0, 0, 0};
        if (!skip_pair(ff, fb)) {
            R t = fb.z - ff.z;
            R tSeg = t / R(kNumSubdivs);
            R g_tot = 0;
            const R inv = R(1) / R(kNumSubdivs);
            for (int s = kNumSubdivs - 1; s >= 0; --s) {
                R c0[3], c1[3], a, cacc[3], A;
                sub_inputs(ff, fb, s, atten, c0, c1, a);
                bool active = seg_integral(tSeg, c0, c1, a, cacc, A);
                R Tin = active ? T / A : T;
                R gcacc[3] = {Tin * gC[0], Tin * gC[1], Tin * gC[2]};
                R gA = Tin * gT;
                if (active) {
                    gT = (gC[0] * cacc[0] + gC[1] * cacc[1] + gC[2] * cacc[2]) + gT * A;
                } else {
                    gA = Tin * gT;  // A == 1 in the forward; derivative through the a->0 limit
                }
                T = Tin;
                R g_t, g_a, g_c0[3], g_c1[3];
                seg_integral_adjoint(tSeg, c0, c1, a, A, gcacc, gA, g_t, g_a, g_c0, g_c1);
                g_tot += g_t * inv;
                R fbg = R(s) * inv, fm = (R(s) + R(0.5)) * inv, fe = (R(s) + R(1)) * inv;
                for (int k = 0; k < 3; ++k) {
                    gcol_f[k] += (R(1) - fbg) * g_c0[k] + (R(1) - fe) * g_c1[k];
                    gcol_b[k] += fbg * g_c0[k] + fe * g_c1[k];
                }
                gcol_f[3] += (R(1) - fm) * g_a * atten;
                gcol_b[3] += fm * g_a * atten;
            }
            gz_f -= g_tot;
            gz_b += g_tot;
        }
        // Fragment i is complete.
        frag_vertex_grads(m, cam, fb.face, px, py, gz_b, gcol_b, prm.use_abs_grad != 0, grad_pos, grad_col);
        fb = ff;
        gz_b = gz_f;
        for (int k = 0; k < 4; ++k) gcol_b[k] = gcol_f[k];
    }
    frag_vertex_grads(m, cam, fb.face, px, py, gz_b, gcol_b, prm.use_abs_grad != 0, grad_pos, grad_col);
}

template <class R>
MeshR<R> make_mesh(const uint32_t* tri, const R* pos, const R* col, int64_t V, const CamConst& cam) {
    MeshR<R> m;
    m.tri = tri;
    m.pos = pos;
    m.col = col;
    m.proj.resize(V);
    for (int64_t v = 0; v < V; ++v) m.proj[v] = project_r<R>(cam, pos[3 * v], pos[3 * v + 1], pos[3 * v + 2]);
    return m;
}

template <class R>
std::vector<ProjF> project_all_f(const R* pos, int64_t V, const CamConst& cam) {
    std::vector<ProjF> pf(V);
    for (int64_t v = 0; v < V; ++v)
        pf[v] = project_f(cam, float(pos[3 * v]), float(pos[3 * v + 1]), float(pos[3 * v + 2]));
    return pf;
}

inline void row_range(const Params& prm, int H, int& r0, int& r1) {
    r0 = std::max(0, prm.row_begin);
    r1 = prm.row_end > 0 ? std::min(H, prm.row_end) : H;
}

template <class R>
int render_impl(const uint32_t* tri, const uint32_t* fbits, int64_t F, const R* pos, const R* col, int64_t V,
                const Camera* camp, const Params* prm, R* image, R* tfinal, uint32_t* term, int64_t* nfrag,
                const float* pos_coverage = nullptr) {
    CamConst cam = make_cam(*camp);
    int r0, r1;
    row_range(*prm, cam.H, r0, r1);
    // Coverage and depth order come from pos_coverage when given (frozen
    // fragment lists for smooth finite differences), else from pos.
    auto pf = pos_coverage ? project_all_f(pos_coverage, V, cam) : project_all_f(pos, V, cam);
    FragLists fl = build_fragments(tri, fbits, F, pf, cam, r0, r1);
    MeshR<R> m = make_mesh(tri, pos, col, V, cam);
    const int W = cam.W;
#pragma omp parallel for schedule(dynamic, 4)
    for (int py = r0; py < r1; ++py) {
        for (int px = 0; px < W; ++px) {
            int64_t p = int64_t(py) * W + px;
            R out[4], Tf;
            uint32_t tm;
            composite_pixel(m, *prm, fl.records.data() + fl.offsets[p], fl.offsets[p + 1] - fl.offsets[p], px,
                            py, out, Tf, tm);
            for (int k = 0; k < 4; ++k) image[4 * p + k] = out[k];
            if (tfinal) tfinal[p] = Tf;
            if (term) term[p] = tm;
        }
    }
    if (nfrag) *nfrag = int64_t(fl.records.size());
    return 0;
}

template <class R>
int adjoint_impl(const uint32_t* tri, const uint32_t* fbits, int64_t F, const R* pos, const R* col, int64_t V,
                 const Camera* camp, const Params* prm, const R* image_adj, R* grad_pos, R* grad_col) {
    CamConst cam = make_cam(*camp);
    int r0, r1;
    row_range(*prm, cam.H, r0, r1);
    auto pf = project_all_f(pos, V, cam);
    FragLists fl = build_fragments(tri, fbits, F, pf, cam, r0, r1);
    MeshR<R> m = make_mesh(tri, pos, col, V, cam);
    const int W = cam.W;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    std::vector<std::vector<R>> gp(nthreads, std::vector<R>(3 * V, R(0)));
    std::vector<std::vector<R>> gc(nthreads, std::vector<R>(4 * V, R(0)));
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
#pragma omp for schedule(dynamic, 4)
        for (int py = r0; py < r1; ++py) {
            for (int px = 0; px < W; ++px) {
                int64_t p = int64_t(py) * W + px;
                const uint64_t* recs = fl.records.data() + fl.offsets[p];
                int64_t n = fl.offsets[p + 1] - fl.offsets[p];
                R out[4], Tf;
                uint32_t tm;
                composite_pixel(m, *prm, recs, n, px, py, out, Tf, tm);
                R g[4] = {image_adj[4 * p], image_adj[4 * p + 1], image_adj[4 * p + 2], image_adj[4 * p + 3]};
                adjoint_pixel(m, cam, *prm, recs, n, px, py, Tf, tm, g, gp[tid].data(), gc[tid].data());
            }
        }
    }
    for (int t = 0; t < nthreads; ++t) {
        for (int64_t i = 0; i < 3 * V; ++i) grad_pos[i] += gp[t][i];
        for (int64_t i = 0; i < 4 * V; ++i) grad_col[i] += gc[t][i];
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Ray-tet path (intersection renderer).  The reference draws the camera-facing
// faces of every tet sorted by depth and intersects each pixel ray with the
// whole tet (Intersect/IntersectRasterization.glsl:139-273,
// RayIntersectionTests.glsl:77-106): one segment per (pixel, tet), Euclidean
// length along the normalised ray, the same 4-sub-segment integral.  Here the
// tets a pixel ray crosses are found by walking through face adjacency: the
// entries come from the pixel's boundary fragments (front-facing boundary
// faces, depth order); from a tet entered through face fe the ray leaves
// through the back face that covers the pixel (the exact fixed-point rule of
// the rasteriser), and continues into the tet on the other side until it
// leaves through a boundary face.
struct WalkTopo {
    const uint32_t* tri;
    const uint32_t* fbits;
    const uint32_t* f2t;
    const uint32_t* tet_faces;
};

constexpr uint32_t kNoTet = 0xffffffffu;

// Face of tet t (other than `skip`) that covers the pixel and faces the camera
// (want_front) or away from it, with respect to t's outward normal.
inline uint32_t tet_face_at(const WalkTopo& tp, const std::vector<ProjF>& pf, uint32_t t, uint32_t skip,
                            bool want_front, int px, int py) {
    for (int j = 0; j < 4; ++j) {
        const uint32_t f = tp.tet_faces[4 * size_t(t) + j];
        if (f == skip) continue;
        int64_t a2;
        if (!face_covers(pf, tp.tri, f, px, py, &a2)) continue;
        const bool front_stored = a2 < 0;
        const bool owner = tp.f2t[2 * size_t(f)] == t;  // stored winding is outward for tetId0
        if ((front_stored == owner) == want_front) return f;
    }
    return kNoTet;
}

inline uint32_t other_tet(const WalkTopo& tp, uint32_t f, uint32_t t) {
    const uint32_t a = tp.f2t[2 * size_t(f)], b = tp.f2t[2 * size_t(f) + 1];
    return a == t ? b : a;
}

struct WalkState {
    uint32_t last_tet = kNoTet, last_entry = kNoTet, last_b = 0, nseg = 0;
};

template <class R>
inline R ray_len_scale(const CamConst& cam, int px, int py) {
    const R f = std::is_same<R, float>::value ? R(cam.f) : R(cam.fd);
    const R dx = (R(px) + R(0.5) - R(cam.cx)) / f, dy = (R(py) + R(0.5) - R(cam.cy)) / f;
    return std::sqrt(R(1) + dx * dx + dy * dy);
}

template <class R>
Frag<R> face_frag(const MeshR<R>& m, uint32_t f, int px, int py) {
    return eval_frag(m, uint64_t(f) << 2, px, py);
}

template <class R>
void walk_composite_pixel(const MeshR<R>& m, const WalkTopo& tp, const std::vector<ProjF>& pf, const CamConst& cam,
                          const Params& prm, const uint64_t* recs, int64_t n, int px, int py, R out[4], R& Tfinal,
                          WalkState& st) {
    R C[3] = {0, 0, 0};
    R T = 1;
    const R scale = ray_len_scale<R>(cam, px, py);
    bool stop = false;
    const uint64_t max_steps = 1ull << 24;
    for (int64_t b = 0; b < n && !stop; ++b) {
        const uint32_t bits = uint32_t(recs[b] & 0xffffffffu);
        const uint32_t fe0 = bits >> 2;
        if (!tp.fbits[fe0] || !(bits & 1u)) continue;  // intervals start at front-facing boundary faces
        uint32_t fe = fe0, t = tp.f2t[2 * size_t(fe0)];
        Frag<R> f0 = face_frag(m, fe, px, py);
        for (uint64_t step = 0; step < max_steps; ++step) {
            const uint32_t fx = tet_face_at(tp, pf, t, fe, /*want_front=*/false, px, py);
            if (fx == kNoTet) break;
            if (prm.use_ert && T < R(prm.ert_thresh)) {
                stop = true;
                break;
            }
            const Frag<R> f1 = face_frag(m, fx, px, py);
            const R tSeg = (f1.z - f0.z) * scale / R(kNumSubdivs);
            for (int s = 0; s < kNumSubdivs; ++s) {
                R c0[3], c1[3], a, cacc[3], A;
                sub_inputs(f0, f1, s, R(prm.attenuation), c0, c1, a);
                if (!seg_integral(tSeg, c0, c1, a, cacc, A)) continue;
                for (int k = 0; k < 3; ++k) C[k] += T * cacc[k];
                T *= A;
            }
            st.last_tet = t;
            st.last_entry = fe;
            st.last_b = uint32_t(b);
            st.nseg++;
            if (tp.fbits[fx]) break;
            const uint32_t tn = other_tet(tp, fx, t);
            if (tn == kNoTet) break;
            t = tn;
            fe = fx;
            f0 = f1;
        }
    }
    Tfinal = T;
    for (int k = 0; k < 3; ++k) out[k] = C[k] + T * R(prm.clear_color[k]);
    out[3] = (R(1) - T) + T * R(prm.clear_color[3]);
}

template <class R>
void walk_adjoint_pixel(const MeshR<R>& m, const WalkTopo& tp, const std::vector<ProjF>& pf, const CamConst& cam,
                        const Params& prm, const uint64_t* recs, int64_t n, int px, int py, R Tfinal,
                        const WalkState& st, const R g[4], R* grad_pos, R* grad_col) {
    if (st.last_tet == kNoTet) return;
    const R atten = R(prm.attenuation);
    const R scale = ray_len_scale<R>(cam, px, py);
    R gC[3] = {g[0], g[1], g[2]};
    R gT = g[0] * R(prm.clear_color[0]) + g[1] * R(prm.clear_color[1]) + g[2] * R(prm.clear_color[2]) +
           g[3] * (R(prm.clear_color[3]) - R(1));
    R T = Tfinal;
    uint32_t t = st.last_tet, fe = st.last_entry;
    int64_t b = st.last_b;
    // Exit face of the current tet and its accumulated (dL/dz, dL/dcolour).
    uint32_t fx = tet_face_at(tp, pf, t, fe, false, px, py);
    R gz_x = 0, gcol_x[4] = {0, 0, 0, 0};
    const uint64_t max_steps = 1ull << 24;
    for (uint64_t step = 0; step < max_steps; ++step) {
        const Frag<R> f0 = face_frag(m, fe, px, py), f1 = face_frag(m, fx, px, py);
        const R tSeg = (f1.z - f0.z) * scale / R(kNumSubdivs);
        R gz_e = 0, gcol_e[4] = {0, 0, 0, 0};
        R g_tot = 0;
        const R inv = R(1) / R(kNumSubdivs);
        for (int s = kNumSubdivs - 1; s >= 0; --s) {
            R c0[3], c1[3], a, cacc[3], A;
            sub_inputs(f0, f1, s, atten, c0, c1, a);
            const bool active = seg_integral(tSeg, c0, c1, a, cacc, A);
            const R Tin = active ? T / A : T;
            R gcacc[3] = {Tin * gC[0], Tin * gC[1], Tin * gC[2]};
            const R gA = Tin * gT;
            if (active) gT = (gC[0] * cacc[0] + gC[1] * cacc[1] + gC[2] * cacc[2]) + gT * A;
            T = Tin;
            R g_t, g_a, g_c0[3], g_c1[3];
            seg_integral_adjoint(tSeg, c0, c1, a, A, gcacc, gA, g_t, g_a, g_c0, g_c1);
            g_tot += g_t * inv;
            const R fbg = R(s) * inv, fm = (R(s) + R(0.5)) * inv, fen = (R(s) + R(1)) * inv;
            for (int k = 0; k < 3; ++k) {
                gcol_e[k] += (R(1) - fbg) * g_c0[k] + (R(1) - fen) * g_c1[k];
                gcol_x[k] += fbg * g_c0[k] + fen * g_c1[k];
            }
            gcol_e[3] += (R(1) - fm) * g_a * atten;
            gcol_x[3] += fm * g_a * atten;
        }
        gz_e -= g_tot * scale;
        gz_x += g_tot * scale;
        frag_vertex_grads(m, cam, fx, px, py, gz_x, gcol_x, prm.use_abs_grad != 0, grad_pos, grad_col);
        if (tp.fbits[fe]) {
            frag_vertex_grads(m, cam, fe, px, py, gz_e, gcol_e, prm.use_abs_grad != 0, grad_pos, grad_col);
            // Previous interval: its exit is the last back-facing boundary fragment before b.
            int64_t bb = b - 1;
            while (bb >= 0) {
                const uint32_t bits = uint32_t(recs[bb] & 0xffffffffu);
                if (tp.fbits[bits >> 2] && !(bits & 1u)) break;
                --bb;
            }
            if (bb < 0) return;
            fx = uint32_t(recs[bb] & 0xffffffffu) >> 2;
            t = tp.f2t[2 * size_t(fx)];
            fe = tet_face_at(tp, pf, t, fx, /*want_front=*/true, px, py);
            if (fe == kNoTet) return;
            // Entry fragment of the previous interval: the last front boundary fragment before bb.
            int64_t be = bb - 1;
            while (be >= 0) {
                const uint32_t bits = uint32_t(recs[be] & 0xffffffffu);
                if (tp.fbits[bits >> 2] && (bits & 1u)) break;
                --be;
            }
            b = be < 0 ? 0 : be;
            gz_x = 0;
            for (int k = 0; k < 4; ++k) gcol_x[k] = 0;
            continue;
        }
        const uint32_t tp_prev = other_tet(tp, fe, t);
        if (tp_prev == kNoTet) return;
        const uint32_t fe_prev = tet_face_at(tp, pf, tp_prev, fe, /*want_front=*/true, px, py);
        if (fe_prev == kNoTet) return;
        fx = fe;
        gz_x = gz_e;
        for (int k = 0; k < 4; ++k) gcol_x[k] = gcol_e[k];
        t = tp_prev;
        fe = fe_prev;
    }
}

template <class R>
int raytet_impl(const uint32_t* tri, const uint32_t* fbits, const uint32_t* f2t, const uint32_t* tet_faces,
                int64_t F, const R* pos, const R* col, int64_t V, const Camera* camp, const Params* prm, R* image,
                R* tfinal, uint32_t* nseg, const R* image_adj, R* grad_pos, R* grad_col, const float* pos_cov) {
    CamConst cam = make_cam(*camp);
    int r0, r1;
    row_range(*prm, cam.H, r0, r1);
    auto pf = pos_cov ? project_all_f(pos_cov, V, cam) : project_all_f(pos, V, cam);
    FragLists fl = build_fragments(tri, fbits, F, pf, cam, r0, r1);
    MeshR<R> m = make_mesh(tri, pos, col, V, cam);
    const WalkTopo tp{tri, fbits, f2t, tet_faces};
    const int W = cam.W;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    std::vector<std::vector<R>> gp, gc;
    if (image_adj) {
        gp.assign(nthreads, std::vector<R>(3 * V, R(0)));
        gc.assign(nthreads, std::vector<R>(4 * V, R(0)));
    }
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
#pragma omp for schedule(dynamic, 4)
        for (int py = r0; py < r1; ++py) {
            for (int px = 0; px < W; ++px) {
                const int64_t p = int64_t(py) * W + px;
                const uint64_t* recs = fl.records.data() + fl.offsets[p];
                const int64_t n = fl.offsets[p + 1] - fl.offsets[p];
                R out[4], Tf;
                WalkState st;
                walk_composite_pixel(m, tp, pf, cam, *prm, recs, n, px, py, out, Tf, st);
                if (image)
                    for (int k = 0; k < 4; ++k) image[4 * p + k] = out[k];
                if (tfinal) tfinal[p] = Tf;
                if (nseg) nseg[p] = st.nseg;
                if (image_adj) {
                    const R g[4] = {image_adj[4 * p], image_adj[4 * p + 1], image_adj[4 * p + 2],
                                    image_adj[4 * p + 3]};
                    walk_adjoint_pixel(m, tp, pf, cam, *prm, recs, n, px, py, Tf, st, g, gp[tid].data(),
                                       gc[tid].data());
                }
            }
        }
    }
    if (image_adj) {
        for (int t = 0; t < nthreads; ++t) {
            for (int64_t i = 0; i < 3 * V; ++i) grad_pos[i] += gp[t][i];
            for (int64_t i = 0; i < 4 * V; ++i) grad_col[i] += gc[t][i];
        }
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Per-cell colours (ColorStorage::PER_CELL).  Forward.glsl:213-246: two
// consecutive fragments bound a segment of the tet both faces belong to
// (tetIdUnion, LinkedListResolve.glsl:85-94; no shared tet = empty space, no
// segment); the segment has that cell's constant colour and density,
// accumulateConst (ForwardCommon.glsl:37-40): A = exp(-a t), C = (1 - A) c,
// with no sub-segments.  Early ray termination is checked before each
// fragment and the termination index is the fragment index where the loop
// stopped (:222-227, 256-259).  The adjoint (Backward.glsl:283-329 with
// accumulateConstAdjoint, BackwardCommon.glsl:100-105) is the exact
// derivative: cell colour gradients per segment, position gradients through
// the two fragment depths.
constexpr uint32_t kInvalidTet = 0xffffffffu;

inline uint32_t tet_union(uint32_t a0, uint32_t a1, uint32_t b0, uint32_t b1) {
    if ((a0 == b0 || a0 == b1) && a0 != kInvalidTet) return a0;
    if ((a1 == b0 || a1 == b1) && a1 != kInvalidTet) return a1;
    return kInvalidTet;
}

template <class R>
R face_depth(const MeshR<R>& m, uint32_t face, int px, int py) {
    const uint32_t i0 = m.tri[3 * face], i1 = m.tri[3 * face + 1], i2 = m.tri[3 * face + 2];
    R lam[3], b[3], z;
    face_bary(m.proj[i0], m.proj[i1], m.proj[i2], R(px) + R(0.5), R(py) + R(0.5), lam, b, z);
    return z;
}

inline uint32_t rec_face(uint64_t rec) { return uint32_t(rec & 0xffffffffu) >> 2; }

template <class R>
void composite_pixel_cells(const MeshR<R>& m, const uint32_t* f2t, const R* ccol, const Params& prm,
                           const uint64_t* recs, int64_t n, int px, int py, R out[4], R& Tfinal, uint32_t& term) {
    const R atten = R(prm.attenuation);
    R C[3] = {0, 0, 0};
    R T = 1, zprev = 0;
    uint32_t pa = kInvalidTet, pb = kInvalidTet;
    int64_t i = 0;
    for (; i < n; ++i) {
        if (prm.use_ert && T < R(prm.ert_thresh)) break;
        const uint32_t face = rec_face(recs[i]);
        const R z = face_depth(m, face, px, py);
        const uint32_t qa = f2t[2 * size_t(face)], qb = f2t[2 * size_t(face) + 1];
        const uint32_t open = tet_union(qa, qb, pa, pb);
        if (open != kInvalidTet) {
            const R* c = ccol + 4 * size_t(open);
            const R A = std::exp(-(c[3] * atten) * (z - zprev));
            for (int k = 0; k < 3; ++k) C[k] += T * (R(1) - A) * c[k];
            T *= A;
        }
        pa = qa;
        pb = qb;
        zprev = z;
    }
    term = uint32_t(i);
    Tfinal = T;
    for (int k = 0; k < 3; ++k) out[k] = C[k] + T * R(prm.clear_color[k]);
    out[3] = (R(1) - T) + T * R(prm.clear_color[3]);
}

template <class R>
void adjoint_pixel_cells(const MeshR<R>& m, const CamConst& cam, const uint32_t* f2t, const R* ccol,
                         const Params& prm, const uint64_t* recs, int64_t n, int px, int py, R Tfinal, uint32_t term,
                         const R g[4], R* grad_pos, R* grad_cell) {
    const int64_t last = (prm.use_ert ? int64_t(term) : n) - 1;  // last fragment visited
    if (last < 1) return;
    const R atten = R(prm.attenuation);
    const bool use_abs = prm.use_abs_grad != 0;
    const R gC[3] = {g[0], g[1], g[2]};
    R gT = g[0] * R(prm.clear_color[0]) + g[1] * R(prm.clear_color[1]) + g[2] * R(prm.clear_color[2]) +
           g[3] * (R(prm.clear_color[3]) - R(1));
    R T = Tfinal;
    const R zero4[4] = {0, 0, 0, 0};
    uint32_t fb = rec_face(recs[last]);
    R zb = face_depth(m, fb, px, py), gz_b = 0;
    for (int64_t i = last; i >= 1; --i) {
        const uint32_t ff = rec_face(recs[i - 1]);
        const R zf = face_depth(m, ff, px, py);
        R gz_f = 0;
        const uint32_t open = tet_union(f2t[2 * size_t(fb)], f2t[2 * size_t(fb) + 1], f2t[2 * size_t(ff)],
                                        f2t[2 * size_t(ff) + 1]);
        if (open != kInvalidTet) {
            const R* c = ccol + 4 * size_t(open);
            const R a = c[3] * atten, t = zb - zf;
            const R A = std::exp(-a * t);
            const R Tin = T / A;
            R gcacc[3], dot_c = 0, dot_cacc = 0;
            for (int k = 0; k < 3; ++k) {
                gcacc[k] = Tin * gC[k];
                dot_c += gcacc[k] * c[k];
                dot_cacc += gC[k] * (R(1) - A) * c[k];
            }
            const R gA = Tin * gT - dot_c;  // dL/dA: through T_out and through C = (1 - A) c
            gT = dot_cacc + gT * A;
            T = Tin;
            const R g_t = gA * (-a * A), g_a = gA * (-t * A);
            R gc[4] = {gcacc[0] * (R(1) - A), gcacc[1] * (R(1) - A), gcacc[2] * (R(1) - A), g_a * atten};
            if (use_abs)
                for (int k = 0; k < 4; ++k) gc[k] = std::fabs(gc[k]);
            for (int k = 0; k < 4; ++k) grad_cell[4 * size_t(open) + k] += gc[k];
            gz_b += g_t;
            gz_f -= g_t;
        }
        frag_vertex_grads(m, cam, fb, px, py, gz_b, zero4, use_abs, grad_pos, static_cast<R*>(nullptr));
        fb = ff;
        zb = zf;
        gz_b = gz_f;
    }
    frag_vertex_grads(m, cam, fb, px, py, gz_b, zero4, use_abs, grad_pos, static_cast<R*>(nullptr));
}

template <class R>
int cells_impl(const uint32_t* tri, const uint32_t* fbits, const uint32_t* f2t, int64_t F, const R* pos,
               const R* ccol, int64_t V, int64_t T, const Camera* camp, const Params* prm, R* image, R* tfinal,
               uint32_t* term, int64_t* nfrag, const R* image_adj, R* grad_pos, R* grad_cell,
               const float* pos_coverage) {
    CamConst cam = make_cam(*camp);
    int r0, r1;
    row_range(*prm, cam.H, r0, r1);
    auto pf = pos_coverage ? project_all_f(pos_coverage, V, cam) : project_all_f(pos, V, cam);
    FragLists fl = build_fragments(tri, fbits, F, pf, cam, r0, r1);
    MeshR<R> m = make_mesh<R>(tri, pos, nullptr, V, cam);
    const int W = cam.W;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    std::vector<std::vector<R>> gp, gc;
    if (image_adj) {
        gp.assign(nthreads, std::vector<R>(3 * V, R(0)));
        gc.assign(nthreads, std::vector<R>(4 * T, R(0)));
    }
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
#pragma omp for schedule(dynamic, 4)
        for (int py = r0; py < r1; ++py) {
            for (int px = 0; px < W; ++px) {
                const int64_t p = int64_t(py) * W + px;
                const uint64_t* recs = fl.records.data() + fl.offsets[p];
                const int64_t n = fl.offsets[p + 1] - fl.offsets[p];
                R out[4], Tf;
                uint32_t tm;
                composite_pixel_cells(m, f2t, ccol, *prm, recs, n, px, py, out, Tf, tm);
                if (image)
                    for (int k = 0; k < 4; ++k) image[4 * p + k] = out[k];
                if (tfinal) tfinal[p] = Tf;
                if (term) term[p] = tm;
                if (image_adj) {
                    const R g[4] = {image_adj[4 * p], image_adj[4 * p + 1], image_adj[4 * p + 2],
                                    image_adj[4 * p + 3]};
                    adjoint_pixel_cells(m, cam, f2t, ccol, *prm, recs, n, px, py, Tf, tm, g, gp[tid].data(),
                                        gc[tid].data());
                }
            }
        }
    }
    if (image_adj) {
        for (int t = 0; t < nthreads; ++t) {
            for (int64_t i = 0; i < 3 * V; ++i) grad_pos[i] += gp[t][i];
            for (int64_t i = 0; i < 4 * T; ++i) grad_cell[i] += gc[t][i];
        }
    }
    if (nfrag) *nfrag = int64_t(fl.records.size());
    return 0;
}

struct TempFace {
    uint32_t v[3];
    uint32_t face_id;
    uint32_t tet_id;
    bool operator<(const TempFace& o) const {
        for (int i = 0; i < 3; ++i)
            if (v[i] != o.v[i]) return v[i] < o.v[i];
        return face_id < o.face_id;
    }
    bool same(const TempFace& o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2]; }
};

}  // namespace

// ---------------------------------------------------------------------------
// Reference mode: the reference's own formulas of the PPLL path, as its GLSL
// states them, on the same fragment sets (this file's fixed-point coverage,
// since the reference's rasteriser is the GPU's).  Used to measure how far
// the exact path (above; the CUDA library follows it) is from what the
// reference computes on the same inputs.  Evaluated in double; the FP32
// storage of the depth buffer value is reproduced.
//
// Forward (Data/Shaders/PPLL/Forward.glsl:35-105, 159-211):
//  - each fragment stores gl_FragCoord.z, the NDC depth interpolated affinely
//    in screen space, as a 32-bit float (LinkedListGather.glsl:97); lists are
//    ordered by it (the 4-ary heap, Forward.glsl:107-114; ties here by face);
//  - depthLinear = zNear zFar / (zFar + z_ndc (zNear - zFar))
//    (Utils/DepthHelper.glsl:72-75);
//  - the world point is the inverse view-projection of (ndc.xy, z_ndc), and
//    the colour weights are unsigned cross-product ratios u = |d21 x (p - p1)|
//    / A, v = |(p - p0) x d20| / A, w = 1 - u - v, A = max(|d20 x d21|, 1e-5)
//    (Forward.glsl:80-103);
//  - accumulateLinearConst returns 0 when a < 1e-6 (ForwardCommon.glsl:42-49);
//  - opacity is blended front to back and the ray stops once
//    alpha > 1 - thresh (Forward.glsl:169-173).
// Adjoint (PPLL/Backward.glsl:107-512, Common/BackwardCommon.glsl:95-251):
//  - back to front from the termination index; per segment only
//    sub-segments s = 3, 2, 1 (Backward.glsl:222), each inverted with
//    alpha_in = (C.a - alpha_out) / (C.a - 1) (:232) and differentiated by
//    accumulateLinearConstAdjoint (:116-133; its getNextFragment clamps the
//    area at 1e-6, Backward.glsl:98);
//  - segmentLengthAdjoint differentiates the Euclidean distance between the
//    two fragments' world points (BackwardCommon.glsl:139-181);
//  - baryAdjoint differentiates u, v with the world point held fixed
//    (:183-251).
namespace refmode {

struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double len(V3 a) { return std::sqrt(dot(a, a)); }

struct Cam {
    CamConst c;
    double inv_view[16];  // column-major inverse of the view matrix
    double zn, zf;
};

inline void invert4(const float* m, double* out) {
    // Gauss-Jordan on a row-major copy of the column-major matrix.
    double a[4][8];
    for (int r = 0; r < 4; ++r)
        for (int k = 0; k < 4; ++k) {
            a[r][k] = double(m[k * 4 + r]);
            a[r][4 + k] = r == k ? 1.0 : 0.0;
        }
    for (int c = 0; c < 4; ++c) {
        int piv = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
        for (int k = 0; k < 8; ++k) std::swap(a[c][k], a[piv][k]);
        const double d = a[c][c];
        for (int k = 0; k < 8; ++k) a[c][k] /= d;
        for (int r = 0; r < 4; ++r) {
            if (r == c) continue;
            const double f = a[r][c];
            for (int k = 0; k < 8; ++k) a[r][k] -= f * a[c][k];
        }
    }
    for (int r = 0; r < 4; ++r)
        for (int k = 0; k < 4; ++k) out[k * 4 + r] = a[r][4 + k];
}

Cam make(const Camera& camera) {
    Cam k;
    k.c = make_cam(camera);
    invert4(camera.view, k.inv_view);
    k.zn = camera.znear;
    k.zf = camera.zfar;
    return k;
}

// NDC depth of view depth ze (perspectiveRH_ZO): zFar (ze - zNear) / ((zFar - zNear) ze).
inline double ndc_of_ze(const Cam& k, double ze) { return k.zf * (ze - k.zn) / ((k.zf - k.zn) * ze); }
inline double lin_depth(const Cam& k, double zndc) { return k.zn * k.zf / (k.zf + zndc * (k.zn - k.zf)); }

// World point of pixel centre (px, py) at NDC depth zndc.
inline V3 unproject(const Cam& k, int px, int py, double zndc) {
    const double ze = lin_depth(k, zndc);
    const double sx = double(px) + 0.5, sy = double(py) + 0.5;
    const double xv = (sx - k.c.cxd) * ze / k.c.fd, yv = -(sy - k.c.cyd) * ze / k.c.fd, zv = -ze;
    const double* M = k.inv_view;
    return {M[0] * xv + M[4] * yv + M[8] * zv + M[12], M[1] * xv + M[5] * yv + M[9] * zv + M[13],
            M[2] * xv + M[6] * yv + M[10] * zv + M[14]};
}

struct Mesh {
    const uint32_t* tri;
    const double* pos;
    const double* col;
    std::vector<ProjR<double>> proj;
};

inline V3 vpos(const Mesh& m, uint32_t v) { return {m.pos[3 * v], m.pos[3 * v + 1], m.pos[3 * v + 2]}; }

struct Frag {
    float zndc;          // the stored depth buffer value
    double depth;        // depthLinear
    V3 p;                // world point
    V3 pv[3];            // face vertices
    double c[3][4];      // vertex colours
    uint32_t vi[3];
    double u, v;
    double col[4];
    bool boundary, front;
};

// gl_FragCoord.z of face f at the pixel centre (screen-affine interpolation
// of the vertices' NDC depths), as stored: a 32-bit float.
inline float frag_zndc(const Mesh& m, const Cam& k, uint32_t f, int px, int py) {
    const ProjR<double>& a = m.proj[m.tri[3 * f]];
    const ProjR<double>& b = m.proj[m.tri[3 * f + 1]];
    const ProjR<double>& c = m.proj[m.tri[3 * f + 2]];
    const double qx = px + 0.5, qy = py + 0.5;
    const double d0x = a.sx - qx, d0y = a.sy - qy, d1x = b.sx - qx, d1y = b.sy - qy, d2x = c.sx - qx,
                 d2y = c.sy - qy;
    const double E0 = d1x * d2y - d1y * d2x, E1 = d2x * d0y - d2y * d0x, E2 = d0x * d1y - d0y * d1x;
    const double A = E0 + E1 + E2;
    return float((E0 * ndc_of_ze(k, a.ze) + E1 * ndc_of_ze(k, b.ze) + E2 * ndc_of_ze(k, c.ze)) / A);
}

inline Frag eval(const Mesh& m, const Cam& k, uint32_t bits, float zndc, int px, int py, double area_floor) {
    Frag fr;
    const uint32_t f = bits >> 2;
    fr.boundary = (bits >> 1) & 1u;
    fr.front = bits & 1u;
    fr.zndc = zndc;
    fr.depth = lin_depth(k, double(zndc));
    fr.p = unproject(k, px, py, double(zndc));
    for (int j = 0; j < 3; ++j) {
        fr.vi[j] = m.tri[3 * f + j];
        fr.pv[j] = vpos(m, fr.vi[j]);
        for (int q = 0; q < 4; ++q) fr.c[j][q] = m.col[4 * size_t(fr.vi[j]) + q];
    }
    const V3 d20 = fr.pv[2] - fr.pv[0], d21 = fr.pv[2] - fr.pv[1];
    const double area = std::max(len(cross(d20, d21)), area_floor);
    fr.u = len(cross(d21, fr.p - fr.pv[1])) / area;
    fr.v = len(cross(fr.p - fr.pv[0], d20)) / area;
    const double w = 1.0 - fr.u - fr.v;
    for (int q = 0; q < 4; ++q) fr.col[q] = fr.c[0][q] * fr.u + fr.c[1][q] * fr.v + fr.c[2][q] * w;
    return fr;
}

// Records of one pixel re-keyed by the stored NDC depth (ties by face).
inline std::vector<std::pair<float, uint32_t>> pixel_list(const Mesh& m, const Cam& k, const uint64_t* recs,
                                                          int64_t n, int px, int py) {
    std::vector<std::pair<float, uint32_t>> l{};
    l.resize(size_t(n));
    for (int64_t i = 0; i < n; ++i) {
        const uint32_t bits = uint32_t(recs[i] & 0xffffffffu);
        l[size_t(i)] = {frag_zndc(m, k, bits >> 2, px, py), bits};
    }
    std::sort(l.begin(), l.end(), [](const std::pair<float, uint32_t>& a, const std::pair<float, uint32_t>& b) {
        return a.first < b.first || (a.first == b.first && (a.second >> 2) < (b.second >> 2));
    });
    return l;
}

// accumulateLinearConst (ForwardCommon.glsl:42-49 / BackwardCommon.glsl:103-110).
inline void acc_lin_const(double t, const double c0[3], const double c1[3], double a, double out[4], double& A) {
    A = std::exp(-a * t);
    if (a < 1e-6) {
        out[0] = out[1] = out[2] = out[3] = 0.0;
        return;
    }
    const double K = (t + 1.0 / a) * A - 1.0 / a;
    for (int q = 0; q < 3; ++q) out[q] = (1.0 - A) * c0[q] + K * (c0[q] - c1[q]);
    out[3] = 1.0 - A;
}

inline bool skip(const Frag& f0, const Frag& f1) {
    return (f0.boundary && !f0.front) && (f1.boundary && f1.front);
}

// Forward of one pixel: premultiplied colour and opacity, termination index.
inline void composite(const Mesh& m, const Cam& k, const Params& prm, const std::vector<std::pair<float, uint32_t>>& l,
                      int px, int py, double ray[4], uint32_t& term) {
    ray[0] = ray[1] = ray[2] = ray[3] = 0.0;
    const size_t n = l.size();
    size_t i = n;
    if (n >= 1) {
        Frag f1 = eval(m, k, l[0].second, l[0].first, px, py, 1e-5), f0;
        for (i = 1; i < n; ++i) {
            if (prm.use_ert && ray[3] > 1.0 - double(prm.ert_thresh)) break;
            f0 = f1;
            f1 = eval(m, k, l[i].second, l[i].first, px, py, 1e-5);
            if (skip(f0, f1)) continue;
            const double tSeg = (f1.depth - f0.depth) / kNumSubdivs;
            for (int s = 0; s < kNumSubdivs; ++s) {
                const double fb = double(s) / kNumSubdivs, fm = (s + 0.5) / kNumSubdivs,
                             fe = (s + 1.0) / kNumSubdivs;
                double c0[3], c1[3], acc[4], A;
                for (int q = 0; q < 3; ++q) {
                    c0[q] = f0.col[q] + (f1.col[q] - f0.col[q]) * fb;
                    c1[q] = f0.col[q] + (f1.col[q] - f0.col[q]) * fe;
                }
                const double alpha = f0.col[3] + (f1.col[3] - f0.col[3]) * fm;
                acc_lin_const(tSeg, c0, c1, alpha * prm.attenuation, acc, A);
                for (int q = 0; q < 3; ++q) ray[q] += (1.0 - ray[3]) * acc[q];
                ray[3] += (1.0 - ray[3]) * acc[3];
            }
        }
    }
    term = uint32_t(i);
}

// d/dp_k of (n . (a x b)) with da/dp_k = al I, db/dp_k = be I: al (b x n) + be (n x a).
inline V3 dcross(V3 n, V3 a, V3 b, double al, double be) { return al * cross(b, n) + be * cross(n, a); }

// baryAdjoint (BackwardCommon.glsl:183-251), world point p fixed.
inline void bary_adjoint(const Frag& fr, const double dc[4], double du, double dv, V3 dp[3], double dcol[3][4]) {
    const V3 p = fr.p, p0 = fr.pv[0], p1 = fr.pv[1], p2 = fr.pv[2];
    du += dc[0] * (fr.c[0][0] - fr.c[2][0]) + dc[1] * (fr.c[0][1] - fr.c[2][1]) + dc[2] * (fr.c[0][2] - fr.c[2][2]) +
          dc[3] * (fr.c[0][3] - fr.c[2][3]);
    dv += dc[0] * (fr.c[1][0] - fr.c[2][0]) + dc[1] * (fr.c[1][1] - fr.c[2][1]) + dc[2] * (fr.c[1][2] - fr.c[2][2]) +
          dc[3] * (fr.c[1][3] - fr.c[2][3]);
    const double w = 1.0 - fr.u - fr.v;
    for (int q = 0; q < 4; ++q) {
        dcol[0][q] = dc[q] * fr.u;
        dcol[1][q] = dc[q] * fr.v;
        dcol[2][q] = dc[q] * w;
    }
    // u = |n1| / |n0|, v = |n2| / |n0| with n0 = (p0 - p2) x (p1 - p2),
    // n1 = (p - p1) x (p1 - p2), n2 = (p - p0) x (p0 - p2); the denominators
    // clamped as in the GLSL (max(f0^1.5, 1e-6), max(sqrt(f), 1e-6)).
    const V3 a0 = p0 - p2, b0 = p1 - p2, n0 = cross(a0, b0);
    const V3 a1 = p - p1, b1 = p1 - p2, n1 = cross(a1, b1);
    const V3 a2 = p - p0, b2 = p0 - p2, n2 = cross(a2, b2);
    const double f0 = dot(n0, n0), f1 = dot(n1, n1), f2 = dot(n2, n2);
    const double den0 = std::max(std::pow(f0, 1.5), 1e-6), den1 = std::max(std::sqrt(f1), 1e-6),
                 den2 = std::max(std::sqrt(f2), 1e-6);
    // n . dn/dp_k for the three vertices.
    const V3 g0[3] = {dcross(n0, a0, b0, 1, 0), dcross(n0, a0, b0, 0, 1), dcross(n0, a0, b0, -1, -1)};
    const V3 g1[3] = {V3{0, 0, 0}, dcross(n1, a1, b1, -1, 1), dcross(n1, a1, b1, 0, -1)};
    const V3 g2[3] = {dcross(n2, a2, b2, -1, 1), V3{0, 0, 0}, dcross(n2, a2, b2, 0, -1)};
    for (int j = 0; j < 3; ++j) {
        const V3 du_dp = (1.0 / (den1 * den0)) * (f0 * g1[j] - f1 * g0[j]);
        const V3 dv_dp = (1.0 / (den2 * den0)) * (f0 * g2[j] - f2 * g0[j]);
        dp[j] = dp[j] + du * du_dp + dv * dv_dp;
    }
}

// segmentLengthAdjoint (BackwardCommon.glsl:139-181): t = |P0 - P1| with
// P_k = u_k p_k0 + v_k p_k1 + w_k p_k2.
inline void seglen_adjoint(const Frag& f0, const Frag& f1, double g, double& du0, double& dv0, double& du1,
                           double& dv1, V3 dp0[3], V3 dp1[3]) {
    const double w0 = 1.0 - f0.u - f0.v, w1 = 1.0 - f1.u - f1.v;
    const V3 P0 = f0.u * f0.pv[0] + f0.v * f0.pv[1] + w0 * f0.pv[2];
    const V3 P1 = f1.u * f1.pv[0] + f1.v * f1.pv[1] + w1 * f1.pv[2];
    const V3 D = P0 - P1;
    const double inv = 1.0 / std::sqrt(std::max(dot(D, D), 1e-6));
    du0 = g * dot(f0.pv[0] - f0.pv[2], D) * inv;
    dv0 = g * dot(f0.pv[1] - f0.pv[2], D) * inv;
    du1 = -g * dot(f1.pv[0] - f1.pv[2], D) * inv;
    dv1 = -g * dot(f1.pv[1] - f1.pv[2], D) * inv;
    dp0[0] = (g * f0.u * inv) * D;
    dp0[1] = (g * f0.v * inv) * D;
    dp0[2] = (g * w0 * inv) * D;
    dp1[0] = (-g * f1.u * inv) * D;
    dp1[1] = (-g * f1.v * inv) * D;
    dp1[2] = (-g * w1 * inv) * D;
}

// Adjoint of one pixel (Backward.glsl:107-512, PER_VERTEX_COLORS).
// skip0: reproduce the loop bound s > 0 of Backward.glsl:222 (false: s >= 0,
// for checks of this restatement).
inline void adjoint(const Mesh& m, const Cam& k, const Params& prm, const std::vector<std::pair<float, uint32_t>>& l,
                    int px, int py, const double ray_out[4], uint32_t term, const double g_in[4], double* grad_pos,
                    double* grad_col, bool skip0) {
    const int64_t n = int64_t(l.size());
    if (n < 2) return;
    const int64_t tidx = prm.use_ert ? n - int64_t(term) : 0;  // farthest layers the forward did not reach
    double ray[4] = {ray_out[0], ray_out[1], ray_out[2], ray_out[3]};
    double dout[4] = {g_in[0], g_in[1], g_in[2], g_in[3]};
    const double inv_n = 1.0 / kNumSubdivs;
    // Back to front: backward index b is forward index n - 1 - b.
    auto frag_b = [&](int64_t b) {
        const auto& e = l[size_t(n - 1 - b)];
        return eval(m, k, e.second, e.first, px, py, 1e-6);
    };
    Frag fr0 = frag_b(0), fr1;
    for (int64_t i = 1; i < n; ++i) {
        if (i > tidx) fr1 = fr0;
        fr0 = frag_b(i);
        if (i <= tidx) continue;
        if (skip(fr0, fr1)) continue;
        double dcf0[4] = {0, 0, 0, 0}, dcf1[4] = {0, 0, 0, 0}, dt = 0.0;
        const double t = fr1.depth - fr0.depth, tSeg = t / kNumSubdivs;
        for (int s = kNumSubdivs - 1; s >= (skip0 ? 1 : 0); --s) {
            const double fb = s * inv_n, fm = (s + 0.5) * inv_n, fe = (s + 1.0) * inv_n;
            double c0[3], c1[3], acc[4], A;
            for (int q = 0; q < 3; ++q) {
                c0[q] = fr0.col[q] + (fr1.col[q] - fr0.col[q]) * fb;
                c1[q] = fr0.col[q] + (fr1.col[q] - fr0.col[q]) * fe;
            }
            const double alpha = fr0.col[3] + (fr1.col[3] - fr0.col[3]) * fm;
            const double a = alpha * prm.attenuation;
            acc_lin_const(tSeg, c0, c1, a, acc, A);
            const double a_in = (acc[3] - ray[3]) / (acc[3] - 1.0);
            double dacc[4];
            for (int q = 0; q < 3; ++q) {
                ray[q] = ray[q] - (1.0 - a_in) * acc[q];
                dacc[q] = (1.0 - a_in) * dout[q];
            }
            dacc[3] = (1.0 - a_in) * dout[3];
            dout[3] = dout[3] * (1.0 - acc[3]) - (dout[0] * acc[0] + dout[1] * acc[1] + dout[2] * acc[2]);
            ray[3] = a_in;
            // accumulateLinearConstAdjoint (BackwardCommon.glsl:116-133), tf = 1 / NUM_SUBDIVS.
            const double tt = tSeg;
            double dot_t = 0.0;
            for (int q = 0; q < 3; ++q) dot_t += dacc[q] * (a * c0[q] + (a * c1[q] - a * c0[q]) * tt) * A;
            dt += inv_n * (dot_t + dacc[3] * a * A);
            double dc0[3], dc1[3], da;
            if (a < 1e-6) {
                da = dacc[3] * tt;
                for (int q = 0; q < 3; ++q) {
                    dc0[q] = dc1[q] = 0.0;
                    da += dacc[q] * (tt * c0[q] + 0.5 * tt * tt * (c1[q] - c0[q]));
                }
            } else {
                const double ia = 1.0 / a, K = (tt + ia) * A - ia;
                da = dacc[3] * tt * A;
                for (int q = 0; q < 3; ++q) {
                    dc0[q] = ((1.0 - A) + K) * dacc[q];
                    dc1[q] = -K * dacc[q];
                    da += dacc[q] * (tt * A * c0[q] + (ia * ia - (tt * tt + ia * ia + tt * ia) * A) * (c0[q] - c1[q]));
                }
            }
            da *= prm.attenuation;
            for (int q = 0; q < 3; ++q) {
                dcf0[q] += (1.0 - fb) * dc0[q] + (1.0 - fe) * dc1[q];
                dcf1[q] += fb * dc0[q] + fe * dc1[q];
            }
            dcf0[3] += (1.0 - fm) * da;
            dcf1[3] += fm * da;
        }
        double du0, dv0, du1, dv1;
        V3 dp0[3], dp1[3];
        seglen_adjoint(fr0, fr1, dt, du0, dv0, du1, dv1, dp0, dp1);
        double dcol0[3][4], dcol1[3][4];
        bary_adjoint(fr0, dcf0, du0, dv0, dp0, dcol0);
        bary_adjoint(fr1, dcf1, du1, dv1, dp1, dcol1);
        const bool ab = prm.use_abs_grad != 0;
        for (int j = 0; j < 3; ++j) {
            const V3 q0 = dp0[j], q1 = dp1[j];
            const double g0[3] = {q0.x, q0.y, q0.z}, g1[3] = {q1.x, q1.y, q1.z};
            for (int c = 0; c < 3; ++c) {
                grad_pos[3 * size_t(fr0.vi[j]) + c] += ab ? std::fabs(g0[c]) : g0[c];
                grad_pos[3 * size_t(fr1.vi[j]) + c] += ab ? std::fabs(g1[c]) : g1[c];
            }
            for (int c = 0; c < 4; ++c) {
                grad_col[4 * size_t(fr0.vi[j]) + c] += ab ? std::fabs(dcol0[j][c]) : dcol0[j][c];
                grad_col[4 * size_t(fr1.vi[j]) + c] += ab ? std::fabs(dcol1[j][c]) : dcol1[j][c];
            }
        }
    }
}

// Forward (and with image_adj, the adjoint) of pixel rows of the prm range.
int run(const uint32_t* tri, const uint32_t* fbits, int64_t F, const float* pos_f, const double* pos,
        const double* col, int64_t V, const Camera* camp, const Params* prm, double* image, uint32_t* term,
        const double* image_adj, double* grad_pos, double* grad_col, bool skip0) {
    const Cam k = make(*camp);
    int r0, r1;
    row_range(*prm, k.c.H, r0, r1);
    auto pf = project_all_f(pos_f, V, k.c);
    FragLists fl = build_fragments(tri, fbits, F, pf, k.c, r0, r1);
    Mesh m{tri, pos, col, {}};
    m.proj.resize(size_t(V));
    for (int64_t v = 0; v < V; ++v) m.proj[size_t(v)] = project_r<double>(k.c, pos[3 * v], pos[3 * v + 1], pos[3 * v + 2]);
    const int W = k.c.W;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    std::vector<std::vector<double>> gp, gc;
    if (image_adj) {
        gp.assign(nthreads, std::vector<double>(3 * size_t(V), 0.0));
        gc.assign(nthreads, std::vector<double>(4 * size_t(V), 0.0));
    }
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
#pragma omp for schedule(dynamic, 4)
        for (int py = r0; py < r1; ++py)
            for (int px = 0; px < W; ++px) {
                const int64_t p = int64_t(py) * W + px;
                const auto l = pixel_list(m, k, fl.records.data() + fl.offsets[p], fl.offsets[p + 1] - fl.offsets[p],
                                          px, py);
                double ray[4];
                uint32_t tm;
                composite(m, k, *prm, l, px, py, ray, tm);
                // Clear colour blended under the premultiplied result, as the exact path does.
                const double T = 1.0 - ray[3];
                if (image)
                    for (int q = 0; q < 4; ++q) image[4 * p + q] = ray[q] + T * double(prm->clear_color[q]);
                if (term) term[p] = tm;
                if (image_adj) {
                    const double g[4] = {image_adj[4 * p], image_adj[4 * p + 1], image_adj[4 * p + 2],
                                         image_adj[4 * p + 3]};
                    adjoint(m, k, *prm, l, px, py, ray, tm, g, gp[tid].data(), gc[tid].data(), skip0);
                }
            }
    }
    if (image_adj)
        for (int t = 0; t < nthreads; ++t) {
            for (int64_t i = 0; i < 3 * V; ++i) grad_pos[i] += gp[t][size_t(i)];
            for (int64_t i = 0; i < 4 * V; ++i) grad_col[i] += gc[t][size_t(i)];
        }
    return 0;
}

}  // namespace refmode

extern "C" {

// buildFacesSlim, src/Tet/TetMesh.cpp:1218-1268 (with TempFace ordering
// :1183-1216 and the device arrays of uploadDataToDevice :560-576): unique
// faces in sorted-vertex-triple order, each keeping the winding of its lowest
// faceId copy; boundary bit per face and per vertex; face -> (tet0, tet1).
// Returns the number of faces F (arrays must hold 4T faces).
int64_t orc_build_faces(const uint32_t* cells, int64_t T, int64_t V, uint32_t* tri_out, uint32_t* face_boundary,
                        uint32_t* face_to_tet, uint32_t* vertex_boundary) {
    std::vector<TempFace> tf(size_t(T) * 4);
    std::vector<uint32_t> wound(size_t(T) * 12);
    for (int64_t c = 0; c < T; ++c) {
        for (int j = 0; j < 4; ++j) {
            uint32_t fid = uint32_t(4 * c + j);
            uint32_t v[3];
            for (int k = 0; k < 3; ++k) v[k] = cells[4 * c + kTetFace[j][k]];
            for (int k = 0; k < 3; ++k) wound[3 * size_t(fid) + k] = v[k];
            std::sort(v, v + 3);
            tf[fid] = TempFace{{v[0], v[1], v[2]}, fid, uint32_t(c)};
        }
    }
    std::sort(tf.begin(), tf.end());
    int64_t F = 0;
    for (size_t i = 0; i < tf.size(); ++i) {
        if (i == 0 || !tf[i].same(tf[i - 1])) {
            for (int k = 0; k < 3; ++k) tri_out[3 * F + k] = wound[3 * size_t(tf[i].face_id) + k];
            face_to_tet[2 * F] = tf[i].tet_id;
            face_to_tet[2 * F + 1] = 0xffffffffu;
            face_boundary[F] = 1;
            ++F;
        } else {
            face_boundary[F - 1] = 0;
            face_to_tet[2 * (F - 1) + 1] = tf[i].tet_id;
        }
    }
    std::memset(vertex_boundary, 0, sizeof(uint32_t) * size_t(V));
    for (int64_t f = 0; f < F; ++f)
        if (face_boundary[f])
            for (int k = 0; k < 3; ++k) vertex_boundary[tri_out[3 * f + k]] = 1;
    return F;
}

// Per-pixel sorted fragment lists (exported like Renderer.get_fragment_buffer /
// get_start_offset_buffer, Module.cpp:960-981, in offsets+records layout).
// Returns Nf; writes offsets[P+1] and records[Nf] when the pointers are non-null
// and records_cap >= Nf.
int64_t orc_fragments(const uint32_t* tri, const uint32_t* fbits, int64_t F, const float* pos, int64_t V,
                      const Camera* camp, int64_t* offsets, uint64_t* records, int64_t records_cap) {
    CamConst cam = make_cam(*camp);
    auto pf = project_all_f(pos, V, cam);
    FragLists fl = build_fragments(tri, fbits, F, pf, cam, 0, cam.H);
    int64_t nf = int64_t(fl.records.size());
    if (offsets) std::memcpy(offsets, fl.offsets.data(), sizeof(int64_t) * fl.offsets.size());
    if (records && records_cap >= nf) std::memcpy(records, fl.records.data(), sizeof(uint64_t) * size_t(nf));
    return nf;
}

// Fragment lists of pixel rows [row_begin, row_end) only (offsets over all
// P + 1 pixels, zero-length lists outside the rows): bounded checks of large
// images.
int64_t orc_fragments_rows(const uint32_t* tri, const uint32_t* fbits, int64_t F, const float* pos, int64_t V,
                           const Camera* camp, int32_t row_begin, int32_t row_end, int64_t* offsets,
                           uint64_t* records, int64_t records_cap) {
    CamConst cam = make_cam(*camp);
    auto pf = project_all_f(pos, V, cam);
    FragLists fl = build_fragments(tri, fbits, F, pf, cam, row_begin, row_end);
    int64_t nf = int64_t(fl.records.size());
    if (offsets) std::memcpy(offsets, fl.offsets.data(), sizeof(int64_t) * fl.offsets.size());
    if (records && records_cap >= nf) std::memcpy(records, fl.records.data(), sizeof(uint64_t) * size_t(nf));
    return nf;
}

// FP32 projection of vertices (sx, sy, ze per vertex) and the snapped coords.
void orc_project_f32(const float* pos, int64_t V, const Camera* camp, float* sxsyze, int32_t* XY,
                     uint8_t* valid) {
    CamConst cam = make_cam(*camp);
    for (int64_t v = 0; v < V; ++v) {
        ProjF p = project_f(cam, pos[3 * v], pos[3 * v + 1], pos[3 * v + 2]);
        sxsyze[3 * v] = p.sx;
        sxsyze[3 * v + 1] = p.sy;
        sxsyze[3 * v + 2] = p.ze;
        XY[2 * v] = p.X;
        XY[2 * v + 1] = p.Y;
        valid[v] = p.valid ? 1 : 0;
    }
}

int orc_render_f64(const uint32_t* tri, const uint32_t* fbits, int64_t F, const double* pos, const double* col,
                   int64_t V, const Camera* cam, const Params* prm, double* image, double* tfinal, uint32_t* term,
                   int64_t* nfrag) {
    return render_impl<double>(tri, fbits, F, pos, col, V, cam, prm, image, tfinal, term, nfrag);
}

// Forward with the fragment lists (coverage and order) of pos_coverage and
// every continuous quantity from pos: the function whose derivative the
// adjoint computes, smooth in pos, for finite-difference checks.
int orc_render_frozen_f64(const uint32_t* tri, const uint32_t* fbits, int64_t F, const float* pos_coverage,
                          const double* pos, const double* col, int64_t V, const Camera* cam, const Params* prm,
                          double* image) {
    return render_impl<double>(tri, fbits, F, pos, col, V, cam, prm, image, nullptr, nullptr, nullptr,
                               pos_coverage);
}

int orc_render_f32(const uint32_t* tri, const uint32_t* fbits, int64_t F, const float* pos, const float* col,
                   int64_t V, const Camera* cam, const Params* prm, float* image, float* tfinal, uint32_t* term,
                   int64_t* nfrag) {
    return render_impl<float>(tri, fbits, F, pos, col, V, cam, prm, image, tfinal, term, nfrag);
}

int orc_adjoint_f64(const uint32_t* tri, const uint32_t* fbits, int64_t F, const double* pos, const double* col,
                    int64_t V, const Camera* cam, const Params* prm, const double* image_adj, double* grad_pos,
                    double* grad_col) {
    return adjoint_impl<double>(tri, fbits, F, pos, col, V, cam, prm, image_adj, grad_pos, grad_col);
}

int orc_adjoint_f32(const uint32_t* tri, const uint32_t* fbits, int64_t F, const float* pos, const float* col,
                    int64_t V, const Camera* cam, const Params* prm, const float* image_adj, float* grad_pos,
                    float* grad_col) {
    return adjoint_impl<float>(tri, fbits, F, pos, col, V, cam, prm, image_adj, grad_pos, grad_col);
}

// tet -> its four unique face indices, in TetFaceTable order (the face of tet
// c opposite vertex tetFaceTable[j][3] is tet_faces[4c + j]).
void orc_tet_faces(const uint32_t* cells, int64_t T, uint32_t* tet_faces) {
    std::vector<TempFace> tf(size_t(T) * 4);
    for (int64_t c = 0; c < T; ++c)
        for (int j = 0; j < 4; ++j) {
            uint32_t v[3];
            for (int k = 0; k < 3; ++k) v[k] = cells[4 * c + kTetFace[j][k]];
            std::sort(v, v + 3);
            tf[4 * c + j] = TempFace{{v[0], v[1], v[2]}, uint32_t(4 * c + j), uint32_t(c)};
        }
    std::sort(tf.begin(), tf.end());
    int64_t F = -1;
    for (size_t i = 0; i < tf.size(); ++i) {
        if (i == 0 || !tf[i].same(tf[i - 1])) ++F;
        tet_faces[tf[i].face_id] = uint32_t(F);
    }
}

// Ray-tet path: forward (image, T_final, segments per pixel) and, with
// image_adj non-null, the exact adjoint added into grad_pos / grad_col.
// pos_cov (nullable): coverage and walk from these float positions (frozen).
int orc_raytet_f64(const uint32_t* tri, const uint32_t* fbits, const uint32_t* f2t, const uint32_t* tet_faces,
                   int64_t F, const double* pos, const double* col, int64_t V, const Camera* cam, const Params* prm,
                   double* image, double* tfinal, uint32_t* nseg, const double* image_adj, double* grad_pos,
                   double* grad_col, const float* pos_cov) {
    return raytet_impl<double>(tri, fbits, f2t, tet_faces, F, pos, col, V, cam, prm, image, tfinal, nseg, image_adj,
                               grad_pos, grad_col, pos_cov);
}

int orc_raytet_f32(const uint32_t* tri, const uint32_t* fbits, const uint32_t* f2t, const uint32_t* tet_faces,
                   int64_t F, const float* pos, const float* col, int64_t V, const Camera* cam, const Params* prm,
                   float* image, float* tfinal, uint32_t* nseg, const float* image_adj, float* grad_pos,
                   float* grad_col, const float* pos_cov) {
    return raytet_impl<float>(tri, fbits, f2t, tet_faces, F, pos, col, V, cam, prm, image, tfinal, nseg, image_adj,
                              grad_pos, grad_col, pos_cov);
}

// Segment integral for closed-form checks (ForwardCommon.glsl:42-49).
void orc_segment_integral(double t, const double* c0, const double* c1, double a, double* out4) {
    double cacc[3], A;
    bool active = seg_integral<double>(t, c0, c1, a, cacc, A);
    for (int k = 0; k < 3; ++k) out4[k] = cacc[k];
    out4[3] = active ? 1.0 - A : 0.0;
}

// Per-cell colours: forward (image, T_final, termination index, #fragments) and,
// with image_adj, the adjoint added into grad_pos [3V] and grad_cell [4T].
// pos_coverage (nullable): fragment lists from these positions (frozen lists).
int orc_cells_f64(const uint32_t* tri, const uint32_t* fbits, const uint32_t* f2t, int64_t F, const double* pos,
                  const double* ccol, int64_t V, int64_t T, const Camera* cam, const Params* prm, double* image,
                  double* tfinal, uint32_t* term, int64_t* nfrag, const double* image_adj, double* grad_pos,
                  double* grad_cell, const float* pos_coverage) {
    return cells_impl<double>(tri, fbits, f2t, F, pos, ccol, V, T, cam, prm, image, tfinal, term, nfrag, image_adj,
                              grad_pos, grad_cell, pos_coverage);
}

// Tet-quality regularizer (Data/Shaders/Optimizer/TetRegularizer.glsl:108-166):
// per tet, q = 6 sqrt(2) V / l_rms^3 with V = -det[p1-p0, p2-p0, p3-p0] / 6
// (:91-93) and l_rms^2 = (sum of squared edge lengths) / 6 (:95-109); penalty
// (lambda / beta) log(1 + exp(-beta q)) whose derivative -lambda / (1 + exp(beta q))
// is :120; dq/dp written from the quotient rule on q = -c D / S^(3/2) with the
// reference's denominator clamp max(S^(5/2), 1e-5) (:125-142).  Adds into
// grad[3V]; returns the penalty summed over tets.
double orc_tet_regularizer(const uint32_t* cells, int64_t T, const double* pos, double lambda, double beta,
                           double* grad) {
    const double c = 12.0 * std::sqrt(3.0);
    double total = 0.0;
    for (int64_t t = 0; t < T; ++t) {
        double p[4][3];
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 3; ++k) p[j][k] = pos[3 * size_t(cells[4 * t + j]) + k];
        double e[4][3];  // e[j] = p[j] - p[0]
        for (int j = 1; j < 4; ++j)
            for (int k = 0; k < 3; ++k) e[j][k] = p[j][k] - p[0][k];
        auto cross = [](const double* a, const double* b, double* o) {
            o[0] = a[1] * b[2] - a[2] * b[1];
            o[1] = a[2] * b[0] - a[0] * b[2];
            o[2] = a[0] * b[1] - a[1] * b[0];
        };
        double dD[4][3];
        cross(e[2], e[3], dD[1]);
        cross(e[3], e[1], dD[2]);
        cross(e[1], e[2], dD[3]);
        for (int k = 0; k < 3; ++k) dD[0][k] = -(dD[1][k] + dD[2][k] + dD[3][k]);
        const double D = dD[3][0] * e[3][0] + dD[3][1] * e[3][1] + dD[3][2] * e[3][2];
        double S = 0.0;
        for (int a = 0; a < 4; ++a)
            for (int b = a + 1; b < 4; ++b)
                for (int k = 0; k < 3; ++k) S += (p[a][k] - p[b][k]) * (p[a][k] - p[b][k]);
        const double q = -c * D / std::pow(S, 1.5);
        const double dLdq = -lambda / (1.0 + std::exp(beta * q));
        const double den = std::max(std::pow(S, 2.5), 1e-5);
        double sum[3] = {0, 0, 0};
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 3; ++k) sum[k] += p[j][k];
        for (int j = 0; j < 4; ++j) {
            const size_t v = cells[4 * t + j];
            for (int k = 0; k < 3; ++k) {
                const double dS = 2.0 * (4.0 * p[j][k] - sum[k]);
                grad[3 * v + k] += dLdq * (-c * S * dD[j][k] + 1.5 * c * D * dS) / den;
            }
        }
        const double z = -beta * q;
        total += (lambda / beta) * (std::max(z, 0.0) + std::log1p(std::exp(-std::fabs(z))));
    }
    return total;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Reference mode (namespace refmode): forward, and the adjoint when image_adj
// is given.  pos_f: the FP32 positions of the coverage rule.  skip0 = 0 runs
// the adjoint over all four sub-segments (a check of this restatement).
int orc_refmode_f64(const uint32_t* tri, const uint32_t* fbits, int64_t F, const float* pos_f, const double* pos,
                    const double* col, int64_t V, const Camera* cam, const Params* prm, double* image,
                    uint32_t* term, const double* image_adj, double* grad_pos, double* grad_col, int32_t skip0) {
    return refmode::run(tri, fbits, F, pos_f, pos, col, V, cam, prm, image, term, image_adj, grad_pos, grad_col,
                        skip0 != 0);
}

// Check hook of the reference mode's baryAdjoint: u, v of world point p on
// face (p0, p1, p2) and their gradients w.r.t. the vertices (p fixed):
// du[3 j + c] = du / d p_j[c], likewise dv.
void orc_refmode_bary_uv(const double* p, const double* p0, const double* p1, const double* p2, double* u,
                         double* v, double* du, double* dv) {
    refmode::Frag fr;
    fr.p = {p[0], p[1], p[2]};
    fr.pv[0] = {p0[0], p0[1], p0[2]};
    fr.pv[1] = {p1[0], p1[1], p1[2]};
    fr.pv[2] = {p2[0], p2[1], p2[2]};
    for (int j = 0; j < 3; ++j)
        for (int q = 0; q < 4; ++q) fr.c[j][q] = 0.0;
    const refmode::V3 d20 = fr.pv[2] - fr.pv[0], d21 = fr.pv[2] - fr.pv[1];
    const double area = std::max(refmode::len(refmode::cross(d20, d21)), 1e-6);
    fr.u = refmode::len(refmode::cross(d21, fr.p - fr.pv[1])) / area;
    fr.v = refmode::len(refmode::cross(fr.p - fr.pv[0], d20)) / area;
    *u = fr.u;
    *v = fr.v;
    const double zero[4] = {0, 0, 0, 0};
    for (int which = 0; which < 2; ++which) {
        refmode::V3 dp[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        double dcol[3][4];
        refmode::bary_adjoint(fr, zero, which == 0 ? 1.0 : 0.0, which == 1 ? 1.0 : 0.0, dp, dcol);
        double* out = which == 0 ? du : dv;
        for (int j = 0; j < 3; ++j) {
            out[3 * j] = dp[j].x;
            out[3 * j + 1] = dp[j].y;
            out[3 * j + 2] = dp[j].z;
        }
    }
}

}  // extern "C"
