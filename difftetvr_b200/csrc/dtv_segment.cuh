// Piecewise-linear colour / constant-density segment integral and its
// adjoint, in a form that keeps full FP32 accuracy for small optical depth.
//
// Reference: accumulateLinearConst (Data/Shaders/Common/ForwardCommon.glsl:42-49)
//   A = exp(-a t),  C = (1 - A) c0 + ((t + 1/a) A - 1/a) (c0 - c1),  alpha = 1 - A
// and accumulateLinearConstAdjoint (Data/Shaders/Common/BackwardCommon.glsl:116-133).
//
// With x = a t the same quantities are written as
//   1 - A = x phi1(x),        phi1(x) = (1 - e^-x) / x
//   K     = (t + 1/a) A - 1/a = -t x psi(x),   psi(x) = (phi1(x) - e^-x) / x
//   dK/da = t^2 chi(x),       chi(x) = (1 - e^-x (1 + x + x^2)) / x^2
// For x < 0.5 phi1, psi and chi come from their Taylor series (derived from
// the exponential series; coefficients below; below x = 1/8 from the one
// series of phi2, degree 8-9 series above), which avoids the cancellation of
// the direct form (~1e-3 relative error in FP32 at a t ~ 1e-4).
// exp and the divisions use the fast hardware approximations (__expf,
// __fdividef: a few ulp), well inside the path's 1e-5 image / 1e-4 gradient
// tolerances; the discrete depth key never goes through this file.
#pragma once
#include "dtv_device.cuh"

namespace dtv {

struct SegTerms {
    float A;     // exp(-x)
    float omA;   // 1 - exp(-x)
    float K;     // (t + 1/a) A - 1/a
    float dK;    // dK/da (seg_terms_adj only)
};

__device__ __forceinline__ float series_phi1(float x) {
    // sum_k (-1)^k x^k / (k+1)!, k = 0..9
    float p = -2.75573192e-7f;
    p = fmaf(p, x, 2.75573192e-6f);
    p = fmaf(p, x, -2.48015873e-5f);
    p = fmaf(p, x, 1.98412698e-4f);
    p = fmaf(p, x, -1.38888889e-3f);
    p = fmaf(p, x, 8.33333333e-3f);
    p = fmaf(p, x, -4.16666667e-2f);
    p = fmaf(p, x, 0.166666667f);
    p = fmaf(p, x, -0.5f);
    p = fmaf(p, x, 1.0f);
    return p;
}

__device__ __forceinline__ float series_psi(float x) {
    // sum_m (-1)^m (m+1) x^m / (m+2)!, m = 0..8
    float p = 2.48015873e-6f;
    p = fmaf(p, x, -2.20458554e-5f);
    p = fmaf(p, x, 1.73611111e-4f);
    p = fmaf(p, x, -1.19047619e-3f);
    p = fmaf(p, x, 6.94444444e-3f);
    p = fmaf(p, x, -3.33333333e-2f);
    p = fmaf(p, x, 0.125f);
    p = fmaf(p, x, -0.333333333f);
    p = fmaf(p, x, 0.5f);
    return p;
}

__device__ __forceinline__ float series_chi(float x) {
    // -sum_m (-1)^m (m+1)^2 x^m / (m+2)!, m = 0..9
    float p = 2.50521084e-6f;
    p = fmaf(p, x, -2.23214286e-5f);
    p = fmaf(p, x, 1.76366843e-4f);
    p = fmaf(p, x, -1.21527778e-3f);
    p = fmaf(p, x, 7.14285714e-3f);
    p = fmaf(p, x, -3.47222222e-2f);
    p = fmaf(p, x, 0.133333333f);
    p = fmaf(p, x, -0.375f);
    p = fmaf(p, x, 0.666666667f);
    p = fmaf(p, x, -0.5f);
    return p;
}

// Below x = 1/8 one series serves all three: with
//   phi2(x) = (e^-x - 1 + x) / x^2 = sum_j (-x)^j / (j+2)!,
// phi1 = 1 - x phi2, psi = phi1 - phi2 (the series of psi is the difference
// of those of phi1 and phi2 term by term) and chi = psi - e^-x (likewise).
// phi2 to degree 5: the first omitted term at x = 1/8 is x^6/8! = 9.5e-11,
// 2e-10 of the value.  Both differences are exact in FP32 (Sterbenz: phi1/2
// <= phi2 <= phi1 and A/2 <= psi <= A for 0 <= x <= 1/8), so psi and chi
// carry only the rounding of their operands (chi: that of A too).  At
// the path's densities and segment lengths nearly every sub-segment has
// x < 1/8.
__device__ __forceinline__ float series_phi2_short(float x) {
    float p = -1.98412698e-4f;
    p = fmaf(p, x, 1.38888889e-3f);
    p = fmaf(p, x, -8.33333333e-3f);
    p = fmaf(p, x, 4.16666667e-2f);
    p = fmaf(p, x, -0.166666667f);
    p = fmaf(p, x, 0.5f);
    return p;
}

// e^x - 1 for |x| < 1/2 from its Taylor series to degree 9 (the first
// omitted term at |x| = 1/2 is x^10 / 10! = 2.7e-10, under 7e-10 of the value).
__device__ __forceinline__ float expm1_half(float x) {
    float p = 2.75573192e-6f;             // 1/9!
    p = fmaf(p, x, 2.48015873e-5f);       // 1/8!
    p = fmaf(p, x, 1.98412698e-4f);       // 1/7!
    p = fmaf(p, x, 1.38888889e-3f);       // 1/6!
    p = fmaf(p, x, 8.33333333e-3f);       // 1/5!
    p = fmaf(p, x, 4.16666667e-2f);       // 1/4!
    p = fmaf(p, x, 0.166666667f);         // 1/3!
    p = fmaf(p, x, 0.5f);                 // 1/2!
    p = fmaf(p, x, 1.0f);
    return x * p;
}

// The x = a t < 1/8 tier of seg_terms / seg_terms_adj alone (no branch), for
// callers that have checked the tier for several sub-segments at once.
// Here A = 1 - (1 - A): one rounding of a value near 1 (within 2^-25), no
// exp evaluation.
__device__ __forceinline__ SegTerms seg_terms_short(float t, float a) {
    SegTerms s;
    const float x = a * t;
    const float phi2 = series_phi2_short(x);
    const float phi1 = fmaf(-x, phi2, 1.0f);
    s.omA = x * phi1;
    s.A = 1.0f - s.omA;
    s.K = -t * x * (phi1 - phi2);
    s.dK = 0.f;
    return s;
}

__device__ __forceinline__ SegTerms seg_terms_adj_short(float t, float a) {
    SegTerms s;
    const float x = a * t;
    const float phi2 = series_phi2_short(x);
    const float phi1 = fmaf(-x, phi2, 1.0f);
    const float psi = phi1 - phi2;
    s.omA = x * phi1;
    s.A = 1.0f - s.omA;
    s.K = -t * x * psi;
    s.dK = t * t * (psi - s.A);
    return s;
}

// The four sub-segments of a segment have independent series terms, so they
// run as two pairs (sub-segments 0,1 and 2,3) of sm_100's two-wide FP32
// instructions (fma2 / mul2 / add2, dtv_device.cuh) at half the issue slots.
struct SegTerms2 {
    float2 A, omA, K, dK;
};

// seg_terms_adj_short (DK: also dK) for two sub-segments: phi2 from its
// series in -x (the same terms as in x with alternating signs, so the same
// value), then phi1 = 1 - x phi2, psi = phi1 - phi2, 1 - A = x phi1,
// K = -t x psi, dK = t^2 (psi - A).
template <bool DK>
__device__ __forceinline__ SegTerms2 seg_terms_short2(float t, float2 a) {
    const float2 x = mul2(a, bc2(t)), nx = mul2(a, bc2(-t));
    float2 p = bc2(1.98412698e-4f);
    p = fma2(p, nx, bc2(1.38888889e-3f));
    p = fma2(p, nx, bc2(8.33333333e-3f));
    p = fma2(p, nx, bc2(4.16666667e-2f));
    p = fma2(p, nx, bc2(0.166666667f));
    p = fma2(p, nx, bc2(0.5f));
    const float2 phi1 = fma2(nx, p, bc2(1.0f));
    const float2 psi = sub2(phi1, p);
    SegTerms2 s;
    s.omA = mul2(x, phi1);
    s.A = sub2(bc2(1.0f), s.omA);
    s.K = mul2(mul2(bc2(-t), x), psi);
    s.dK = DK ? mul2(bc2(t * t), sub2(psi, s.A)) : bc2(0.f);
    return s;
}

// 1 - e^-x without cancellation (x phi1(x) for |x| < 1/8).
__device__ __forceinline__ float one_minus_exp(float x) {
    if (fabsf(x) < 0.125f) return x * fmaf(-x, series_phi2_short(x), 1.0f);
    return 1.0f - __expf(-x);
}

// e^x - 1 without cancellation (series for |x| < 1/2).
__device__ __forceinline__ float expm1_signed(float x) {
    if (fabsf(x) < 0.5f) return expm1_half(x);
    return __expf(x) - 1.0f;
}

// Transmittance carried along a pixel ray as an unevaluated float-float sum
// hi + lo.  A segment of optical depth x lowers T by T (1 - e^-x); at low
// density that is far below the spacing of FP32 values near T (2^-24 T): a
// plain FP32 T would round each decrement, or lose it entirely once it is
// under half that spacing (a ray through thousands of nearly transparent
// segments would keep T = 1).  Each segment's decrement (or, back to front,
// increment) is applied with an error-free sum, the error kept in lo.
struct TransF {
    float hi, lo;
};

// T += d for |d| <= |T.hi| (Fast2Sum), renormalised.
__device__ __forceinline__ void trans_add_small(TransF& T, float d) {
    const float s = __fadd_rn(T.hi, d);
    const float e = __fadd_rn(__fsub_rn(T.hi, s), d);
    const float lo = __fadd_rn(T.lo, e);
    T.hi = __fadd_rn(s, lo);
    T.lo = __fsub_rn(lo, __fsub_rn(T.hi, s));
}

// T += d for any d (TwoSum), renormalised.
__device__ __forceinline__ void trans_add(TransF& T, float d) {
    const float s = __fadd_rn(T.hi, d);
    const float bb = __fsub_rn(s, T.hi);
    const float e = __fadd_rn(__fsub_rn(T.hi, __fsub_rn(s, bb)), __fsub_rn(d, bb));
    const float lo = __fadd_rn(T.lo, e);
    T.hi = __fadd_rn(s, lo);
    T.lo = __fsub_rn(lo, __fsub_rn(T.hi, s));
}

// Forward terms; caller guarantees a > 0.  (The reference drops a < 1e-6; the
// continuous value kept here differs from that by at most a t.)
__device__ __forceinline__ SegTerms seg_terms(float t, float a) {
    const float x = a * t;
    if (x < 0.125f) return seg_terms_short(t, a);
    SegTerms s;
    s.A = __expf(-x);
    if (x < 0.5f) {
        s.omA = x * series_phi1(x);
        s.K = -t * x * series_psi(x);
    } else {
        s.omA = 1.0f - s.A;
        const float phi1 = __fdividef(s.omA, x);
        s.K = -t * (phi1 - s.A);
    }
    s.dK = 0.f;
    return s;
}

// Forward terms and dK/da in one pass (adjoint); caller guarantees a > 0.
__device__ __forceinline__ SegTerms seg_terms_adj(float t, float a) {
    const float x = a * t;
    if (x < 0.125f) return seg_terms_adj_short(t, a);
    SegTerms s;
    s.A = __expf(-x);
    float chi;
    if (x < 0.5f) {
        s.omA = x * series_phi1(x);
        s.K = -t * x * series_psi(x);
        chi = series_chi(x);
    } else {
        s.omA = 1.0f - s.A;
        const float ix = __fdividef(1.0f, x);
        s.K = -t * (s.omA * ix - s.A);
        chi = (s.omA - x * s.A * (1.0f + x)) * ix * ix;
    }
    s.dK = t * t * chi;
    return s;
}

}  // namespace dtv
