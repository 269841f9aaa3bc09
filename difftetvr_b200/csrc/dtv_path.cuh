// Per-face and per-pixel bodies of the hot path, shared by the single-view
// kernels (dtv_kernels.cu) and the batched multi-view kernels (dtv_batch.cu).
#pragma once
#include <type_traits>
#include "dtv_device.cuh"
#include "dtv_segment.cuh"

namespace dtv {

using u64 = unsigned long long;
constexpr int kTile = 16;  // composite / adjoint pixel tile (16 x 16 threads)

// ---------------------------------------------------------------------------
// (a)+(b) face rasterisation, warp-cooperative.  Each lane of a warp sets up
// one face (projected fixed-point vertices, orientation, clipped bounding box)
// into shared memory; the warp then takes the faces one at a time.  Each box
// row of a face meets it in one interval of pixel centres, found exactly per
// row (row_span).  The count (one thread per face) adds +1 / -1 at the ends of
// each row's interval to a per-row difference array in `counts`, which
// row_prefix_warp turns into per-pixel counts; the fill (one warp per face)
// spreads the covered pixels of the face over the warp's lanes and writes
// each record at offsets[p] + (--counts[p]),
// leaving counts zeroed for the next render.  Only pixel rows [row0, row1) are
// visited (row bands of a render whose lists do not fit the fragment budget at
// once).
//
// Coverage: edge functions in 1/256-pixel fixed point, evaluated relative to
// the centre of the box's first pixel (edge functions are translation
// invariant, so the values are the exact ones).  For boxes under 64 px
// (2^14 units) on each side every term is below 2^29 and 32-bit integers are
// exact; larger faces use 64 bits.  Both give identical coverage.
template <typename I>
__device__ __forceinline__ bool edge_in(I E, I dx, I dy) {
    return (E > 0) || (E == 0 && ((dy < 0) || (dy == 0 && dx > 0)));
}

struct __align__(16) RasterJob {
    int ax0, ay0, ax1, ay1, ax2, ay2;  // vertices, relative to the first pixel centre; E > 0 inside
    int px0, py0, bw, bh;              // first pixel and size of the clipped bounding box
    uint32_t bits;                     // record low word: face << 2 | boundary << 1 | front
    uint32_t v0, v1, v2;               // vertex rows of vproj (depth key)
    int W;                             // image width (pixel rows of counts / offsets)
    int wide;                          // edge functions need 64 bits
    u64 pix_base;                      // first pixel of the image in counts / offsets
};

// Setup of face f (vertex indices local to vfix; vproj rows = vert_base + index).
__device__ __forceinline__ bool raster_setup(uint32_t f, const uint4* __restrict__ faces,
                                             const int2* __restrict__ vfix, uint32_t vert_base, int W, int row0,
                                             int row1, u64 pix_base, RasterJob& J) {
    const uint4 fc = faces[f];
    const int2 q0 = vfix[fc.x], q1 = vfix[fc.y], q2 = vfix[fc.z];
    if (q0.x == kInvalidFix || q1.x == kInvalidFix || q2.x == kInvalidFix) return false;
    const long long X0 = q0.x, Y0 = q0.y, X1 = q1.x, Y1 = q1.y, X2 = q2.x, Y2 = q2.y;
    const long long area2 = (X1 - X0) * (Y2 - Y0) - (Y1 - Y0) * (X2 - X0);
    if (area2 == 0) return false;
    const long long minX = min(X0, min(X1, X2)), maxX = max(X0, max(X1, X2));
    const long long minY = min(Y0, min(Y1, Y2)), maxY = max(Y0, max(Y1, Y2));
    const int px0 = int(max(0LL, ceil_div256(minX - 128)));
    const int px1 = int(min((long long)W - 1, floor_div256(maxX - 128)));
    const int py0 = int(max((long long)row0, ceil_div256(minY - 128)));
    const int py1 = int(min((long long)row1 - 1, floor_div256(maxY - 128)));
    if (px0 > px1 || py0 > py1) return false;
    const long long Xs = 256LL * px0 + 128, Ys = 256LL * py0 + 128;
    // Counter-clockwise order (E > 0 inside): swap vertices 1 and 2 of a front face.
    const bool front = area2 < 0;
    J.ax0 = int(X0 - Xs);
    J.ay0 = int(Y0 - Ys);
    J.ax1 = int((front ? X2 : X1) - Xs);
    J.ay1 = int((front ? Y2 : Y1) - Ys);
    J.ax2 = int((front ? X1 : X2) - Xs);
    J.ay2 = int((front ? Y1 : Y2) - Ys);
    J.px0 = px0;
    J.py0 = py0;
    J.bw = px1 - px0 + 1;
    J.bh = py1 - py0 + 1;
    J.bits = (f << 2) | ((fc.w & 1u) << 1) | (front ? 1u : 0u);
    J.v0 = vert_base + fc.x;
    J.v1 = vert_base + fc.y;
    J.v2 = vert_base + fc.z;
    J.W = W;
    J.wide = (maxX - minX < (1LL << 14) && maxY - minY < (1LL << 14)) ? 0 : 1;
    J.pix_base = pix_base;
    return true;
}

// Edge function of one edge over the box, with the coverage tie rule folded
// in: for integer E, "E > 0, or E == 0 and the edge is a top-left edge
// (dy < 0, or dy == 0 and dx > 0)" is "E + t - 1 >= 0" with t = 1 for a
// top-left edge, 0 otherwise.  T(c, r) = base + sx c + sy r is that shifted
// value at pixel (c, r) of the box, so a pixel is covered iff the three
// values are all non-negative, i.e. iff the sign bit of their OR is clear.
template <typename I>
struct EdgeT {
    I base, sx, sy;
    __device__ __forceinline__ void set(I ax, I ay, I bx, I by) {  // edge a -> b
        const I dx = bx - ax, dy = by - ay;
        const I t = ((dy < 0) || (dy == 0 && dx > 0)) ? I(1) : I(0);
        base = dy * ax - dx * ay + t - I(1);  // E at the origin: dx (0 - ay) - dy (0 - ax)
        sx = -dy * I(256);
        sy = dx * I(256);
    }
    __device__ __forceinline__ I at(int c, int r) const { return base + sx * I(c) + sy * I(r); }
};

// Exact column range of box row r under one edge: T(c, r) = q + sx c >= 0
// with q = base + sy r is c >= -q / sx (sx > 0) or c <= -q / sx (sx < 0);
// sx = 0 makes the row all-in or all-out.  The bound is estimated in FP32
// (relative error a few 2^-24: under 0.01 px for every bound inside a box of
// at most 2^14 px, clamped to [-2, bw + 1] beyond it) and corrected by one
// exact integer test on each side, so lo / hi are the exact first / last
// columns the edge admits.
template <typename I>
__device__ __forceinline__ void span_edge(const EdgeT<I>& e, float inv_sx, int r, int bw, int& lo, int& hi) {
    const I q = e.base + e.sy * I(r);
    if (e.sx == I(0)) {
        if (q < I(0)) {
            lo = bw;
            hi = -1;
        }
        return;
    }
    const float b = fminf(fmaxf(-float(q) * inv_sx, -2.f), float(bw) + 1.f);
    if (e.sx > I(0)) {
        int c = int(ceilf(b));  // first column with T >= 0, up to one off
        if (q + e.sx * I(c - 1) >= I(0))
            --c;
        else if (q + e.sx * I(c) < I(0))
            ++c;
        lo = max(lo, c);
    } else {
        int c = int(floorf(b));  // last column with T >= 0, up to one off
        if (q + e.sx * I(c + 1) >= I(0))
            ++c;
        else if (q + e.sx * I(c) < I(0))
            --c;
        hi = min(hi, c);
    }
}

// Covered columns [xl, xl + len) of box row r (len 0: none): exactly the
// pixels whose centres pass all three edge tests, since a row meets a
// triangle in one interval.
template <typename I>
__device__ __forceinline__ int row_span(const EdgeT<I>& e0, const EdgeT<I>& e1, const EdgeT<I>& e2, float i0,
                                        float i1, float i2, int r, int bw, int& xl) {
    int lo = 0, hi = bw - 1;
    span_edge(e0, i0, r, bw, lo, hi);
    span_edge(e1, i1, r, bw, lo, hi);
    span_edge(e2, i2, r, bw, lo, hi);
    xl = lo;
    return max(0, hi - lo + 1);
}

struct FaceEdges {
    // Counter-clockwise edges e0: 1 -> 2, e1: 2 -> 0, e2: 0 -> 1, and their
    // column-step reciprocals for the FP32 span estimates.
    template <typename I>
    __device__ __forceinline__ static void make(const RasterJob& J, EdgeT<I>& e0, EdgeT<I>& e1, EdgeT<I>& e2,
                                                float& i0, float& i1, float& i2) {
        e0.set(I(J.ax1), I(J.ay1), I(J.ax2), I(J.ay2));
        e1.set(I(J.ax2), I(J.ay2), I(J.ax0), I(J.ay0));
        e2.set(I(J.ax0), I(J.ay0), I(J.ax1), I(J.ay1));
        i0 = e0.sx != I(0) ? __frcp_rn(float(e0.sx)) : 0.f;
        i1 = e1.sx != I(0) ? __frcp_rn(float(e1.sx)) : 0.f;
        i2 = e2.sx != I(0) ? __frcp_rn(float(e2.sx)) : 0.f;
    }
};

// Count pass over one face, one thread: each box row's exact span adds +1 at
// its first pixel and -1 after its last one (when that is still in the image
// row) to a per-row difference array held in `counts` (u32, modulo 2^32);
// row_prefix_warp turns it into per-pixel counts.  Two atomics per face row
// instead of one per covered pixel, and no per-face warp work: a face has
// about eleven rows at the path's sizes.
template <typename I>
__device__ __forceinline__ void count_face(const RasterJob& J, uint32_t* __restrict__ counts) {
    EdgeT<I> e0, e1, e2;
    float i0, i1, i2;
    FaceEdges::make(J, e0, e1, e2, i0, i1, i2);
    uint32_t* row = counts + J.pix_base + u64(J.py0) * u64(J.W) + u64(J.px0);
    for (int r = 0; r < J.bh; ++r, row += J.W) {
        int xl;
        const int len = row_span(e0, e1, e2, i0, i1, i2, r, J.bw, xl);
        if (len > 0) {
            atomicAdd(row + xl, 1u);
            if (J.px0 + xl + len < J.W) atomicAdd(row + xl + len, 0xffffffffu);
        }
    }
}

// Per-row inclusive prefix, in place, of the count pass's difference array
// (u32 arithmetic modulo 2^32, so the -1 entries wrap and the sums come out
// exact): one warp per image row.
__device__ __forceinline__ void row_prefix_warp(uint32_t* row, int W, int lane) {
    uint32_t carry = 0;
    for (int x0 = 0; x0 < W; x0 += 32) {
        const int x = x0 + lane;
        uint32_t v = x < W ? row[x] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += t;
        }
        v += carry;
        if (x < W) row[x] = v;
        carry = __shfl_sync(0xffffffffu, v, 31);
    }
}

// Fill of U covered pixels per lane per step: offset loads, counter atomics
// and depth keys of all U before the stores.  A counter already at zero
// (which matching count and fill spans never leave) skips the store, so a
// record is never written outside its list.
template <typename I, int U>
__device__ __forceinline__ void fill_pixels(const RasterJob& J, const int (&c)[U], const int (&r)[U],
                                            const bool (&valid)[U], u64 pbase, const float4& va, const float4& vb,
                                            const float4& vc, uint32_t* __restrict__ counts,
                                            const u64* __restrict__ offsets, u64* __restrict__ records) {
    uint32_t slot[U];
    u64 off[U];
    float z[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
        if (valid[k]) {
            const u64 p = pbase + uint32_t(r[k] * J.W + c[k]);
            off[k] = offsets[p];
            slot[k] = atomicSub(&counts[p], 1u);
            z[k] = depth_key(va, vb, vc, float(J.px0 + c[k]) + 0.5f, float(J.py0 + r[k]) + 0.5f);
        }
    }
#pragma unroll
    for (int k = 0; k < U; ++k)
        if (valid[k] && slot[k] != 0u) records[off[k] + slot[k] - 1u] = (u64(__float_as_uint(z[k])) << 32) | J.bits;
}

// Fill of one face by the warp: it takes the box rows 32 at a time (lane =
// row), finds each row's exact span, and spreads the concatenated spans over
// its lanes (slot s -> row by a binary search of the spans' exclusive prefix
// sums), so every lane slot is a covered pixel.
template <bool FILL, typename I>
__device__ __forceinline__ void raster_job(const RasterJob& J, int lane, const float4* __restrict__ vproj,
                                           uint32_t* __restrict__ counts, const u64* __restrict__ offsets,
                                           u64* __restrict__ records) {
    static_assert(FILL, "the count pass runs one face per thread (count_face)");
    {
        constexpr int U = sizeof(I) == 4 ? 2 : 1;  // one pixel per step on the rare 64-bit path
        EdgeT<I> e0, e1, e2;
        float i0, i1, i2;
        FaceEdges::make(J, e0, e1, e2, i0, i1, i2);
        const u64 pbase = J.pix_base + u64(J.py0) * u64(J.W) + u64(J.px0);
        const float4 va = vproj[J.v0], vb = vproj[J.v1], vc = vproj[J.v2];
        for (int r0 = 0; r0 < J.bh; r0 += 32) {
            const int r = r0 + lane;
            int xl = 0, len = 0;
            if (r < J.bh) len = row_span(e0, e1, e2, i0, i1, i2, r, J.bw, xl);
            int incl = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const int excl = incl - len;
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            for (int s0 = 0; s0 < total; s0 += 32 * U) {
                int c[U], rr[U];
                bool valid[U];
#pragma unroll
                for (int k = 0; k < U; ++k) {
                    const int sl = s0 + 32 * k + lane;
                    int i = 0;  // last row whose span starts at or before slot sl
#pragma unroll
                    for (int step = 16; step >= 1; step >>= 1)
                        if (__shfl_sync(0xffffffffu, excl, i + step) <= sl) i += step;
                    valid[k] = sl < total;
                    rr[k] = r0 + i;
                    c[k] = __shfl_sync(0xffffffffu, xl, i) + (sl - __shfl_sync(0xffffffffu, excl, i));
                }
                fill_pixels<I, U>(J, c, rr, valid, pbase, va, vb, vc, counts, offsets, records);
            }
        }
    }
}

// The warp's jobs (one per lane that has one, `live` the ballot), one at a time.
// The 32-bit and 64-bit faces go to separate launches (WIDE), so that the
// common 32-bit kernel keeps the register count of its own path.
template <bool FILL, bool WIDE>
__device__ __forceinline__ void raster_warp(const RasterJob* jobs, uint32_t live, int lane,
                                            const float4* __restrict__ vproj, uint32_t* __restrict__ counts,
                                            const u64* __restrict__ offsets, u64* __restrict__ records) {
    __syncwarp();
    while (live) {
        const int k = __ffs(live) - 1;
        live &= live - 1;
        const RasterJob J = jobs[k];
        raster_job<FILL, typename std::conditional<WIDE, long long, int>::type>(J, lane, vproj, counts, offsets,
                                                                                records);
    }
}

// ---------------------------------------------------------------------------
// Fragment evaluation shared by composite and adjoint.
struct FragV {
    float z;
    float4 col;
    uint32_t face;
    uint32_t bits;
    uint32_t v0, v1, v2;
};

// Fragment values from the record's low word (face << 2 | bits) and the
// face's vertex indices.
__device__ __forceinline__ FragV load_frag_face(uint32_t lo, const uint4& fc, float qx, float qy,
                                                const VGeo* __restrict__ vgeo, const float4* __restrict__ colors) {
    FragV fr;
    fr.face = lo >> 2;
    fr.bits = lo & 3u;
    fr.v0 = fc.x;
    fr.v1 = fc.y;
    fr.v2 = fc.z;
    const VGeo a = vgeo[fc.x], b = vgeo[fc.y], c = vgeo[fc.z];
    float bary[3];
    face_bary(a, b, c, qx, qy, bary, fr.z);  // depth and colour from the same weights
    const float4 c0 = colors[fc.x], c1 = colors[fc.y], c2 = colors[fc.z];
    // (r, g) and (b, a) as FP32 pairs.
    const float2 b0 = bc2(bary[0]), b1 = bc2(bary[1]), b2 = bc2(bary[2]);
    const float2 rg = fma2(b2, make_float2(c2.x, c2.y),
                           fma2(b1, make_float2(c1.x, c1.y), mul2(b0, make_float2(c0.x, c0.y))));
    const float2 ba = fma2(b2, make_float2(c2.z, c2.w),
                           fma2(b1, make_float2(c1.z, c1.w), mul2(b0, make_float2(c0.z, c0.w))));
    fr.col = make_float4(rg.x, rg.y, ba.x, ba.y);
    return fr;
}

__device__ __forceinline__ FragV load_frag(u64 rec, float qx, float qy, const uint4* __restrict__ faces,
                                           const VGeo* __restrict__ vgeo, const float4* __restrict__ colors) {
    const uint32_t lo = uint32_t(rec);
    return load_frag_face(lo, faces[lo >> 2], qx, qy, vgeo, colors);
}

// Low word of record i of a list (the face and its two flag bits).
__device__ __forceinline__ uint32_t record_lo(const u64* __restrict__ records, u64 i) {
    return reinterpret_cast<const uint32_t*>(records)[2 * i];
}

// ---------------------------------------------------------------------------
// Whether every sub-segment of a segment has a > 0 and x = a t < 1/8 (the
// short tier).  The sub-segment densities are affine in s, so their extremes
// are at the end sub-segments (the inner ones can exceed them only by
// rounding, where the series is still accurate).
__device__ __forceinline__ bool short_tier_of(const float (&av)[kNumSubdivs], float tSeg) {
    const float lo = fminf(av[0], av[kNumSubdivs - 1]), hi = fmaxf(av[0], av[kNumSubdivs - 1]);
    return (lo > 0.f) & (hi * tSeg < 0.125f);
}

// One segment of a pixel's ray between a front fragment (colour cf) and a back
// fragment (colour cb): the 4-sub-segment integral (ForwardCommon.glsl:42-49
// per sub-segment, colour and density linear along the segment), front to
// back.  Per sub-segment starting at fraction s, c0 = cf + s (cb - cf) and
// c1 - c0 = (cb - cf) / 4, so C += T ((1 - A) c0 - (K / 4) (cb - cf)).
// When every sub-segment has a > 0 and a t < 1/8 (nearly all of them at the
// path's densities) the four sets of terms are independent straight-line code
// (seg_terms_short, the same arithmetic seg_terms picks for that tier), which
// the scheduler interleaves; otherwise each sub-segment takes seg_terms.
__device__ __forceinline__ void segment_composite(float tSeg, const float4& cf, const float4& cb, float atten,
                                                  float& C0, float& C1, float& C2, TransF& T) {
    const float d0 = cb.x - cf.x, d1 = cb.y - cf.y, d2 = cb.z - cf.z, dw = cb.w - cf.w;
    float av[kNumSubdivs];
#pragma unroll
    for (int s = 0; s < kNumSubdivs; ++s) av[s] = (cf.w + dw * (0.25f * (s + 0.5f))) * atten;
    const bool short_tier = short_tier_of(av, tSeg);
    // Sub-segment s adds w (cf + fs d) - k d per channel; summed over the
    // sub-segments that is cf sum(w) + d sum(w fs - k), two scalars.
    float ws = 0.f, ds = 0.f;
    if (short_tier) {
        // Two-wide: sub-segments (0, 1) and (2, 3).  Entry transmittances
        // front to back by the FMA step, then the weights w = Ts (1 - A) and
        // k = Ts K / 4 of both pairs.
        const SegTerms2 s01 = seg_terms_short2<false>(tSeg, make_float2(av[0], av[1]));
        const SegTerms2 s23 = seg_terms_short2<false>(tSeg, make_float2(av[2], av[3]));
        const float T0 = T.hi;
        const float T1 = __fmaf_rn(-T0, s01.omA.x, T0);
        const float T2 = __fmaf_rn(-T1, s01.omA.y, T1);
        const float T3 = __fmaf_rn(-T2, s23.omA.x, T2);
        const float2 w01 = mul2(make_float2(T0, T1), s01.omA), w23 = mul2(make_float2(T2, T3), s23.omA);
        const float2 k01 = mul2(make_float2(T0, T1), s01.K), k23 = mul2(make_float2(T2, T3), s23.K);
        ws = hsum2(add2(w01, w23));
        // sum(w fs) - sum(Ts K) / 4
        const float2 wf = fma2(w23, make_float2(0.5f, 0.75f), mul2(w01, make_float2(0.f, 0.25f)));
        ds = __fmaf_rn(hsum2(add2(k01, k23)), -0.25f, hsum2(wf));
        trans_add_small(T, -ws);
        C0 += cf.x * ws + d0 * ds;
        C1 += cf.y * ws + d1 * ds;
        C2 += cf.z * ws + d2 * ds;
        return;
    }
    SegTerms st[kNumSubdivs];
    {
        // a <= 0 contributes nothing: A = 1, 1 - A = K = 0.
#pragma unroll
        for (int s = 0; s < kNumSubdivs; ++s) st[s] = av[s] > 0.f ? seg_terms(tSeg, av[s]) : SegTerms{1.f, 0.f, 0.f, 0.f};
    }
    // Inside the segment the sub-segments' entry transmittances follow in
    // FP32 from T.hi (Ts = Ts - Ts (1 - A) in one FMA); the segment lowers T
    // by exactly the sum of its sub-segment weights ws, applied to the
    // float-float T.
    float Ts = T.hi;
#pragma unroll
    for (int s = 0; s < kNumSubdivs; ++s) {
        const float w = Ts * st[s].omA, k = Ts * (0.25f * st[s].K);
        ws += w;
        ds += w * (0.25f * s) - k;
        Ts = __fmaf_rn(-Ts, st[s].omA, Ts);
    }
    trans_add_small(T, -ws);
    C0 += cf.x * ws + d0 * ds;
    C1 += cf.y * ws + d1 * ds;
    C2 += cf.z * ws + d2 * ds;
}

// Final pixel value over the clear colour (alpha = 1 - T taken from the
// float-float T, so a nearly transparent pixel keeps its small alpha) and the
// final transmittance for the adjoint.
__device__ __forceinline__ void write_pixel(float4* __restrict__ image, float* __restrict__ tfinal, size_t p,
                                            float C0, float C1, float C2, const TransF& T, const ShadeDev& sh) {
    const float alpha = __fsub_rn(__fsub_rn(1.f, T.hi), T.lo);
    image[p] = make_float4(C0 + T.hi * sh.clear[0], C1 + T.hi * sh.clear[1], C2 + T.hi * sh.clear[2],
                           alpha + T.hi * sh.clear[3]);
    tfinal[p] = T.hi + T.lo;
}

// ---------------------------------------------------------------------------
// (d) front-to-back compositing, one thread per pixel (16x16 pixel tiles).
// Forward.glsl:159-211 with early ray termination (:169-173) and the
// termination index (:256-259); final transmittance is kept for the adjoint.
__device__ __forceinline__ void composite_pixel(
    int px, int py, int W, const u64* __restrict__ offsets, const u64* __restrict__ records,
    const uint4* __restrict__ faces, const VGeo* __restrict__ vgeo, const float4* __restrict__ colors,
    const ShadeDev& sh, float4* __restrict__ image, float* __restrict__ tfinal, uint32_t* __restrict__ term) {
    const size_t p = size_t(py) * W + px;
    const u64 beg = offsets[p];
    const uint32_t n = uint32_t(offsets[p + 1] - beg);
    const float qx = float(px) + 0.5f, qy = float(py) + 0.5f;
    float C0 = 0.f, C1 = 0.f, C2 = 0.f;
    TransF T{1.f, 0.f};
    uint32_t i = n;
    if (n >= 2) {
        FragV f1 = load_frag(records[beg], qx, qy, faces, vgeo, colors), f0;
        for (i = 1; i < n; ++i) {
            if (sh.use_ert && T.hi < sh.ert_thresh) break;
            f0 = f1;
            f1 = load_frag(records[beg + i], qx, qy, faces, vgeo, colors);
            if (skip_pair(f0.bits, f1.bits)) continue;
            segment_composite((f1.z - f0.z) * 0.25f, f0.col, f1.col, sh.atten, C0, C1, C2, T);
        }
    }
    write_pixel(image, tfinal, p, C0, C1, C2, T, sh);
    term[p] = i;
}

// ---------------------------------------------------------------------------
// (f) adjoint.  Back to front from the termination index; transmittance is
// rebuilt from the final value (T = T_final e^X, TransBack); per fragment the depth and
// colour adjoints of its two segments are summed and pushed through the
// screen-space barycentrics and the projection to the face's three vertices.
// Vertex gradient accumulation: the 7 values of a vertex (position xyz, pad,
// colour rgba) share one 32-byte row of an interleaved buffer and are added
// with two float4 vector atomics, so each vertex update touches one L2 sector
// (scalar atomics into the [V,3] / [V,4] layout touch about three).
// Vertex gradient sinks.  A fragment's colour adjoint is the pixel's colour
// adjoint gC times a scalar (segment_adjoint), so a vertex's contribution from
// one pixel is its position gradient xyz, a weight s1 (colour rgb = gC s1)
// and the alpha gradient s2; set_pixel() gives the sink gC (|gC| for absolute
// gradients, whose s1 is then the absolute weight).
struct GradAcc {
    static constexpr bool kOrdered = false;
    float4* rows;   // [V][2]: position xyz, pad; colour rgba
    float g0 = 0.f, g1 = 0.f, g2 = 0.f;

    __device__ __forceinline__ void set_pixel(float a0, float a1, float a2) { g0 = a0; g1 = a1; g2 = a2; }
    __device__ __forceinline__ void add_face(const uint32_t (&v)[3], const float4 (&gp)[3], const float (&s2)[3]) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            atomicAdd(rows + 2 * size_t(v[j]), make_float4(gp[j].x, gp[j].y, gp[j].z, 0.f));
            atomicAdd(rows + 2 * size_t(v[j]) + 1, make_float4(g0 * gp[j].w, g1 * gp[j].w, g2 * gp[j].w, s2[j]));
        }
    }
    __device__ __forceinline__ void flush() {}
};

// Vertex-row accumulator with a per-thread cache of the three vertices of the
// last face it was given.  Consecutive fragments of a pixel's list bound one
// tet, so their faces share an edge: each new face usually brings one new
// vertex and retires one, and only the retired vertex's row goes to global
// memory (two float4 atomics instead of six per fragment; the gradient
// atomics bound the adjoint otherwise).  The cached values (position xyz and
// colour weight in a float4, alpha in a float) live in shared memory: slot s
// of thread t at c4[t + s * stride], c1[t + s * stride]; flush() writes the
// remaining ones at the end of the pixel.  (A block-wide shared-memory table
// behind it, summing the tile's pixels with shared-memory atomics, and a
// warp-wide merge of equal retired vertices both measured slower.)  It takes
// faces in their stored vertex order and finds each vertex's slot by id; the
// screen-space adjoints use the ordered caches below (no search), this one
// serves the world-space rows of absolute-value gradients.
struct VertCache {
    static constexpr bool kOrdered = false;
    static constexpr uint32_t kNone = 0xffffffffu;
    float4* rows;   // [V][2] global rows
    float4* c4;     // this thread's slot 0: position xyz, colour weight
    float* c1;      // this thread's slot 0: alpha
    int stride;     // threads of the block
    float g0 = 0.f, g1 = 0.f, g2 = 0.f;
    uint32_t id0 = kNone, id1 = kNone, id2 = kNone;

    __device__ __forceinline__ void set_pixel(float a0, float a1, float a2) { g0 = a0; g1 = a1; g2 = a2; }
    __device__ __forceinline__ void spill(int s, uint32_t v) const {
        if (v == kNone) return;
        spill_held(s, v);
    }
    __device__ __forceinline__ void spill_held(int s, uint32_t v) const {
        const float4 q = c4[s * stride];
        const float a = c1[s * stride];
        atomicAdd(rows + 2 * size_t(v), make_float4(q.x, q.y, q.z, 0.f));
        atomicAdd(rows + 2 * size_t(v) + 1, make_float4(g0 * q.w, g1 * q.w, g2 * q.w, a));
    }
    // The same steps for every lane (no branch on which slot a vertex is in):
    // the retired slots are spilled in a loop over the retire mask (one pass
    // on most fragments: each new face usually retires one vertex), and each
    // of the face's vertices adds into its slot, a new one into the lowest
    // free slot (the load of its old value predicated off).
    __device__ __forceinline__ void add_face(const uint32_t (&v)[3], const float4 (&gp)[3], const float (&s2)[3]) {
        int m[3];  // cache slot holding each vertex of the face, -1 if none
        uint32_t used = 0u;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            m[k] = v[k] == id0 ? 0 : (v[k] == id1 ? 1 : (v[k] == id2 ? 2 : -1));
            used |= m[k] >= 0 ? (1u << m[k]) : 0u;
        }
        const uint32_t held = uint32_t(id0 != kNone) | (uint32_t(id1 != kNone) << 1) | (uint32_t(id2 != kNone) << 2);
        uint32_t retire = held & ~used;
        while (retire) {
            const int s = __ffs(retire) - 1;
            retire &= retire - 1u;
            spill_held(s, s == 0 ? id0 : (s == 1 ? id1 : id2));
        }
        uint32_t free = ~used & 7u;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const bool hit = m[k] >= 0;
            const int s = hit ? m[k] : __ffs(free) - 1;
            free = hit ? free : (free & (free - 1u));
            const int o = s * stride;
            float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
            float a = 0.f;
            if (hit) {
                q = c4[o];
                a = c1[o];
            }
            c4[o] = make_float4(q.x + gp[k].x, q.y + gp[k].y, q.z + gp[k].z, q.w + gp[k].w);
            c1[o] = a + s2[k];
            id0 = (!hit && s == 0) ? v[k] : id0;
            id1 = (!hit && s == 1) ? v[k] : id1;
            id2 = (!hit && s == 2) ? v[k] : id2;
        }
    }
    __device__ __forceinline__ void flush() {
        spill(0, id0);
        spill(1, id1);
        spill(2, id2);
        id0 = id1 = id2 = kNone;
    }
};

// Vertex order of a fragment's face relative to the face processed just
// before it (w, in its own order): each vertex the two faces share keeps its
// position in w, and the face's other vertices take the remaining positions
// in their order.  Returns the order in `out` and a 3-bit mask of the
// positions whose vertex continues from w.  Consecutive fragments of a list
// usually bound one tet and share an edge, so one position changes per
// fragment and a cache of the three vertex rows needs no search.
__device__ __forceinline__ uint32_t order_like(const uint32_t (&w)[3], uint32_t y0, uint32_t y1, uint32_t y2,
                                               uint32_t (&out)[3]) {
    const bool e00 = w[0] == y0, e01 = w[0] == y1, e02 = w[0] == y2;
    const bool e10 = w[1] == y0, e11 = w[1] == y1, e12 = w[1] == y2;
    const bool e20 = w[2] == y0, e21 = w[2] == y1, e22 = w[2] == y2;
    const bool m0 = e00 | e01 | e02, m1 = e10 | e11 | e12, m2 = e20 | e21 | e22;
    const bool u0 = e00 | e10 | e20, u1 = e01 | e11 | e21;
    // The first and second of the face's vertices that w does not hold.
    const uint32_t n1 = !u0 ? y0 : (!u1 ? y1 : y2);
    const uint32_t n2 = (!u0 && !u1) ? y1 : y2;
    out[0] = m0 ? w[0] : n1;
    out[1] = m1 ? w[1] : (m0 ? n1 : n2);
    const int free_before = int(!m0) + int(!m1);
    out[2] = m2 ? w[2] : (free_before == 0 ? n1 : (free_before == 1 ? n2 : y2));
    return uint32_t(m0) | (uint32_t(m1) << 1) | (uint32_t(m2) << 2);
}

// Vertex-row accumulator for faces given in order_like order: position s of
// each face is cache slot s, so a face adds into its slots directly.  The
// order of the next face is known when a face is added (its keep mask), so a
// slot whose vertex does not continue is written to global memory (two float4
// atomics) right after that add, with the face's own vertex ids; the cache
// holds no ids.  Rows held in registers.
struct OrderedRows {
    static constexpr bool kOrdered = true;
    float4* rows;   // [V][2] global rows
    float g0 = 0.f, g1 = 0.f, g2 = 0.f;
    float4 p[3];
    float a[3];

    __device__ __forceinline__ void set_pixel(float a0, float a1, float a2) { g0 = a0; g1 = a1; g2 = a2; }
    __device__ __forceinline__ void put(uint32_t v, const float4& q, float al) const {
        atomicAdd(rows + 2 * size_t(v), make_float4(q.x, q.y, q.z, 0.f));
        atomicAdd(rows + 2 * size_t(v) + 1, make_float4(g0 * q.w, g1 * q.w, g2 * q.w, al));
    }
    // Face v (ordered; keep: the slots continuing from the previous face)
    // adds its rows; slots not in keep_next (the next face's keep mask, 0 for
    // the last face) are written out.
    __device__ __forceinline__ void add_ordered(const uint32_t (&v)[3], uint32_t keep, uint32_t keep_next,
                                                const float4 (&gp)[3], const float (&s2)[3]) {
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const bool k = (keep >> s) & 1u;
            p[s] = k ? make_float4(p[s].x + gp[s].x, p[s].y + gp[s].y, p[s].z + gp[s].z, p[s].w + gp[s].w) : gp[s];
            a[s] = k ? a[s] + s2[s] : s2[s];
            if (!((keep_next >> s) & 1u)) put(v[s], p[s], a[s]);
        }
    }
    // The slots a face added with keep_next left open, when no next face
    // follows.
    __device__ __forceinline__ void close(const uint32_t (&v)[3], uint32_t keep_next) const {
#pragma unroll
        for (int s = 0; s < 3; ++s)
            if ((keep_next >> s) & 1u) put(v[s], p[s], a[s]);
    }
    __device__ __forceinline__ void flush() {}
};

// OrderedRows with the rows in shared memory (slot s of thread t at
// c4[t + s * stride], c1[t + s * stride]), for kernels whose other state
// leaves no registers for them.
struct OrderedRowsSmem {
    static constexpr bool kOrdered = true;
    float4* rows;
    float4* c4;
    float* c1;
    int stride;
    float g0 = 0.f, g1 = 0.f, g2 = 0.f;

    __device__ __forceinline__ void set_pixel(float a0, float a1, float a2) { g0 = a0; g1 = a1; g2 = a2; }
    __device__ __forceinline__ void put(uint32_t v, const float4& q, float al) const {
        atomicAdd(rows + 2 * size_t(v), make_float4(q.x, q.y, q.z, 0.f));
        atomicAdd(rows + 2 * size_t(v) + 1, make_float4(g0 * q.w, g1 * q.w, g2 * q.w, al));
    }
    __device__ __forceinline__ void add_ordered(const uint32_t (&v)[3], uint32_t keep, uint32_t keep_next,
                                                const float4 (&gp)[3], const float (&s2)[3]) {
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            float4 q = gp[s];
            float al = s2[s];
            if ((keep >> s) & 1u) {
                const float4 o = c4[s * stride];
                q = make_float4(o.x + q.x, o.y + q.y, o.z + q.z, o.w + q.w);
                al += c1[s * stride];
            }
            if ((keep_next >> s) & 1u) {
                c4[s * stride] = q;
                c1[s * stride] = al;
            } else {
                put(v[s], q, al);
            }
        }
    }
    __device__ __forceinline__ void close(const uint32_t (&v)[3], uint32_t keep_next) const {
#pragma unroll
        for (int s = 0; s < 3; ++s)
            if ((keep_next >> s) & 1u) put(v[s], c4[s * stride], c1[s * stride]);
    }
    __device__ __forceinline__ void flush() {}
};

// Vertex gradients of one fragment from its depth adjoint gz, its colour
// adjoint gC w (gC = (g0, g1, g2), the pixel's) and its alpha adjoint ga,
// through the perspective-correct barycentrics and the projection.  With
// SCREEN the position part stops at the vertex's screen-space adjoints
// (d/dsx, d/dsy, d/d(1/ze)): the projection is linear in them with
// coefficients of the vertex alone, so it is applied once per vertex when the
// rows are scattered (screen_to_world) -- valid for one camera per row buffer
// and without absolute-value gradients.
template <class Acc, bool SCREEN = false>
__device__ __forceinline__ void frag_vertex_grads(const FragV& fr, float qx, float qy,
                                                  const VGeo* __restrict__ vgeo,
                                                  const float4* __restrict__ colors, const CamDev& cam,
                                                  float gz, float g0, float g1, float g2, float w, float ga,
                                                  bool use_abs, Acc& acc) {
    const float4 gcol = make_float4(g0 * w, g1 * w, g2 * w, ga);
    const uint32_t vi[3] = {fr.v0, fr.v1, fr.v2};
    VGeo P[3];
    float4 Cv[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        P[j] = vgeo[vi[j]];
        Cv[j] = colors[vi[j]];
    }
    FaceInterp fi;
    face_interp(P[0], P[1], P[2], qx, qy, fi);
    const float* dx = fi.dx;
    const float* dy = fi.dy;
    const float zb = fi.zb;
    float gb[3], sb = 0.f;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        gb[j] = gcol.x * Cv[j].x + gcol.y * Cv[j].y + gcol.z * Cv[j].z + gcol.w * Cv[j].w;
        sb += gb[j] * fi.bary[j];
    }
    const float gzz = fi.clamped ? 0.f : gz * zb * zb;
    float glam[3], giz[3], sl = 0.f;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const float gu = zb * (gb[j] - sb) - gzz;
        glam[j] = gu * P[j].iz;
        giz[j] = gu * fi.lam[j];
        sl += glam[j] * fi.lam[j];
    }
    const float invA = __fdividef(1.0f, fi.A);
    float gE[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) gE[j] = (glam[j] - sl) * invA;
    float gsx[3], gsy[3];
    gsx[0] = -gE[1] * dy[2] + gE[2] * dy[1];
    gsy[0] = gE[1] * dx[2] - gE[2] * dx[1];
    gsx[1] = gE[0] * dy[2] - gE[2] * dy[0];
    gsy[1] = -gE[0] * dx[2] + gE[2] * dx[0];
    gsx[2] = -gE[0] * dy[1] + gE[1] * dy[0];
    gsy[2] = gE[0] * dx[1] - gE[1] * dx[0];
    const float* V = cam.V;
    float4 gpv[3];
    float gav[3];
    if constexpr (SCREEN) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            gpv[j] = make_float4(gsx[j], gsy[j], giz[j], w * fi.bary[j]);
            gav[j] = ga * fi.bary[j];
        }
    } else {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float iz = P[j].iz;
            const float gxv = gsx[j] * cam.f * iz;
            const float gyv = -gsy[j] * cam.f * iz;
            const float giz_t = giz[j] + cam.f * (gsx[j] * P[j].xv - gsy[j] * P[j].yv);
            const float gzv = giz_t * iz * iz;
            float gp0 = V[0] * gxv + V[1] * gyv + V[2] * gzv;
            float gp1 = V[4] * gxv + V[5] * gyv + V[6] * gzv;
            float gp2 = V[8] * gxv + V[9] * gyv + V[10] * gzv;
            float s1 = w * fi.bary[j], s2 = ga * fi.bary[j];
            if (use_abs) {
                gp0 = fabsf(gp0); gp1 = fabsf(gp1); gp2 = fabsf(gp2);
                s1 = fabsf(s1);
                s2 = fabsf(s2);
            }
            gpv[j] = make_float4(gp0, gp1, gp2, s1);
            gav[j] = s2;
        }
    }
    if constexpr (!Acc::kOrdered) acc.add_face(vi, gpv, gav);  // ordered caches take carried fragments only
}

// Transmittance rebuilt back to front for the adjoint: T = tf e^X, with tf the
// pixel's final transmittance and X the optical depth between the current
// point and the ray's end (the sum of the sub-segment optical depths a t,
// a > 0, already walked).  A sum of non-negative terms keeps every small step
// (a ray of thousands of nearly transparent segments keeps its increments),
// and one exponential per segment replaces a compensated update.  `cur` is
// the current value, tf e^X.
struct TransBack {
    float tf, X, cur;
    __device__ __forceinline__ explicit TransBack(float t) : tf(t), X(0.f), cur(t) {}
    __device__ __forceinline__ void advance(float dX) {
        X += dX;
        cur = tf * __expf(X);
    }
};

// Adjoint of one segment of a pixel's ray between a front fragment (colour
// cf) and a back fragment (colour cb), the 4-sub-segment integral taken back
// to front.  T holds the transmittance after the segment and is advanced to
// the one before it (its optical depth grows by the segment's); gT is the
// running transmittance adjoint.
//
// The pixel's colour adjoint gC = dL/dC.rgb enters every colour term through
// dot products, so the sub-segment math runs on scalars: P0 = gC . c0 and
// D = gC . (c1 - c0) for sub-segment colours c0 -> c1 (P0 and D are linear in
// pf = gC . cf.rgb and pb = gC . cb.rgb), and the colour adjoint of each
// fragment is gC times a scalar weight.  With A = exp(-a t), 1 - A and
// K = (t + 1/a) A - 1/a (dtv_segment.cuh), C = (1 - A) c0 - K (c1 - c0):
//   gT_in  = (1 - A) P0 - K D + gT A
//   dL/dt  = a T_out (P0 + t D - gT)        dL/da = T_in (t A (P0 - gT) - dK/da D)
//   colour weights: front += T_in ((1 - s) (1 - A) + K/4), back += T_in (s (1 - A) - K/4)
// for a sub-segment starting at fraction s of the segment.  A sub-segment with
// a <= 0 is dropped by the forward; its gradient is the a -> 0+ limit
// (BackwardCommon.glsl:121-125) so a density clamped at zero can grow again.
// Outputs (added): g_tot = dL/d(segment length), the colour weights wf / wb and
// the alpha adjoints af / ab of the front / back fragment.
__device__ __forceinline__ void segment_adjoint(float tSeg, float cfw, float cbw, float pf, float pb, float atten,
                                                TransBack& T, TransF& gT, float& g_tot, float& wf, float& wb,
                                                float& af, float& ab) {
    const float dp = pb - pf, D = 0.25f * dp, dw = cbw - cfw;
    float av[kNumSubdivs];
#pragma unroll
    for (int s = 0; s < kNumSubdivs; ++s) av[s] = (cfw + dw * (0.25f * (s + 0.5f))) * atten;
    const bool short_tier = short_tier_of(av, tSeg);
    // One sub-segment, back to front; st is used only when a > 0.  (This
    // path runs when some sub-segment of the segment has x >= 1/8: T and gT
    // change by large steps there; T steps by 1 / A inside the segment and is
    // rebuilt from the optical depth at its end.)
    float Th = T.cur, Xseg = 0.f;
    auto step = [&](int s, const SegTerms& st, bool dense) {
        const float fs = 0.25f * s, fm = 0.25f * (s + 0.5f);
        const float P0 = pf + fs * dp;
        const float a = av[s];
        float g_a;
        if (dense) {
            const float iA = __fdividef(1.f, st.A);
            const float Tin = Th * iA;
            const float gTo = gT.hi;
            gT.hi = st.omA * P0 - st.K * D + gTo * st.A;
            gT.lo *= st.A;
            g_tot += 0.25f * (a * Th) * (P0 + tSeg * D - gTo);
            g_a = Tin * (tSeg * st.A * (P0 - gTo) - st.dK * D);
            Th = Tin;
            Xseg += a * tSeg;
            const float qK = 0.25f * st.K, tw = Tin * st.omA;
            wf += (1.f - fs) * tw + Tin * qK;
            wb += fs * tw - Tin * qK;
        } else {
            g_a = Th * (tSeg * (P0 - gT.hi) + 0.5f * tSeg * tSeg * D);
        }
        af += (1.f - fm) * g_a * atten;
        ab += fm * g_a * atten;
    };
    // Same tiers as segment_composite: straight-line terms when all four
    // sub-segments are in the short tier (seg_terms_adj's arithmetic there).
    // There every x = a t < 1/8: the optical depth grows by X = x0 + x1 + x2 +
    // x3, giving the transmittance in front of the segment, and each
    // sub-segment's entry transmittance follows front to back by the
    // forward's own FMA step.  The
    // transmittance adjoint gT (= gTo A + (1 - A) P0 - K D per sub-segment)
    // runs in FP32 from gT.hi inside the segment and its total change over the
    // segment is added to the float-float gT.  The constant factors (1/4 of
    // the length adjoint, the attenuation of the alpha adjoints) are applied
    // once per segment.
    if (short_tier) {
        // Two-wide: sub-segments (0, 1) and (2, 3) as pairs.
        const float2 av01 = make_float2(av[0], av[1]), av23 = make_float2(av[2], av[3]);
        const SegTerms2 s01 = seg_terms_short2<true>(tSeg, av01);
        const SegTerms2 s23 = seg_terms_short2<true>(tSeg, av23);
        const float Tout_seg = T.cur;
        T.advance((av[0] + av[1] + av[2] + av[3]) * tSeg);
        const float Tin0 = T.cur;
        const float Tin1 = __fmaf_rn(-Tin0, s01.omA.x, Tin0);
        const float Tin2 = __fmaf_rn(-Tin1, s01.omA.y, Tin1);
        const float Tin3 = __fmaf_rn(-Tin2, s23.omA.x, Tin2);
        const float2 Tin01 = make_float2(Tin0, Tin1), Tin23 = make_float2(Tin2, Tin3);
        const float2 Tout01 = make_float2(Tin1, Tin2), Tout23 = make_float2(Tin3, Tout_seg);
        // P0 = pf + fs dp and c = (1 - A) P0 - K D per sub-segment.
        const float2 P01 = fma2(make_float2(0.f, 0.25f), bc2(dp), bc2(pf));
        const float2 P23 = fma2(make_float2(0.5f, 0.75f), bc2(dp), bc2(pf));
        const float2 c01 = fma2(s01.K, bc2(-D), mul2(s01.omA, P01));
        const float2 c23 = fma2(s23.K, bc2(-D), mul2(s23.omA, P23));
        // Transmittance adjoint back to front: gTo (A - 1) + c per sub-segment.
        const float g3 = gT.hi;
        const float d3 = __fmaf_rn(-g3, s23.omA.y, c23.y);
        const float g2 = g3 + d3;
        const float d2 = __fmaf_rn(-g2, s23.omA.x, c23.x);
        const float g1 = g2 + d2;
        const float d1 = __fmaf_rn(-g1, s01.omA.y, c01.y);
        const float g0 = g1 + d1;
        const float d0 = __fmaf_rn(-g0, s01.omA.x, c01.x);
        const float2 gTo01 = make_float2(g0, g1), gTo23 = make_float2(g2, g3);
        // Length adjoint: sum a Tout (P0 + t D - gTo).
        const float tD = tSeg * D;
        const float2 gl2 = fma2(mul2(av23, Tout23), sub2(add2(P23, bc2(tD)), gTo23),
                                mul2(mul2(av01, Tout01), sub2(add2(P01, bc2(tD)), gTo01)));
        // Alpha adjoints: Tin (t A (P0 - gTo) - dK D), split front / back.
        const float2 ga01 = mul2(Tin01, fma2(s01.dK, bc2(-D), mul2(mul2(bc2(tSeg), s01.A), sub2(P01, gTo01))));
        const float2 ga23 = mul2(Tin23, fma2(s23.dK, bc2(-D), mul2(mul2(bc2(tSeg), s23.A), sub2(P23, gTo23))));
        const float2 gaf2 = fma2(make_float2(0.375f, 0.125f), ga23, mul2(make_float2(0.875f, 0.625f), ga01));
        const float2 gab2 = fma2(make_float2(0.625f, 0.875f), ga23, mul2(make_float2(0.125f, 0.375f), ga01));
        // Colour weights: front += sum((1 - fs) tw + Tin K / 4), back +=
        // sum(fs tw - Tin K / 4), from three sums.
        const float2 tw01 = mul2(Tin01, s01.omA), tw23 = mul2(Tin23, s23.omA);
        const float stw = hsum2(add2(tw01, tw23));
        const float sftw = hsum2(fma2(make_float2(0.5f, 0.75f), tw23, mul2(make_float2(0.f, 0.25f), tw01)));
        const float sk = hsum2(fma2(Tin23, s23.K, mul2(Tin01, s01.K)));
        trans_add(gT, ((d3 + d2) + d1) + d0);
        g_tot += 0.25f * hsum2(gl2);
        wf += (stw - sftw) + 0.25f * sk;
        wb += sftw - 0.25f * sk;
        af += hsum2(gaf2) * atten;
        ab += hsum2(gab2) * atten;
        return;
    }
#pragma unroll
    for (int s = kNumSubdivs - 1; s >= 0; --s) {
        if (av[s] > 0.f)
            step(s, seg_terms_adj(tSeg, av[s]), true);
        else
            step(s, SegTerms{}, false);
    }
    T.advance(Xseg);
}

__device__ __forceinline__ void segment_adjoint(float tSeg, const float4& cf, const float4& cb, float pf, float pb,
                                                float atten, TransBack& T, TransF& gT, float& g_tot, float& wf,
                                                float& wb, float& af, float& ab) {
    segment_adjoint(tSeg, cf.w, cb.w, pf, pb, atten, T, gT, g_tot, wf, wb, af, ab);
}

// Position gradients of one fragment from its depth adjoint alone (per-cell
// colours: the fragment carries no colour, so only the depth path of
// frag_vertex_grads remains).  One float4 atomic per vertex (position row).
__device__ __forceinline__ void frag_position_grads(const uint4& fc, float qx, float qy,
                                                    const VGeo* __restrict__ vgeo, const CamDev& cam, float gz,
                                                    bool use_abs, float4* __restrict__ rows) {
    const uint32_t vi[3] = {fc.x, fc.y, fc.z};
    VGeo P[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) P[j] = vgeo[vi[j]];
    FaceInterp fi;
    face_interp(P[0], P[1], P[2], qx, qy, fi);
    if (fi.clamped) return;  // the depth is clamped to a vertex depth: no dependence
    const float gzz = gz * fi.zb * fi.zb;
    float glam[3], giz[3], sl = 0.f;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        glam[j] = -gzz * P[j].iz;
        giz[j] = -gzz * fi.lam[j];
        sl += glam[j] * fi.lam[j];
    }
    const float invA = __fdividef(1.0f, fi.A);
    float gE[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) gE[j] = (glam[j] - sl) * invA;
    const float* dx = fi.dx;
    const float* dy = fi.dy;
    float gsx[3], gsy[3];
    gsx[0] = -gE[1] * dy[2] + gE[2] * dy[1];
    gsy[0] = gE[1] * dx[2] - gE[2] * dx[1];
    gsx[1] = gE[0] * dy[2] - gE[2] * dy[0];
    gsy[1] = -gE[0] * dx[2] + gE[2] * dx[0];
    gsx[2] = -gE[0] * dy[1] + gE[1] * dy[0];
    gsy[2] = gE[0] * dx[1] - gE[1] * dx[0];
    const float* V = cam.V;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const float iz = P[j].iz;
        const float gxv = gsx[j] * cam.f * iz;
        const float gyv = -gsy[j] * cam.f * iz;
        const float gzv = (giz[j] + cam.f * (gsx[j] * P[j].xv - gsy[j] * P[j].yv)) * iz * iz;
        float gp0 = V[0] * gxv + V[1] * gyv + V[2] * gzv;
        float gp1 = V[4] * gxv + V[5] * gyv + V[6] * gzv;
        float gp2 = V[8] * gxv + V[9] * gyv + V[10] * gzv;
        if (use_abs) {
            gp0 = fabsf(gp0);
            gp1 = fabsf(gp1);
            gp2 = fabsf(gp2);
        }
        atomicAdd(rows + 2 * size_t(vi[j]), make_float4(gp0, gp1, gp2, 0.f));
    }
}

// World-space position gradient of a vertex from its summed screen-space
// adjoints a = (d/dsx, d/dsy, d/d(1/ze)) (frag_vertex_grads with SCREEN).
__device__ __forceinline__ float3 screen_to_world(const float4& a, const VGeo& P, const CamDev& cam) {
    const float iz = P.iz;
    const float gxv = a.x * cam.f * iz;
    const float gyv = -a.y * cam.f * iz;
    const float gzv = (a.z + cam.f * (a.x * P.xv - a.y * P.yv)) * iz * iz;
    const float* V = cam.V;
    return make_float3(V[0] * gxv + V[1] * gyv + V[2] * gzv, V[4] * gxv + V[5] * gyv + V[6] * gzv,
                       V[8] * gxv + V[9] * gyv + V[10] * gzv);
}

// A fragment of the screen-space adjoint with what its vertex gradients need:
// the interpolation state of face_interp and its vertices' colours reduced by
// the pixel's colour adjoint gC.  A fragment's gradients are taken one step
// after it is loaded (its back segment and its front segment must both be
// done), so carrying this state spares the second gather of its three
// vertices and the second solve.  Its depth and alpha are those of
// load_frag_face (same expressions), so the adjoint walks the forward's
// transmittances; gC . colour is the barycentric sum of the reduced vertex
// colours.
struct FragG {
    uint32_t v[3];
    uint32_t bits;
    float z, alpha, pcol;            // depth, alpha, gC . colour.rgb
    float lam[3], iz[3], dx[3], dy[3];
    float invA, zb, zz;              // 1 / sum(E), 1 / sum(lam iz), zb^2 (0 when the depth is clamped)
    float pc[3], cw[3];              // gC . vertex colour rgb, vertex alpha
};

__device__ __forceinline__ FragG load_frag_g(uint32_t lo, uint32_t v0, uint32_t v1, uint32_t v2, uint32_t keep,
                                             float qx, float qy, const VGeo* __restrict__ vgeo,
                                             const float4* __restrict__ colors, float gC0, float gC1, float gC2) {
    FragG f;
    f.v[0] = v0;
    f.v[1] = v1;
    f.v[2] = v2;
    const VGeo a = vgeo[v0], b = vgeo[v1], c = vgeo[v2];
    FaceInterp fi;
    face_interp(a, b, c, qx, qy, fi);
    f.bits = (lo & 3u) | (keep << 2);
    const float4 c0 = colors[v0], c1 = colors[v1], c2 = colors[v2];
    const float* bary = fi.bary;
    f.z = fi.z;
    f.alpha = bary[0] * c0.w + bary[1] * c1.w + bary[2] * c2.w;
    f.iz[0] = a.iz;
    f.iz[1] = b.iz;
    f.iz[2] = c.iz;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        f.lam[j] = fi.lam[j];
        f.dx[j] = fi.dx[j];
        f.dy[j] = fi.dy[j];
    }
    f.invA = __fdividef(1.0f, fi.A);
    f.zb = fi.zb;
    f.zz = fi.clamped ? 0.f : fi.zb * fi.zb;
    f.pc[0] = gC0 * c0.x + gC1 * c0.y + gC2 * c0.z;
    f.pc[1] = gC0 * c1.x + gC1 * c1.y + gC2 * c1.z;
    f.pc[2] = gC0 * c2.x + gC1 * c2.y + gC2 * c2.z;
    f.pcol = bary[0] * f.pc[0] + bary[1] * f.pc[1] + bary[2] * f.pc[2];
    f.cw[0] = c0.w;
    f.cw[1] = c1.w;
    f.cw[2] = c2.w;
    return f;
}

__device__ __forceinline__ FragG load_frag_g(uint32_t lo, const uint4& fc, float qx, float qy,
                                             const VGeo* __restrict__ vgeo, const float4* __restrict__ colors,
                                             float gC0, float gC1, float gC2) {
    return load_frag_g(lo, fc.x, fc.y, fc.z, 0u, qx, qy, vgeo, colors, gC0, gC1, gC2);
}

// frag_vertex_grads with SCREEN from a carried fragment: depth adjoint gz,
// colour weight w (colour adjoint = gC w) and alpha adjoint ga.
template <class Acc>
__device__ __forceinline__ void frag_grads_carried(const FragG& f, float gz, float w, float ga, uint32_t keep_next,
                                                   Acc& acc) {
    float bary[3], gb[3], sb = 0.f;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        bary[j] = (f.lam[j] * f.iz[j]) * f.zb;
        gb[j] = w * f.pc[j] + ga * f.cw[j];
        sb += gb[j] * bary[j];
    }
    const float gzz = gz * f.zz;
    float glam[3], giz[3], sl = 0.f;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const float gu = f.zb * (gb[j] - sb) - gzz;
        glam[j] = gu * f.iz[j];
        giz[j] = gu * f.lam[j];
        sl += glam[j] * f.lam[j];
    }
    float gE[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) gE[j] = (glam[j] - sl) * f.invA;
    const float* dx = f.dx;
    const float* dy = f.dy;
    float4 gpv[3];
    float gav[3];
    gpv[0] = make_float4(-gE[1] * dy[2] + gE[2] * dy[1], gE[1] * dx[2] - gE[2] * dx[1], giz[0], w * bary[0]);
    gpv[1] = make_float4(gE[0] * dy[2] - gE[2] * dy[0], -gE[0] * dx[2] + gE[2] * dx[0], giz[1], w * bary[1]);
    gpv[2] = make_float4(-gE[0] * dy[1] + gE[1] * dy[0], gE[0] * dx[1] - gE[1] * dx[0], giz[2], w * bary[2]);
#pragma unroll
    for (int j = 0; j < 3; ++j) gav[j] = ga * bary[j];
    if constexpr (Acc::kOrdered)
        acc.add_ordered(f.v, f.bits >> 2, keep_next, gpv, gav);
    else
        acc.add_face(f.v, gpv, gav);
}

// adjoint_pixel for screen-space rows (no absolute gradients), on carried
// fragments.
template <class Acc>
__device__ __forceinline__ void adjoint_pixel_carried(
    int px, int py, const u64* __restrict__ offsets, const u64* __restrict__ records, const uint4* __restrict__ faces,
    const VGeo* __restrict__ vgeo, const float4* __restrict__ colors, int W, const ShadeDev& sh,
    const float4* __restrict__ dimage, const float* __restrict__ tfinal, const uint32_t* __restrict__ term,
    Acc& acc) {
    const size_t p = size_t(py) * W + px;
    const u64 beg = offsets[p];
    const uint32_t n = uint32_t(offsets[p + 1] - beg);
    if (n < 2) return;
    const float4 g = dimage[p];
    if (g.x == 0.f && g.y == 0.f && g.z == 0.f && g.w == 0.f) return;
    const float qx = float(px) + 0.5f, qy = float(py) + 0.5f;
    const float gC0 = g.x, gC1 = g.y, gC2 = g.z;
    TransF gT{g.x * sh.clear[0] + g.y * sh.clear[1] + g.z * sh.clear[2] + g.w * (sh.clear[3] - 1.f), 0.f};
    TransBack T(tfinal[p]);
    const int last = sh.use_ert ? int(term[p]) - 1 : int(n) - 1;
    if (last < 1) return;
    const float atten = sh.atten;
    acc.set_pixel(gC0, gC1, gC2);
    // Dependent loads record -> face -> vertex rows software-pipelined as in
    // adjoint_pixel.
    const uint32_t lo_b = record_lo(records, beg + last);
    FragG fb = load_frag_g(lo_b, faces[lo_b >> 2], qx, qy, vgeo, colors, gC0, gC1, gC2);
    uint32_t lo_f = record_lo(records, beg + last - 1);
    uint4 fc_f = faces[lo_f >> 2];
    uint32_t lo_n = last >= 2 ? record_lo(records, beg + last - 2) : 0u;
    float gz_b = 0.f, wb = 0.f, ab = 0.f;
    for (int i = last; i >= 1; --i) {
        FragG ff;
        if constexpr (Acc::kOrdered) {
            uint32_t pv[3];
            const uint32_t keep = order_like(fb.v, fc_f.x, fc_f.y, fc_f.z, pv);
            ff = load_frag_g(lo_f, pv[0], pv[1], pv[2], keep, qx, qy, vgeo, colors, gC0, gC1, gC2);
        } else {
            ff = load_frag_g(lo_f, fc_f, qx, qy, vgeo, colors, gC0, gC1, gC2);
        }
        if (i >= 2) {
            fc_f = faces[lo_n >> 2];
            lo_f = lo_n;
            if (i >= 3) lo_n = record_lo(records, beg + i - 3);
        }
        float gz_f = 0.f, wf = 0.f, af = 0.f;
        if (!skip_pair(ff.bits, fb.bits)) {
            float g_tot = 0.f;
            segment_adjoint((fb.z - ff.z) * 0.25f, ff.alpha, fb.alpha, ff.pcol, fb.pcol, atten, T, gT, g_tot, wf,
                            wb, af, ab);
            gz_f -= g_tot;
            gz_b += g_tot;
        }
        frag_grads_carried(fb, gz_b, wb, ab, ff.bits >> 2, acc);
        fb = ff;
        gz_b = gz_f;
        wb = wf;
        ab = af;
    }
    frag_grads_carried(fb, gz_b, wb, ab, 0u, acc);
    acc.flush();
}

template <class Acc, bool SCREEN = false>
__device__ __forceinline__ void adjoint_pixel(
    int px, int py, const u64* __restrict__ offsets, const u64* __restrict__ records, const uint4* __restrict__ faces,
    const VGeo* __restrict__ vgeo, const float4* __restrict__ colors, int W, const CamDev& cam, const ShadeDev& sh,
    const float4* __restrict__ dimage, const float* __restrict__ tfinal, const uint32_t* __restrict__ term,
    Acc& acc) {
    if constexpr (SCREEN) {
        adjoint_pixel_carried(px, py, offsets, records, faces, vgeo, colors, W, sh, dimage, tfinal, term, acc);
        return;
    }
    const size_t p = size_t(py) * W + px;
    const u64 beg = offsets[p];
    const uint32_t n = uint32_t(offsets[p + 1] - beg);
    if (n < 2) return;
    const float4 g = dimage[p];
    if (g.x == 0.f && g.y == 0.f && g.z == 0.f && g.w == 0.f) return;
    const float qx = float(px) + 0.5f, qy = float(py) + 0.5f;
    const float gC0 = g.x, gC1 = g.y, gC2 = g.z;
    TransF gT{g.x * sh.clear[0] + g.y * sh.clear[1] + g.z * sh.clear[2] + g.w * (sh.clear[3] - 1.f), 0.f};
    TransBack T(tfinal[p]);
    const int last = sh.use_ert ? int(term[p]) - 1 : int(n) - 1;
    if (last < 1) return;
    const float atten = sh.atten;
    const bool use_abs = sh.use_abs_grad != 0;
    if (use_abs)
        acc.set_pixel(fabsf(gC0), fabsf(gC1), fabsf(gC2));
    else
        acc.set_pixel(gC0, gC1, gC2);
    // The dependent loads record -> face -> vertex rows are software-pipelined:
    // while fragment i's segment is processed, the face of fragment i-2 and the
    // record of fragment i-3 are already in flight.
    FragV fb = load_frag(records[beg + last], qx, qy, faces, vgeo, colors);
    uint32_t lo_f = record_lo(records, beg + last - 1);
    uint4 fc_f = faces[lo_f >> 2];
    uint32_t lo_n = last >= 2 ? record_lo(records, beg + last - 2) : 0u;
    // Per fragment: depth adjoint, colour weight (colour adjoint = gC x weight)
    // and alpha adjoint, of the back fragment (b) and the front one (f).
    float pb = gC0 * fb.col.x + gC1 * fb.col.y + gC2 * fb.col.z;
    float gz_b = 0.f, wb = 0.f, ab = 0.f;
    for (int i = last; i >= 1; --i) {
        const FragV ff = load_frag_face(lo_f, fc_f, qx, qy, vgeo, colors);
        if (i >= 2) {
            fc_f = faces[lo_n >> 2];
            lo_f = lo_n;
            if (i >= 3) lo_n = record_lo(records, beg + i - 3);
        }
        const float pf = gC0 * ff.col.x + gC1 * ff.col.y + gC2 * ff.col.z;
        float gz_f = 0.f, wf = 0.f, af = 0.f;
        if (!skip_pair(ff.bits, fb.bits)) {
            float g_tot = 0.f;
            segment_adjoint((fb.z - ff.z) * 0.25f, ff.col, fb.col, pf, pb, atten, T, gT, g_tot, wf, wb, af, ab);
            gz_f -= g_tot;
            gz_b += g_tot;
        }
        frag_vertex_grads<Acc, SCREEN>(fb, qx, qy, vgeo, colors, cam, gz_b, gC0, gC1, gC2, wb, ab, use_abs, acc);
        fb = ff;
        pb = pf;
        gz_b = gz_f;
        wb = wf;
        ab = af;
    }
    frag_vertex_grads<Acc, SCREEN>(fb, qx, qy, vgeo, colors, cam, gz_b, gC0, gC1, gC2, wb, ab, use_abs, acc);
    acc.flush();
}


}  // namespace dtv
