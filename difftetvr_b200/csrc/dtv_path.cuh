// Per-face and per-pixel bodies of the hot path, shared by the single-view
// kernels (dtv_kernels.cu) and the batched multi-view kernels (dtv_batch.cu).
#pragma once
#include "dtv_device.cuh"
#include "dtv_segment.cuh"

namespace dtv {

using u64 = unsigned long long;
constexpr int kTile = 16;  // composite / adjoint pixel tile (16 x 16 threads)

// ---------------------------------------------------------------------------
// (a)+(b) face rasterisation.  One thread per face walks the pixel centres of
// the face's bounding box with incrementally updated integer edge functions in
// 1/256-pixel fixed point.  COUNT mode increments the per-pixel counter; FILL
// mode writes the record at offsets[p] + (--counts[p]), leaving counts zeroed
// for the next render.  Only pixel rows [row0, row1) are visited (row bands of
// a render whose lists do not fit the fragment budget at once).
//
// Edge functions are translation invariant, so they are evaluated relative to
// the bounding-box corner: for boxes under 64 px (2^14 fixed-point units) on
// each side every product is below 2^29 and the exact values fit in 32-bit
// integers (half the ALU work of the 64-bit form); larger faces use 64 bits.
// Both give identical coverage.
template <typename I>
__device__ __forceinline__ bool edge_in(I E, I dx, I dy) {
    return (E > 0) || (E == 0 && ((dy < 0) || (dy == 0 && dx > 0)));
}

template <bool FILL, typename I>
__device__ __forceinline__ void raster_box(const uint4& fc, uint32_t bits, I ax0, I ay0, I ax1, I ay1, I ax2, I ay2,
                                           I Xs, I Ys, int px0, int px1, int py0, int py1,
                                           const float4* __restrict__ vproj, int W, uint32_t* __restrict__ counts,
                                           const u64* __restrict__ offsets, u64* __restrict__ records) {
    // Edges e0: a1->a2, e1: a2->a0, e2: a0->a1; (Xs, Ys) is the centre of
    // pixel (px0, py0) in the same (possibly box-relative) coordinates.
    const I dx0 = ax2 - ax1, dy0 = ay2 - ay1;
    const I dx1 = ax0 - ax2, dy1 = ay0 - ay2;
    const I dx2 = ax1 - ax0, dy2 = ay1 - ay0;
    I E0r = dx0 * (Ys - ay1) - dy0 * (Xs - ax1);
    I E1r = dx1 * (Ys - ay2) - dy1 * (Xs - ax2);
    I E2r = dx2 * (Ys - ay0) - dy2 * (Xs - ax0);
    float4 va, vb, vc;
    if (FILL) {
        va = vproj[fc.x];
        vb = vproj[fc.y];
        vc = vproj[fc.z];
    }
    // Four pixels of a row per step: their coverage tests, depth keys, counter
    // atomics and offset loads are independent and issue back to back before
    // the record stores (the fill is bound by atomic round trips otherwise).
    const I sx0 = -dy0 * I(256), sx1 = -dy1 * I(256), sx2 = -dy2 * I(256);
    for (int py = py0; py <= py1; ++py) {
        I E0 = E0r, E1 = E1r, E2 = E2r;
        const size_t row = size_t(py) * W;
        for (int px = px0; px <= px1; px += 4) {
            bool in[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                in[k] = (px + k <= px1) && edge_in<I>(E0 + I(k) * sx0, dx0, dy0) &&
                        edge_in<I>(E1 + I(k) * sx1, dx1, dy1) && edge_in<I>(E2 + I(k) * sx2, dx2, dy2);
            if (FILL) {
                uint32_t slot[4];
                u64 off[4];
                float z[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (in[k]) {
                        const size_t p = row + px + k;
                        off[k] = offsets[p];
                        slot[k] = atomicSub(&counts[p], 1u);
                        z[k] = depth_key(va, vb, vc, float(px + k) + 0.5f, float(py) + 0.5f);
                    }
                }
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (in[k]) records[off[k] + slot[k] - 1u] = (u64(__float_as_uint(z[k])) << 32) | bits;
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (in[k]) atomicAdd(&counts[row + px + k], 1u);
            }
            E0 += I(4) * sx0;
            E1 += I(4) * sx1;
            E2 += I(4) * sx2;
        }
        E0r += dx0 * I(256);
        E1r += dx1 * I(256);
        E2r += dx2 * I(256);
    }
}

template <bool FILL>
__device__ __forceinline__ void raster_face(uint32_t f, const uint4* __restrict__ faces,
                                            const float4* __restrict__ vproj, const int2* __restrict__ vfix,
                                            int W, int row0, int row1, uint32_t* __restrict__ counts,
                                            const u64* __restrict__ offsets, u64* __restrict__ records) {
    const uint4 fc = faces[f];
    const int2 q0 = vfix[fc.x], q1 = vfix[fc.y], q2 = vfix[fc.z];
    if (q0.x == kInvalidFix || q1.x == kInvalidFix || q2.x == kInvalidFix) return;
    const long long X0 = q0.x, Y0 = q0.y, X1 = q1.x, Y1 = q1.y, X2 = q2.x, Y2 = q2.y;
    const long long area2 = (X1 - X0) * (Y2 - Y0) - (Y1 - Y0) * (X2 - X0);
    if (area2 == 0) return;
    const uint32_t front = area2 < 0 ? 1u : 0u;
    const uint32_t bits = (f << 2) | ((fc.w & 1u) << 1) | front;
    long long ax1 = X1, ay1 = Y1, ax2 = X2, ay2 = Y2;
    if (area2 < 0) {
        ax1 = X2; ay1 = Y2;
        ax2 = X1; ay2 = Y1;
    }
    const long long minX = min(X0, min(X1, X2)), maxX = max(X0, max(X1, X2));
    const long long minY = min(Y0, min(Y1, Y2)), maxY = max(Y0, max(Y1, Y2));
    const int px0 = int(max(0LL, ceil_div256(minX - 128)));
    const int px1 = int(min((long long)W - 1, floor_div256(maxX - 128)));
    const int py0 = int(max((long long)row0, ceil_div256(minY - 128)));
    const int py1 = int(min((long long)row1 - 1, floor_div256(maxY - 128)));
    if (px0 > px1 || py0 > py1) return;
    const long long Xs = 256LL * px0 + 128, Ys = 256LL * py0 + 128;
    if (maxX - minX < (1LL << 14) && maxY - minY < (1LL << 14)) {
        raster_box<FILL, int>(fc, bits, int(X0 - minX), int(Y0 - minY), int(ax1 - minX), int(ay1 - minY),
                              int(ax2 - minX), int(ay2 - minY), int(Xs - minX), int(Ys - minY), px0, px1, py0, py1,
                              vproj, W, counts, offsets, records);
    } else {
        raster_box<FILL, long long>(fc, bits, X0, Y0, ax1, ay1, ax2, ay2, Xs, Ys, px0, px1, py0, py1, vproj, W,
                                    counts, offsets, records);
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

__device__ __forceinline__ FragV load_frag(u64 rec, float qx, float qy, const uint4* __restrict__ faces,
                                           const VGeo* __restrict__ vgeo, const float4* __restrict__ colors) {
    FragV fr;
    const uint32_t lo = uint32_t(rec);
    fr.face = lo >> 2;
    fr.bits = lo & 3u;
    const uint4 fc = faces[fr.face];
    fr.v0 = fc.x;
    fr.v1 = fc.y;
    fr.v2 = fc.z;
    const VGeo a = vgeo[fc.x], b = vgeo[fc.y], c = vgeo[fc.z];
    float bary[3];
    face_bary(a, b, c, qx, qy, bary, fr.z);  // depth and colour from the same weights
    const float4 c0 = colors[fc.x], c1 = colors[fc.y], c2 = colors[fc.z];
    fr.col = make_float4(bary[0] * c0.x + bary[1] * c1.x + bary[2] * c2.x,
                         bary[0] * c0.y + bary[1] * c1.y + bary[2] * c2.y,
                         bary[0] * c0.z + bary[1] * c1.z + bary[2] * c2.z,
                         bary[0] * c0.w + bary[1] * c1.w + bary[2] * c2.w);
    return fr;
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
    float C0 = 0.f, C1 = 0.f, C2 = 0.f, T = 1.f;
    uint32_t i = n;
    if (n >= 2) {
        FragV f1 = load_frag(records[beg], qx, qy, faces, vgeo, colors), f0;
        for (i = 1; i < n; ++i) {
            if (sh.use_ert && T < sh.ert_thresh) break;
            f0 = f1;
            f1 = load_frag(records[beg + i], qx, qy, faces, vgeo, colors);
            if (skip_pair(f0.bits, f1.bits)) continue;
            const float tSeg = (f1.z - f0.z) * 0.25f;
#pragma unroll
            for (int s = 0; s < kNumSubdivs; ++s) {
                const float fb = 0.25f * s, fm = 0.25f * (s + 0.5f), fe = 0.25f * (s + 1);
                const float4 c0 = lerp4(f0.col, f1.col, fb);
                const float4 c1 = lerp4(f0.col, f1.col, fe);
                const float a = (f0.col.w + (f1.col.w - f0.col.w) * fm) * sh.atten;
                if (!(a > 0.f)) continue;  // a <= 0 contributes nothing
                const SegTerms st = seg_terms(tSeg, a);
                C0 += T * (st.omA * c0.x + st.K * (c0.x - c1.x));
                C1 += T * (st.omA * c0.y + st.K * (c0.y - c1.y));
                C2 += T * (st.omA * c0.z + st.K * (c0.z - c1.z));
                T *= st.A;
            }
        }
    }
    image[p] = make_float4(C0 + T * sh.clear[0], C1 + T * sh.clear[1], C2 + T * sh.clear[2],
                           (1.f - T) + T * sh.clear[3]);
    tfinal[p] = T;
    term[p] = i;
}

// ---------------------------------------------------------------------------
// (f) adjoint.  Back to front from the termination index; transmittance is
// rebuilt from the final value (T_in = T_out / A); per fragment the depth and
// colour adjoints of its two segments are summed and pushed through the
// screen-space barycentrics and the projection to the face's three vertices.
// Vertex gradient accumulation: the 7 values of a vertex (position xyz, pad,
// colour rgba) share one 32-byte row of an interleaved buffer and are added
// with two float4 vector atomics, so each vertex update touches one L2 sector
// (scalar atomics into the [V,3] / [V,4] layout touch about three).
struct GradAcc {
    float4* rows;   // [V][2]

    __device__ __forceinline__ void add(uint32_t v, float gp0, float gp1, float gp2, float4 gc) const {
        atomicAdd(rows + 2 * size_t(v), make_float4(gp0, gp1, gp2, 0.f));
        atomicAdd(rows + 2 * size_t(v) + 1, gc);
    }
};

__device__ __forceinline__ void frag_vertex_grads(const FragV& fr, float qx, float qy,
                                                  const VGeo* __restrict__ vgeo,
                                                  const float4* __restrict__ colors, const CamDev& cam,
                                                  float gz, float4 gcol, bool use_abs, const GradAcc& acc) {
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
        float4 gc = f4scale(gcol, fi.bary[j]);
        if (use_abs) {
            gp0 = fabsf(gp0); gp1 = fabsf(gp1); gp2 = fabsf(gp2);
            gc = make_float4(fabsf(gc.x), fabsf(gc.y), fabsf(gc.z), fabsf(gc.w));
        }
        acc.add(vi[j], gp0, gp1, gp2, gc);
    }
}

// Adjoint of one sub-segment (colour c0 -> c1, density a, length tSeg) of
// the 4-sub-segment integral.  T holds the transmittance after the segment and
// is rebuilt in place to the one before it (T_in = T_out / A); gT is the
// running transmittance adjoint.  Outputs: dL/dtSeg, dL/da and the colour
// adjoints of both sub-segment ends.
__device__ __forceinline__ void sub_segment_adjoint(float tSeg, float a, float4 c0, float4 c1, float gC0, float gC1,
                                                    float gC2, float& T, float& gT, float& g_t, float& g_a,
                                                    float& gc0x, float& gc0y, float& gc0z, float& gc1x, float& gc1y,
                                                    float& gc1z) {
    if (a > 0.f) {
        const SegTerms st = seg_terms_adj(tSeg, a);
        const float cx = st.omA * c0.x + st.K * (c0.x - c1.x);
        const float cy = st.omA * c0.y + st.K * (c0.y - c1.y);
        const float cz = st.omA * c0.z + st.K * (c0.z - c1.z);
        const float Tin = __fdividef(T, st.A);
        const float gax = Tin * gC0, gay = Tin * gC1, gaz = Tin * gC2;
        const float gA = Tin * gT;
        gT = (gC0 * cx + gC1 * cy + gC2 * cz) + gT * st.A;
        T = Tin;
        const float aA = a * st.A;
        g_t = gax * (aA * (c0.x + tSeg * (c1.x - c0.x))) + gay * (aA * (c0.y + tSeg * (c1.y - c0.y))) +
              gaz * (aA * (c0.z + tSeg * (c1.z - c0.z))) - gA * aA;
        const float dK = st.dK;
        const float tA = tSeg * st.A;
        g_a = gax * (tA * c0.x + dK * (c0.x - c1.x)) + gay * (tA * c0.y + dK * (c0.y - c1.y)) +
              gaz * (tA * c0.z + dK * (c0.z - c1.z)) - gA * tA;
        const float k0 = st.omA + st.K;
        gc0x = k0 * gax; gc0y = k0 * gay; gc0z = k0 * gaz;
        gc1x = -st.K * gax; gc1y = -st.K * gay; gc1z = -st.K * gaz;
    } else {
        // The forward drops the sub-segment for a <= 0; the gradient is the
        // a -> 0+ limit (BackwardCommon.glsl:121-125) so a density clamped at
        // zero can grow again.
        const float gax = T * gC0, gay = T * gC1, gaz = T * gC2, gA = T * gT;
        g_t = 0.f;
        g_a = gax * (tSeg * c0.x + 0.5f * tSeg * tSeg * (c1.x - c0.x)) +
              gay * (tSeg * c0.y + 0.5f * tSeg * tSeg * (c1.y - c0.y)) +
              gaz * (tSeg * c0.z + 0.5f * tSeg * tSeg * (c1.z - c0.z)) - gA * tSeg;
        gc0x = gc0y = gc0z = gc1x = gc1y = gc1z = 0.f;
    }
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

__device__ __forceinline__ void adjoint_pixel(
    int px, int py, const u64* __restrict__ offsets, const u64* __restrict__ records, const uint4* __restrict__ faces,
    const VGeo* __restrict__ vgeo, const float4* __restrict__ colors, int W, const CamDev& cam, const ShadeDev& sh,
    const float4* __restrict__ dimage, const float* __restrict__ tfinal, const uint32_t* __restrict__ term,
    const GradAcc& acc) {
    const size_t p = size_t(py) * W + px;
    const u64 beg = offsets[p];
    const uint32_t n = uint32_t(offsets[p + 1] - beg);
    if (n < 2) return;
    const float4 g = dimage[p];
    if (g.x == 0.f && g.y == 0.f && g.z == 0.f && g.w == 0.f) return;
    const float qx = float(px) + 0.5f, qy = float(py) + 0.5f;
    const float gC0 = g.x, gC1 = g.y, gC2 = g.z;
    float gT = g.x * sh.clear[0] + g.y * sh.clear[1] + g.z * sh.clear[2] + g.w * (sh.clear[3] - 1.f);
    float T = tfinal[p];
    const int last = sh.use_ert ? int(term[p]) - 1 : int(n) - 1;
    if (last < 1) return;
    const float atten = sh.atten;
    const bool use_abs = sh.use_abs_grad != 0;
    FragV fb = load_frag(records[beg + last], qx, qy, faces, vgeo, colors);
    float gz_b = 0.f;
    float4 gcol_b = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = last; i >= 1; --i) {
        const FragV ff = load_frag(records[beg + i - 1], qx, qy, faces, vgeo, colors);
        float gz_f = 0.f;
        float4 gcol_f = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!skip_pair(ff.bits, fb.bits)) {
            const float tSeg = (fb.z - ff.z) * 0.25f;
            float g_tot = 0.f;
#pragma unroll
            for (int s = kNumSubdivs - 1; s >= 0; --s) {
                const float fbg = 0.25f * s, fm = 0.25f * (s + 0.5f), fe = 0.25f * (s + 1);
                const float4 c0 = lerp4(ff.col, fb.col, fbg);
                const float4 c1 = lerp4(ff.col, fb.col, fe);
                const float a = (ff.col.w + (fb.col.w - ff.col.w) * fm) * atten;
                float g_t, g_a, gc0x, gc0y, gc0z, gc1x, gc1y, gc1z;
                sub_segment_adjoint(tSeg, a, c0, c1, gC0, gC1, gC2, T, gT, g_t, g_a, gc0x, gc0y, gc0z, gc1x, gc1y,
                                    gc1z);
                g_tot += 0.25f * g_t;
                gcol_f.x += (1.f - fbg) * gc0x + (1.f - fe) * gc1x;
                gcol_f.y += (1.f - fbg) * gc0y + (1.f - fe) * gc1y;
                gcol_f.z += (1.f - fbg) * gc0z + (1.f - fe) * gc1z;
                gcol_b.x += fbg * gc0x + fe * gc1x;
                gcol_b.y += fbg * gc0y + fe * gc1y;
                gcol_b.z += fbg * gc0z + fe * gc1z;
                gcol_f.w += (1.f - fm) * g_a * atten;
                gcol_b.w += fm * g_a * atten;
            }
            gz_f -= g_tot;
            gz_b += g_tot;
        }
        frag_vertex_grads(fb, qx, qy, vgeo, colors, cam, gz_b, gcol_b, use_abs, acc);
        fb = ff;
        gz_b = gz_f;
        gcol_b = gcol_f;
    }
    frag_vertex_grads(fb, qx, qy, vgeo, colors, cam, gz_b, gcol_b, use_abs, acc);
}


}  // namespace dtv
