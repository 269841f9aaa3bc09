// Ray-tet path (the reference's intersection renderer) by traversal through
// face adjacency.
//
// Reference: TetMeshRendererIntersection::render (TetMeshRendererIntersection.cpp:
// 603-707) draws the camera-facing faces of every tet, sorted by depth, and
// intersects each pixel ray with the whole tet (IntersectRasterization.glsl:
// 139-273, intersectRayTet in RayIntersectionTests.glsl:77-106): one segment
// per (pixel, tet), Euclidean length along the normalised ray, the 4-sub-segment
// integral; its adjoint (AdjointIntersectRasterization.glsl:111-362) runs
// front to back under pixel interlock.
//
// Here each pixel thread finds the tets its ray crosses by walking the mesh:
// intervals start at the pixel's front-facing boundary fragments (a small
// count / scan / fill / sort over the boundary faces only); from a tet entered
// through face fe the ray leaves through the back face that covers the pixel
// under the rasteriser's exact fixed-point rule, and continues into the tet on
// the other side of that face until it leaves through a boundary face.  No
// per-fragment storage exists beyond the boundary lists; the adjoint walks the
// same tets backwards (previous tet = the one across the entry face), so the
// backward pass needs no stored lists either.  Walks are bounded by the tet
// count (a malformed mesh cannot loop forever).
#include "dtv_internal.h"
#include "dtv_path.cuh"

namespace dtv {

constexpr uint32_t kNoTet = 0xffffffffu;

// Exact coverage of the pixel centre by a triangle (the rasteriser's rule),
// vertices relative to the pixel centre, `swap`: the given order winds
// clockwise.  With every vertex within 2^14 fixed-point units (64 px) of the
// centre the edge functions are exact in 32-bit integers, otherwise in 64
// bits; both give the raster's coverage.  No early exits, so a warp's lanes
// stay together.
template <typename I>
__device__ __forceinline__ bool covers_rel(I r0x, I r0y, I r1x, I r1y, I r2x, I r2y, bool swap) {
    // Vertices relative to the pixel centre; the orientation-normalised order
    // is (0, 1, 2), or (0, 2, 1) when the stored winding is clockwise.
    const I a1x = swap ? r2x : r1x, a1y = swap ? r2y : r1y;
    const I a2x = swap ? r1x : r2x, a2y = swap ? r1y : r2y;
    const I dx0 = a2x - a1x, dy0 = a2y - a1y;
    const I dx1 = r0x - a2x, dy1 = r0y - a2y;
    const I dx2 = a1x - r0x, dy2 = a1y - r0y;
    // E = dx (Yc - ay) - dy (Xc - ax) with the pixel centre at the origin.
    const I E0 = dy0 * a1x - dx0 * a1y;
    const I E1 = dy1 * a2x - dx1 * a2y;
    const I E2 = dy2 * r0x - dx2 * r0y;
    return edge_in<I>(E0, dx0, dy0) & edge_in<I>(E1, dx1, dy1) & edge_in<I>(E2, dx2, dy2);
}

// Per-tet topology for the walk: the unique face ids of a tet's four faces
// (face j = local vertices kTetFaceTable[j] = {0,1,2}, {1,0,3}, {0,2,3},
// {2,1,3}), its vertex ids, and per face the bit that turns the on-screen
// winding of the tet's own vertex order into "faces the camera as seen from
// this tet" (the mesh builder's tet_flip; 0 for consistently oriented meshes).
struct TetTopo {
    const uint4* tet_faces;
    const uint4* cells;
    const uint8_t* flip;
};

// Face of tet t (not `skip`) covering the pixel that faces the camera
// (want_front) or away from it with respect to t's outward normal; the first
// such face in the tet's face order.  All four faces are evaluated from the
// tet's four projected vertices (4 vertex loads instead of 12, and no face or
// face->tet loads); coverage is the rasteriser's rule (covers_rel normalises
// the winding, and the normalised triangle's directed edges do not depend on
// the starting vertex).
// A tet's row of the walk tables (loaded ahead of its face search by the
// walks, so that the loads overlap the previous segment's work).
struct TetRow {
    uint4 tf;       // face ids
    uint4 cv;       // vertex ids
    uint32_t flip;  // face-side bits
};

__device__ __forceinline__ TetRow load_tet(const TetTopo& tt, uint32_t t) {
    return TetRow{tt.tet_faces[t], tt.cells[t], uint32_t(tt.flip[t])};
}

__device__ __forceinline__ uint32_t tet_face_of(const TetRow& tr, const int2* __restrict__ vfix, uint32_t skip,
                                                bool want_front, int px, int py) {
    const uint4 tf = tr.tf;
    const uint4 cv = tr.cv;
    const uint32_t flip = tr.flip;
    const uint32_t fs[4] = {tf.x, tf.y, tf.z, tf.w};
    const int2 q[4] = {vfix[cv.x], vfix[cv.y], vfix[cv.z], vfix[cv.w]};
    uint32_t found = kNoTet;
    // All four vertices projected and within 2^14 units of the centre (nearly
    // every step): 32-bit integers are exact.  The tet's four faces share its
    // six edges, so six edge functions K_uv = r_u x r_v (vertex positions
    // relative to the pixel centre, u < v) and their tie-rule bits decide all
    // four faces: a face's doubled area is the sum of its three directed
    // edges' functions, the reversed edge of a non-degenerate edge owns the
    // centre exactly when the edge does not, and a face with a degenerate
    // edge has zero area and is skipped.  Same values and decisions as
    // covers_rel on each face.
    const bool projected = (q[0].x != kInvalidFix) & (q[1].x != kInvalidFix) & (q[2].x != kInvalidFix) &
                           (q[3].x != kInvalidFix) & (px < (1 << 22)) & (py < (1 << 22));
    if (projected) {
        const int Xc = 256 * px + 128, Yc = 256 * py + 128;
        int ix[4], iy[4], mm = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            ix[k] = q[k].x - Xc;
            iy[k] = q[k].y - Yc;
            mm = max(mm, max(abs(ix[k]), abs(iy[k])));
        }
        if (mm < (1 << 14)) {
            const int K01 = ix[0] * iy[1] - iy[0] * ix[1], K02 = ix[0] * iy[2] - iy[0] * ix[2];
            const int K03 = ix[0] * iy[3] - iy[0] * ix[3], K12 = ix[1] * iy[2] - iy[1] * ix[2];
            const int K13 = ix[1] * iy[3] - iy[1] * ix[3], K23 = ix[2] * iy[3] - iy[2] * ix[3];
            const bool f01 = edge_in<int>(K01, ix[1] - ix[0], iy[1] - iy[0]);
            const bool f02 = edge_in<int>(K02, ix[2] - ix[0], iy[2] - iy[0]);
            const bool f03 = edge_in<int>(K03, ix[3] - ix[0], iy[3] - iy[0]);
            const bool f12 = edge_in<int>(K12, ix[2] - ix[1], iy[2] - iy[1]);
            const bool f13 = edge_in<int>(K13, ix[3] - ix[1], iy[3] - iy[1]);
            const bool f23 = edge_in<int>(K23, ix[3] - ix[2], iy[3] - iy[2]);
            // Face j = (A, B, C): directed edges B->C, C->A, A->B.
            const int ar[4] = {K12 - K02 + K01, K03 - K13 - K01, K23 - K03 + K02, K13 - K23 - K12};
            const bool e0[4] = {f12, f03, f23, f13}, e1[4] = {!f02, !f13, !f03, !f23}, e2[4] = {f01, !f01, f02, !f12};
#pragma unroll
            for (int j = 3; j >= 0; --j) {
                const bool sw = ar[j] < 0;  // clockwise: every directed edge reversed
                const bool in = sw ? !(e0[j] | e1[j] | e2[j]) : (e0[j] & e1[j] & e2[j]);
                const bool front = sw != (((flip >> j) & 1u) != 0u);
                const bool match = fs[j] != skip && ar[j] != 0 && in && front == want_front;
                found = match ? fs[j] : found;  // descending j: the smallest matching j wins
            }
            return found;
        }
    }
    const long long Xc = 256LL * px + 128, Yc = 256LL * py + 128;
    long long rx[4], ry[4];
    bool ok[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        ok[k] = q[k].x != kInvalidFix;
        rx[k] = (long long)q[k].x - Xc;
        ry[k] = (long long)q[k].y - Yc;
    }
    constexpr int A[4] = {0, 1, 0, 2}, B[4] = {1, 0, 2, 1}, C[4] = {2, 3, 3, 3};
#pragma unroll
    for (int j = 3; j >= 0; --j) {
        const int a = A[j], b = B[j], c = C[j];
        const long long area2 = (rx[b] - rx[a]) * (ry[c] - ry[a]) - (ry[b] - ry[a]) * (rx[c] - rx[a]);
        const long long m = max(max(max(llabs(rx[a]), llabs(ry[a])), max(llabs(rx[b]), llabs(ry[b]))),
                                max(llabs(rx[c]), llabs(ry[c])));
        bool in;
        if (m < (1LL << 14))
            in = covers_rel<int>(int(rx[a]), int(ry[a]), int(rx[b]), int(ry[b]), int(rx[c]), int(ry[c]), area2 < 0);
        else
            in = covers_rel<long long>(rx[a], ry[a], rx[b], ry[b], rx[c], ry[c], area2 < 0);
        const bool front = (area2 < 0) != (((flip >> j) & 1u) != 0u);
        const bool match = fs[j] != skip && ok[a] && ok[b] && ok[c] && area2 != 0 && in && front == want_front;
        found = match ? fs[j] : found;  // descending j: the smallest matching j wins
    }
    return found;
}

__device__ __forceinline__ uint32_t tet_face_at(const TetTopo& tt, const int2* __restrict__ vfix, uint32_t t,
                                                uint32_t skip, bool want_front, int px, int py) {
    return tet_face_of(load_tet(tt, t), vfix, skip, want_front, px, py);
}

__device__ __forceinline__ uint32_t other_tet(const uint32_t* __restrict__ f2t, uint32_t f, uint32_t t) {
    const uint32_t a = f2t[2 * size_t(f)], b = f2t[2 * size_t(f) + 1];
    return a == t ? b : a;
}

// Length of the pixel ray per unit of view depth (|d| with d.z_view = -1).
__device__ __forceinline__ float ray_scale(const CamDev& cam, float qx, float qy) {
    const float dx = (qx - cam.cx) / cam.f, dy = (qy - cam.cy) / cam.f;
    return sqrtf(1.f + dx * dx + dy * dy);
}

// The forward walk in 16 x 8 pixel blocks, five per SM (96 registers): the
// walk is bound by the latency of its tet -> faces -> vertices chain, and 20
// warps per SM hide more of it than 16 at 110 registers (3.59 -> 3.22 ms at
// 64^3 / 1024^2).
constexpr int kWalkRows = 8;
constexpr int kWalkThreads = kTile * kWalkRows;
__global__ void __launch_bounds__(kWalkThreads, 5) k_walk_composite(
    const u64* __restrict__ b_offsets, const u64* __restrict__ b_records, const uint32_t* __restrict__ bf_global,
    const uint4* __restrict__ faces, const uint32_t* __restrict__ f2t, TetTopo tt, uint32_t num_tets, const int2* __restrict__ vfix, const VGeo* __restrict__ vgeo,
    const float4* __restrict__ colors, CamDev cam, ShadeDev sh, float4* __restrict__ image,
    float* __restrict__ tfinal, uint4* __restrict__ wstate) {
    const int px = blockIdx.x * kTile + (threadIdx.x % kTile);
    const int py = blockIdx.y * kWalkRows + (threadIdx.x / kTile);
    if (px >= cam.W || py >= cam.H) return;
    const size_t p = size_t(py) * cam.W + px;
    const u64 beg = b_offsets[p];
    const uint32_t nb = uint32_t(b_offsets[p + 1] - beg);
    const float qx = float(px) + 0.5f, qy = float(py) + 0.5f;
    const float scale = ray_scale(cam, qx, qy);
    float C0 = 0.f, C1 = 0.f, C2 = 0.f;
    TransF T{1.f, 0.f};
    uint32_t last_tet = kNoTet, last_entry = kNoTet, last_b = 0, nseg = 0;
    bool stop = false;
    for (uint32_t b = 0; b < nb && !stop; ++b) {
        const uint32_t bits = uint32_t(b_records[beg + b]);
        if (!(bits & 1u)) continue;  // intervals start at front-facing boundary faces
        uint32_t fe = bf_global[bits >> 2];
        uint32_t t = f2t[2 * size_t(fe)];
        FragV f0 = load_frag(u64(fe) << 2, qx, qy, faces, vgeo, colors);
        TetRow tr = load_tet(tt, t);
        for (uint32_t step = 0; step <= num_tets; ++step) {
            const uint32_t fx = tet_face_of(tr, vfix, fe, false, px, py);
            if (fx == kNoTet) break;
            if (sh.use_ert && T.hi < sh.ert_thresh) {
                stop = true;
                break;
            }
            // The next tet and its table row are fetched before this segment
            // is composited, so their loads overlap the exit face's vertex loads.
            const uint4 fcx = faces[fx];
            const uint32_t tn = other_tet(f2t, fx, t);
            const bool more = !(fcx.w & 1u) && tn != kNoTet;  // not leaving the mesh
            TetRow tr_next{};
            if (more) tr_next = load_tet(tt, tn);
            const FragV f1 = load_frag_face(fx << 2, fcx, qx, qy, vgeo, colors);
            segment_composite((f1.z - f0.z) * scale * 0.25f, f0.col, f1.col, sh.atten, C0, C1, C2, T);
            last_tet = t;
            last_entry = fe;
            last_b = b;
            ++nseg;
            if (!more) break;
            t = tn;
            fe = fx;
            f0 = f1;
            tr = tr_next;
        }
    }
    write_pixel(image, tfinal, p, C0, C1, C2, T, sh);
    wstate[p] = make_uint4(last_tet, last_entry, last_b, nseg);
}

// The walk adjoint with screen-space rows on carried fragments (FragG): the
// exit fragment of a tet is the entry fragment of the one walked before it,
// so each step loads and solves one face, and a fragment's gradients are taken
// from the state kept since its load.  Same steps and values as the general
// loop in k_walk_adjoint.
template <class Acc>
__device__ __forceinline__ void walk_adjoint_carried(
    const u64* __restrict__ b_records, u64 beg, const uint32_t* __restrict__ bf_global,
    const uint4* __restrict__ faces, const uint32_t* __restrict__ f2t, const TetTopo& tt, uint32_t num_tets,
    const int2* __restrict__ vfix, const VGeo* __restrict__ vgeo, const float4* __restrict__ colors, int px, int py,
    float scale, float atten, float gC0, float gC1, float gC2, TransBack T, TransF gT, uint32_t t, uint32_t fe,
    uint32_t fx, int b, Acc& acc) {
    const float qx = float(px) + 0.5f, qy = float(py) + 0.5f;
    FragG fX = load_frag_g(fx << 2, faces[fx], qx, qy, vgeo, colors, gC0, gC1, gC2);
    float gz_x = 0.f, wx = 0.f, ax = 0.f;
    // Cache slots the last added fragment left open for the next one; shared
    // vertices keep their slot, so fX (the last added fragment, or the one it
    // was kept for) names them when the walk ends.
    uint32_t open = 0u;
    for (uint32_t step = 0; step <= num_tets; ++step) {
        // The tet behind the entry face and its table row are fetched first, so
        // their loads overlap the entry face's vertex loads and this step's math.
        const uint4 fce = faces[fe];
        const uint32_t tprev = other_tet(f2t, fe, t);
        const bool inner = !(fce.w & 1u) && tprev != kNoTet;
        TetRow trp{};
        if (inner) trp = load_tet(tt, tprev);
        // The entry face shares an edge with the exit face (one tet): its
        // vertices in the exit face's order for the ordered row cache.
        uint32_t pv[3];
        const uint32_t keep = order_like(fX.v, fce.x, fce.y, fce.z, pv);
        const FragG fE = load_frag_g(fe << 2, pv[0], pv[1], pv[2], keep, qx, qy, vgeo, colors, gC0, gC1, gC2);
        const float tSeg = (fX.z - fE.z) * scale * 0.25f;
        float g_tot = 0.f, we = 0.f, ae = 0.f;
        segment_adjoint(tSeg, fE.alpha, fX.alpha, fE.pcol, fX.pcol, atten, T, gT, g_tot, we, wx, ae, ax);
        const float gz_e = -g_tot * scale;
        gz_x += g_tot * scale;
        const bool leaving = fce.w & 1u;
        frag_grads_carried(fX, gz_x, wx, ax, keep, acc);
        if (leaving) {
            frag_grads_carried(fE, gz_e, we, ae, 0u, acc);
            open = 0u;
            // Previous interval: its exit is the last back-facing boundary fragment before b.
            int bb = b - 1;
            while (bb >= 0 && (uint32_t(b_records[beg + bb]) & 1u)) --bb;
            if (bb < 0) break;
            fx = bf_global[uint32_t(b_records[beg + bb]) >> 2];
            t = f2t[2 * size_t(fx)];
            fe = tet_face_at(tt, vfix, t, fx, true, px, py);
            if (fe == kNoTet) break;
            int be = bb - 1;
            while (be >= 0 && !(uint32_t(b_records[beg + be]) & 1u)) --be;
            b = be < 0 ? 0 : be;
            fX = load_frag_g(fx << 2, faces[fx], qx, qy, vgeo, colors, gC0, gC1, gC2);
            gz_x = 0.f;
            wx = 0.f;
            ax = 0.f;
            continue;
        }
        open = keep;
        if (!inner) break;
        const uint32_t feprev = tet_face_of(trp, vfix, fe, true, px, py);
        if (feprev == kNoTet) break;
        fX = fE;
        gz_x = gz_e;
        wx = we;
        ax = ae;
        t = tprev;
        fe = feprev;
    }
    acc.close(fX.v, open);
    acc.flush();
}

template <bool SCREEN>
__global__ void __launch_bounds__(kTile * kTile, 2) k_walk_adjoint(
    const u64* __restrict__ b_offsets, const u64* __restrict__ b_records, const uint32_t* __restrict__ bf_global,
    const uint4* __restrict__ faces, const uint32_t* __restrict__ f2t, TetTopo tt, uint32_t num_tets, const int2* __restrict__ vfix, const VGeo* __restrict__ vgeo,
    const float4* __restrict__ colors, CamDev cam, ShadeDev sh, const float4* __restrict__ dimage,
    const float* __restrict__ tfinal, const uint4* __restrict__ wstate, float4* __restrict__ grad_rows) {
    const int px = blockIdx.x * kTile + (threadIdx.x % kTile);
    const int py = blockIdx.y * kTile + (threadIdx.x / kTile);
    if (px >= cam.W || py >= cam.H) return;
    const size_t p = size_t(py) * cam.W + px;
    const uint4 ws = wstate[p];
    if (ws.x == kNoTet) return;
    const float4 g = dimage[p];
    if (g.x == 0.f && g.y == 0.f && g.z == 0.f && g.w == 0.f) return;
    const bool use_abs = sh.use_abs_grad != 0;
    const u64 beg = b_offsets[p];
    const float qx = float(px) + 0.5f, qy = float(py) + 0.5f;
    const float scale = ray_scale(cam, qx, qy);
    const float atten = sh.atten;
    const float gC0 = g.x, gC1 = g.y, gC2 = g.z;
    TransF gT{g.x * sh.clear[0] + g.y * sh.clear[1] + g.z * sh.clear[2] + g.w * (sh.clear[3] - 1.f), 0.f};
    TransBack T(tfinal[p]);
    uint32_t t = ws.x, fe = ws.y;
    int b = int(ws.z);
    uint32_t fx = tet_face_at(tt, vfix, t, fe, false, px, py);
    if (fx == kNoTet) return;
    if constexpr (SCREEN) {
        __shared__ float4 vcache4[3 * kTile * kTile];
        __shared__ float vcache1[3 * kTile * kTile];
        OrderedRowsSmem acc{grad_rows, vcache4 + threadIdx.x, vcache1 + threadIdx.x, kTile * kTile};
        acc.set_pixel(gC0, gC1, gC2);
        walk_adjoint_carried(b_records, beg, bf_global, faces, f2t, tt, num_tets, vfix, vgeo, colors, px, py, scale,
                             atten, gC0, gC1, gC2, T, gT, t, fe, fx, b, acc);
        return;
    }
    // Vertex rows straight to global memory (absolute gradients, world rows).
    GradAcc acc{grad_rows};
    if (use_abs)
        acc.set_pixel(fabsf(gC0), fabsf(gC1), fabsf(gC2));
    else
        acc.set_pixel(gC0, gC1, gC2);
    // Per fragment: depth adjoint, colour weight (colour adjoint = gC x weight)
    // and alpha adjoint of the exit (x) and entry (e) fragments of the tet.
    float gz_x = 0.f, wx = 0.f, ax = 0.f;
    for (uint32_t step = 0; step <= num_tets; ++step) {
        const FragV f0 = load_frag(u64(fe) << 2, qx, qy, faces, vgeo, colors);
        const FragV f1 = load_frag(u64(fx) << 2, qx, qy, faces, vgeo, colors);
        const float tSeg = (f1.z - f0.z) * scale * 0.25f;
        const float p0 = gC0 * f0.col.x + gC1 * f0.col.y + gC2 * f0.col.z;
        const float p1 = gC0 * f1.col.x + gC1 * f1.col.y + gC2 * f1.col.z;
        float g_tot = 0.f, we = 0.f, ae = 0.f;
        segment_adjoint(tSeg, f0.col, f1.col, p0, p1, atten, T, gT, g_tot, we, wx, ae, ax);
        float gz_e = -g_tot * scale;
        gz_x += g_tot * scale;
        frag_vertex_grads<GradAcc, SCREEN>(f1, qx, qy, vgeo, colors, cam, gz_x, gC0, gC1, gC2, wx, ax, use_abs, acc);
        if (faces[fe].w & 1u) {
            frag_vertex_grads<GradAcc, SCREEN>(f0, qx, qy, vgeo, colors, cam, gz_e, gC0, gC1, gC2, we, ae, use_abs,
                                               acc);
            // Previous interval: its exit is the last back-facing boundary fragment before b.
            int bb = b - 1;
            while (bb >= 0 && (uint32_t(b_records[beg + bb]) & 1u)) --bb;
            if (bb < 0) break;
            fx = bf_global[uint32_t(b_records[beg + bb]) >> 2];
            t = f2t[2 * size_t(fx)];
            fe = tet_face_at(tt, vfix, t, fx, true, px, py);
            if (fe == kNoTet) break;
            int be = bb - 1;
            while (be >= 0 && !(uint32_t(b_records[beg + be]) & 1u)) --be;
            b = be < 0 ? 0 : be;
            gz_x = 0.f;
            wx = 0.f;
            ax = 0.f;
            continue;
        }
        const uint32_t tprev = other_tet(f2t, fe, t);
        if (tprev == kNoTet) break;
        const uint32_t feprev = tet_face_at(tt, vfix, tprev, fe, true, px, py);
        if (feprev == kNoTet) break;
        fx = fe;
        gz_x = gz_e;
        wx = we;
        ax = ae;
        t = tprev;
        fe = feprev;
    }
    acc.flush();
}

void launch_walk_composite(const u64* b_offsets, const u64* b_records, const uint32_t* bf_global,
                           const uint4* faces, const uint32_t* face_to_tet, const uint32_t* tet_faces,
                           const uint32_t* cells, const uint8_t* tet_flip, uint32_t num_tets, const int2* vfix, const VGeo* vgeo, const float4* colors,
                           const CamDev& cam, const ShadeDev& sh, float4* image, float* tfinal, uint4* wstate,
                           cudaStream_t s) {
    dim3 grid((cam.W + kTile - 1) / kTile, (cam.H + kWalkRows - 1) / kWalkRows);
    const TetTopo tt{reinterpret_cast<const uint4*>(tet_faces), reinterpret_cast<const uint4*>(cells), tet_flip};
    k_walk_composite<<<grid, kWalkThreads, 0, s>>>(b_offsets, b_records, bf_global, faces, face_to_tet, tt,
                                                    num_tets, vfix, vgeo, colors, cam, sh, image, tfinal, wstate);
}

void launch_walk_adjoint(const u64* b_offsets, const u64* b_records, const uint32_t* bf_global, const uint4* faces,
                         const uint32_t* face_to_tet, const uint32_t* tet_faces, const uint32_t* cells,
                         const uint8_t* tet_flip, uint32_t num_tets,
                         const int2* vfix, const VGeo* vgeo, const float4* colors, const CamDev& cam,
                         const ShadeDev& sh, const float4* dimage, const float* tfinal, const uint4* wstate,
                         uint32_t V, float4* grad_rows, float* grad_pos, float4* grad_col, cudaStream_t s) {
    cudaMemsetAsync(grad_rows, 0, sizeof(float4) * 2 * size_t(V), s);
    dim3 grid((cam.W + kTile - 1) / kTile, (cam.H + kTile - 1) / kTile);
    const TetTopo tt{reinterpret_cast<const uint4*>(tet_faces), reinterpret_cast<const uint4*>(cells), tet_flip};
    // Screen-space position rows unless absolute gradients are asked for
    // (frag_vertex_grads); the scatter converts them per vertex.
    if (sh.use_abs_grad)
        k_walk_adjoint<false><<<grid, kTile * kTile, 0, s>>>(b_offsets, b_records, bf_global, faces, face_to_tet,
                                                             tt, num_tets, vfix, vgeo, colors, cam, sh, dimage,
                                                             tfinal, wstate, grad_rows);
    else
        k_walk_adjoint<true><<<grid, kTile * kTile, 0, s>>>(b_offsets, b_records, bf_global, faces, face_to_tet,
                                                            tt, num_tets, vfix, vgeo, colors, cam, sh, dimage,
                                                            tfinal, wstate, grad_rows);
    launch_scatter_grads(grad_rows, V, grad_pos, grad_col, s, sh.use_abs_grad ? nullptr : vgeo, &cam);
}

}  // namespace dtv
