// Per-cell colours (ColorStorage::PER_CELL) on the fragment-list path.
//
// Reference: Forward.glsl:213-246 and Backward.glsl:283-329 (the
// !PER_VERTEX_COLORS branches), tetIdUnion (LinkedListResolve.glsl:85-94),
// accumulateConst / accumulateConstAdjoint (ForwardCommon.glsl:37-40,
// BackwardCommon.glsl:95-105).  Two consecutive fragments of a pixel's sorted
// list bound a segment of the tet both faces belong to; a pair of faces with
// no common tet (empty space between boundary faces, or a ray crossing an
// edge) contributes nothing.  The segment has the cell's constant colour c and
// density a = c.a * attenuation:  A = exp(-a t),  C = (1 - A) c.  Early ray
// termination is checked before each fragment; the termination index is the
// fragment index where the loop stopped.
//
// The adjoint runs back to front from the termination index with
// T_in = T_out / A, adds each segment's colour adjoint into the cell's
// gradient (one float4 atomic) and pushes the two fragment-depth adjoints to
// the face vertices' positions.  Without absolute gradients each fragment's
// face interpolation is computed once and carried to the next step (FragP),
// and the vertices' screen-space position adjoints go through the ordered
// register rows (order_like, as the per-vertex adjoint); k_scatter_positions
// converts them to world space per vertex.  With absolute gradients every
// fragment adds |world-space contribution| per vertex (frag_position_grads).
#include "dtv_internal.h"
#include "dtv_path.cuh"

namespace dtv {

constexpr uint32_t kInvalidCell = 0xffffffffu;

__device__ __forceinline__ uint32_t tet_union(uint2 a, uint2 b) {
    if ((a.x == b.x || a.x == b.y) && a.x != kInvalidCell) return a.x;
    if ((a.y == b.x || a.y == b.y) && a.y != kInvalidCell) return a.y;
    return kInvalidCell;
}

__device__ __forceinline__ float face_depth(const uint4& fc, const VGeo* __restrict__ vgeo, float qx, float qy) {
    float bary[3], z;
    face_bary(vgeo[fc.x], vgeo[fc.y], vgeo[fc.z], qx, qy, bary, z);
    return z;
}

__global__ void __launch_bounds__(kTile * kTile) k_composite_cells(
    const u64* __restrict__ offsets, const u64* __restrict__ records, const uint4* __restrict__ faces,
    const uint2* __restrict__ f2t, const VGeo* __restrict__ vgeo, const float4* __restrict__ cell_colors, int W,
    int row0, int row1, ShadeDev sh, float4* __restrict__ image, float* __restrict__ tfinal,
    uint32_t* __restrict__ term) {
    const int px = blockIdx.x * kTile + (threadIdx.x % kTile);
    const int py = row0 + int(blockIdx.y) * kTile + int(threadIdx.x / kTile);
    if (px >= W || py >= row1) return;
    const size_t p = size_t(py) * W + px;
    const u64 beg = offsets[p];
    const uint32_t n = uint32_t(offsets[p + 1] - beg);
    const float qx = float(px) + 0.5f, qy = float(py) + 0.5f;
    float C0 = 0.f, C1 = 0.f, C2 = 0.f, zprev = 0.f;
    TransF T{1.f, 0.f};  // float-float transmittance (dtv_segment.cuh)
    uint2 prev = make_uint2(kInvalidCell, kInvalidCell);
    uint32_t i = 0;
    for (; i < n; ++i) {
        if (sh.use_ert && T.hi < sh.ert_thresh) break;
        const uint32_t face = uint32_t(records[beg + i]) >> 2;
        const float z = face_depth(faces[face], vgeo, qx, qy);
        const uint2 cur = f2t[face];
        const uint32_t open = tet_union(cur, prev);
        if (open != kInvalidCell) {
            const float4 c = cell_colors[open];
            const float w = T.hi * one_minus_exp((c.w * sh.atten) * (z - zprev));
            C0 += w * c.x;
            C1 += w * c.y;
            C2 += w * c.z;
            trans_add(T, -w);
        }
        prev = cur;
        zprev = z;
    }
    write_pixel(image, tfinal, p, C0, C1, C2, T, sh);
    term[p] = i;
}

// A fragment's face interpolation for its position gradients (the
// interpolation state of face_interp; z is the depth the composite used).
struct FragP {
    uint32_t v[3];
    uint32_t keep;                   // slots continuing from the previous fragment's face (order_like)
    uint2 tets;                      // the face's cells (face_to_tet)
    float z;
    float lam[3], iz[3], dx[3], dy[3];
    float invA, zz;                  // 1 / sum(E); zb^2, 0 when the depth is clamped
};

__device__ __forceinline__ FragP load_frag_p(const uint32_t (&v)[3], uint32_t keep, uint2 tets, float qx, float qy,
                                             const VGeo* __restrict__ vgeo) {
    FragP f;
#pragma unroll
    for (int j = 0; j < 3; ++j) f.v[j] = v[j];
    f.keep = keep;
    f.tets = tets;
    const VGeo a = vgeo[v[0]], b = vgeo[v[1]], c = vgeo[v[2]];
    FaceInterp fi;
    face_interp(a, b, c, qx, qy, fi);
    f.z = fi.z;
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
    f.zz = fi.clamped ? 0.f : fi.zb * fi.zb;
    return f;
}

// Screen-space position rows of three ordered slots (OrderedRows without the
// colour row): a slot the next face does not continue is written out with one
// float4 atomic (d/dsx, d/dsy, d/d(1/ze), 0).
struct OrderedPosRows {
    float4* rows;  // [V][2] rows; the position row of vertex v is rows[2 v]
    float3 p[3];
    __device__ __forceinline__ void put(uint32_t v, const float3& q) const {
        atomicAdd(rows + 2 * size_t(v), make_float4(q.x, q.y, q.z, 0.f));
    }
    __device__ __forceinline__ void add_ordered(const uint32_t (&v)[3], uint32_t keep, uint32_t keep_next,
                                                const float3 (&gp)[3]) {
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            p[s] = ((keep >> s) & 1u) ? make_float3(p[s].x + gp[s].x, p[s].y + gp[s].y, p[s].z + gp[s].z) : gp[s];
            if (!((keep_next >> s) & 1u)) put(v[s], p[s]);
        }
    }
};

// Position adjoints of a carried fragment from its depth adjoint gz (the depth
// path of frag_position_grads, left in screen space).
__device__ __forceinline__ void frag_pos_carried(const FragP& f, float gz, uint32_t keep_next, OrderedPosRows& acc) {
    const float gzz = gz * f.zz;
    float glam[3], giz[3], sl = 0.f;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        glam[j] = -gzz * f.iz[j];
        giz[j] = -gzz * f.lam[j];
        sl += glam[j] * f.lam[j];
    }
    float gE[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) gE[j] = (glam[j] - sl) * f.invA;
    const float* dx = f.dx;
    const float* dy = f.dy;
    float3 gp[3];
    gp[0] = make_float3(-gE[1] * dy[2] + gE[2] * dy[1], gE[1] * dx[2] - gE[2] * dx[1], giz[0]);
    gp[1] = make_float3(gE[0] * dy[2] - gE[2] * dy[0], -gE[0] * dx[2] + gE[2] * dx[0], giz[1]);
    gp[2] = make_float3(-gE[0] * dy[1] + gE[1] * dy[0], gE[0] * dx[1] - gE[1] * dx[0], giz[2]);
    acc.add_ordered(f.v, f.keep, keep_next, gp);
}

// Segment of a pixel's back-to-front walk between fragments with cells pf
// (front) and pb (back) at depths zf < zb: transmittance and its adjoint
// stepped back over the segment, the cell colour adjoint added into
// grad_cells, and the depth adjoint g_t of the segment's length returned
// (0 when the two faces share no cell).
__device__ __forceinline__ float cell_segment_adjoint(uint2 pf, uint2 pb, float zf, float zb,
                                                      const float4* __restrict__ cell_colors, float atten,
                                                      bool use_abs, const float4& g, TransF& T, TransF& gT,
                                                      float4* __restrict__ grad_cells) {
    const uint32_t open = tet_union(pb, pf);
    if (open == kInvalidCell) return 0.f;
    const float4 c = cell_colors[open];
    const float a = c.w * atten, t = zb - zf;
    const float x = a * t;
    const float oma = one_minus_exp(x), A = fabsf(x) < 0.125f ? 1.f - oma : __expf(-x);
    trans_add(T, T.hi * expm1_signed(x));  // T_in = T_out / A
    const float Tin = T.hi;
    const float gx = Tin * g.x, gy = Tin * g.y, gzc = Tin * g.z;
    const float gA = Tin * gT.hi - (gx * c.x + gy * c.y + gzc * c.z);
    trans_add(gT, oma * ((g.x * c.x + g.y * c.y + g.z * c.z) - gT.hi));  // gT A + (1 - A) gC . c
    const float g_a = gA * (-t * A);
    float4 gc = make_float4(gx * oma, gy * oma, gzc * oma, g_a * atten);
    if (use_abs) gc = make_float4(fabsf(gc.x), fabsf(gc.y), fabsf(gc.z), fabsf(gc.w));
    atomicAdd(grad_cells + open, gc);
    return gA * (-a * A);
}

// 16 x 8 pixel blocks: the carried screen-space variant fits five per SM
// (at most 102 registers, no spills).
constexpr int kCellRows = 8;
template <bool SCREEN>
__global__ void __launch_bounds__(kTile * kCellRows, SCREEN ? 5 : 4) k_adjoint_cells(
    const u64* __restrict__ offsets, const u64* __restrict__ records, const uint4* __restrict__ faces,
    const uint2* __restrict__ f2t, const VGeo* __restrict__ vgeo, const float4* __restrict__ cell_colors, int W,
    int row0, int row1, CamDev cam, ShadeDev sh, const float4* __restrict__ dimage, const float* __restrict__ tfinal,
    const uint32_t* __restrict__ term, float4* __restrict__ grad_rows, float4* __restrict__ grad_cells) {
    const int px = blockIdx.x * kTile + (threadIdx.x % kTile);
    const int py = row0 + int(blockIdx.y) * kCellRows + int(threadIdx.x / kTile);
    if (px >= W || py >= row1) return;
    const size_t p = size_t(py) * W + px;
    const u64 beg = offsets[p];
    const uint32_t n = uint32_t(offsets[p + 1] - beg);
    const int last = int(sh.use_ert ? term[p] : n) - 1;  // last fragment visited
    if (last < 1) return;
    const float4 g = dimage[p];
    if (g.x == 0.f && g.y == 0.f && g.z == 0.f && g.w == 0.f) return;
    const float qx = float(px) + 0.5f, qy = float(py) + 0.5f;
    const bool use_abs = sh.use_abs_grad != 0;
    const float atten = sh.atten;
    // Float-float transmittance and its adjoint (dtv_segment.cuh).
    TransF gT{g.x * sh.clear[0] + g.y * sh.clear[1] + g.z * sh.clear[2] + g.w * (sh.clear[3] - 1.f), 0.f};
    TransF T{tfinal[p], 0.f};
    if constexpr (SCREEN) {
        // Dependent loads record -> face -> vertex rows one step ahead, as in
        // adjoint_pixel_carried.
        OrderedPosRows acc{grad_rows};
        const uint32_t fbi = uint32_t(records[beg + last]) >> 2;
        const uint4 fcb = faces[fbi];
        const uint32_t vb[3] = {fcb.x, fcb.y, fcb.z};
        FragP fb = load_frag_p(vb, 0u, f2t[fbi], qx, qy, vgeo);
        uint32_t ffi = uint32_t(records[beg + last - 1]) >> 2;
        uint4 fc_f = faces[ffi];
        uint2 pf_f = f2t[ffi];
        uint32_t fni = last >= 2 ? uint32_t(records[beg + last - 2]) >> 2 : 0u;
        float gz_b = 0.f;
        for (int i = last; i >= 1; --i) {
            uint32_t pv[3];
            const uint32_t keep = order_like(fb.v, fc_f.x, fc_f.y, fc_f.z, pv);
            const FragP ff = load_frag_p(pv, keep, pf_f, qx, qy, vgeo);
            if (i >= 2) {
                fc_f = faces[fni];
                pf_f = f2t[fni];
                if (i >= 3) fni = uint32_t(records[beg + i - 3]) >> 2;
            }
            const float g_t = cell_segment_adjoint(ff.tets, fb.tets, ff.z, fb.z, cell_colors, atten, false, g, T, gT,
                                                   grad_cells);
            frag_pos_carried(fb, gz_b + g_t, ff.keep, acc);
            fb = ff;
            gz_b = -g_t;
        }
        frag_pos_carried(fb, gz_b, 0u, acc);
        return;
    }
    uint32_t fbi = uint32_t(records[beg + last]) >> 2;
    uint4 fb = faces[fbi];
    uint2 pb = f2t[fbi];
    float zb = face_depth(fb, vgeo, qx, qy), gz_b = 0.f;
    for (int i = last; i >= 1; --i) {
        const uint32_t ffi = uint32_t(records[beg + i - 1]) >> 2;
        const uint4 ff = faces[ffi];
        const uint2 pf = f2t[ffi];
        const float zf = face_depth(ff, vgeo, qx, qy);
        const float g_t = cell_segment_adjoint(pf, pb, zf, zb, cell_colors, atten, use_abs, g, T, gT, grad_cells);
        gz_b += g_t;
        frag_position_grads(fb, qx, qy, vgeo, cam, gz_b, use_abs, grad_rows);
        fb = ff;
        pb = pf;
        zb = zf;
        gz_b = -g_t;
    }
    frag_position_grads(fb, qx, qy, vgeo, cam, gz_b, use_abs, grad_rows);
}

template <bool SCREEN>
__global__ void __launch_bounds__(256) k_scatter_positions(const float4* __restrict__ rows, uint32_t V,
                                                           float* __restrict__ grad_pos,
                                                           const VGeo* __restrict__ vgeo, CamDev cam) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    float4 a = rows[2 * size_t(v)];
    if (SCREEN) {
        const float3 w = screen_to_world(a, vgeo[v], cam);
        a = make_float4(w.x, w.y, w.z, 0.f);
    }
    float* gp = grad_pos + 3 * size_t(v);
    gp[0] += a.x;
    gp[1] += a.y;
    gp[2] += a.z;
}

void launch_composite_cells(const u64* offsets, const u64* records, const uint4* faces, const uint32_t* face_to_tet,
                            const VGeo* vgeo, const float4* cell_colors, int W, int H, const ShadeDev& sh,
                            float4* image, float* tfinal, uint32_t* term, cudaStream_t s, int row0, int row1) {
    if (row1 < 0) row1 = H;
    if (row1 <= row0) return;
    dim3 grid((W + kTile - 1) / kTile, (row1 - row0 + kTile - 1) / kTile);
    k_composite_cells<<<grid, kTile * kTile, 0, s>>>(offsets, records, faces,
                                                     reinterpret_cast<const uint2*>(face_to_tet), vgeo, cell_colors, W,
                                                     row0, row1, sh, image, tfinal, term);
}

void launch_adjoint_cells_rows(const u64* offsets, const u64* records, const uint4* faces,
                               const uint32_t* face_to_tet, const VGeo* vgeo, const float4* cell_colors,
                               const CamDev& cam, const ShadeDev& sh, const float4* dimage, const float* tfinal,
                               const uint32_t* term, int row0, int row1, float4* grad_rows, float4* grad_cells,
                               cudaStream_t s) {
    if (row1 <= row0) return;
    dim3 grid((cam.W + kTile - 1) / kTile, (row1 - row0 + kCellRows - 1) / kCellRows);
    if (sh.use_abs_grad)
        k_adjoint_cells<false><<<grid, kTile * kCellRows, 0, s>>>(offsets, records, faces,
                                                              reinterpret_cast<const uint2*>(face_to_tet), vgeo,
                                                              cell_colors, cam.W, row0, row1, cam, sh, dimage, tfinal,
                                                              term, grad_rows, grad_cells);
    else
        k_adjoint_cells<true><<<grid, kTile * kCellRows, 0, s>>>(offsets, records, faces,
                                                             reinterpret_cast<const uint2*>(face_to_tet), vgeo,
                                                             cell_colors, cam.W, row0, row1, cam, sh, dimage, tfinal,
                                                             term, grad_rows, grad_cells);
}

void launch_scatter_positions(const float4* grad_rows, uint32_t V, float* grad_pos, cudaStream_t s,
                              const VGeo* vgeo, const CamDev* cam) {
    if (V == 0) return;
    if (vgeo)
        k_scatter_positions<true><<<(V + 255) / 256, 256, 0, s>>>(grad_rows, V, grad_pos, vgeo, *cam);
    else
        k_scatter_positions<false><<<(V + 255) / 256, 256, 0, s>>>(grad_rows, V, grad_pos, nullptr, CamDev{});
}

}  // namespace dtv
