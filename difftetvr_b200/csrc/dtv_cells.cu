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
// the face vertices' positions (frag_position_grads).
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

__global__ void __launch_bounds__(kTile * kTile) k_adjoint_cells(
    const u64* __restrict__ offsets, const u64* __restrict__ records, const uint4* __restrict__ faces,
    const uint2* __restrict__ f2t, const VGeo* __restrict__ vgeo, const float4* __restrict__ cell_colors, int W,
    int row0, int row1, CamDev cam, ShadeDev sh, const float4* __restrict__ dimage, const float* __restrict__ tfinal,
    const uint32_t* __restrict__ term, float4* __restrict__ grad_rows, float4* __restrict__ grad_cells) {
    const int px = blockIdx.x * kTile + (threadIdx.x % kTile);
    const int py = row0 + int(blockIdx.y) * kTile + int(threadIdx.x / kTile);
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
    uint32_t fbi = uint32_t(records[beg + last]) >> 2;
    uint4 fb = faces[fbi];
    uint2 pb = f2t[fbi];
    float zb = face_depth(fb, vgeo, qx, qy), gz_b = 0.f;
    for (int i = last; i >= 1; --i) {
        const uint32_t ffi = uint32_t(records[beg + i - 1]) >> 2;
        const uint4 ff = faces[ffi];
        const uint2 pf = f2t[ffi];
        const float zf = face_depth(ff, vgeo, qx, qy);
        float gz_f = 0.f;
        const uint32_t open = tet_union(pb, pf);
        if (open != kInvalidCell) {
            const float4 c = cell_colors[open];
            const float a = c.w * atten, t = zb - zf;
            const float x = a * t;
            const float oma = one_minus_exp(x), A = fabsf(x) < 0.125f ? 1.f - oma : __expf(-x);
            trans_add(T, T.hi * expm1_signed(x));  // T_in = T_out / A
            const float Tin = T.hi;
            const float gx = Tin * g.x, gy = Tin * g.y, gzc = Tin * g.z;
            const float gA = Tin * gT.hi - (gx * c.x + gy * c.y + gzc * c.z);
            trans_add(gT, oma * ((g.x * c.x + g.y * c.y + g.z * c.z) - gT.hi));  // gT A + (1 - A) gC . c
            const float g_t = gA * (-a * A), g_a = gA * (-t * A);
            float4 gc = make_float4(gx * oma, gy * oma, gzc * oma, g_a * atten);
            if (use_abs) gc = make_float4(fabsf(gc.x), fabsf(gc.y), fabsf(gc.z), fabsf(gc.w));
            atomicAdd(grad_cells + open, gc);
            gz_b += g_t;
            gz_f -= g_t;
        }
        frag_position_grads(fb, qx, qy, vgeo, cam, gz_b, use_abs, grad_rows);
        fb = ff;
        pb = pf;
        zb = zf;
        gz_b = gz_f;
    }
    frag_position_grads(fb, qx, qy, vgeo, cam, gz_b, use_abs, grad_rows);
}

__global__ void __launch_bounds__(256) k_scatter_positions(const float4* __restrict__ rows, uint32_t V,
                                                           float* __restrict__ grad_pos) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const float4 a = rows[2 * size_t(v)];
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
    dim3 grid((cam.W + kTile - 1) / kTile, (row1 - row0 + kTile - 1) / kTile);
    k_adjoint_cells<<<grid, kTile * kTile, 0, s>>>(offsets, records, faces,
                                                   reinterpret_cast<const uint2*>(face_to_tet), vgeo, cell_colors,
                                                   cam.W, row0, row1, cam, sh, dimage, tfinal, term, grad_rows,
                                                   grad_cells);
}

void launch_scatter_positions(const float4* grad_rows, uint32_t V, float* grad_pos, cudaStream_t s) {
    if (V) k_scatter_positions<<<(V + 255) / 256, 256, 0, s>>>(grad_rows, V, grad_pos);
}

}  // namespace dtv
