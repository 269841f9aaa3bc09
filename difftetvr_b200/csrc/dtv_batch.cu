// Batched multi-view / multi-mesh rendering, adjoint and training step.
//
// Many camera views of meshes of uneven size go through the hot path with one
// launch per stage: every stage runs over a flattened index space of
// (view, item) pairs - projected vertices, faces, pixels, 16x16 pixel tiles -
// with a grid-stride loop, and finds its view by binary search in a small
// descriptor table.  The per-pixel counters, offsets and fragment records of
// all views share one buffer, so one scan and one sort cover the batch.
//
// The training step (render -> fused L2 loss -> adjoint -> Adam of every mesh)
// can be captured once in a CUDA graph and replayed.  The record buffer then
// has a fixed capacity: a guard after the scan flags an overflow, every later
// kernel of the step returns immediately when the flag is set, the host sees
// the flag at the end of the step and reruns that step uncaptured with a
// larger buffer, then recaptures.  View descriptors (cameras, image and
// target pointers) are read from device memory, so they can change between
// replays without a new capture; a change of view count or sizes recaptures.
//
// The reference renders one view per call (TetMeshRendererPPLL::render /
// renderAdjoint, TetMeshRendererPPLL.cpp:671-724) and steps its optimizer per
// parameter buffer (OptimizerPass.cpp:120-177); the batched forms have no
// separate counterpart there.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include "difftetvr_b200.h"
#include "dtv_host.h"
#include "dtv_internal.h"
#include "dtv_path.cuh"

namespace dtv {

struct BatchView {
    CamDev cam;
    const uint4* faces;
    const float* positions;
    const float4* colors;
    float4* image;
    float4* dimage;            // image adjoint: read by the adjoint, written by the fused loss
    const float4* target;      // fused-loss target (nullable)
    u64 vert_base, face_base, pix_base, tile_base, grad_base;
    uint32_t V, F, W, H, tiles_x;
    int32_t grad_slot;         // -1: no gradient for this view
    float loss_scale;          // 1 / (W * H * 4)  (torch.nn.MSELoss, mean)
};

// Rows of the interleaved gradient accumulator that belong to one slot, and
// what the optimizer / scatter does with them.
struct BatchSlot {
    u64 row_base;
    uint32_t V;
    float* grad_pos;           // [V][3] (scatter adds here)
    float4* grad_col;          // [V]
    // training step (dtv_batch_train_step)
    float* pos;                // [V][3] parameters
    float4* col;               // [V]
    float* m_pos;              // Adam state [V][3]
    float* v_pos;
    float4* m_col;             // [V]
    float4* v_col;
    const uint32_t* boundary;  // per-vertex boundary bits (fixed-boundary modes)
};

template <typename Getter>
__device__ __forceinline__ int find_index(u64 g, int n, Getter base) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (base(mid) <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ bool batch_ok(const uint32_t* ok) { return ok == nullptr || *ok != 0u; }

// View of item g for kernels with one item per thread: one search for the
// block's first item (the same loads for every thread of the block), then a
// forward walk for the few threads past a view boundary.
template <typename Getter>
__device__ __forceinline__ int view_of_item(u64 g, u64 block_first, int n, Getter base) {
    int v = find_index(block_first, n, base);
    while (v + 1 < n && base(v + 1) <= g) ++v;
    return v;
}

__global__ void __launch_bounds__(256) kb_project(const BatchView* __restrict__ views, int nviews, u64 total,
                                                  float4* __restrict__ vproj, int2* __restrict__ vfix,
                                                  VGeo* __restrict__ vgeo) {
    const u64 first = u64(blockIdx.x) * blockDim.x;
    const u64 g = first + threadIdx.x;
    if (g < total) {
        const int v = view_of_item(g, first, nviews, [&](int i) { return views[i].vert_base; });
        const BatchView& bv = views[v];
        const u64 k = g - bv.vert_base;
        const float x = bv.positions[3 * k], y = bv.positions[3 * k + 1], z = bv.positions[3 * k + 2];
        int2 fx;
        vproj[g] = project_vertex(bv.cam, x, y, z, fx);
        vfix[g] = fx;
        vgeo[g] = project_vertex_geo(bv.cam, x, y, z, fx);
    }
}

// Row-band order of the batch fill (launch_fill_order for one view): items
// (view faces) grouped by the band of 2^shift pixels of the concatenated
// views' pixels that holds the start of the face's first covered row, the
// shift putting about kFillBandBytes of records in a band.  The shift comes
// from the scanned total on the device (no host read in a captured step).
__device__ __forceinline__ int kb_band_shift(const u64* __restrict__ offsets, u64 tot_pixels) {
    const u64 nf = offsets[tot_pixels];
    const u64 target = nf ? (kFillBandBytes / sizeof(u64)) * tot_pixels / nf : tot_pixels;
    int shift = target ? 63 - __clzll((long long)target) : 0;
    while (((tot_pixels - 1) >> shift) >= u64(kFillBands)) ++shift;
    return shift;
}

__device__ __forceinline__ int kb_face_band(const BatchView* __restrict__ views, int nviews, u64 g,
                                            const int2* __restrict__ vfix, int shift) {
    const int v = find_index(g, nviews, [&](int i) { return views[i].face_base; });
    const BatchView& bv = views[v];
    const uint4 fc = bv.faces[g - bv.face_base];
    const int2* vf = vfix + bv.vert_base;
    const int2 q0 = vf[fc.x], q1 = vf[fc.y], q2 = vf[fc.z];
    if (q0.x == kInvalidFix || q1.x == kInvalidFix || q2.x == kInvalidFix) return 0;
    const long long minY = min(q0.y, min(q1.y, q2.y));
    const long long py0 = min((long long)bv.H - 1, max(0LL, ceil_div256(minY - 128)));
    return int(min(u64(kFillBands - 1), (bv.pix_base + u64(py0) * bv.W) >> shift));
}

__global__ void __launch_bounds__(256) kb_band_count(const BatchView* __restrict__ views, int nviews, u64 total,
                                                     const int2* __restrict__ vfix, const u64* __restrict__ offsets,
                                                     u64 tot_pixels, uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[kFillBands];
    for (int b = threadIdx.x; b < kFillBands; b += blockDim.x) h[b] = 0u;
    __syncthreads();
    const u64 g = u64(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g < total) atomicAdd(&h[kb_face_band(views, nviews, g, vfix, kb_band_shift(offsets, tot_pixels))], 1u);
    __syncthreads();
    for (int b = threadIdx.x; b < kFillBands; b += blockDim.x)
        if (h[b]) atomicAdd(&hist[b], h[b]);
}

__global__ void __launch_bounds__(256) kb_band_scatter(const BatchView* __restrict__ views, int nviews, u64 total,
                                                       const int2* __restrict__ vfix, const u64* __restrict__ offsets,
                                                       u64 tot_pixels, uint32_t* __restrict__ cursor,
                                                       uint32_t* __restrict__ order) {
    __shared__ uint32_t h[kFillBands], base[kFillBands];
    for (int b = threadIdx.x; b < kFillBands; b += blockDim.x) h[b] = 0u;
    __syncthreads();
    const u64 g = u64(blockIdx.x) * blockDim.x + threadIdx.x;
    int band = 0;
    uint32_t rank = 0;
    if (g < total) {
        band = kb_face_band(views, nviews, g, vfix, kb_band_shift(offsets, tot_pixels));
        rank = atomicAdd(&h[band], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < kFillBands; b += blockDim.x)
        if (h[b]) base[b] = atomicAdd(&cursor[b], h[b]);
    __syncthreads();
    if (g < total) order[base[band] + rank] = uint32_t(g);
}

template <bool FILL, bool WIDE>
__global__ void __launch_bounds__(128) kb_raster(const BatchView* __restrict__ views, int nviews, u64 total,
                                                 const float4* __restrict__ vproj, const int2* __restrict__ vfix,
                                                 uint32_t* __restrict__ counts, const u64* __restrict__ offsets,
                                                 u64* __restrict__ records, const uint32_t* __restrict__ ok,
                                                 const uint32_t* __restrict__ order,
                                                 uint32_t* __restrict__ wide_list) {
    if (FILL && !batch_ok(ok)) return;
    const u64 first = u64(blockIdx.x) * blockDim.x;
    const u64 i = first + threadIdx.x;
    bool set = false, live = false;
    RasterJob J;
    u64 g = 0;
    if (i < total) {
        g = order ? u64(order[i]) : i;
        const int v = order ? find_index(g, nviews, [&](int k) { return views[k].face_base; })
                            : view_of_item(g, first, nviews, [&](int k) { return views[k].face_base; });
        const BatchView& bv = views[v];
        set = raster_setup(uint32_t(g - bv.face_base), bv.faces, vfix + bv.vert_base, uint32_t(bv.vert_base),
                           int(bv.W), 0, int(bv.H), bv.pix_base, J);
        live = set && (J.wide != 0) == WIDE;
    }
    if constexpr (!FILL) {
        if (live) count_face<typename std::conditional<WIDE, long long, int>::type>(J, counts);
        if (!WIDE && wide_list) {
            // The items of the 64-bit path, for its count and fill launches
            // (wide_list[0] = how many, then the items).
            const bool wide = set && J.wide != 0;
            const unsigned m = __ballot_sync(0xffffffffu, wide);
            if (m) {
                const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
                uint32_t base = 0;
                if (lane == leader) base = atomicAdd(wide_list, uint32_t(__popc(m)));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (wide) wide_list[1 + base + __popc(m & ((1u << lane) - 1u))] = uint32_t(g);
            }
        }
    } else {
        __shared__ RasterJob jobs[4][32];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (live) jobs[w][lane] = J;
        raster_warp<FILL, WIDE>(jobs[w], __ballot_sync(0xffffffffu, live), lane, vproj, counts, offsets, records);
    }
}

// The 64-bit items listed by the count (wide_list), 32 per warp and step over
// a fixed grid: the count (one thread per face) or the fill (raster_warp).
template <bool FILL>
__global__ void __launch_bounds__(128) kb_raster_listed(const BatchView* __restrict__ views, int nviews,
                                                        const float4* __restrict__ vproj,
                                                        const int2* __restrict__ vfix,
                                                        uint32_t* __restrict__ counts,
                                                        const u64* __restrict__ offsets, u64* __restrict__ records,
                                                        const uint32_t* __restrict__ ok,
                                                        const uint32_t* __restrict__ wide_list) {
    if (FILL && !batch_ok(ok)) return;
    __shared__ RasterJob jobs[4][32];
    const uint32_t n = wide_list[0];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + uint32_t(w) * 32u; base < n; base += stride) {
        const uint32_t i = base + uint32_t(lane);
        RasterJob J;
        bool live = false;
        if (i < n) {
            const u64 g = wide_list[1 + i];
            const int v = find_index(g, nviews, [&](int k) { return views[k].face_base; });
            const BatchView& bv = views[v];
            live = raster_setup(uint32_t(g - bv.face_base), bv.faces, vfix + bv.vert_base, uint32_t(bv.vert_base),
                                int(bv.W), 0, int(bv.H), bv.pix_base, J) &&
                   J.wide != 0;
        }
        if constexpr (!FILL) {
            if (live) count_face<long long>(J, counts);
        } else {
            if (live) jobs[w][lane] = J;
            raster_warp<FILL, true>(jobs[w], __ballot_sync(0xffffffffu, live), lane, vproj, counts, offsets,
                                    records);
            __syncwarp();  // every lane is done with this step's jobs before the next step writes them
        }
    }
}

// Per-row prefix of the count pass's difference arrays, one view per grid row.
__global__ void __launch_bounds__(256) kb_row_prefix(const BatchView* __restrict__ views,
                                                     uint32_t* __restrict__ counts) {
    const BatchView& bv = views[blockIdx.y];
    const uint32_t row = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (row < bv.H) row_prefix_warp(counts + bv.pix_base + size_t(row) * bv.W, int(bv.W), threadIdx.x & 31);
}

// ok = (records fit the buffer); *total_out = number of records.
__global__ void kb_check_capacity(const u64* __restrict__ offsets_end, u64 capacity, uint32_t* __restrict__ ok,
                                  u64* __restrict__ total_out) {
    const u64 total = *offsets_end;
    *ok = total <= capacity ? 1u : 0u;
    *total_out = total;
}

// On overflow the fill does not run, so clear the counters it would have consumed.
__global__ void __launch_bounds__(256) kb_clear_counts(uint32_t* __restrict__ counts, u64 n,
                                                       const uint32_t* __restrict__ ok) {
    if (batch_ok(ok)) return;
    for (u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += u64(gridDim.x) * blockDim.x) counts[i] = 0;
}

__device__ __forceinline__ bool tile_pixel(const BatchView* views, int nviews, int& v, int& px, int& py) {
    v = find_index(blockIdx.x, nviews, [&](int i) { return views[i].tile_base; });
    const BatchView& bv = views[v];
    const uint32_t t = uint32_t(blockIdx.x - bv.tile_base);
    px = int((t % bv.tiles_x) * kTile + threadIdx.x % kTile);
    py = int((t / bv.tiles_x) * kTile + threadIdx.x / kTile);
    return px < int(bv.W) && py < int(bv.H);
}

__global__ void __launch_bounds__(kTile * kTile) kb_composite(const BatchView* __restrict__ views, int nviews,
                                                              const u64* __restrict__ offsets,
                                                              const u64* __restrict__ records,
                                                              const VGeo* __restrict__ vgeo, ShadeDev sh,
                                                              float* __restrict__ tfinal,
                                                              uint32_t* __restrict__ term,
                                                              const uint32_t* __restrict__ ok) {
    if (!batch_ok(ok)) return;
    int v, px, py;
    if (!tile_pixel(views, nviews, v, px, py)) return;
    const BatchView& bv = views[v];
    composite_pixel(px, py, int(bv.W), offsets + bv.pix_base, records, bv.faces, vgeo + bv.vert_base, bv.colors, sh,
                    bv.image, tfinal + bv.pix_base, term + bv.pix_base);
}

// Fused L2 loss of every view with a target: dimage = 2 s (image - target),
// loss += s * sum (image - target)^2 with s = 1 / (4 W H).
__global__ void __launch_bounds__(256) kb_loss(const BatchView* __restrict__ views, int nviews, u64 total_pixels,
                                               float* __restrict__ loss, const uint32_t* __restrict__ ok) {
    if (!batch_ok(ok)) return;
    __shared__ float sm[8];
    float acc = 0.f;
    for (u64 g = u64(blockIdx.x) * blockDim.x + threadIdx.x; g < total_pixels; g += u64(gridDim.x) * blockDim.x) {
        const int v = find_index(g, nviews, [&](int i) { return views[i].pix_base; });
        const BatchView& bv = views[v];
        if (!bv.target || !bv.dimage) continue;
        const u64 p = g - bv.pix_base;
        const float4 a = bv.image[p], b = bv.target[p];
        const float4 d = make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
        const float s2 = 2.f * bv.loss_scale;
        bv.dimage[p] = make_float4(s2 * d.x, s2 * d.y, s2 * d.z, s2 * d.w);
        acc += bv.loss_scale * (d.x * d.x + d.y * d.y + d.z * d.z + d.w * d.w);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) atomicAdd(loss, v);
    }
}

// SCREEN: each view adds screen-space adjoint rows of its own camera into
// view_rows (at its vert_base), which kb_view_rows projects and adds into the
// slots' rows; otherwise world-space rows go straight to the slot (views of
// one mesh share them).
template <bool SCREEN>
__global__ void __launch_bounds__(kTile * kTile, 2) kb_adjoint(const BatchView* __restrict__ views, int nviews,
                                                            const u64* __restrict__ offsets,
                                                            const u64* __restrict__ records,
                                                            const VGeo* __restrict__ vgeo, ShadeDev sh,
                                                            const float* __restrict__ tfinal,
                                                            const uint32_t* __restrict__ term,
                                                            float4* __restrict__ grad_rows,
                                                            float4* __restrict__ view_rows,
                                                            const uint32_t* __restrict__ ok) {
    __shared__ float4 vcache4[3 * kTile * kTile];
    __shared__ float vcache1[3 * kTile * kTile];
    if (!batch_ok(ok)) return;
    int v, px, py;
    if (!tile_pixel(views, nviews, v, px, py)) return;
    const BatchView& bv = views[v];
    if (bv.grad_slot < 0 || bv.dimage == nullptr) return;
    float4* rows = SCREEN ? view_rows + 2 * bv.vert_base : grad_rows + 2 * bv.grad_base;
    if constexpr (SCREEN) {
        OrderedRowsSmem acc{rows, vcache4 + threadIdx.x, vcache1 + threadIdx.x, kTile * kTile};
        adjoint_pixel<OrderedRowsSmem, SCREEN>(px, py, offsets + bv.pix_base, records, bv.faces, vgeo + bv.vert_base,
                                           bv.colors, int(bv.W), bv.cam, sh, bv.dimage, tfinal + bv.pix_base,
                                           term + bv.pix_base, acc);
    } else {
        VertCache acc{rows, vcache4 + threadIdx.x, vcache1 + threadIdx.x, kTile * kTile};
        adjoint_pixel<VertCache, SCREEN>(px, py, offsets + bv.pix_base, records, bv.faces, vgeo + bv.vert_base,
                                         bv.colors, int(bv.W), bv.cam, sh, bv.dimage, tfinal + bv.pix_base,
                                         term + bv.pix_base, acc);
    }
}

// Screen-space rows of every view with a gradient slot -> world-space rows
// of the slot (one thread per view vertex; untouched vertices skipped).
__global__ void __launch_bounds__(256) kb_view_rows(const BatchView* __restrict__ views, int nviews, u64 total,
                                                    const VGeo* __restrict__ vgeo,
                                                    const float4* __restrict__ view_rows,
                                                    float4* __restrict__ grad_rows, const uint32_t* __restrict__ ok) {
    if (!batch_ok(ok)) return;
    const u64 first = u64(blockIdx.x) * blockDim.x;
    const u64 g = first + threadIdx.x;
    if (g >= total) return;
    const int v = view_of_item(g, first, nviews, [&](int i) { return views[i].vert_base; });
    const BatchView& bv = views[v];
    if (bv.grad_slot < 0 || bv.dimage == nullptr) return;
    const float4 a = view_rows[2 * g], c = view_rows[2 * g + 1];
    if (a.x == 0.f && a.y == 0.f && a.z == 0.f && c.x == 0.f && c.y == 0.f && c.z == 0.f && c.w == 0.f) return;
    const float3 w = screen_to_world(a, vgeo[g], bv.cam);
    float4* row = grad_rows + 2 * (bv.grad_base + (g - bv.vert_base));
    atomicAdd(row, make_float4(w.x, w.y, w.z, 0.f));
    atomicAdd(row + 1, c);
}

// Adds each slot's accumulated rows into its gradient buffers.
__global__ void __launch_bounds__(256) kb_scatter(const BatchSlot* __restrict__ slots, int nslots, u64 total_rows,
                                                  const float4* __restrict__ rows) {
    for (u64 g = u64(blockIdx.x) * blockDim.x + threadIdx.x; g < total_rows; g += u64(gridDim.x) * blockDim.x) {
        const int si = find_index(g, nslots, [&](int i) { return slots[i].row_base; });
        const BatchSlot& sl = slots[si];
        const u64 v = g - sl.row_base;
        const float4 a = rows[2 * g], b = rows[2 * g + 1];
        float* gp = sl.grad_pos + 3 * v;
        gp[0] += a.x;
        gp[1] += a.y;
        gp[2] += a.z;
        const float4 c = sl.grad_col[v];
        sl.grad_col[v] = make_float4(c.x + b.x, c.y + b.y, c.z + b.z, c.w + b.w);
    }
}

struct AdamConst {
    float lr_pos, lr_col, b1, b2, eps;
    int clamp_colors;      // 0 none, 1 max(.,0) (train.py:352-356), 2 rgb [0,1] alpha >= 0 (Optimizer.glsl:161-167)
    int fixed_mode;        // 0 none, 1 zero boundary position gradients, 2 skip boundary positions
};

__device__ __forceinline__ float adam_update(float p, float g, float& m, float& v, float lr, const AdamConst& a,
                                             float bc1, float sbc2) {
    m = a.b1 * m + (1.f - a.b1) * g;
    v = a.b2 * v + (1.f - a.b2) * g * g;
    return p - (lr / bc1) * (m / (sqrtf(v) / sbc2 + a.eps));
}

// Adam on every mesh's positions and colours straight from the gradient rows
// (one thread per vertex; the step counter lives on the device so a captured
// graph replays with the right bias correction).
__global__ void __launch_bounds__(256) kb_adam_rows(const BatchSlot* __restrict__ slots, int nslots, u64 total_rows,
                                                    const float4* __restrict__ rows, AdamConst a,
                                                    const int* __restrict__ step, const uint32_t* __restrict__ ok) {
    if (!batch_ok(ok)) return;
    const float t = float(*step + 1);
    const float bc1 = 1.f - powf(a.b1, t);
    const float sbc2 = sqrtf(1.f - powf(a.b2, t));
    for (u64 g = u64(blockIdx.x) * blockDim.x + threadIdx.x; g < total_rows; g += u64(gridDim.x) * blockDim.x) {
        const int si = find_index(g, nslots, [&](int i) { return slots[i].row_base; });
        const BatchSlot& sl = slots[si];
        const u64 v = g - sl.row_base;
        float4 gp = rows[2 * g];
        const float4 gc = rows[2 * g + 1];
        const bool fixed = a.fixed_mode != 0 && sl.boundary != nullptr && sl.boundary[v] != 0u;
        if (!(fixed && a.fixed_mode == 2)) {
            if (fixed) gp = make_float4(0.f, 0.f, 0.f, 0.f);
            float* p = sl.pos + 3 * v;
            float* m = sl.m_pos + 3 * v;
            float* w = sl.v_pos + 3 * v;
            const float g3[3] = {gp.x, gp.y, gp.z};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float mk = m[k], wk = w[k];
                p[k] = adam_update(p[k], g3[k], mk, wk, a.lr_pos, a, bc1, sbc2);
                m[k] = mk;
                w[k] = wk;
            }
        }
        float4 c = sl.col[v], mc = sl.m_col[v], vc = sl.v_col[v];
        c.x = adam_update(c.x, gc.x, mc.x, vc.x, a.lr_col, a, bc1, sbc2);
        c.y = adam_update(c.y, gc.y, mc.y, vc.y, a.lr_col, a, bc1, sbc2);
        c.z = adam_update(c.z, gc.z, mc.z, vc.z, a.lr_col, a, bc1, sbc2);
        c.w = adam_update(c.w, gc.w, mc.w, vc.w, a.lr_col, a, bc1, sbc2);
        if (a.clamp_colors == 1) {
            c = make_float4(fmaxf(c.x, 0.f), fmaxf(c.y, 0.f), fmaxf(c.z, 0.f), fmaxf(c.w, 0.f));
        } else if (a.clamp_colors == 2) {
            c = make_float4(fminf(fmaxf(c.x, 0.f), 1.f), fminf(fmaxf(c.y, 0.f), 1.f), fminf(fmaxf(c.z, 0.f), 1.f),
                            fmaxf(c.w, 0.f));
        }
        sl.col[v] = c;
        sl.m_col[v] = mc;
        sl.v_col[v] = vc;
    }
}

__global__ void kb_step_increment(int* __restrict__ step, const uint32_t* __restrict__ ok) {
    if (batch_ok(ok)) *step += 1;
}

static unsigned grid_for(u64 n, unsigned threads, unsigned cap_blocks) {
    u64 b = (n + threads - 1) / threads;
    if (b == 0) b = 1;
    return unsigned(b < cap_blocks ? b : cap_blocks);
}

}  // namespace dtv

using namespace dtv_host;
using dtv::BatchSlot;
using dtv::BatchView;

struct dtv_batch {
    struct MeshEntry {
        const dtv_mesh* mesh = nullptr;
        float* pos = nullptr;
        float* col = nullptr;
        uint64_t V = 0, F = 0;
        const uint4* faces = nullptr;
        const uint32_t* boundary = nullptr;
        // training state (allocated on the first train step)
        DevBuf<float> m_pos, v_pos;
        DevBuf<float4> m_col, v_col;
    };
    std::vector<MeshEntry> meshes;
    // per-batch scratch
    DevBuf<BatchView> d_views;
    DevBuf<BatchSlot> d_slots;
    BatchView* h_views = nullptr;    // pinned staging
    BatchSlot* h_slots = nullptr;
    size_t h_views_cap = 0, h_slots_cap = 0;
    cudaEvent_t staging_free = nullptr;
    DevBuf<float4> vproj;
    DevBuf<int2> vfix;
    DevBuf<dtv::VGeo> vgeo;
    DevBuf<uint32_t> counts;
    DevBuf<u64> offsets;
    DevBuf<u64> records;
    DevBuf<u64> scan;
    DevBuf<float> tfinal;
    DevBuf<uint32_t> term;
    DevBuf<uint32_t> long_list;
    DevBuf<uint32_t> ok;
    DevBuf<u64> total;
    DevBuf<float4> grad_rows;
    DevBuf<uint32_t> fill_order;    // items (view faces) in row-band order for the fill
    DevBuf<uint32_t> band_scratch;  // band counts and cursors of fill_order
    DevBuf<uint32_t> wide_list;     // [0] = n, then the items of the 64-bit raster path (count -> fill)
    DevBuf<float4> view_rows;  // [tot_verts][2]: screen-space adjoint rows of each view (at its vert_base)
    DevBuf<float4> dimage_internal;
    DevBuf<float> loss;
    DevBuf<int> step;
    uint32_t* h_ok = nullptr;        // pinned
    u64* h_total = nullptr;
    // shapes of the last render (for the adjoint)
    int nviews = 0;
    u64 tot_verts = 0, tot_faces = 0, tot_pixels = 0, tot_tiles = 0, tot_rows = 0;
    uint32_t max_height = 0;  // tallest view (grid of the count's row prefix)
    dtv::ShadeDev sh{};
    bool have_render = false;
    u64 last_fragments = 0;
    // graph
    bool use_graph = false;
    cudaGraphExec_t exec = nullptr;
    std::vector<u64> graph_sig;
    u64 capacity = 0;
    uint64_t steps_rerun = 0;
    uint32_t sort_surrogate_classes = dtv::kSortSurrogateDefault;
    uint32_t sort_bucket_classes = dtv::kSortBucketDefault;
    bool async_render = false;  // last render enqueued without a host sync (capacity-guarded)
};

namespace {

void ensure_pinned(void** p, size_t& cap, size_t bytes) {
    if (*p && cap >= bytes) return;
    if (*p) DTV_CK(cudaFreeHost(*p));
    *p = nullptr;
    DTV_CK(cudaMallocHost(p, bytes));
    cap = bytes;
}

// Builds the descriptor table for `views`; returns the totals.
void build_views(dtv_batch* b, int nviews, const dtv_batch_view* views, bool train, bool internal_dimage) {
    require(nviews > 0, "need at least one view");
    ensure_pinned(reinterpret_cast<void**>(&b->h_views), b->h_views_cap, sizeof(BatchView) * size_t(nviews));
    if (b->staging_free) DTV_CK(cudaEventSynchronize(b->staging_free));
    u64 vb = 0, fb = 0, pb = 0, tb = 0;
    for (int i = 0; i < nviews; ++i) {
        const dtv_batch_view& in = views[i];
        require(in.mesh >= 0 && in.mesh < int(b->meshes.size()), "view mesh index out of range");
        const auto& me = b->meshes[size_t(in.mesh)];
        const dtv_camera& c = in.camera;
        require(c.width > 0 && c.height > 0 && c.width <= 16384 && c.height <= 16384, "viewport size out of range");
        require(c.znear > 0.f && c.zfar > c.znear, "need 0 < znear < zfar");
        require(c.fovy > 0.f && c.fovy < 3.14159f, "fovy must be in (0, pi)");
        require(in.d_image != nullptr && (reinterpret_cast<uintptr_t>(in.d_image) & 15u) == 0,
                "d_image must be non-null and 16-byte aligned");
        BatchView bv{};
        bv.cam = dtv::camera_constants(c);
        bv.faces = me.faces;
        bv.positions = me.pos;
        bv.colors = reinterpret_cast<const float4*>(me.col);
        bv.image = reinterpret_cast<float4*>(in.d_image);
        bv.target = reinterpret_cast<const float4*>(in.d_target);
        bv.dimage = reinterpret_cast<float4*>(in.d_image_adjoint);
        bv.V = uint32_t(me.V);
        bv.F = uint32_t(me.F);
        bv.W = uint32_t(c.width);
        bv.H = uint32_t(c.height);
        bv.tiles_x = uint32_t((c.width + dtv::kTile - 1) / dtv::kTile);
        bv.vert_base = vb;
        bv.face_base = fb;
        bv.pix_base = pb;
        bv.tile_base = tb;
        bv.grad_slot = train ? in.mesh : in.grad_slot;
        bv.loss_scale = 1.0f / float(4.0 * double(c.width) * double(c.height));
        vb += me.V;
        fb += me.F;
        pb += u64(c.width) * u64(c.height);
        tb += u64(bv.tiles_x) * u64((c.height + dtv::kTile - 1) / dtv::kTile);
        b->h_views[i] = bv;
    }
    (void)internal_dimage;
    require(vb < (u64(1) << 32), "a batch holds fewer than 2^32 vertices in total");
    require(fb < (u64(1) << 32), "a batch holds fewer than 2^32 faces in total");
    b->nviews = nviews;
    b->tot_verts = vb;
    b->tot_faces = fb;
    b->tot_pixels = pb;
    b->tot_tiles = tb;
    uint32_t mh = 0;
    for (int i = 0; i < nviews; ++i) mh = std::max(mh, b->h_views[i].H);
    b->max_height = mh;
}

void ensure_scratch(dtv_batch* b, cudaStream_t s) {
    b->d_views.ensure(size_t(b->nviews), s);
    b->vproj.ensure(b->tot_verts ? b->tot_verts : 1, s);
    b->vfix.ensure(b->tot_verts ? b->tot_verts : 1, s);
    b->vgeo.ensure(b->tot_verts ? b->tot_verts : 1, s);
    b->view_rows.ensure(2 * (b->tot_verts ? b->tot_verts : 1), s);
    b->fill_order.ensure(b->tot_faces ? b->tot_faces : 1, s);
    b->band_scratch.ensure(2 * dtv::kFillBands, s);
    b->wide_list.ensure(b->tot_faces + 1, s);
    b->counts.ensure(b->tot_pixels, s, /*zero_new=*/true);
    b->offsets.ensure(b->tot_pixels + 1, s);
    b->scan.ensure(dtv::scan_scratch_elems(b->tot_pixels), s);
    b->tfinal.ensure(b->tot_pixels, s);
    b->term.ensure(b->tot_pixels, s);
    b->long_list.ensure(dtv::sort_scratch_elems(b->tot_pixels), s);
    b->ok.ensure(1, s);
    b->total.ensure(1, s);
    b->loss.ensure(1, s);
    if (!b->h_ok) {
        DTV_CK(cudaMallocHost(&b->h_ok, sizeof(uint32_t)));
        DTV_CK(cudaMallocHost(&b->h_total, sizeof(u64)));
        DTV_CK(cudaEventCreateWithFlags(&b->staging_free, cudaEventDisableTiming));
    }
}

void upload_views(dtv_batch* b, cudaStream_t s) {
    DTV_CK(cudaMemcpyAsync(b->d_views.ptr, b->h_views, sizeof(BatchView) * size_t(b->nviews), cudaMemcpyHostToDevice,
                           s));
    DTV_CK(cudaEventRecord(b->staging_free, s));
}

// Count (FILL false) or fill pass over every view's faces: the 32-bit faces,
// then the 64-bit ones (kb_raster); the count's difference arrays are then
// summed along each view's rows (kb_row_prefix).
template <bool FILL>
void launch_kb_raster(dtv_batch* b, const uint32_t* okp, cudaStream_t s) {
    using namespace dtv;
    const unsigned blocks = grid_for(b->tot_faces, 128, 0x7fffffffu);
    const uint32_t* order = nullptr;
    if (FILL && b->tot_faces) {
        const unsigned ob = grid_for(b->tot_faces, 256, 0x7fffffffu);
        DTV_CK(cudaMemsetAsync(b->band_scratch.ptr, 0, kFillBands * sizeof(uint32_t), s));
        kb_band_count<<<ob, 256, 0, s>>>(b->d_views.ptr, b->nviews, b->tot_faces, b->vfix.ptr, b->offsets.ptr,
                                         b->tot_pixels, b->band_scratch.ptr);
        launch_band_scan(b->band_scratch.ptr, b->band_scratch.ptr + kFillBands, s);
        kb_band_scatter<<<ob, 256, 0, s>>>(b->d_views.ptr, b->nviews, b->tot_faces, b->vfix.ptr, b->offsets.ptr,
                                           b->tot_pixels, b->band_scratch.ptr + kFillBands, b->fill_order.ptr);
        order = b->fill_order.ptr;
    }
    // The count lists the 64-bit items; the 64-bit count and the fill that
    // follows walk that list instead of setting up every item again.
    if (!FILL) DTV_CK(cudaMemsetAsync(b->wide_list.ptr, 0, sizeof(uint32_t), s));
    kb_raster<FILL, false><<<blocks, 128, 0, s>>>(b->d_views.ptr, b->nviews, b->tot_faces, b->vproj.ptr,
                                                  b->vfix.ptr, b->counts.ptr, FILL ? b->offsets.ptr : nullptr,
                                                  FILL ? b->records.ptr : nullptr, okp, order,
                                                  FILL ? nullptr : b->wide_list.ptr);
    kb_raster_listed<FILL><<<148, 128, 0, s>>>(b->d_views.ptr, b->nviews, b->vproj.ptr, b->vfix.ptr, b->counts.ptr,
                                               FILL ? b->offsets.ptr : nullptr, FILL ? b->records.ptr : nullptr, okp,
                                               b->wide_list.ptr);
    if (!FILL) {
        dim3 grid(unsigned(b->max_height + 7) / 8, unsigned(b->nviews));
        kb_row_prefix<<<grid, 256, 0, s>>>(b->d_views.ptr, b->counts.ptr);
    }
}

// Adjoint of every view with a gradient slot into the slots' rows (which the
// caller has cleared): screen-space view rows projected per vertex, or
// world-space rows directly for absolute-value gradients.
void enqueue_adjoint(dtv_batch* b, const dtv::ShadeDev& sh, const uint32_t* okp, cudaStream_t s) {
    using namespace dtv;
    if (sh.use_abs_grad) {
        kb_adjoint<false><<<unsigned(b->tot_tiles), kTile * kTile, 0, s>>>(
            b->d_views.ptr, b->nviews, b->offsets.ptr, b->records.ptr, b->vgeo.ptr, sh, b->tfinal.ptr, b->term.ptr,
            b->grad_rows.ptr, b->view_rows.ptr, okp);
        return;
    }
    DTV_CK(cudaMemsetAsync(b->view_rows.ptr, 0, sizeof(float4) * 2 * size_t(b->tot_verts), s));
    kb_adjoint<true><<<unsigned(b->tot_tiles), kTile * kTile, 0, s>>>(
        b->d_views.ptr, b->nviews, b->offsets.ptr, b->records.ptr, b->vgeo.ptr, sh, b->tfinal.ptr, b->term.ptr,
        b->grad_rows.ptr, b->view_rows.ptr, okp);
    kb_view_rows<<<grid_for(b->tot_verts, 256, 0x7fffffffu), 256, 0, s>>>(
        b->d_views.ptr, b->nviews, b->tot_verts, b->vgeo.ptr, b->view_rows.ptr, b->grad_rows.ptr, okp);
}

// Enqueues project, count, scan, [capacity guard], fill, sort, composite.
// With `guarded`, kernels after the scan run only if the records fit.
void enqueue_forward(dtv_batch* b, const dtv::ShadeDev& sh, bool guarded, cudaStream_t s) {
    using namespace dtv;
    const uint32_t* okp = guarded ? b->ok.ptr : nullptr;
    kb_project<<<grid_for(b->tot_verts, 256, 0x7fffffffu), 256, 0, s>>>(b->d_views.ptr, b->nviews, b->tot_verts,
                                                                        b->vproj.ptr, b->vfix.ptr, b->vgeo.ptr);
    launch_kb_raster<false>(b, nullptr, s);
    launch_scan(b->counts.ptr, b->tot_pixels, b->offsets.ptr, b->scan.ptr, s);
    if (guarded) {
        kb_check_capacity<<<1, 1, 0, s>>>(b->offsets.ptr + b->tot_pixels, b->capacity, b->ok.ptr, b->total.ptr);
        kb_clear_counts<<<grid_for(b->tot_pixels, 256, 148 * 16), 256, 0, s>>>(b->counts.ptr, b->tot_pixels, okp);
    }
    launch_kb_raster<true>(b, okp, s);
    launch_sort(b->offsets.ptr, b->records.ptr, uint32_t(b->tot_pixels), b->long_list.ptr, s, okp,
                b->sort_surrogate_classes, b->sort_bucket_classes);
    kb_composite<<<unsigned(b->tot_tiles), kTile * kTile, 0, s>>>(b->d_views.ptr, b->nviews, b->offsets.ptr,
                                                                  b->records.ptr, b->vgeo.ptr, sh, b->tfinal.ptr,
                                                                  b->term.ptr, okp);
    check_launch("batch forward");
}

}  // namespace

extern "C" {

int32_t dtv_batch_create(dtv_batch** out) {
    return guarded([&] {
        require(out != nullptr, "out is null");
        *out = new dtv_batch();
    });
}

int32_t dtv_batch_set_tuning(dtv_batch* b, const dtv_tuning* t) {
    return guarded([&] {
        require(b && t, "null pointer");
        require((t->sort_surrogate_classes & ~0x1eu) == 0 && (t->sort_bucket_classes & ~0x3eu) == 0,
                "sort class masks: surrogate bits 1..4, bucket bits 1..5");
        if ((b->sort_surrogate_classes != t->sort_surrogate_classes ||
             b->sort_bucket_classes != t->sort_bucket_classes) && b->exec) {
            // The captured step holds the old sort launches.
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
            b->graph_sig.clear();
        }
        b->sort_surrogate_classes = t->sort_surrogate_classes;
        b->sort_bucket_classes = t->sort_bucket_classes;
    });
}

int32_t dtv_batch_get_tuning(const dtv_batch* b, dtv_tuning* t) {
    return guarded([&] {
        require(b && t, "null pointer");
        *t = dtv_tuning{0, 0, b->sort_surrogate_classes, b->sort_bucket_classes};
    });
}

int32_t dtv_batch_reserve(dtv_batch* b, uint64_t max_views, uint64_t max_vertices, uint64_t max_pixels,
                          uint64_t max_fragments, uint64_t max_grad_vertices, dtv_stream stream) {
    return guarded([&] {
        require(b != nullptr, "batch is null");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t nv = size_t(max_views ? max_views : 1);
        ensure_pinned(reinterpret_cast<void**>(&b->h_views), b->h_views_cap, sizeof(BatchView) * nv);
        ensure_pinned(reinterpret_cast<void**>(&b->h_slots), b->h_slots_cap, sizeof(BatchSlot) * nv);
        b->d_views.ensure(nv, s);
        b->d_slots.ensure(nv, s);
        const u64 V = max_vertices ? max_vertices : 1, P = max_pixels ? max_pixels : 1;
        b->vproj.ensure(V, s);
        b->vfix.ensure(V, s);
        b->vgeo.ensure(V, s);
        b->view_rows.ensure(2 * V, s);
        // Fill order: a Kuhn-grid tet mesh has about 12 faces per vertex; a
        // batch with more faces grows it at its first render.
        b->fill_order.ensure(13 * V, s);
        b->band_scratch.ensure(2 * dtv::kFillBands, s);
        b->wide_list.ensure(13 * V + 1, s);
        b->counts.ensure(P, s, /*zero_new=*/true);
        b->offsets.ensure(P + 1, s);
        b->scan.ensure(dtv::scan_scratch_elems(P), s);
        b->tfinal.ensure(P, s);
        b->term.ensure(P, s);
        b->long_list.ensure(dtv::sort_scratch_elems(P), s);
        b->records.ensure(max_fragments ? max_fragments : 1, s);
        b->grad_rows.ensure(2 * (max_grad_vertices ? max_grad_vertices : 1), s);
        b->ok.ensure(1, s);
        b->total.ensure(1, s);
        b->loss.ensure(1, s);
        if (!b->h_ok) {
            DTV_CK(cudaMallocHost(&b->h_ok, sizeof(uint32_t)));
            DTV_CK(cudaMallocHost(&b->h_total, sizeof(u64)));
            DTV_CK(cudaEventCreateWithFlags(&b->staging_free, cudaEventDisableTiming));
        }
        DTV_CK(cudaStreamSynchronize(s));
    });
}

int32_t dtv_batch_destroy(dtv_batch* b) {
    if (!b) return DTV_OK;
    cudaDeviceSynchronize();
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (auto& me : b->meshes) {
        me.m_pos.release();
        me.v_pos.release();
        me.m_col.release();
        me.v_col.release();
    }
    b->d_views.release();
    b->d_slots.release();
    b->vproj.release();
    b->vfix.release();
    b->vgeo.release();
    b->counts.release();
    b->offsets.release();
    b->records.release();
    b->scan.release();
    b->tfinal.release();
    b->term.release();
    b->long_list.release();
    b->ok.release();
    b->total.release();
    b->grad_rows.release();
    b->view_rows.release();
    b->fill_order.release();
    b->band_scratch.release();
    b->wide_list.release();
    b->dimage_internal.release();
    b->loss.release();
    b->step.release();
    if (b->h_views) cudaFreeHost(b->h_views);
    if (b->h_slots) cudaFreeHost(b->h_slots);
    if (b->h_ok) cudaFreeHost(b->h_ok);
    if (b->h_total) cudaFreeHost(b->h_total);
    if (b->staging_free) cudaEventDestroy(b->staging_free);
    delete b;
    return DTV_OK;
}

int32_t dtv_batch_set_meshes(dtv_batch* b, int32_t num_meshes, const dtv_mesh* const* meshes,
                             float* const* d_positions, float* const* d_colors) {
    return guarded([&] {
        require(b && num_meshes > 0 && meshes && d_positions && d_colors, "null argument");
        std::vector<dtv_batch::MeshEntry> me;
        me.resize(static_cast<size_t>(num_meshes));
        for (int i = 0; i < num_meshes; ++i) {
            require(meshes[i] && d_positions[i] && d_colors[i], "null mesh, positions or colours");
            require((reinterpret_cast<uintptr_t>(d_colors[i]) & 15u) == 0, "colours must be 16-byte aligned");
            const dtv::MeshView mv = dtv::mesh_view(meshes[i]);
            me[size_t(i)].mesh = meshes[i];
            me[size_t(i)].pos = d_positions[i];
            me[size_t(i)].col = d_colors[i];
            me[size_t(i)].V = mv.num_vertices;
            me[size_t(i)].F = mv.num_faces;
            me[size_t(i)].faces = mv.faces;
            const uint32_t* vb = nullptr;
            dtv_mesh_vertex_boundary_device(meshes[i], &vb);
            me[size_t(i)].boundary = vb;
        }
        // Keep the optimizer state of meshes that stay (same handle and pointers).
        for (size_t i = 0; i < me.size() && i < b->meshes.size(); ++i) {
            auto& old = b->meshes[i];
            if (old.mesh == me[i].mesh && old.pos == me[i].pos && old.col == me[i].col) {
                std::swap(me[i].m_pos, old.m_pos);
                std::swap(me[i].v_pos, old.v_pos);
                std::swap(me[i].m_col, old.m_col);
                std::swap(me[i].v_col, old.v_col);
            }
        }
        for (auto& old : b->meshes) {
            old.m_pos.release();
            old.v_pos.release();
            old.m_col.release();
            old.v_col.release();
        }
        b->meshes = std::move(me);
        if (b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        b->graph_sig.clear();
        b->have_render = false;
    });
}

int32_t dtv_batch_render(dtv_batch* b, int32_t num_views, const dtv_batch_view* views,
                         const dtv_render_params* params, dtv_stream stream) {
    return guarded([&] {
        require(b && views && params, "null argument");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        b->have_render = false;
        build_views(b, num_views, views, /*train=*/false, false);
        ensure_scratch(b, s);
        b->sh = dtv::shade_constants(*params);
        upload_views(b, s);
        // Count and scan, then size the record buffer exactly (one host sync).
        using namespace dtv;
        kb_project<<<grid_for(b->tot_verts, 256, 0x7fffffffu), 256, 0, s>>>(b->d_views.ptr, b->nviews,
                                                                            b->tot_verts, b->vproj.ptr, b->vfix.ptr,
                                                                            b->vgeo.ptr);
        launch_kb_raster<false>(b, nullptr, s);
        launch_scan(b->counts.ptr, b->tot_pixels, b->offsets.ptr, b->scan.ptr, s);
        check_launch("batch count");
        DTV_CK(cudaMemcpyAsync(b->h_total, b->offsets.ptr + b->tot_pixels, sizeof(u64), cudaMemcpyDeviceToHost, s));
        DTV_CK(cudaStreamSynchronize(s));
        const u64 nf = *b->h_total;
        if (params->fragment_budget_bytes && nf * sizeof(u64) > params->fragment_budget_bytes) {
            DTV_CK(cudaMemsetAsync(b->counts.ptr, 0, sizeof(uint32_t) * b->tot_pixels, s));
            throw DtvError(DTV_ERR_BUDGET, "batch needs " + std::to_string(nf) + " fragments, over the budget");
        }
        try {
            b->records.ensure(nf ? nf : 1, s, false, 1.25);
        } catch (...) {
            cudaMemsetAsync(b->counts.ptr, 0, sizeof(uint32_t) * b->tot_pixels, s);
            throw;
        }
        launch_kb_raster<true>(b, nullptr, s);
        launch_sort(b->offsets.ptr, b->records.ptr, uint32_t(b->tot_pixels), b->long_list.ptr, s, nullptr, b->sort_surrogate_classes, b->sort_bucket_classes);
        kb_composite<<<unsigned(b->tot_tiles), kTile * kTile, 0, s>>>(b->d_views.ptr, b->nviews, b->offsets.ptr,
                                                                      b->records.ptr, b->vgeo.ptr, b->sh,
                                                                      b->tfinal.ptr, b->term.ptr, nullptr);
        check_launch("batch render");
        b->last_fragments = nf;
        b->have_render = true;
        b->async_render = false;
    });
}

int32_t dtv_batch_render_async(dtv_batch* b, int32_t num_views, const dtv_batch_view* views,
                               const dtv_render_params* params, dtv_stream stream) {
    return guarded([&] {
        require(b && views && params, "null argument");
        if (b->records.cap == 0)
            throw DtvError(DTV_ERR_STATE, "dtv_batch_render_async needs record capacity (dtv_batch_reserve)");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        b->have_render = false;
        build_views(b, num_views, views, /*train=*/false, false);
        ensure_scratch(b, s);
        b->sh = dtv::shade_constants(*params);
        upload_views(b, s);
        b->capacity = b->records.cap;
        enqueue_forward(b, b->sh, /*guarded=*/true, s);
        DTV_CK(cudaMemcpyAsync(b->h_ok, b->ok.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        DTV_CK(cudaMemcpyAsync(b->h_total, b->total.ptr, sizeof(u64), cudaMemcpyDeviceToHost, s));
        b->have_render = true;
        b->async_render = true;
    });
}

int32_t dtv_batch_render_status(const dtv_batch* b, int32_t* fits, uint64_t* num_fragments) {
    return guarded([&] {
        require(b && fits && num_fragments, "null pointer");
        if (!b->have_render || !b->async_render)
            throw DtvError(DTV_ERR_STATE, "no dtv_batch_render_async to report on");
        *fits = *b->h_ok != 0u ? 1 : 0;
        *num_fragments = *b->h_total;
    });
}

int32_t dtv_batch_render_adjoint(dtv_batch* b, int32_t num_views, const dtv_batch_view* views, int32_t num_slots,
                                 const dtv_batch_grad_slot* slots, int32_t use_abs_grad, dtv_stream stream) {
    return guarded([&] {
        require(b && views && (num_slots == 0 || slots), "null argument");
        if (!b->have_render) throw DtvError(DTV_ERR_STATE, "dtv_batch_render_adjoint before dtv_batch_render");
        if (num_views != b->nviews) throw DtvError(DTV_ERR_ARG, "view count differs from the last dtv_batch_render");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        // Slot table: rows per slot = vertices of its mesh.
        ensure_pinned(reinterpret_cast<void**>(&b->h_slots), b->h_slots_cap,
                      sizeof(BatchSlot) * size_t(num_slots > 0 ? num_slots : 1));
        u64 rows = 0;
        std::vector<u64> slot_base;
        slot_base.resize(static_cast<size_t>(num_slots));
        for (int i = 0; i < num_slots; ++i) {
            require(slots[i].mesh >= 0 && slots[i].mesh < int(b->meshes.size()), "slot mesh index out of range");
            require(slots[i].d_grad_positions && slots[i].d_grad_colors, "null slot gradient pointer");
            require((reinterpret_cast<uintptr_t>(slots[i].d_grad_colors) & 15u) == 0,
                    "slot colour gradients must be 16-byte aligned");
            BatchSlot sl{};
            sl.row_base = rows;
            sl.V = uint32_t(b->meshes[size_t(slots[i].mesh)].V);
            sl.grad_pos = slots[i].d_grad_positions;
            sl.grad_col = reinterpret_cast<float4*>(slots[i].d_grad_colors);
            b->h_slots[i] = sl;
            slot_base[size_t(i)] = rows;
            rows += sl.V;
        }
        // Point every view with a slot at its rows (the view table lives on the device).
        DTV_CK(cudaEventSynchronize(b->staging_free));
        for (int v = 0; v < b->nviews; ++v) {
            BatchView& bv = b->h_views[v];
            bv.grad_slot = views[v].grad_slot;
            bv.dimage = reinterpret_cast<float4*>(views[v].d_image_adjoint);
            if (bv.grad_slot >= 0)
                require(bv.dimage != nullptr && (reinterpret_cast<uintptr_t>(bv.dimage) & 15u) == 0,
                        "a view with a grad slot needs a 16-byte aligned d_image_adjoint");
            const int sl = bv.grad_slot;
            if (sl >= num_slots) throw DtvError(DTV_ERR_ARG, "view grad_slot out of range");
            if (sl >= 0) {
                if (b->h_slots[sl].V != bv.V) throw DtvError(DTV_ERR_ARG, "view and its grad slot use different meshes");
                bv.grad_base = slot_base[size_t(sl)];
            }
        }
        upload_views(b, s);
        b->d_slots.ensure(size_t(num_slots > 0 ? num_slots : 1), s);
        if (num_slots > 0)
            DTV_CK(cudaMemcpyAsync(b->d_slots.ptr, b->h_slots, sizeof(BatchSlot) * size_t(num_slots),
                                   cudaMemcpyHostToDevice, s));
        b->grad_rows.ensure(2 * (rows ? rows : 1), s);
        DTV_CK(cudaMemsetAsync(b->grad_rows.ptr, 0, sizeof(float4) * 2 * size_t(rows), s));
        dtv::ShadeDev sh = b->sh;
        sh.use_abs_grad = use_abs_grad ? 1 : 0;
        using namespace dtv;
        const uint32_t* okp = b->async_render ? b->ok.ptr : nullptr;
        enqueue_adjoint(b, sh, okp, s);
        if (rows)
            kb_scatter<<<grid_for(rows, 256, 148 * 16), 256, 0, s>>>(b->d_slots.ptr, num_slots, rows,
                                                                     b->grad_rows.ptr);
        check_launch("batch adjoint");
        DTV_CK(cudaEventRecord(b->staging_free, s));
    });
}

}  // extern "C"

namespace {

void enqueue_train_body(dtv_batch* b, const dtv::AdamConst& ac, int nslots, cudaStream_t s) {
    using namespace dtv;
    enqueue_forward(b, b->sh, /*guarded=*/true, s);
    DTV_CK(cudaMemsetAsync(b->loss.ptr, 0, sizeof(float), s));
    kb_loss<<<grid_for(b->tot_pixels, 256, 148 * 8), 256, 0, s>>>(b->d_views.ptr, b->nviews, b->tot_pixels,
                                                                  b->loss.ptr, b->ok.ptr);
    DTV_CK(cudaMemsetAsync(b->grad_rows.ptr, 0, sizeof(float4) * 2 * size_t(b->tot_rows), s));
    enqueue_adjoint(b, b->sh, b->ok.ptr, s);
    kb_adam_rows<<<grid_for(b->tot_rows, 256, 148 * 16), 256, 0, s>>>(b->d_slots.ptr, nslots, b->tot_rows,
                                                                      b->grad_rows.ptr, ac, b->step.ptr, b->ok.ptr);
    kb_step_increment<<<1, 1, 0, s>>>(b->step.ptr, b->ok.ptr);
    check_launch("batch train step");
}

std::vector<u64> train_signature(const dtv_batch* b, const dtv::AdamConst& ac, int nslots) {
    std::vector<u64> sig = {u64(b->nviews), b->tot_verts, b->tot_faces, b->tot_pixels, b->tot_tiles, b->tot_rows,
                            u64(b->max_height),
                            b->capacity, u64(nslots), u64(uintptr_t(b->records.ptr)),
                            u64(uintptr_t(b->dimage_internal.ptr)), u64(uintptr_t(b->grad_rows.ptr)),
                            u64(uintptr_t(b->view_rows.ptr)), u64(uintptr_t(b->wide_list.ptr))};
    const uint32_t* shw = reinterpret_cast<const uint32_t*>(&b->sh);
    for (size_t i = 0; i < sizeof(b->sh) / 4; ++i) sig.push_back(shw[i]);
    const uint32_t* acw = reinterpret_cast<const uint32_t*>(&ac);
    for (size_t i = 0; i < sizeof(ac) / 4; ++i) sig.push_back(acw[i]);
    return sig;
}

}  // namespace

extern "C" {

int32_t dtv_batch_set_graph(dtv_batch* b, int32_t enable) {
    return guarded([&] {
        require(b != nullptr, "batch is null");
        b->use_graph = enable != 0;
        if (!b->use_graph && b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
            b->graph_sig.clear();
        }
    });
}

int32_t dtv_batch_train_step(dtv_batch* b, int32_t num_views, const dtv_batch_view* views,
                             const dtv_render_params* params, const dtv_batch_optim* opt, float* d_loss,
                             dtv_stream stream) {
    return guarded([&] {
        require(b && views && params && opt, "null argument");
        require(opt->clamp_colors >= 0 && opt->clamp_colors <= 2, "clamp_colors must be 0, 1 or 2");
        require(opt->fixed_boundary >= 0 && opt->fixed_boundary <= 2, "fixed_boundary must be 0, 1 or 2");
        cudaStream_t user = static_cast<cudaStream_t>(stream);
        b->have_render = false;
        build_views(b, num_views, views, /*train=*/true, true);
        for (int i = 0; i < num_views; ++i)
            require(views[i].d_target != nullptr, "every view of a training step needs d_target");
        ensure_scratch(b, user);
        b->sh = dtv::shade_constants(*params);
        // One gradient slot per mesh; Adam state per mesh.
        const int nslots = int(b->meshes.size());
        ensure_pinned(reinterpret_cast<void**>(&b->h_slots), b->h_slots_cap, sizeof(BatchSlot) * size_t(nslots));
        u64 rows = 0;
        std::vector<u64> mesh_rows;
        mesh_rows.resize(static_cast<size_t>(nslots));
        for (int m = 0; m < nslots; ++m) {
            auto& me = b->meshes[size_t(m)];
            if (me.m_pos.ensure(3 * me.V, user, true) | me.v_pos.ensure(3 * me.V, user, true) |
                me.m_col.ensure(me.V, user, true) | me.v_col.ensure(me.V, user, true)) {
                // fresh optimizer state
            }
            BatchSlot sl{};
            sl.row_base = rows;
            sl.V = uint32_t(me.V);
            sl.pos = me.pos;
            sl.col = reinterpret_cast<float4*>(me.col);
            sl.m_pos = me.m_pos.ptr;
            sl.v_pos = me.v_pos.ptr;
            sl.m_col = me.m_col.ptr;
            sl.v_col = me.v_col.ptr;
            sl.boundary = me.boundary;
            b->h_slots[m] = sl;
            mesh_rows[size_t(m)] = rows;
            rows += me.V;
        }
        b->tot_rows = rows;
        b->grad_rows.ensure(2 * (rows ? rows : 1), user);
        b->dimage_internal.ensure(b->tot_pixels, user);
        if (b->step.ensure(1, user, true)) {
        }
        for (int v = 0; v < b->nviews; ++v) {
            BatchView& bv = b->h_views[v];
            bv.grad_base = mesh_rows[size_t(bv.grad_slot)];
            if (!bv.dimage) bv.dimage = b->dimage_internal.ptr + bv.pix_base;
        }
        b->d_slots.ensure(size_t(nslots), user);
        dtv::AdamConst ac{opt->lr_positions, opt->lr_colors, opt->beta1, opt->beta2, opt->eps, opt->clamp_colors,
                          opt->fixed_boundary};
        // Work runs on an internal stream (graph capture is not allowed on the
        // legacy default stream), ordered after / before the caller's stream.
        static thread_local cudaStream_t ws = nullptr;
        static thread_local cudaEvent_t ev_in = nullptr, ev_out = nullptr;
        if (!ws) {
            DTV_CK(cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking));
            DTV_CK(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
            DTV_CK(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
        }
        DTV_CK(cudaEventRecord(ev_in, user));
        DTV_CK(cudaStreamWaitEvent(ws, ev_in, 0));
        auto run = [&](bool try_graph) {
            upload_views(b, ws);
            DTV_CK(cudaMemcpyAsync(b->d_slots.ptr, b->h_slots, sizeof(BatchSlot) * size_t(nslots),
                                   cudaMemcpyHostToDevice, ws));
            if (try_graph && b->use_graph && b->capacity > 0) {
                const std::vector<u64> sig = train_signature(b, ac, nslots);
                if (!b->exec || sig != b->graph_sig) {
                    if (b->exec) {
                        cudaGraphExecDestroy(b->exec);
                        b->exec = nullptr;
                    }
                    cudaGraph_t g = nullptr;
                    DTV_CK(cudaStreamBeginCapture(ws, cudaStreamCaptureModeThreadLocal));
                    try {
                        enqueue_train_body(b, ac, nslots, ws);
                    } catch (...) {
                        cudaStreamEndCapture(ws, &g);
                        if (g) cudaGraphDestroy(g);
                        throw;
                    }
                    DTV_CK(cudaStreamEndCapture(ws, &g));
                    cudaError_t e = cudaGraphInstantiate(&b->exec, g, 0);
                    cudaGraphDestroy(g);
                    if (e != cudaSuccess) {
                        b->exec = nullptr;
                        throw DtvError(DTV_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
                    }
                    b->graph_sig = sig;
                }
                DTV_CK(cudaGraphLaunch(b->exec, ws));
            } else {
                enqueue_train_body(b, ac, nslots, ws);
            }
            DTV_CK(cudaMemcpyAsync(b->h_ok, b->ok.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, ws));
            DTV_CK(cudaMemcpyAsync(b->h_total, b->total.ptr, sizeof(u64), cudaMemcpyDeviceToHost, ws));
            DTV_CK(cudaStreamSynchronize(ws));
            return *b->h_ok != 0u;
        };
        bool done = run(true);
        if (!done) {
            // Records did not fit: grow, rerun this step uncaptured, recapture next time.
            const u64 need = *b->h_total;
            b->capacity = u64(double(need) * 1.25) + 1024;
            b->records.ensure(b->capacity, ws);
            b->capacity = b->records.cap;
            if (b->exec) {
                cudaGraphExecDestroy(b->exec);
                b->exec = nullptr;
            }
            b->graph_sig.clear();
            if (b->last_fragments != 0) b->steps_rerun++;
            done = run(false);
            if (!done) throw DtvError(DTV_ERR_STATE, "batch records overflowed after resizing");
        }
        b->last_fragments = *b->h_total;
        if (d_loss) DTV_CK(cudaMemcpyAsync(d_loss, b->loss.ptr, sizeof(float), cudaMemcpyDeviceToDevice, ws));
        DTV_CK(cudaEventRecord(ev_out, ws));
        DTV_CK(cudaStreamWaitEvent(user, ev_out, 0));
        b->have_render = true;
    });
}

int32_t dtv_batch_get_info(const dtv_batch* b, uint64_t* num_fragments, uint64_t* capacity, uint64_t* steps_rerun,
                           int32_t* graph_active) {
    return guarded([&] {
        require(b != nullptr, "batch is null");
        if (num_fragments) *num_fragments = b->last_fragments;
        if (capacity) *capacity = b->capacity;
        if (steps_rerun) *steps_rerun = b->steps_rerun;
        if (graph_active) *graph_active = b->exec != nullptr ? 1 : 0;
    });
}

}  // extern "C"
