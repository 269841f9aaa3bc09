// sm_100a kernels of the tetrahedral volume-rendering hot path:
//   project -> raster count -> exclusive scan -> raster fill -> per-pixel sort
//   -> front-to-back composite;  adjoint;  L2 loss;  Adam.
// The PPLL linked lists of the reference (LinkedListGather.glsl) become a
// count / prefix-scan / fill layout of 8-byte records in HBM:
//   record = (fp32 view-depth bits << 32) | (face << 2) | (boundary << 1) | front
// sorted per pixel by the 64-bit value (depth, then face index).
#include "dtv_internal.h"
#include "dtv_segment.cuh"

namespace dtv {

using u64 = unsigned long long;
constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------
// (a) vertex projection (LinkedListGather.glsl:55-68, split into view
// transform + perspective divide; FP32 with fixed rounding).
__global__ void __launch_bounds__(256) k_project(const float* __restrict__ pos, uint32_t V, CamDev cam,
                                                 float4* __restrict__ vproj, int2* __restrict__ vfix,
                                                 VGeo* __restrict__ vgeo) {
    uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    float x = pos[3 * size_t(v)], y = pos[3 * size_t(v) + 1], z = pos[3 * size_t(v) + 2];
    int2 fx;
    vproj[v] = project_vertex(cam, x, y, z, fx);
    vfix[v] = fx;
    vgeo[v] = project_vertex_geo(cam, x, y, z);
}

void launch_project(const float* pos, uint32_t V, const CamDev& cam, float4* vproj, int2* vfix, VGeo* vgeo,
                    cudaStream_t s) {
    if (V == 0) return;
    k_project<<<(V + 255) / 256, 256, 0, s>>>(pos, V, cam, vproj, vfix, vgeo);
}

// ---------------------------------------------------------------------------
// (a)+(b) face rasterisation.  One thread per face walks the pixel centres of
// the face's bounding box with incrementally updated int64 edge functions in
// 1/256-pixel fixed point.  COUNT mode increments the per-pixel counter; FILL
// mode writes the record at offsets[p] + (--counts[p]), leaving counts zeroed
// for the next render.
template <bool FILL>
__global__ void __launch_bounds__(128) k_raster(const uint4* __restrict__ faces, uint32_t F,
                                                const float4* __restrict__ vproj, const int2* __restrict__ vfix,
                                                int W, int H, uint32_t* __restrict__ counts,
                                                const u64* __restrict__ offsets, u64* __restrict__ records) {
    uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const uint4 fc = faces[f];
    const int2 q0 = vfix[fc.x], q1 = vfix[fc.y], q2 = vfix[fc.z];
    if (q0.x == kInvalidFix || q1.x == kInvalidFix || q2.x == kInvalidFix) return;
    const long long X0 = q0.x, Y0 = q0.y, X1 = q1.x, Y1 = q1.y, X2 = q2.x, Y2 = q2.y;
    const long long area2 = (X1 - X0) * (Y2 - Y0) - (Y1 - Y0) * (X2 - X0);
    if (area2 == 0) return;
    const uint32_t front = area2 < 0 ? 1u : 0u;
    const uint32_t bits = (f << 2) | ((fc.w & 1u) << 1) | front;
    long long ax0 = X0, ay0 = Y0, ax1 = X1, ay1 = Y1, ax2 = X2, ay2 = Y2;
    if (area2 < 0) {
        ax1 = X2; ay1 = Y2;
        ax2 = X1; ay2 = Y1;
    }
    const long long minX = min(X0, min(X1, X2)), maxX = max(X0, max(X1, X2));
    const long long minY = min(Y0, min(Y1, Y2)), maxY = max(Y0, max(Y1, Y2));
    const int px0 = int(max(0LL, ceil_div256(minX - 128)));
    const int px1 = int(min((long long)W - 1, floor_div256(maxX - 128)));
    const int py0 = int(max(0LL, ceil_div256(minY - 128)));
    const int py1 = int(min((long long)H - 1, floor_div256(maxY - 128)));
    if (px0 > px1 || py0 > py1) return;
    // Edges e0: a1->a2, e1: a2->a0, e2: a0->a1.
    const long long dx0 = ax2 - ax1, dy0 = ay2 - ay1;
    const long long dx1 = ax0 - ax2, dy1 = ay0 - ay2;
    const long long dx2 = ax1 - ax0, dy2 = ay1 - ay0;
    const long long Xs = 256LL * px0 + 128, Ys = 256LL * py0 + 128;
    long long E0r = dx0 * (Ys - ay1) - dy0 * (Xs - ax1);
    long long E1r = dx1 * (Ys - ay2) - dy1 * (Xs - ax2);
    long long E2r = dx2 * (Ys - ay0) - dy2 * (Xs - ax0);
    float4 va, vb, vc;
    if (FILL) {
        va = vproj[fc.x];
        vb = vproj[fc.y];
        vc = vproj[fc.z];
    }
    for (int py = py0; py <= py1; ++py) {
        long long E0 = E0r, E1 = E1r, E2 = E2r;
        for (int px = px0; px <= px1; ++px) {
            if (edge_inside(E0, dx0, dy0) && edge_inside(E1, dx1, dy1) && edge_inside(E2, dx2, dy2)) {
                const size_t p = size_t(py) * W + px;
                if (FILL) {
                    const float z = depth_key(va, vb, vc, float(px) + 0.5f, float(py) + 0.5f);
                    const uint32_t slot = atomicSub(&counts[p], 1u) - 1u;
                    records[offsets[p] + slot] = (u64(__float_as_uint(z)) << 32) | bits;
                } else {
                    atomicAdd(&counts[p], 1u);
                }
            }
            E0 -= dy0 * 256;
            E1 -= dy1 * 256;
            E2 -= dy2 * 256;
        }
        E0r += dx0 * 256;
        E1r += dx1 * 256;
        E2r += dx2 * 256;
    }
}

void launch_raster_count(const uint4* faces, uint32_t F, const float4* vproj, const int2* vfix, int W, int H,
                         uint32_t* counts, cudaStream_t s) {
    if (F == 0) return;
    k_raster<false><<<(F + 127) / 128, 128, 0, s>>>(faces, F, vproj, vfix, W, H, counts, nullptr, nullptr);
}

void launch_raster_fill(const uint4* faces, uint32_t F, const float4* vproj, const int2* vfix, int W, int H,
                        uint32_t* counts, const u64* offsets, u64* records, cudaStream_t s) {
    if (F == 0) return;
    k_raster<true><<<(F + 127) / 128, 128, 0, s>>>(faces, F, vproj, vfix, W, H, counts, offsets, records);
}

// ---------------------------------------------------------------------------
// Exclusive scan of the per-pixel counts (u32) into u64 offsets[n+1].
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr uint64_t kScanTile = uint64_t(kScanThreads) * kScanItems;

__device__ __forceinline__ u64 block_exclusive_scan(u64 v, u64* sm, u64& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    u64 x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        u64 y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sm[wid] = x;
    __syncthreads();
    if (wid == 0) {
        u64 w = lane < nw ? sm[lane] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            u64 y = __shfl_up_sync(kFull, w, o);
            if (lane >= o) w += y;
        }
        sm[lane] = w;
    }
    __syncthreads();
    const u64 prefix = wid > 0 ? sm[wid - 1] : 0ull;
    total = sm[nw - 1];
    __syncthreads();
    return prefix + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const uint32_t* __restrict__ in, uint64_t n,
                                                              u64* __restrict__ block_sums) {
    __shared__ u64 sm[32];
    const uint64_t base = uint64_t(blockIdx.x) * kScanTile + uint64_t(threadIdx.x) * kScanItems;
    u64 s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) s += in[base + k];
    u64 total;
    block_exclusive_scan(s, sm, total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_mid(u64* __restrict__ block_sums, uint64_t nb,
                                                           u64* __restrict__ out_total) {
    __shared__ u64 sm[32];
    u64 carry = 0;
    for (uint64_t start = 0; start < nb; start += kScanThreads) {
        const uint64_t i = start + threadIdx.x;
        u64 v = i < nb ? block_sums[i] : 0ull;
        u64 total;
        u64 ex = block_exclusive_scan(v, sm, total);
        if (i < nb) block_sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) *out_total = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_final(const uint32_t* __restrict__ in, uint64_t n,
                                                             const u64* __restrict__ block_offsets,
                                                             u64* __restrict__ out) {
    __shared__ u64 sm[32];
    const uint64_t base = uint64_t(blockIdx.x) * kScanTile + uint64_t(threadIdx.x) * kScanItems;
    uint32_t v[kScanItems];
    u64 s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0u;
        s += v[k];
    }
    u64 total;
    u64 run = block_exclusive_scan(s, sm, total) + block_offsets[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
}

size_t scan_scratch_elems(uint64_t n) { return size_t((n + kScanTile - 1) / kScanTile) + 1; }

void launch_scan(const uint32_t* counts, uint64_t n, u64* offsets, u64* scratch, cudaStream_t s) {
    const uint64_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 0) {
        cudaMemsetAsync(offsets, 0, sizeof(u64), s);
        return;
    }
    k_scan_reduce<<<unsigned(nb), kScanThreads, 0, s>>>(counts, n, scratch);
    k_scan_mid<<<1, kScanThreads, 0, s>>>(scratch, nb, offsets + n);
    k_scan_final<<<unsigned(nb), kScanThreads, 0, s>>>(counts, n, scratch, offsets);
}

// ---------------------------------------------------------------------------
// (c) per-pixel depth sort.  Lists of <= 32 records: one warp, one record per
// lane, bitonic network over shuffles.  Lists of <= kSortWarpCap: one warp,
// bitonic sort in shared memory.  Longer lists are queued for one block each.
__device__ __forceinline__ u64 umin64(u64 a, u64 b) { return a < b ? a : b; }
__device__ __forceinline__ u64 umax64(u64 a, u64 b) { return a < b ? b : a; }

__device__ __forceinline__ u64 bitonic32(u64 v, int lane) {
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const u64 o = __shfl_xor_sync(kFull, v, j);
            const bool up = (lane & k) == 0;
            const bool lower = (lane & j) == 0;
            v = (lower == up) ? umin64(v, o) : umax64(v, o);
        }
    }
    return v;
}

// Bitonic sort of N = 32*K records held in registers, K consecutive records
// per lane (record i lives in lane i / K, register i % K).  Stages with
// partner distance j < K stay inside a lane; the others exchange registers
// with lane ^ (j / K) through shuffles.
template <int K>
__device__ __forceinline__ void warp_sort_regs(u64 (&v)[K], int lane) {
#pragma unroll
    for (int k = 2; k <= 32 * K; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j < K) {
#pragma unroll
                for (int r = 0; r < K; ++r) {
                    const int l = r ^ j;
                    if (l > r) {
                        const int i = lane * K + r;
                        const bool up = (i & k) == 0;
                        const u64 a = v[r], b = v[l];
                        const bool sw = (a > b) == up;
                        v[r] = sw ? b : a;
                        v[l] = sw ? a : b;
                    }
                }
            } else {
                const int lm = j / K;
                const bool lower = (lane & lm) == 0;
#pragma unroll
                for (int r = 0; r < K; ++r) {
                    const int i = lane * K + r;
                    const bool up = (i & k) == 0;
                    const u64 o = __shfl_xor_sync(kFull, v[r], lm);
                    v[r] = (lower == up) ? umin64(v[r], o) : umax64(v[r], o);
                }
            }
        }
    }
}

template <int K>
__device__ __forceinline__ void warp_sort_list(u64* r, uint32_t n, int lane) {
    u64 v[K];
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const uint32_t i = uint32_t(lane) * K + q;
        v[q] = i < n ? r[i] : ~0ull;
    }
    warp_sort_regs<K>(v, lane);
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const uint32_t i = uint32_t(lane) * K + q;
        if (i < n) r[i] = v[q];
    }
}

template <bool BLOCK>
__device__ __forceinline__ void bitonic_smem(u64* s, uint32_t N, uint32_t tid, uint32_t nthr) {
    for (uint32_t k = 2; k <= N; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t t = tid; t < (N >> 1); t += nthr) {
                const uint32_t i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
                const uint32_t l = i + j;
                const bool up = (i & k) == 0;
                const u64 a = s[i], b = s[l];
                if ((a > b) == up) {
                    s[i] = b;
                    s[l] = a;
                }
            }
            if (BLOCK) __syncthreads(); else __syncwarp();
        }
    }
}

constexpr int kSortWarps = 8;

__global__ void __launch_bounds__(kSortWarps * 32) k_sort_warp(const u64* __restrict__ offsets, u64* records,
                                                                uint32_t P, uint32_t* __restrict__ long_list,
                                                                uint32_t* __restrict__ flags) {
    extern __shared__ u64 sm_sort[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t p = blockIdx.x * kSortWarps + warp;
    if (p >= P) return;
    const u64 beg = offsets[p];
    const uint32_t n = uint32_t(offsets[p + 1] - beg);
    if (n <= 1) return;
    u64* r = records + beg;
    if (n <= 32) {
        u64 v = lane < int(n) ? r[lane] : ~0ull;
        v = bitonic32(v, lane);
        if (lane < int(n)) r[lane] = v;
        return;
    }
    if (n <= 64) { warp_sort_list<2>(r, n, lane); return; }
    if (n <= 128) { warp_sort_list<4>(r, n, lane); return; }
    if (n <= 256) { warp_sort_list<8>(r, n, lane); return; }
    if (n <= 512) { warp_sort_list<16>(r, n, lane); return; }
    if (n > kSortWarpCap) {
        if (lane == 0) {
            uint32_t idx = atomicAdd(&flags[0], 1u);
            long_list[idx] = p;
        }
        return;
    }
    u64* s = sm_sort + size_t(warp) * kSortWarpCap;
    uint32_t N = 64;
    while (N < n) N <<= 1;
    for (uint32_t i = lane; i < N; i += 32) s[i] = i < n ? r[i] : ~0ull;
    __syncwarp();
    bitonic_smem<false>(s, N, lane, 32);
    for (uint32_t i = lane; i < n; i += 32) r[i] = s[i];
}

__global__ void __launch_bounds__(1024) k_sort_long(const u64* __restrict__ offsets, u64* records,
                                                    const uint32_t* __restrict__ long_list,
                                                    uint32_t* __restrict__ flags) {
    extern __shared__ u64 sm_sort[];
    const uint32_t num_long = flags[0];
    for (uint32_t li = blockIdx.x; li < num_long; li += gridDim.x) {
        const uint32_t p = long_list[li];
        const u64 beg = offsets[p];
        const uint32_t n = uint32_t(offsets[p + 1] - beg);
        if (n > kSortBlockCap) {
            if (threadIdx.x == 0) atomicExch(&flags[1], 1u);
            continue;
        }
        u64* r = records + beg;
        uint32_t N = 64;
        while (N < n) N <<= 1;
        for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) sm_sort[i] = i < n ? r[i] : ~0ull;
        __syncthreads();
        bitonic_smem<true>(sm_sort, N, threadIdx.x, blockDim.x);
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) r[i] = sm_sort[i];
        __syncthreads();
    }
}

void launch_sort(const u64* offsets, u64* records, uint32_t P, uint32_t* long_list, uint32_t* flags,
                 cudaStream_t s) {
    static bool attr_set = false;
    const size_t smem = size_t(kSortWarps) * kSortWarpCap * sizeof(u64);
    if (!attr_set) {
        cudaFuncSetAttribute(k_sort_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        cudaFuncSetAttribute(k_sort_long, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(kSortBlockCap * sizeof(u64)));
        attr_set = true;
    }
    if (P == 0) return;
    k_sort_warp<<<(P + kSortWarps - 1) / kSortWarps, kSortWarps * 32, smem, s>>>(offsets, records, P, long_list,
                                                                                 flags);
}

void launch_sort_long(const u64* offsets, u64* records, const uint32_t* long_list, uint32_t /*num_long*/,
                      uint32_t* flags, cudaStream_t s) {
    k_sort_long<<<296, 1024, kSortBlockCap * sizeof(u64), s>>>(offsets, records, long_list, flags);
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
constexpr int kTile = 16;

__global__ void __launch_bounds__(kTile * kTile) k_composite(
    const u64* __restrict__ offsets, const u64* __restrict__ records, const uint4* __restrict__ faces,
    const VGeo* __restrict__ vgeo, const float4* __restrict__ colors, int W, int H, ShadeDev sh,
    float4* __restrict__ image, float* __restrict__ tfinal, uint32_t* __restrict__ term) {
    const int px = blockIdx.x * kTile + (threadIdx.x % kTile);
    const int py = blockIdx.y * kTile + (threadIdx.x / kTile);
    if (px >= W || py >= H) return;
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

void launch_composite(const u64* offsets, const u64* records, const uint4* faces, const VGeo* vgeo,
                      const float4* colors, int W, int H, const ShadeDev& sh, float4* image, float* tfinal,
                      uint32_t* term, cudaStream_t s) {
    dim3 grid((W + kTile - 1) / kTile, (H + kTile - 1) / kTile);
    k_composite<<<grid, kTile * kTile, 0, s>>>(offsets, records, faces, vgeo, colors, W, H, sh, image, tfinal,
                                               term);
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
    const float invA = 1.0f / fi.A;
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
                if (a > 0.f) {
                    const SegTerms st = seg_terms(tSeg, a);
                    const float cx = st.omA * c0.x + st.K * (c0.x - c1.x);
                    const float cy = st.omA * c0.y + st.K * (c0.y - c1.y);
                    const float cz = st.omA * c0.z + st.K * (c0.z - c1.z);
                    const float Tin = T / st.A;
                    const float gax = Tin * gC0, gay = Tin * gC1, gaz = Tin * gC2;
                    const float gA = Tin * gT;
                    gT = (gC0 * cx + gC1 * cy + gC2 * cz) + gT * st.A;
                    T = Tin;
                    const float aA = a * st.A;
                    g_t = gax * (aA * (c0.x + tSeg * (c1.x - c0.x))) + gay * (aA * (c0.y + tSeg * (c1.y - c0.y))) +
                          gaz * (aA * (c0.z + tSeg * (c1.z - c0.z))) - gA * aA;
                    const float dK = seg_dK_da(tSeg, a, st);
                    const float tA = tSeg * st.A;
                    g_a = gax * (tA * c0.x + dK * (c0.x - c1.x)) + gay * (tA * c0.y + dK * (c0.y - c1.y)) +
                          gaz * (tA * c0.z + dK * (c0.z - c1.z)) - gA * tA;
                    const float k0 = st.omA + st.K;
                    gc0x = k0 * gax; gc0y = k0 * gay; gc0z = k0 * gaz;
                    gc1x = -st.K * gax; gc1y = -st.K * gay; gc1z = -st.K * gaz;
                } else {
                    // The forward drops the sub-segment for a <= 0; the gradient
                    // is the a -> 0+ limit (BackwardCommon.glsl:121-125) so a
                    // density clamped at zero can grow again.
                    const float gax = T * gC0, gay = T * gC1, gaz = T * gC2, gA = T * gT;
                    g_t = 0.f;
                    g_a = gax * (tSeg * c0.x + 0.5f * tSeg * tSeg * (c1.x - c0.x)) +
                          gay * (tSeg * c0.y + 0.5f * tSeg * tSeg * (c1.y - c0.y)) +
                          gaz * (tSeg * c0.z + 0.5f * tSeg * tSeg * (c1.z - c0.z)) - gA * tSeg;
                    gc0x = gc0y = gc0z = gc1x = gc1y = gc1z = 0.f;
                }
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


__global__ void __launch_bounds__(kTile * kTile) k_adjoint(
    const u64* __restrict__ offsets, const u64* __restrict__ records, const uint4* __restrict__ faces,
    const VGeo* __restrict__ vgeo, const float4* __restrict__ colors, int W, int H, CamDev cam, ShadeDev sh,
    const float4* __restrict__ dimage, const float* __restrict__ tfinal, const uint32_t* __restrict__ term,
    float4* __restrict__ grad_rows) {
    const int px = blockIdx.x * kTile + (threadIdx.x % kTile);
    const int py = blockIdx.y * kTile + (threadIdx.x / kTile);
    if (px >= W || py >= H) return;
    adjoint_pixel(px, py, offsets, records, faces, vgeo, colors, W, cam, sh, dimage, tfinal, term,
                  GradAcc{grad_rows});
}

// Adds the interleaved rows into the caller's gradient buffers.
__global__ void __launch_bounds__(256) k_scatter_grads(const float4* __restrict__ rows, uint32_t V,
                                                       float* __restrict__ grad_pos,
                                                       float4* __restrict__ grad_col) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const float4 a = rows[2 * size_t(v)], b = rows[2 * size_t(v) + 1];
    float* gp = grad_pos + 3 * size_t(v);
    gp[0] += a.x;
    gp[1] += a.y;
    gp[2] += a.z;
    float4 c = grad_col[v];
    grad_col[v] = make_float4(c.x + b.x, c.y + b.y, c.z + b.z, c.w + b.w);
}

void launch_adjoint(const u64* offsets, const u64* records, const uint4* faces, const VGeo* vgeo,
                    const float4* colors, const CamDev& cam, const ShadeDev& sh, const float4* dimage,
                    const float* tfinal, const uint32_t* term, uint32_t V, float4* grad_rows, float* grad_pos,
                    float4* grad_col, cudaStream_t s) {
    cudaMemsetAsync(grad_rows, 0, sizeof(float4) * 2 * size_t(V), s);
    dim3 grid((cam.W + kTile - 1) / kTile, (cam.H + kTile - 1) / kTile);
    k_adjoint<<<grid, kTile * kTile, 0, s>>>(offsets, records, faces, vgeo, colors, cam.W, cam.H, cam, sh, dimage,
                                             tfinal, term, grad_rows);
    if (V) k_scatter_grads<<<(V + 255) / 256, 256, 0, s>>>(grad_rows, V, grad_pos, grad_col);
}

// ---------------------------------------------------------------------------
// L2 loss and its image adjoint (Data/Shaders/Optimizer/Loss.glsl:242-248;
// torch.nn.MSELoss in pytests/train.py:321-326): adjoint = 2 * scale * (x - y),
// loss += scale * sum (x - y)^2.
__global__ void __launch_bounds__(256) k_loss_l2(const float* __restrict__ img, const float* __restrict__ tgt,
                                                 uint64_t n, float scale, float* __restrict__ adj,
                                                 float* __restrict__ loss) {
    __shared__ float sm[8];
    float acc = 0.f;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const float d = img[i] - tgt[i];
        if (adj) adj[i] = 2.f * scale * d;
        acc += d * d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
        if (threadIdx.x == 0 && loss) atomicAdd(loss, scale * v);
    }
}

void launch_loss_l2(const float* image, const float* target, uint64_t n, float scale, float* adjoint,
                    float* loss_accum, cudaStream_t s) {
    if (n == 0) return;
    uint64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_loss_l2<<<unsigned(blocks), 256, 0, s>>>(image, target, n, scale, adjoint, loss_accum);
}

// ---------------------------------------------------------------------------
// (g) Adam (torch.optim.Adam as used by pytests/train.py:318; the same update
// as Data/Shaders/Optimizer/Optimizer.glsl:147-168).
//   fixed mode 1: zero the gradient of fixed entries (train.py:349-350)
//   fixed mode 2: leave fixed entries untouched (Optimizer.glsl:141-145)
//   clamp mode 1: p = max(p, 0) (train.py:352-356)
//   clamp mode 2: rgb in [0,1], alpha >= 0 for stride-4 colours (Optimizer.glsl:161-167)
__global__ void __launch_bounds__(256) k_adam(float* __restrict__ param, const float* __restrict__ grad,
                                              float* __restrict__ m, float* __restrict__ v, uint64_t n, float lr,
                                              float b1, float b2, float eps, float bc1, float bc2, int clamp_mode,
                                              const uint32_t* __restrict__ fixed_mask, int fixed_mode, int stride) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        float g = grad[i];
        if (fixed_mask && fixed_mode != 0 && fixed_mask[i / uint64_t(stride)] != 0u) {
            if (fixed_mode == 2) continue;
            g = 0.f;
        }
        const float mt = b1 * m[i] + (1.f - b1) * g;
        const float vt = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mt;
        v[i] = vt;
        const float denom = sqrtf(vt) / sqrtf(bc2) + eps;
        float p = param[i] - (lr / bc1) * (mt / denom);
        if (clamp_mode == 1) {
            p = fmaxf(p, 0.f);
        } else if (clamp_mode == 2) {
            p = (i % 4 == 3) ? fmaxf(p, 0.f) : fminf(fmaxf(p, 0.f), 1.f);
        }
        param[i] = p;
    }
}

void launch_adam(float* param, const float* grad, float* m, float* v, uint64_t n, float lr, float beta1,
                 float beta2, float eps, float bc1, float bc2, int clamp_mode, const uint32_t* fixed_mask,
                 int fixed_mode, int stride, cudaStream_t s) {
    if (n == 0) return;
    uint64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_adam<<<unsigned(blocks), 256, 0, s>>>(param, grad, m, v, n, lr, beta1, beta2, eps, bc1, bc2, clamp_mode,
                                            fixed_mask, fixed_mask ? fixed_mode : 0, stride > 0 ? stride : 1);
}

}  // namespace dtv
