// sm_100a kernels of the tetrahedral volume-rendering hot path:
//   project -> raster count -> exclusive scan -> raster fill -> per-pixel sort
//   -> front-to-back composite;  adjoint;  L2 loss;  Adam.
// The PPLL linked lists of the reference (LinkedListGather.glsl) become a
// count / prefix-scan / fill layout of 8-byte records in HBM:
//   record = (fp32 view-depth bits << 32) | (face << 2) | (boundary << 1) | front
// sorted per pixel by the 64-bit value (depth, then face index).
#include <algorithm>
#include "dtv_internal.h"
#include "dtv_path.cuh"

namespace dtv {

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
    vgeo[v] = project_vertex_geo(cam, x, y, z, fx);
}

void launch_project(const float* pos, uint32_t V, const CamDev& cam, float4* vproj, int2* vfix, VGeo* vgeo,
                    cudaStream_t s) {
    if (V == 0) return;
    k_project<<<(V + 255) / 256, 256, 0, s>>>(pos, V, cam, vproj, vfix, vgeo);
}

// (a)+(b) face rasterisation: 32 faces per warp, the warp's lanes spread over
// each face's pixels in turn (raster_warp, dtv_path.cuh).
constexpr int kRasterWarps = 4;

template <bool FILL, bool WIDE>
__global__ void __launch_bounds__(32 * kRasterWarps) k_raster(const uint4* __restrict__ faces, uint32_t F,
                                                              const float4* __restrict__ vproj,
                                                              const int2* __restrict__ vfix, int W, int row0, int row1,
                                                              uint32_t* __restrict__ counts,
                                                              const u64* __restrict__ offsets,
                                                              u64* __restrict__ records,
                                                              const uint32_t* __restrict__ order,
                                                              uint32_t* __restrict__ wide_list) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t f = (order && i < F) ? order[i] : i;
    RasterJob J;
    const bool set = i < F && raster_setup(f, faces, vfix, 0u, W, row0, row1, 0ull, J);
    const bool live = set && (J.wide != 0) == WIDE;
    if constexpr (!FILL) {
        if (live) count_face<typename std::conditional<WIDE, long long, int>::type>(J, counts);
        if (!WIDE && wide_list) {
            // The faces of the 64-bit path, for its count and fill launches
            // (wide_list[0] = how many, then the face ids).
            const bool wide = set && J.wide != 0;
            const unsigned m = __ballot_sync(kFull, wide);
            if (m) {
                const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
                uint32_t base = 0;
                if (lane == leader) base = atomicAdd(wide_list, uint32_t(__popc(m)));
                base = __shfl_sync(kFull, base, leader);
                if (wide) wide_list[1 + base + __popc(m & ((1u << lane) - 1u))] = f;
            }
        }
    } else {
        __shared__ RasterJob jobs[kRasterWarps][32];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (live) jobs[w][lane] = J;
        raster_warp<FILL, WIDE>(jobs[w], __ballot_sync(kFull, live), lane, vproj, counts, offsets, records);
    }
}

// The 64-bit faces listed by the count (wide_list), 32 per warp and step over
// a fixed grid: the count (one thread per face) or the fill (raster_warp).
template <bool FILL>
__global__ void __launch_bounds__(32 * kRasterWarps) k_raster_listed(const uint4* __restrict__ faces,
                                                                     const float4* __restrict__ vproj,
                                                                     const int2* __restrict__ vfix, int W, int row0,
                                                                     int row1, uint32_t* __restrict__ counts,
                                                                     const u64* __restrict__ offsets,
                                                                     u64* __restrict__ records,
                                                                     const uint32_t* __restrict__ wide_list) {
    __shared__ RasterJob jobs[kRasterWarps][32];
    const uint32_t n = wide_list[0];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + uint32_t(w) * 32u; base < n; base += stride) {
        const uint32_t i = base + uint32_t(lane);
        RasterJob J;
        const bool live = i < n && raster_setup(wide_list[1 + i], faces, vfix, 0u, W, row0, row1, 0ull, J) &&
                          J.wide != 0;
        if constexpr (!FILL) {
            if (live) count_face<long long>(J, counts);
        } else {
            if (live) jobs[w][lane] = J;
            raster_warp<FILL, true>(jobs[w], __ballot_sync(kFull, live), lane, vproj, counts, offsets, records);
            __syncwarp();  // every lane is done with this step's jobs before the next step writes them
        }
    }
}

constexpr unsigned kListedBlocks = 148;

// Difference array of the count pass -> per-pixel counts, rows [row0, row1).
__global__ void __launch_bounds__(256) k_row_prefix(uint32_t* __restrict__ counts, int W, int row0, int row1) {
    const int row = row0 + int(blockIdx.x) * 8 + int(threadIdx.x >> 5);
    if (row < row1) row_prefix_warp(counts + size_t(row) * W, W, threadIdx.x & 31);
}

void launch_raster_count(const uint4* faces, uint32_t F, const float4* vproj, const int2* vfix, int W, int H,
                         uint32_t* counts, cudaStream_t s, int row0, int row1, uint32_t* wide_list) {
    if (F == 0) return;
    if (row1 < 0) row1 = H;
    if (row1 <= row0) return;
    const unsigned blocks = (F + 32 * kRasterWarps - 1) / (32 * kRasterWarps);
    if (wide_list) cudaMemsetAsync(wide_list, 0, sizeof(uint32_t), s);
    k_raster<false, false><<<blocks, 32 * kRasterWarps, 0, s>>>(faces, F, vproj, vfix, W, row0, row1, counts, nullptr,
                                                                nullptr, nullptr, wide_list);
    if (wide_list)
        k_raster_listed<false><<<kListedBlocks, 32 * kRasterWarps, 0, s>>>(faces, vproj, vfix, W, row0, row1, counts,
                                                                           nullptr, nullptr, wide_list);
    else
        k_raster<false, true><<<blocks, 32 * kRasterWarps, 0, s>>>(faces, F, vproj, vfix, W, row0, row1, counts,
                                                                   nullptr, nullptr, nullptr, nullptr);
    k_row_prefix<<<unsigned(row1 - row0 + 7) / 8, 256, 0, s>>>(counts, W, row0, row1);
}

void launch_raster_fill(const uint4* faces, uint32_t F, const float4* vproj, const int2* vfix, int W, int H,
                        uint32_t* counts, const u64* offsets, u64* records, cudaStream_t s, int row0, int row1,
                        const uint32_t* order, const uint32_t* wide_list) {
    if (F == 0) return;
    if (row1 < 0) row1 = H;
    const unsigned blocks = (F + 32 * kRasterWarps - 1) / (32 * kRasterWarps);
    k_raster<true, false><<<blocks, 32 * kRasterWarps, 0, s>>>(faces, F, vproj, vfix, W, row0, row1, counts, offsets,
                                                               records, order, nullptr);
    if (wide_list)
        k_raster_listed<true><<<kListedBlocks, 32 * kRasterWarps, 0, s>>>(faces, vproj, vfix, W, row0, row1, counts,
                                                                          offsets, records, wide_list);
    else
        k_raster<true, true><<<blocks, 32 * kRasterWarps, 0, s>>>(faces, F, vproj, vfix, W, row0, row1, counts,
                                                                  offsets, records, order, nullptr);
}

// ---------------------------------------------------------------------------
// Face order of the fill: faces grouped by the band of 2^shift image rows
// that holds their first covered row.  In face-index order every pixel's list
// receives records throughout the fill, so each 32-byte sector of the record
// buffer (four records) is written piecemeal and leaves L2 partly written
// (a DRAM read to merge, and the sector written again).  Band by band, the
// lists being written at any time belong to a few bands whose records fit in
// L2 until their sectors are complete.  The order within a band is arbitrary:
// the per-pixel sort makes the lists canonical.
__device__ __forceinline__ int fill_band(uint32_t f, const uint4* __restrict__ faces, const int2* __restrict__ vfix,
                                         int H, int shift) {
    const uint4 fc = faces[f];
    const int2 q0 = vfix[fc.x], q1 = vfix[fc.y], q2 = vfix[fc.z];
    if (q0.x == kInvalidFix || q1.x == kInvalidFix || q2.x == kInvalidFix) return 0;
    const long long minY = min(q0.y, min(q1.y, q2.y));
    const long long py0 = ceil_div256(minY - 128);
    return int(min((long long)H - 1, max(0LL, py0))) >> shift;
}

__global__ void __launch_bounds__(256) k_band_count(const uint4* __restrict__ faces, uint32_t F,
                                                    const int2* __restrict__ vfix, int H, int shift,
                                                    uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[kFillBands];
    for (int b = threadIdx.x; b < kFillBands; b += blockDim.x) h[b] = 0u;
    __syncthreads();
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < F) atomicAdd(&h[fill_band(f, faces, vfix, H, shift)], 1u);
    __syncthreads();
    for (int b = threadIdx.x; b < kFillBands; b += blockDim.x)
        if (h[b]) atomicAdd(&hist[b], h[b]);
}

// hist[b] -> exclusive prefix in cursor[b] (one warp).
__global__ void k_band_scan(const uint32_t* __restrict__ hist, uint32_t* __restrict__ cursor) {
    const int lane = threadIdx.x;
    uint32_t carry = 0;
    for (int b0 = 0; b0 < kFillBands; b0 += 32) {
        const uint32_t v = hist[b0 + lane];
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += t;
        }
        cursor[b0 + lane] = carry + incl - v;
        carry += __shfl_sync(kFull, incl, 31);
    }
}

__global__ void __launch_bounds__(256) k_band_scatter(const uint4* __restrict__ faces, uint32_t F,
                                                      const int2* __restrict__ vfix, int H, int shift,
                                                      uint32_t* __restrict__ cursor, uint32_t* __restrict__ order) {
    __shared__ uint32_t h[kFillBands], base[kFillBands];
    for (int b = threadIdx.x; b < kFillBands; b += blockDim.x) h[b] = 0u;
    __syncthreads();
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    int band = 0;
    uint32_t rank = 0;
    if (f < F) {
        band = fill_band(f, faces, vfix, H, shift);
        rank = atomicAdd(&h[band], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < kFillBands; b += blockDim.x)
        if (h[b]) base[b] = atomicAdd(&cursor[b], h[b]);
    __syncthreads();
    if (f < F) order[base[band] + rank] = f;
}

// Largest band of 2^shift rows whose records (nf over H rows on average) stay
// under kFillBandBytes, with at most kFillBands bands.
void launch_band_scan(const uint32_t* hist, uint32_t* cursor, cudaStream_t s) {
    k_band_scan<<<1, 32, 0, s>>>(hist, cursor);
}

int fill_band_shift(int H, uint64_t nf) {
    const double per_row = double(nf) * sizeof(u64) / double(H > 0 ? H : 1);
    int shift = 0;
    while (shift < 30 && per_row * double(2u << shift) <= double(kFillBandBytes)) ++shift;
    while (((H - 1) >> shift) >= kFillBands) ++shift;
    return shift;
}

void launch_fill_order(const uint4* faces, uint32_t F, const int2* vfix, int H, uint64_t nf, uint32_t* order,
                       uint32_t* band_scratch, cudaStream_t s) {
    if (F == 0) return;
    const int shift = fill_band_shift(H, nf);
    const unsigned blocks = (F + 255) / 256;
    cudaMemsetAsync(band_scratch, 0, kFillBands * sizeof(uint32_t), s);
    k_band_count<<<blocks, 256, 0, s>>>(faces, F, vfix, H, shift, band_scratch);
    launch_band_scan(band_scratch, band_scratch + kFillBands, s);
    k_band_scatter<<<blocks, 256, 0, s>>>(faces, F, vfix, H, shift, band_scratch + kFillBands, order);
}

// ---------------------------------------------------------------------------
// Exclusive scan of the per-pixel counts (u32) into u64 offsets[n+1].
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
static_assert(uint64_t(kScanThreads) * kScanItems == kScanTile, "scan tile and scan_scratch_elems disagree");

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

// Bitonic sort of 32 K keys of 32 bits in registers (layout as warp_sort_regs):
// each compare-exchange is one min and one max, each exchange one shuffle.
template <int K>
__device__ __forceinline__ void warp_sort_regs32(uint32_t (&v)[K], int lane) {
#pragma unroll
    for (int k = 2; k <= 32 * K; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j < K) {
#pragma unroll
                for (int r = 0; r < K; ++r) {
                    const int l = r ^ j;
                    if (l > r) {
                        const bool up = ((lane * K + r) & k) == 0;
                        const uint32_t a = v[r], b = v[l];
                        const uint32_t mn = min(a, b), mx = max(a, b);
                        v[r] = up ? mn : mx;
                        v[l] = up ? mx : mn;
                    }
                }
            } else {
                const int lm = j / K;
                const bool lower = (lane & lm) == 0;
#pragma unroll
                for (int r = 0; r < K; ++r) {
                    const bool up = ((lane * K + r) & k) == 0;
                    const uint32_t o = __shfl_xor_sync(kFull, v[r], lm);
                    v[r] = (lower == up) ? min(v[r], o) : max(v[r], o);
                }
            }
        }
    }
}

// Sort of one list of n <= 32 K records (n <= 4096) through 32-bit surrogate
// keys: (depth quantised to 20 bits over the list's depth range) << 12 | list
// index.  Quantisation is monotone, so after sorting the keys and gathering
// the records by index, only runs of equal quantised depth can be out of
// order; odd-even transposition passes on the full 64-bit records restore
// the exact (depth, face) order.  A list that is not in order after
// kFixPasses passes (e.g. all depths equal) goes to the block sort.
constexpr int kFixPasses = 16;

template <int K>
__device__ __forceinline__ bool fixup_pass(u64 (&v)[K], int lane, int parity) {
    bool swapped = false;
#pragma unroll
    for (int q = parity; q + 1 < K; q += 2) {
        if (v[q] > v[q + 1]) {
            const u64 t = v[q];
            v[q] = v[q + 1];
            v[q + 1] = t;
            swapped = true;
        }
    }
    if (parity == 1) {
        // Pair across the lane boundary: (lane, K-1) and (lane + 1, 0).
        const u64 next0 = __shfl_down_sync(kFull, v[0], 1);
        const u64 prevL = __shfl_up_sync(kFull, v[K - 1], 1);
        const bool has_next = lane < 31, has_prev = lane > 0;
        if (has_next && v[K - 1] > next0) {
            v[K - 1] = next0;
            swapped = true;
        }
        if (has_prev && prevL > v[0]) v[0] = prevL;
    }
    return swapped;
}

// Returns false when the list is not yet in order (the caller queues it for
// the block sort, which runs later on the same stream).
template <int K>
__device__ __forceinline__ bool warp_sort_list_q(u64* r, uint32_t n, int lane) {
    constexpr uint32_t kLevels = 1u << 20;
    float dmin = 3.4e38f, dmax = 0.f;
    uint32_t key[K];
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const uint32_t i = uint32_t(lane) * K + q;
        if (i < n) {
            const float d = __uint_as_float(uint32_t(r[i] >> 32));
            dmin = fminf(dmin, d);
            dmax = fmaxf(dmax, d);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dmin = fminf(dmin, __shfl_xor_sync(kFull, dmin, o));
        dmax = fmaxf(dmax, __shfl_xor_sync(kFull, dmax, o));
    }
    const float scale = dmax > dmin ? float(kLevels - 1) / (dmax - dmin) : 0.f;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const uint32_t i = uint32_t(lane) * K + q;
        if (i < n) {
            const float d = __uint_as_float(uint32_t(r[i] >> 32));
            const uint32_t qd = min(uint32_t((d - dmin) * scale), kLevels - 1u);
            key[q] = (qd << 12) | i;
        } else {
            key[q] = 0xffffffffu;
        }
    }
    warp_sort_regs32<K>(key, lane);
    u64 v[K];
#pragma unroll
    for (int q = 0; q < K; ++q) v[q] = key[q] != 0xffffffffu ? r[key[q] & 0xfffu] : ~0ull;
    bool sorted = false;
    for (int pass = 0; pass < kFixPasses; ++pass) {
        const bool s0 = fixup_pass<K>(v, lane, 0);
        const bool s1 = fixup_pass<K>(v, lane, 1);
        if (!__any_sync(kFull, s0 || s1)) {
            sorted = true;
            break;
        }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const uint32_t i = uint32_t(lane) * K + q;
        if (i < n) r[i] = v[q];
    }
    return sorted;
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

// Length classes of the per-pixel lists.  A classification pass appends each
// pixel with n >= 2 records to the list of its class (warp-aggregated
// atomics); one kernel per class then sorts its lists, so each is compiled
// with only the registers its class needs.  Class 8: lists of 2..kSortTinyMax
// records, one thread per list (sorting network in registers).  Classes 0..4:
// one warp per list, 32 K records in registers (K = 1, 2, 4, 8, 16; class 0
// from kSortTinyMax + 1 records); class 5: one warp per list, bitonic in
// shared memory (<= kSortWarpCap); class 6: one block per list
// (<= kSortBlockCap); class 7: one block per longer list, in place (merge
// stages over global memory), so no list length is refused.
// Scratch layout (u32): [0, 16) class counts, then kSortClasses lists of P.
constexpr int kSortGridBlocks = 148 * 8;
constexpr uint32_t kSortTinyMax = 8;
constexpr int kSortTinyClass = 8;

__device__ __forceinline__ int sort_class(uint32_t n) {
    if (n <= 32) return 0;
    if (n <= 64) return 1;
    if (n <= 128) return 2;
    if (n <= 256) return 3;
    if (n <= 512) return 4;
    if (n <= kSortWarpCap) return 5;
    return 6;
}

__global__ void __launch_bounds__(256) k_sort_classify(const u64* __restrict__ offsets, uint32_t P,
                                                       uint32_t* __restrict__ scratch,
                                                       const uint32_t* __restrict__ ok) {
    if (ok && *ok == 0u) return;
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    int c = -1;
    if (p < P) {
        const u64 n = offsets[p + 1] - offsets[p];
        if (n > kSortBlockCap)
            c = 7;
        else if (n > kSortTinyMax)
            c = sort_class(uint32_t(n));
        else if (n > 1)
            c = kSortTinyClass;
    }
    const unsigned act = __ballot_sync(kFull, c >= 0);
    if (c < 0) return;
    const unsigned peers = __match_any_sync(act, c);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&scratch[c], uint32_t(__popc(peers)));
    base = __shfl_sync(peers, base, leader);
    const uint32_t rank = uint32_t(__popc(peers & ((1u << lane) - 1u)));
    scratch[16 + size_t(c) * P + base + rank] = p;
}

// Class 8: one thread per list of 2..8 records.  The records (padded with
// ~0, above every record) go through Batcher's odd-even merge network for
// eight inputs (19 compare-exchanges of the 64-bit values, depth 6), and the
// first n are stored back.  Lists this short are what the ray-tet path's
// boundary lists and the silhouettes of the list path hold; one warp each
// (class 0) spends a 32-lane bitonic network on two or four records.
__device__ __forceinline__ void cmp_exch(u64& a, u64& b) {
    const u64 lo = a < b ? a : b, hi = a < b ? b : a;
    a = lo;
    b = hi;
}

__global__ void __launch_bounds__(256) k_sort_class_tiny(const u64* __restrict__ offsets, u64* records,
                                                         const uint32_t* __restrict__ items,
                                                         const uint32_t* __restrict__ count,
                                                         const uint32_t* __restrict__ ok) {
    static_assert(kSortTinyMax == 8, "the network below sorts eight values");
    if (ok && *ok == 0u) return;
    const uint32_t num = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < num; i += gridDim.x * blockDim.x) {
        const uint32_t p = items[i];
        const u64 beg = offsets[p];
        const int n = int(offsets[p + 1] - beg);
        u64* r = records + beg;
        u64 v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = q < n ? r[q] : ~0ull;
        cmp_exch(v[0], v[1]); cmp_exch(v[2], v[3]); cmp_exch(v[4], v[5]); cmp_exch(v[6], v[7]);
        cmp_exch(v[0], v[2]); cmp_exch(v[1], v[3]); cmp_exch(v[4], v[6]); cmp_exch(v[5], v[7]);
        cmp_exch(v[1], v[2]); cmp_exch(v[5], v[6]);
        cmp_exch(v[0], v[4]); cmp_exch(v[1], v[5]); cmp_exch(v[2], v[6]); cmp_exch(v[3], v[7]);
        cmp_exch(v[2], v[4]); cmp_exch(v[3], v[5]);
        cmp_exch(v[1], v[2]); cmp_exch(v[3], v[4]); cmp_exch(v[5], v[6]);
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (q < n) r[q] = v[q];
    }
}

// Classes 0..4: K records per lane in registers (K = 1: bitonic over shuffles).
template <int K, bool Q>
__global__ void __launch_bounds__(kSortWarps * 32, K >= 16 ? 2 : 1) k_sort_class_regs(const u64* __restrict__ offsets, u64* records,
                                                                     const uint32_t* __restrict__ items,
                                                                     const uint32_t* __restrict__ count,
                                                                     uint32_t* __restrict__ redo_count,
                                                                     uint32_t* __restrict__ redo_items,
                                                                     const uint32_t* __restrict__ ok) {
    if (ok && *ok == 0u) return;
    const uint32_t num = *count;
    const int lane = threadIdx.x & 31;
    for (uint32_t i = blockIdx.x * kSortWarps + (threadIdx.x >> 5); i < num; i += gridDim.x * kSortWarps) {
        const uint32_t p = items[i];
        const u64 beg = offsets[p];
        const uint32_t n = uint32_t(offsets[p + 1] - beg);
        u64* r = records + beg;
        if (K == 1) {
            u64 v = lane < int(n) ? r[lane] : ~0ull;
            v = bitonic32(v, lane);
            if (lane < int(n)) r[lane] = v;
        } else if (!Q) {
            warp_sort_list<K>(r, n, lane);
        } else if (!warp_sort_list_q<K>(r, n, lane) && lane == 0) {
            redo_items[atomicAdd(redo_count, 1u)] = p;
        }
    }
}

// Classes 2..4 by distribution: one warp per list of n <= 32 K records.
// Each record goes to bucket floor((depth - min) * n / (max - min)) of n
// buckets (monotone in the depth), buckets are counted (shared-memory
// atomics), scanned and scattered in shared memory, so only records of one
// bucket can be out of order; the odd-even passes of the surrogate-key sort
// then restore the exact (depth, face) order, and a list that needs more than
// kFixPasses passes goes to the block sort.  About 30 instructions per record
// against the bitonic network's log2(N) (log2(N) + 1) / 2 stages.  Shared
// arrays are skewed (one pad element per 16 records, per 32 counters) so
// the lane-strided accesses hit distinct banks.
__device__ __forceinline__ uint32_t skew16(uint32_t i) { return i + (i >> 4); }
__device__ __forceinline__ uint32_t skew32(uint32_t i) { return i + (i >> 5); }

template <int K>
__host__ __device__ constexpr int bucket_warps() { return K >= 16 ? 4 : 8; }

template <int K>
__global__ void __launch_bounds__(bucket_warps<K>() * 32) k_sort_class_bucket(
    const u64* __restrict__ offsets, u64* records, const uint32_t* __restrict__ items,
    const uint32_t* __restrict__ count, uint32_t* __restrict__ redo_count, uint32_t* __restrict__ redo_items,
    const uint32_t* __restrict__ ok) {
    constexpr int N = 32 * K, W = bucket_warps<K>();
    __shared__ u64 sbuf[W][N + N / 16];
    __shared__ uint32_t scnt[W][N + N / 32];
    if (ok && *ok == 0u) return;
    const uint32_t num = *count;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    u64* buf = sbuf[w];
    uint32_t* cnt = scnt[w];
    for (uint32_t it = blockIdx.x * W + w; it < num; it += gridDim.x * W) {
        const uint32_t p = items[it];
        const u64 beg = offsets[p];
        const uint32_t n = uint32_t(offsets[p + 1] - beg);
        u64* r = records + beg;
        u64 v[K];
        float dmin = 3.4e38f, dmax = 0.f;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const uint32_t i = uint32_t(q * 32 + lane);
            v[q] = i < n ? r[i] : ~0ull;
            cnt[skew32(uint32_t(lane * K + q))] = 0u;
            if (i < n) {
                const float d = __uint_as_float(uint32_t(v[q] >> 32));
                dmin = fminf(dmin, d);
                dmax = fmaxf(dmax, d);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dmin = fminf(dmin, __shfl_xor_sync(kFull, dmin, o));
            dmax = fmaxf(dmax, __shfl_xor_sync(kFull, dmax, o));
        }
        const float scale = dmax > dmin ? float(n) / (dmax - dmin) : 0.f;
        __syncwarp();
        uint32_t b[K], rk[K];
#pragma unroll
        for (int q = 0; q < K; ++q) {
            if (uint32_t(q * 32 + lane) < n) {
                const float d = __uint_as_float(uint32_t(v[q] >> 32));
                b[q] = min(uint32_t((d - dmin) * scale), n - 1u);
                rk[q] = atomicAdd(&cnt[skew32(b[q])], 1u);
            }
        }
        __syncwarp();
        // Exclusive scan of the counts: lane owns buckets [K lane, K lane + K).
        uint32_t c[K], tot = 0;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            c[q] = tot;
            tot += cnt[skew32(uint32_t(lane * K + q))];
        }
        uint32_t incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += t;
        }
        const uint32_t base = incl - tot;
#pragma unroll
        for (int q = 0; q < K; ++q) cnt[skew32(uint32_t(lane * K + q))] = base + c[q];
        __syncwarp();
#pragma unroll
        for (int q = 0; q < K; ++q)
            if (uint32_t(q * 32 + lane) < n) buf[skew16(cnt[skew32(b[q])] + rk[q])] = v[q];
        __syncwarp();
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const uint32_t i = uint32_t(lane * K + q);
            v[q] = i < n ? buf[skew16(i)] : ~0ull;
        }
        bool sorted = false;
        for (int pass = 0; pass < kFixPasses; ++pass) {
            const bool s0 = fixup_pass<K>(v, lane, 0);
            const bool s1 = fixup_pass<K>(v, lane, 1);
            if (!__any_sync(kFull, s0 || s1)) {
                sorted = true;
                break;
            }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < K; ++q) buf[skew16(uint32_t(lane * K + q))] = v[q];
        __syncwarp();
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const uint32_t i = uint32_t(q * 32 + lane);
            if (i < n) r[i] = buf[skew16(i)];
        }
        if (!sorted && lane == 0) redo_items[atomicAdd(redo_count, 1u)] = p;
        __syncwarp();
    }
}

// Class 5: one warp per list, bitonic in shared memory.
__global__ void __launch_bounds__(kSortWarps * 32) k_sort_class_smem(const u64* __restrict__ offsets, u64* records,
                                                                     const uint32_t* __restrict__ items,
                                                                     const uint32_t* __restrict__ count,
                                                                     const uint32_t* __restrict__ ok) {
    if (ok && *ok == 0u) return;
    extern __shared__ u64 sm_sort[];
    const uint32_t num = *count;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u64* s = sm_sort + size_t(warp) * kSortWarpCap;
    for (uint32_t i = blockIdx.x * kSortWarps + warp; i < num; i += gridDim.x * kSortWarps) {
        const uint32_t p = items[i];
        const u64 beg = offsets[p];
        const uint32_t n = uint32_t(offsets[p + 1] - beg);
        u64* r = records + beg;
        uint32_t N = 64;
        while (N < n) N <<= 1;
        for (uint32_t j = lane; j < N; j += 32) s[j] = j < n ? r[j] : ~0ull;
        __syncwarp();
        bitonic_smem<false>(s, N, lane, 32);
        for (uint32_t j = lane; j < n; j += 32) r[j] = s[j];
        __syncwarp();
    }
}

// Class 5 by distribution: one warp per list of 513..1024 records in shared
// memory.  Records are bucketed by depth over the list's range (n buckets,
// bucket index monotone in the depth; equal depths share a bucket), the
// buckets counted, scanned and scattered with shared-memory atomics, and each
// bucket put in exact (depth, face) order by an insertion sort on the 64-bit
// records.  Buckets hold about one record each; a list whose largest bucket
// exceeds kBucketInsertMax records (depths clustered) is sorted by the
// bitonic network instead.  O(n) work against the network's
// O(n log^2 n).
constexpr int kSortBucketWarps = 4;
constexpr uint32_t kBucketInsertMax = 64;

__global__ void __launch_bounds__(kSortBucketWarps * 32) k_sort_class_smem_bucket(
    const u64* __restrict__ offsets, u64* records, const uint32_t* __restrict__ items,
    const uint32_t* __restrict__ count, const uint32_t* __restrict__ ok) {
    if (ok && *ok == 0u) return;
    extern __shared__ u64 sm_sort[];
    constexpr uint32_t C = kSortWarpCap;
    const uint32_t num = *count;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u64* in = sm_sort + size_t(warp) * (2 * C + C / 2);
    u64* out = in + C;
    uint32_t* cnt = reinterpret_cast<uint32_t*>(out + C);
    for (uint32_t it = blockIdx.x * kSortBucketWarps + warp; it < num; it += gridDim.x * kSortBucketWarps) {
        const uint32_t p = items[it];
        const u64 beg = offsets[p];
        const uint32_t n = uint32_t(offsets[p + 1] - beg);
        u64* r = records + beg;
        float dmin = 3.4e38f, dmax = 0.f;
        for (uint32_t j = lane; j < n; j += 32) {
            const u64 v = r[j];
            in[j] = v;
            const float d = __uint_as_float(uint32_t(v >> 32));
            dmin = fminf(dmin, d);
            dmax = fmaxf(dmax, d);
            cnt[j] = 0u;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dmin = fminf(dmin, __shfl_xor_sync(kFull, dmin, o));
            dmax = fmaxf(dmax, __shfl_xor_sync(kFull, dmax, o));
        }
        const float scale = dmax > dmin ? float(n) / (dmax - dmin) : 0.f;
        __syncwarp();
        auto bucket = [&](u64 v) {
            return min(uint32_t((__uint_as_float(uint32_t(v >> 32)) - dmin) * scale), n - 1u);
        };
        for (uint32_t j = lane; j < n; j += 32) atomicAdd(&cnt[bucket(in[j])], 1u);
        __syncwarp();
        // Exclusive scan of the counts; lane owns counters [lane * k, lane * k + k).
        const uint32_t k = (n + 31) / 32, c0 = min(uint32_t(lane) * k, n), c1 = min(c0 + k, n);
        uint32_t tot = 0, mx = 0;
        for (uint32_t b = c0; b < c1; ++b) {
            tot += cnt[b];
            mx = max(mx, cnt[b]);
        }
        uint32_t incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += t;
            mx = max(mx, __shfl_xor_sync(kFull, mx, o));
        }
        if (mx > kBucketInsertMax) {
            // Clustered depths: the bitonic network on the list padded to 1024.
            for (uint32_t j = n + lane; j < C; j += 32) in[j] = ~0ull;
            __syncwarp();
            bitonic_smem<false>(in, C, lane, 32);
            for (uint32_t j = lane; j < n; j += 32) r[j] = in[j];
            __syncwarp();
            continue;
        }
        uint32_t run = incl - tot;
        for (uint32_t b = c0; b < c1; ++b) {
            const uint32_t c = cnt[b];
            cnt[b] = run;
            run += c;
        }
        __syncwarp();
        for (uint32_t j = lane; j < n; j += 32) {
            const u64 v = in[j];
            out[atomicAdd(&cnt[bucket(v)], 1u)] = v;
        }
        __syncwarp();
        // cnt[b] is now the end of bucket b (the start of bucket b + 1).
        for (uint32_t b = lane; b < n; b += 32) {
            const uint32_t s0 = b ? cnt[b - 1] : 0u, s1 = cnt[b];
            for (uint32_t i = s0 + 1; i < s1; ++i) {
                const u64 v = out[i];
                uint32_t j = i;
                while (j > s0 && out[j - 1] > v) {
                    out[j] = out[j - 1];
                    --j;
                }
                out[j] = v;
            }
        }
        __syncwarp();
        for (uint32_t j = lane; j < n; j += 32) r[j] = out[j];
        __syncwarp();
    }
}

// Class 6: one block per list.
__global__ void __launch_bounds__(1024) k_sort_class_block(const u64* __restrict__ offsets, u64* records,
                                                           const uint32_t* __restrict__ items,
                                                           const uint32_t* __restrict__ count,
                                                           const uint32_t* __restrict__ ok) {
    if (ok && *ok == 0u) return;
    extern __shared__ u64 sm_sort[];
    const uint32_t num = *count;
    for (uint32_t i = blockIdx.x; i < num; i += gridDim.x) {
        const uint32_t p = items[i];
        const u64 beg = offsets[p];
        const uint32_t n = uint32_t(offsets[p + 1] - beg);
        u64* r = records + beg;
        uint32_t N = 64;
        while (N < n) N <<= 1;
        for (uint32_t j = threadIdx.x; j < N; j += blockDim.x) sm_sort[j] = j < n ? r[j] : ~0ull;
        __syncthreads();
        bitonic_smem<true>(sm_sort, N, threadIdx.x, blockDim.x);
        for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) r[j] = sm_sort[j];
        __syncthreads();
    }
}

// Class 7: lists longer than kSortBlockCap, one block per list, in place.
// An ascending-only bitonic network over the list padded (in thought) with
// +infinity to N = 2^m records: stage k compares i with i ^ (k - 1) (the
// mirrored partner in its block of k), then i with i ^ j for j = k/4 .. 1.
// Every comparator (i, l), i < l, keeps the smaller record at i, so the
// padding never moves and comparators that reach past the list are skipped.
// Chunks of C = kSortBlockCap records are sorted whole in shared memory;
// each later stage (k = 2C .. N) runs its comparators of distance >= C over
// global memory and the rest chunk by chunk in shared memory.  Records are
// distinct (a face meets a pixel once), so the order is the total order of
// the 64-bit values.
__device__ __forceinline__ void cmpswap_global(u64* r, u64 i, u64 l) {
    const u64 a = r[i], b = r[l];
    if (a > b) {
        r[i] = b;
        r[l] = a;
    }
}

__global__ void __launch_bounds__(1024) k_sort_class_long(const u64* __restrict__ offsets, u64* records,
                                                          const uint32_t* __restrict__ items,
                                                          const uint32_t* __restrict__ count,
                                                          const uint32_t* __restrict__ ok) {
    if (ok && *ok == 0u) return;
    extern __shared__ u64 sm_sort[];
    constexpr u64 C = kSortBlockCap;
    const uint32_t num = *count;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    for (uint32_t it = blockIdx.x; it < num; it += gridDim.x) {
        const uint32_t p = items[it];
        const u64 beg = offsets[p];
        const u64 n = offsets[p + 1] - beg;
        u64* r = records + beg;
        u64 N = C;
        while (N < n) N <<= 1;
        // Stages k <= C: each chunk sorted in shared memory.
        for (u64 c0 = 0; c0 < n; c0 += C) {
            const u64 m = min(C, n - c0);
            for (uint32_t j = tid; j < C; j += nthr) sm_sort[j] = j < m ? r[c0 + j] : ~0ull;
            __syncthreads();
            bitonic_smem<true>(sm_sort, uint32_t(C), tid, nthr);
            for (uint32_t j = tid; j < m; j += nthr) r[c0 + j] = sm_sort[j];
            __syncthreads();
        }
        for (u64 k = 2 * C; k <= N; k <<= 1) {
            // Mirror step of stage k, then the half-cleaners of distance >= C.
            const u64 h = k >> 1;
            for (u64 t = tid; t < (N >> 1); t += nthr) {
                const u64 b = (t & ~(h - 1)) << 1, o = t & (h - 1);  // block of k, offset in its lower half
                const u64 l = b + (k - 1 - o);
                if (l < n) cmpswap_global(r, b + o, l);
            }
            __syncthreads();
            for (u64 j = k >> 2; j >= C; j >>= 1) {
                for (u64 t = tid; t < (N >> 1); t += nthr) {
                    const u64 i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
                    if (i + j < n) cmpswap_global(r, i, i + j);
                }
                __syncthreads();
            }
            // Half-cleaners of distance < C stay inside one chunk.
            for (u64 c0 = 0; c0 < n; c0 += C) {
                const u64 m = min(C, n - c0);
                for (uint32_t j = tid; j < C; j += nthr) sm_sort[j] = j < m ? r[c0 + j] : ~0ull;
                __syncthreads();
                for (uint32_t j = uint32_t(C >> 1); j > 0; j >>= 1) {
                    for (uint32_t t = tid; t < uint32_t(C >> 1); t += nthr) {
                        const uint32_t i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
                        const u64 a = sm_sort[i], b = sm_sort[i + j];
                        if (a > b) {
                            sm_sort[i] = b;
                            sm_sort[i + j] = a;
                        }
                    }
                    __syncthreads();
                }
                for (uint32_t j = tid; j < m; j += nthr) r[c0 + j] = sm_sort[j];
                __syncthreads();
            }
        }
    }
}

static_assert(kSortClasses == 9, "k_sort_classify assigns classes 0..8");

template <int K>
void sort_class(int method, unsigned g, const u64* offsets, u64* records, const uint32_t* items,
                const uint32_t* count, uint32_t* redo_n, uint32_t* redo, const uint32_t* ok, cudaStream_t s) {
    if (method == 2)
        k_sort_class_bucket<K><<<g, bucket_warps<K>() * 32, 0, s>>>(offsets, records, items, count, redo_n, redo, ok);
    else if (method == 1)
        k_sort_class_regs<K, true><<<g, kSortWarps * 32, 0, s>>>(offsets, records, items, count, redo_n, redo, ok);
    else
        k_sort_class_regs<K, false><<<g, kSortWarps * 32, 0, s>>>(offsets, records, items, count, redo_n, redo, ok);
}

void launch_sort(const u64* offsets, u64* records, uint32_t P, uint32_t* scratch, cudaStream_t s,
                 const uint32_t* ok, uint32_t surrogate_classes, uint32_t bucket_classes) {
    static bool attr_set = false;
    const size_t smem_warp = size_t(kSortWarps) * kSortWarpCap * sizeof(u64);
    const size_t smem_bucket = size_t(kSortBucketWarps) * (2 * kSortWarpCap + kSortWarpCap / 2) * sizeof(u64);
    const size_t smem_block = size_t(kSortBlockCap) * sizeof(u64);
    if (!attr_set) {
        cudaFuncSetAttribute(k_sort_class_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_warp));
        cudaFuncSetAttribute(k_sort_class_smem_bucket, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smem_bucket));
        cudaFuncSetAttribute(k_sort_class_block, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_block));
        cudaFuncSetAttribute(k_sort_class_long, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_block));
        attr_set = true;
    }
    if (P == 0) return;
    cudaMemsetAsync(scratch, 0, 16 * sizeof(uint32_t), s);
    k_sort_classify<<<(P + 255) / 256, 256, 0, s>>>(offsets, P, scratch, ok);
    auto items = [&](int c) { return scratch + 16 + size_t(c) * P; };
    const unsigned g = unsigned(std::min<uint64_t>(kSortGridBlocks, (uint64_t(P) + kSortWarps - 1) / kSortWarps));
    // Lists the register sorts leave unsettled join the block-sort class (6).
    uint32_t* redo_n = scratch + 6;
    uint32_t* redo = items(6);
    // Per class: 2 = distribution sort, 1 = surrogate keys, 0 = 64-bit bitonic.
    auto q = [&](int c) {
        return ((bucket_classes >> c) & 1u) ? 2 : (((surrogate_classes >> c) & 1u) ? 1 : 0);
    };
    k_sort_class_tiny<<<kSortGridBlocks / 2, 256, 0, s>>>(offsets, records, items(kSortTinyClass),
                                                          scratch + kSortTinyClass, ok);
    k_sort_class_regs<1, false><<<g, kSortWarps * 32, 0, s>>>(offsets, records, items(0), scratch + 0, redo_n, redo,
                                                              ok);
    sort_class<2>(q(1), g, offsets, records, items(1), scratch + 1, redo_n, redo, ok, s);
    sort_class<4>(q(2), g, offsets, records, items(2), scratch + 2, redo_n, redo, ok, s);
    sort_class<8>(q(3), g, offsets, records, items(3), scratch + 3, redo_n, redo, ok, s);
    sort_class<16>(q(4), g, offsets, records, items(4), scratch + 4, redo_n, redo, ok, s);
    if ((bucket_classes >> 5) & 1u)
        k_sort_class_smem_bucket<<<296, kSortBucketWarps * 32, smem_bucket, s>>>(offsets, records, items(5),
                                                                                 scratch + 5, ok);
    else
        k_sort_class_smem<<<std::min(g, 296u), kSortWarps * 32, smem_warp, s>>>(offsets, records, items(5),
                                                                                scratch + 5, ok);
    k_sort_class_block<<<296, 1024, smem_block, s>>>(offsets, records, items(6), scratch + 6, ok);
    k_sort_class_long<<<148, 1024, smem_block, s>>>(offsets, records, items(7), scratch + 7, ok);
}

// ---------------------------------------------------------------------------
// (d) front-to-back compositing, one thread per pixel (composite_pixel).
// Pixel tiles of 256 threads: TX x (256 / TX) pixels (tile index 0: 16 x 16,
// 1: 32 x 8, 2: 8 x 32; chosen by the renderer's tuning).
template <int TX>
__global__ void __launch_bounds__(256) k_composite(
    const u64* __restrict__ offsets, const u64* __restrict__ records, const uint4* __restrict__ faces,
    const VGeo* __restrict__ vgeo, const float4* __restrict__ colors, int W, int row0, int row1, ShadeDev sh,
    float4* __restrict__ image, float* __restrict__ tfinal, uint32_t* __restrict__ term) {
    constexpr int TY = 256 / TX;
    const int px = blockIdx.x * TX + (threadIdx.x % TX);
    const int py = row0 + int(blockIdx.y) * TY + int(threadIdx.x / TX);
    if (px < W && py < row1)
        composite_pixel(px, py, W, offsets, records, faces, vgeo, colors, sh, image, tfinal, term);
}

template <int TX>
void composite_tiles(const u64* offsets, const u64* records, const uint4* faces, const VGeo* vgeo,
                     const float4* colors, int W, int row0, int row1, const ShadeDev& sh, float4* image,
                     float* tfinal, uint32_t* term, cudaStream_t s) {
    constexpr int TY = 256 / TX;
    dim3 grid((W + TX - 1) / TX, (row1 - row0 + TY - 1) / TY);
    k_composite<TX><<<grid, 256, 0, s>>>(offsets, records, faces, vgeo, colors, W, row0, row1, sh, image, tfinal,
                                         term);
}

void launch_composite(const u64* offsets, const u64* records, const uint4* faces, const VGeo* vgeo,
                      const float4* colors, int W, int H, const ShadeDev& sh, float4* image, float* tfinal,
                      uint32_t* term, cudaStream_t s, int row0, int row1, int tile) {
    if (row1 < 0) row1 = H;
    if (row1 <= row0) return;
    if (tile == 1)
        composite_tiles<32>(offsets, records, faces, vgeo, colors, W, row0, row1, sh, image, tfinal, term, s);
    else if (tile == 2)
        composite_tiles<8>(offsets, records, faces, vgeo, colors, W, row0, row1, sh, image, tfinal, term, s);
    else
        composite_tiles<16>(offsets, records, faces, vgeo, colors, W, row0, row1, sh, image, tfinal, term, s);
}

// ---------------------------------------------------------------------------
// (f) adjoint (adjoint_pixel).  Blocks of 128 threads (TX x 128 / TX pixels, four
// blocks per SM at 128 registers): measured 1.5 % faster than 256-thread blocks
// at two per SM, the same occupancy with finer scheduling of uneven lists.
constexpr int kAdjThreads = 128;
template <int TX, bool SCREEN>
__global__ void __launch_bounds__(kAdjThreads, 2 * 256 / kAdjThreads) k_adjoint(
    const u64* __restrict__ offsets, const u64* __restrict__ records, const uint4* __restrict__ faces,
    const VGeo* __restrict__ vgeo, const float4* __restrict__ colors, int W, int row0, int row1, CamDev cam,
    ShadeDev sh, const float4* __restrict__ dimage, const float* __restrict__ tfinal,
    const uint32_t* __restrict__ term, float4* __restrict__ grad_rows) {
    __shared__ float4 vcache4[3 * kAdjThreads];
    __shared__ float vcache1[3 * kAdjThreads];
    constexpr int TY = kAdjThreads / TX;
    const int px = blockIdx.x * TX + (threadIdx.x % TX);
    const int py = row0 + int(blockIdx.y) * TY + int(threadIdx.x / TX);
    if (px >= W || py >= row1) return;
    // Screen-space rows: the ordered register cache (order_like); world-space
    // rows (absolute gradients): the shared-memory cache.
    if constexpr (SCREEN) {
        OrderedRows acc{grad_rows};
        adjoint_pixel<OrderedRows, SCREEN>(px, py, offsets, records, faces, vgeo, colors, W, cam, sh, dimage, tfinal,
                                           term, acc);
    } else {
        VertCache acc{grad_rows, vcache4 + threadIdx.x, vcache1 + threadIdx.x, kAdjThreads};
        adjoint_pixel<VertCache, SCREEN>(px, py, offsets, records, faces, vgeo, colors, W, cam, sh, dimage, tfinal,
                                         term, acc);
    }
}

// Adds the interleaved rows into the caller's gradient buffers (SCREEN: the
// position rows hold screen-space adjoints, converted here per vertex).
template <bool SCREEN>
__global__ void __launch_bounds__(256) k_scatter_grads(const float4* __restrict__ rows, uint32_t V,
                                                       float* __restrict__ grad_pos,
                                                       float4* __restrict__ grad_col,
                                                       const VGeo* __restrict__ vgeo, CamDev cam) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    float4 a = rows[2 * size_t(v)];
    const float4 b = rows[2 * size_t(v) + 1];
    if (SCREEN) {
        const float3 w = screen_to_world(a, vgeo[v], cam);
        a = make_float4(w.x, w.y, w.z, 0.f);
    }
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
    launch_adjoint_rows(offsets, records, faces, vgeo, colors, cam, sh, dimage, tfinal, term, 0, cam.H, grad_rows,
                        s);
    launch_scatter_grads(grad_rows, V, grad_pos, grad_col, s, sh.use_abs_grad ? nullptr : vgeo, &cam);
}

template <int TX>
void adjoint_tiles(const u64* offsets, const u64* records, const uint4* faces, const VGeo* vgeo,
                   const float4* colors, const CamDev& cam, const ShadeDev& sh, const float4* dimage,
                   const float* tfinal, const uint32_t* term, int row0, int row1, float4* grad_rows, cudaStream_t s) {
    constexpr int TY = kAdjThreads / TX;
    dim3 grid((cam.W + TX - 1) / TX, (row1 - row0 + TY - 1) / TY);
    // Rows in screen space unless absolute gradients are asked for (see
    // frag_vertex_grads); launch_scatter_grads converts with the same rule.
    if (sh.use_abs_grad)
        k_adjoint<TX, false><<<grid, kAdjThreads, 0, s>>>(offsets, records, faces, vgeo, colors, cam.W, row0, row1, cam, sh,
                                                  dimage, tfinal, term, grad_rows);
    else
        k_adjoint<TX, true><<<grid, kAdjThreads, 0, s>>>(offsets, records, faces, vgeo, colors, cam.W, row0, row1, cam, sh,
                                                 dimage, tfinal, term, grad_rows);
}

void launch_adjoint_rows(const u64* offsets, const u64* records, const uint4* faces, const VGeo* vgeo,
                         const float4* colors, const CamDev& cam, const ShadeDev& sh, const float4* dimage,
                         const float* tfinal, const uint32_t* term, int row0, int row1, float4* grad_rows,
                         cudaStream_t s, int tile) {
    if (row1 <= row0) return;
    if (tile == 1)
        adjoint_tiles<32>(offsets, records, faces, vgeo, colors, cam, sh, dimage, tfinal, term, row0, row1, grad_rows,
                          s);
    else if (tile == 2)
        adjoint_tiles<8>(offsets, records, faces, vgeo, colors, cam, sh, dimage, tfinal, term, row0, row1, grad_rows,
                         s);
    else
        adjoint_tiles<16>(offsets, records, faces, vgeo, colors, cam, sh, dimage, tfinal, term, row0, row1, grad_rows,
                          s);
}

void launch_scatter_grads(const float4* grad_rows, uint32_t V, float* grad_pos, float4* grad_col, cudaStream_t s,
                          const VGeo* screen_vgeo, const CamDev* cam) {
    if (!V) return;
    if (screen_vgeo)
        k_scatter_grads<true><<<(V + 255) / 256, 256, 0, s>>>(grad_rows, V, grad_pos, grad_col, screen_vgeo, *cam);
    else
        k_scatter_grads<false><<<(V + 255) / 256, 256, 0, s>>>(grad_rows, V, grad_pos, grad_col, nullptr, CamDev{});
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
