// Allocation-free forward render.
//
// Some callers cannot allocate device memory while they render: code running
// inside a host framework that owns the device heap and forbids cudaMalloc
// (cudaMalloc / cudaFree also synchronise the device, which latency-bound
// serving loops avoid after start-up), or code whose memory plan is fixed
// before the first frame.  dtv_render_noalloc gives them the forward render
// of dtv_renderer_render with every scratch buffer (vertex projections,
// per-pixel counters and offsets, the fragment records, per-pixel state)
// carved out of one file-scope device array of fixed size, so the call itself
// allocates nothing.  The same kernels run as in dtv_renderer_render.
//
// Limits (requests beyond them are rejected before any device work):
//   vertices  <= 65,536
//   pixels    <= 65,536 (e.g. 256 x 256)
//   fragments <= 4,194,304 (checked after the exact count of the scan)
// The array is about 39 MiB and every GPU that loads this library holds it
// until the process exits.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address with cudaGetSymbolAddress (a host-side name of a
// __device__ array is not a device address) and caches it per device; make
// that first call before any stream capture.
//
// All calls share the one array and it keeps the last call's contents: each
// call clears what must start at zero (the per-pixel counters; the sort
// clears its own class counters).  Calls that overlap on the GPU (other
// streams, other host threads) race on the array; serialise them.
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include "difftetvr_b200.h"
#include "dtv_internal.h"

namespace {

constexpr uint64_t kNaMaxVertices = 65536;
constexpr uint64_t kNaMaxPixels = 65536;
constexpr uint64_t kNaMaxFragments = uint64_t(4) << 20;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
// The scan and sort scratch sizes come from the same constexpr functions the
// allocating path uses, so a change of their tiling cannot overrun a region.
constexpr size_t kNaScanElems = dtv::scan_scratch_elems(kNaMaxPixels);
constexpr size_t kNaSortElems = dtv::sort_scratch_elems(kNaMaxPixels);

constexpr size_t kOffVproj = 0;
constexpr size_t kOffVfix = align256(kOffVproj + sizeof(float4) * kNaMaxVertices);
constexpr size_t kOffVgeo = align256(kOffVfix + sizeof(int2) * kNaMaxVertices);
constexpr size_t kOffCounts = align256(kOffVgeo + sizeof(dtv::VGeo) * kNaMaxVertices);
constexpr size_t kOffOffsets = align256(kOffCounts + sizeof(uint32_t) * kNaMaxPixels);
constexpr size_t kOffScan = align256(kOffOffsets + sizeof(unsigned long long) * (kNaMaxPixels + 1));
constexpr size_t kOffTfinal = align256(kOffScan + sizeof(unsigned long long) * kNaScanElems);
constexpr size_t kOffTerm = align256(kOffTfinal + sizeof(float) * kNaMaxPixels);
constexpr size_t kOffLong = align256(kOffTerm + sizeof(uint32_t) * kNaMaxPixels);
constexpr size_t kOffRecords = align256(kOffLong + sizeof(uint32_t) * kNaSortElems);
constexpr size_t kNaScratchBytes = align256(kOffRecords + sizeof(unsigned long long) * kNaMaxFragments);
static_assert(kNaScratchBytes < (size_t(48) << 20), "fixed scratch of the allocation-free render grew past 48 MiB");

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaScratchBytes];

namespace {

std::mutex g_noalloc_mutex;
constexpr int kMaxDevices = 64;
void* g_noalloc_ptr[kMaxDevices] = {};

struct NaError : std::runtime_error {
    int32_t code;
    NaError(int32_t c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define NA_CK(expr)                                                                                   \
    do {                                                                                              \
        cudaError_t err__ = (expr);                                                                   \
        if (err__ != cudaSuccess)                                                                     \
            throw NaError(DTV_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(err__));      \
    } while (0)

// Device address of the scratch array on the current device (looked up once).
unsigned char* noalloc_scratch() {
    int dev = 0;
    NA_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw NaError(DTV_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        NA_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = p;
    }
    return static_cast<unsigned char*>(g_noalloc_ptr[dev]);
}

}  // namespace

extern "C" int32_t dtv_render_noalloc(const dtv_mesh* mesh, const float* d_positions, const float* d_colors,
                                      const dtv_camera* camera, const dtv_render_params* params, float* d_image,
                                      dtv_stream stream) {
    try {
        if (!mesh || !camera || !params) throw NaError(DTV_ERR_ARG, "null handle or struct");
        if (!d_positions || !d_colors || !d_image) throw NaError(DTV_ERR_ARG, "null device pointer");
        if ((reinterpret_cast<uintptr_t>(d_colors) & 15u) || (reinterpret_cast<uintptr_t>(d_image) & 15u))
            throw NaError(DTV_ERR_ARG, "colors and image must be 16-byte aligned");
        if (camera->width <= 0 || camera->height <= 0)
            throw NaError(DTV_ERR_ARG, "viewport size must be positive");
        if (!(camera->znear > 0.f && camera->zfar > camera->znear))
            throw NaError(DTV_ERR_ARG, "need 0 < znear < zfar");
        if (!(camera->fovy > 0.f && camera->fovy < 3.14159f)) throw NaError(DTV_ERR_ARG, "fovy must be in (0, pi)");
        const dtv::MeshView mv = dtv::mesh_view(mesh);
        const uint64_t P = uint64_t(camera->width) * uint64_t(camera->height);
        if (mv.num_vertices > kNaMaxVertices)
            throw NaError(DTV_ERR_ARG, "dtv_render_noalloc: " + std::to_string(mv.num_vertices) +
                                           " vertices exceed the fixed scratch limit of " +
                                           std::to_string(kNaMaxVertices));
        if (P > kNaMaxPixels)
            throw NaError(DTV_ERR_ARG, "dtv_render_noalloc: " + std::to_string(P) +
                                           " pixels exceed the fixed scratch limit of " +
                                           std::to_string(kNaMaxPixels));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        unsigned char* base = noalloc_scratch();
        auto* vproj = reinterpret_cast<float4*>(base + kOffVproj);
        auto* vfix = reinterpret_cast<int2*>(base + kOffVfix);
        auto* vgeo = reinterpret_cast<dtv::VGeo*>(base + kOffVgeo);
        auto* counts = reinterpret_cast<uint32_t*>(base + kOffCounts);
        auto* offsets = reinterpret_cast<unsigned long long*>(base + kOffOffsets);
        auto* scan = reinterpret_cast<unsigned long long*>(base + kOffScan);
        auto* tfinal = reinterpret_cast<float*>(base + kOffTfinal);
        auto* term = reinterpret_cast<uint32_t*>(base + kOffTerm);
        auto* long_list = reinterpret_cast<uint32_t*>(base + kOffLong);
        auto* records = reinterpret_cast<unsigned long long*>(base + kOffRecords);

        const dtv::CamDev cam = dtv::camera_constants(*camera);
        const dtv::ShadeDev sh = dtv::shade_constants(*params);
        const int W = camera->width, H = camera->height;
        // The array keeps the previous call's contents: counters start at zero.
        NA_CK(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * P, s));
        dtv::launch_project(d_positions, uint32_t(mv.num_vertices), cam, vproj, vfix, vgeo, s);
        dtv::launch_raster_count(mv.faces, uint32_t(mv.num_faces), vproj, vfix, W, H, counts, s);
        dtv::launch_scan(counts, P, offsets, scan, s);
        NA_CK(cudaGetLastError());
        unsigned long long nf = 0;
        NA_CK(cudaMemcpyAsync(&nf, offsets + P, sizeof(nf), cudaMemcpyDeviceToHost, s));
        NA_CK(cudaStreamSynchronize(s));
        if (nf > kNaMaxFragments)
            throw NaError(DTV_ERR_BUDGET, "dtv_render_noalloc: " + std::to_string(nf) +
                                              " fragments exceed the fixed scratch limit of " +
                                              std::to_string(kNaMaxFragments));
        if (params->fragment_budget_bytes && nf * sizeof(unsigned long long) > params->fragment_budget_bytes)
            throw NaError(DTV_ERR_BUDGET, "dtv_render_noalloc: fragments exceed fragment_budget_bytes");
        dtv::launch_raster_fill(mv.faces, uint32_t(mv.num_faces), vproj, vfix, W, H, counts, offsets, records, s);
        dtv::launch_sort(offsets, records, uint32_t(P), long_list, s);
        dtv::launch_composite(offsets, records, mv.faces, vgeo, reinterpret_cast<const float4*>(d_colors), W, H, sh,
                              reinterpret_cast<float4*>(d_image), tfinal, term, s);
        NA_CK(cudaGetLastError());
        return DTV_OK;
    } catch (const NaError& e) {
        dtv_set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        dtv_set_last_error(e.what());
        return DTV_ERR_STATE;
    }
}
