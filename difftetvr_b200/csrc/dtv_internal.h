// Internal host-side declarations shared by the C-ABI layer and the kernel
// launch wrappers.  Not part of the public interface (include/difftetvr_b200.h).
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "dtv_types.h"

namespace dtv {

// Face record on the device: three vertex indices (winding of the lowest
// faceId copy, TetMesh.cpp:1249-1252) and the boundary bit in .w.
struct MeshHost {
    uint64_t num_cells = 0, num_vertices = 0, num_faces = 0;
    std::vector<uint32_t> tri;            // 3F
    std::vector<uint32_t> face_boundary;  // F
    std::vector<uint32_t> face_to_tet;    // 2F
    std::vector<uint32_t> vertex_boundary;// V
    std::vector<uint32_t> cells;          // 4T
    std::vector<uint32_t> tet_faces;      // 4T: unique face index of face j of tet c (TetFaceTable order)
    // T: bit j set when face j's side seen from tet c is not given by the
    // winding of c's own vertex order (the shared face's stored winding, as
    // read with the owner rule, disagrees with c's order: inconsistently
    // oriented neighbours); 0 for a consistently oriented mesh.
    std::vector<uint8_t> tet_flip;
};

// Builds faces from cells (restates buildFacesSlim, TetMesh.cpp:1218-1268).
void build_faces(const uint32_t* cells, uint64_t T, uint64_t V, MeshHost& out);

// Launch wrappers (dtv_kernels.cu).  All run on `s`.
void launch_project(const float* pos, uint32_t V, const CamDev& cam, float4* vproj, int2* vfix, VGeo* vgeo,
                    cudaStream_t s);
// Pixel rows [row0, row1) only (row1 < 0: all rows).  wide_list (u32[F + 1],
// optional): the count lists the faces of the 64-bit path there, and the
// 64-bit count and the fill that follows (same rows) walk that list instead of
// setting up every face again; without it both 64-bit launches cover all F.
void launch_raster_count(const uint4* faces, uint32_t F, const float4* vproj, const int2* vfix, int W, int H,
                         uint32_t* counts, cudaStream_t s, int row0 = 0, int row1 = -1,
                         uint32_t* wide_list = nullptr);
void launch_raster_fill(const uint4* faces, uint32_t F, const float4* vproj, const int2* vfix, int W, int H,
                        uint32_t* counts, const unsigned long long* offsets, unsigned long long* records,
                        cudaStream_t s, int row0 = 0, int row1 = -1, const uint32_t* order = nullptr,
                        const uint32_t* wide_list = nullptr);
// Order of the faces for the fill, grouped by row bands of about
// kFillBandBytes of records each (nf records over H rows; order: F entries;
// band_scratch: 2 * kFillBands entries).
constexpr int kFillBands = 512;
constexpr uint64_t kFillBandBytes = 24ull << 20;
void launch_fill_order(const uint4* faces, uint32_t F, const int2* vfix, int H, uint64_t nf, uint32_t* order,
                       uint32_t* band_scratch, cudaStream_t s);
// Exclusive prefix of kFillBands band counts (one warp).
void launch_band_scan(const uint32_t* hist, uint32_t* cursor, cudaStream_t s);
// Exclusive scan of counts[n] into offsets[n+1]; scratch must hold scan_scratch_elems(n) u64.
constexpr uint64_t kScanTile = 4096;  // counts per scan block (1024 threads x 4)
constexpr size_t scan_scratch_elems(uint64_t n) { return size_t((n + kScanTile - 1) / kScanTile) + 1; }
void launch_scan(const uint32_t* counts, uint64_t n, unsigned long long* offsets, unsigned long long* scratch,
                 cudaStream_t s);
// Per-pixel sort of the lists of P pixels, any length.  scratch holds
// sort_scratch_elems(P) u32 (length-class counts and lists).  With a non-null
// `ok`, the sort does nothing when *ok == 0 (batched steps whose records
// overflowed the buffer).
constexpr int kSortClasses = 9;  // list-length classes (dtv_kernels.cu)
constexpr size_t sort_scratch_elems(uint64_t P) { return 16 + size_t(kSortClasses) * size_t(P); }
// surrogate_classes: bit c set = list-length class c (1..4: up to 64, 128,
// 256, 512 records) is sorted through 32-bit surrogate keys, else through the
// 64-bit network (same result either way).
constexpr uint32_t kSortSurrogateDefault = 0x1eu;
constexpr uint32_t kSortBucketDefault = 0x3cu;  // classes sorted by distribution (bit c: class c, 2..5)
void launch_sort(const unsigned long long* offsets, unsigned long long* records, uint32_t P, uint32_t* scratch,
                 cudaStream_t s, const uint32_t* ok = nullptr,
                 uint32_t surrogate_classes = kSortSurrogateDefault, uint32_t bucket_classes = kSortBucketDefault);
constexpr uint32_t kSortWarpCap = 1024;    // elements per warp list sorted in shared memory
constexpr uint32_t kSortBlockCap = 16384;  // elements per block-sorted list / chunk of a longer one (128 KiB shared memory)

// tile: pixel tile of the 256-thread blocks (0: 16 x 16, 1: 32 x 8, 2: 8 x 32).
void launch_composite(const unsigned long long* offsets, const unsigned long long* records, const uint4* faces,
                      const VGeo* vgeo, const float4* colors, int W, int H, const ShadeDev& sh, float4* image,
                      float* tfinal, uint32_t* term, cudaStream_t s, int row0 = 0, int row1 = -1, int tile = 0);
void launch_adjoint(const unsigned long long* offsets, const unsigned long long* records, const uint4* faces,
                    const VGeo* vgeo, const float4* colors, const CamDev& cam, const ShadeDev& sh,
                    const float4* dimage, const float* tfinal, const uint32_t* term, uint32_t V,
                    float4* grad_rows, float* grad_pos, float4* grad_col, cudaStream_t s);
// Adjoint of pixel rows [row0, row1) into grad_rows (no clearing, no scatter).
void launch_adjoint_rows(const unsigned long long* offsets, const unsigned long long* records, const uint4* faces,
                         const VGeo* vgeo, const float4* colors, const CamDev& cam, const ShadeDev& sh,
                         const float4* dimage, const float* tfinal, const uint32_t* term, int row0, int row1,
                         float4* grad_rows, cudaStream_t s, int tile = 0);
// Adds the interleaved [V][2] gradient rows into grad_pos [V,3] / grad_col [V,4].
// screen_vgeo / cam: rows hold screen-space position adjoints of that camera
// (the list adjoint without absolute gradients); nullptr: world-space rows.
void launch_scatter_grads(const float4* grad_rows, uint32_t V, float* grad_pos, float4* grad_col, cudaStream_t s,
                          const VGeo* screen_vgeo = nullptr, const CamDev* cam = nullptr);

void launch_loss_l2(const float* image, const float* target, uint64_t n, float scale, float* adjoint,
                    float* loss_accum, cudaStream_t s);
void launch_adam(float* param, const float* grad, float* m, float* v, uint64_t n, float lr, float beta1,
                 float beta2, float eps, float bc1, float bc2, int clamp_mode, const uint32_t* fixed_mask,
                 int fixed_mode, int stride, cudaStream_t s);

// Per-cell colours (dtv_cells.cu): cell_colors f32[4T]; rows [row0, row1).
void launch_composite_cells(const unsigned long long* offsets, const unsigned long long* records, const uint4* faces,
                            const uint32_t* face_to_tet, const VGeo* vgeo, const float4* cell_colors, int W, int H,
                            const ShadeDev& sh, float4* image, float* tfinal, uint32_t* term, cudaStream_t s,
                            int row0, int row1);
void launch_adjoint_cells_rows(const unsigned long long* offsets, const unsigned long long* records,
                               const uint4* faces, const uint32_t* face_to_tet, const VGeo* vgeo,
                               const float4* cell_colors, const CamDev& cam, const ShadeDev& sh, const float4* dimage,
                               const float* tfinal, const uint32_t* term, int row0, int row1, float4* grad_rows,
                               float4* grad_cells, cudaStream_t s);
// Adds the position part of the [V][2] gradient rows into grad_pos [V,3]
// (vgeo non-null: the rows hold screen-space adjoints, converted per vertex
// with the render's camera, as the per-cell adjoint leaves them without
// absolute gradients).
void launch_scatter_positions(const float4* grad_rows, uint32_t V, float* grad_pos, cudaStream_t s,
                              const VGeo* vgeo = nullptr, const CamDev* cam = nullptr);

// Ray-tet path (dtv_raytet.cu).
void launch_walk_composite(const unsigned long long* b_offsets, const unsigned long long* b_records,
                           const uint32_t* bf_global, const uint4* faces, const uint32_t* face_to_tet,
                           const uint32_t* tet_faces, const uint32_t* cells, const uint8_t* tet_flip,
                           uint32_t num_tets, const int2* vfix, const VGeo* vgeo,
                           const float4* colors, const CamDev& cam, const ShadeDev& sh, float4* image,
                           float* tfinal, uint4* wstate, cudaStream_t s);
void launch_walk_adjoint(const unsigned long long* b_offsets, const unsigned long long* b_records,
                         const uint32_t* bf_global, const uint4* faces, const uint32_t* face_to_tet,
                         const uint32_t* tet_faces, const uint32_t* cells, const uint8_t* tet_flip,
                         uint32_t num_tets, const int2* vfix, const VGeo* vgeo,
                         const float4* colors, const CamDev& cam, const ShadeDev& sh, const float4* dimage,
                         const float* tfinal, const uint4* wstate, uint32_t V, float4* grad_rows, float* grad_pos,
                         float4* grad_col, cudaStream_t s);

// Accessors used by the allocation-free entry point (dtv_noalloc.cu); they
// expose what dtv_renderer_render derives from its arguments.
struct MeshView {
    const uint4* faces;
    uint64_t num_faces;
    uint64_t num_vertices;
};

}  // namespace dtv

struct dtv_mesh;
struct dtv_camera;
struct dtv_render_params;

namespace dtv {
MeshView mesh_view(const dtv_mesh* m);
uint64_t mesh_num_cells(const dtv_mesh* m);
const uint32_t* mesh_cells_device(const dtv_mesh* m);  // u32[4T], 16-byte aligned
CamDev camera_constants(const dtv_camera& c);
ShadeDev shade_constants(const dtv_render_params& p);
}  // namespace dtv

// Sets the message returned by dtv_last_error_string() on this thread.
void dtv_set_last_error(const std::string& msg);
