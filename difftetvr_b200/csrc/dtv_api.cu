// C ABI of the B200-native tetrahedral volume-rendering path (see
// include/difftetvr_b200.h).  Host orchestration: buffers, stage order, the
// one host synchronisation per render (the exact fragment count from the scan
// sizes the record buffer), error reporting.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>
#include "difftetvr_b200.h"
#include "dtv_host.h"
#include "dtv_internal.h"

extern "C" int32_t dtv_build_hex_mesh_impl(const float* mn, const float* mx, uint32_t xs, uint32_t ys,
                                           uint32_t zs, uint32_t* cells, float* positions);

namespace {

using namespace dtv_host;
using u64 = unsigned long long;

thread_local std::string g_last_error;

dtv::CamDev make_cam(const dtv_camera& c) {
    dtv::CamDev k;
    std::memcpy(k.V, c.view, sizeof(k.V));
    // Host set-up: the focal constant in double, split into an FP32 pair for
    // the device (the discrete path uses f alone).
    const double tanh = std::tan(0.5 * double(c.fovy));
    const double fd = 0.5 * double(c.height) / tanh;
    k.f = float(fd);
    k.f_lo = float(fd - double(k.f));
    k.cx = 0.5f * float(c.width);
    k.cy = 0.5f * float(c.height);
    k.znear = c.znear;
    k.zfar = c.zfar;
    k.W = c.width;
    k.H = c.height;
    return k;
}

dtv::ShadeDev make_shade(const dtv_render_params& p) {
    dtv::ShadeDev s;
    s.atten = p.attenuation;
    s.ert_thresh = p.early_ray_out_thresh;
    s.use_ert = p.use_early_ray_termination ? 1 : 0;
    s.use_abs_grad = p.use_abs_grad ? 1 : 0;
    for (int k = 0; k < 4; ++k) s.clear[k] = p.clear_color[k];
    return s;
}

enum Stage { kProject = 0, kCount, kScan, kFill, kSort, kComposite, kAdjoint, kNumStages };

}  // namespace

struct dtv_mesh {
    dtv::MeshHost host;
    uint4* d_faces = nullptr;
    uint32_t* d_vertex_boundary = nullptr;
    uint32_t* d_face_to_tet = nullptr;
    uint32_t* d_cells = nullptr;
    // Ray-tet path: per-tet face ids and the boundary faces as their own
    // face set (rasterised alone; record face field k -> global face bf_global[k]).
    uint32_t* d_tet_faces = nullptr;   // 4T
    uint8_t* d_tet_flip = nullptr;     // T (MeshHost::tet_flip)
    uint4* d_bfaces = nullptr;         // Nb
    uint32_t* d_bf_global = nullptr;   // Nb
    std::vector<uint32_t> bf_global;   // host copy
};

struct dtv_renderer {
    int32_t type = DTV_RENDERER_PPLL;
    DevBuf<float4> vproj;
    DevBuf<int2> vfix;
    DevBuf<dtv::VGeo> vgeo;
    DevBuf<uint32_t> counts;
    DevBuf<u64> offsets;
    DevBuf<u64> records;
    DevBuf<u64> scan_scratch;
    DevBuf<float> tfinal;
    DevBuf<uint32_t> term;
    DevBuf<uint32_t> long_list;     // sort scratch (length classes)
    DevBuf<float4> grad_rows;     // [V][2] interleaved vertex gradient accumulator
    // Row bands [row0, row1) of the last render when its lists exceeded the
    // fragment budget (each band's lists are rebuilt by the adjoint); empty
    // when the lists are stored whole.
    std::vector<std::pair<int, int>> bands;
    bool cells = false;           // last render used per-cell colours
    dtv_tuning tuning{0, 0, dtv::kSortSurrogateDefault, dtv::kSortBucketDefault};
    u64* h_rowoff = nullptr;      // pinned row-start offsets (H+1)
    size_t h_rowoff_cap = 0;
    DevBuf<uint32_t> fill_order;    // faces in row-band order for the fill
    DevBuf<uint32_t> band_scratch;  // band counts and cursors of fill_order
    DevBuf<uint32_t> wide_list;     // [0] = n, then the faces of the 64-bit raster path (count -> fill)
    DevBuf<uint4> wstate;         // ray-tet path: (last tet, its entry face, boundary entry index, segments)
    u64* h_nf = nullptr;          // pinned
    // State of the last render.
    bool have_render = false;
    const dtv_mesh* mesh = nullptr;
    dtv::CamDev cam{};
    dtv::ShadeDev sh{};
    uint64_t P = 0, V = 0, nf = 0;
    // Stage timing.
    bool timing = false;
    cudaEvent_t ev[kNumStages + 2] = {};  // render: 0..6, adjoint: 7..8
    float stage_ms[kNumStages] = {};
    bool adjoint_timed = false;
};

namespace {

void rec_event(dtv_renderer* r, int idx, cudaStream_t s) {
    if (r->timing) DTV_CK(cudaEventRecord(r->ev[idx], s));
}

// Splits the image into row bands whose fragment records each fit `cap`
// (greedy, from the row-start offsets of the full scan).  Returns the largest
// band's record count.
uint64_t plan_bands(dtv_renderer* r, int W, int H, uint64_t cap, cudaStream_t s) {
    if (r->h_rowoff_cap < size_t(H) + 1) {
        if (r->h_rowoff) cudaFreeHost(r->h_rowoff);
        r->h_rowoff = nullptr;
        r->h_rowoff_cap = 0;
        DTV_CK(cudaMallocHost(&r->h_rowoff, sizeof(u64) * (size_t(H) + 1)));
        r->h_rowoff_cap = size_t(H) + 1;
    }
    // offsets[y * W] for y = 0..H: a strided copy of one u64 per row.
    DTV_CK(cudaMemcpy2DAsync(r->h_rowoff, sizeof(u64), r->offsets.ptr, sizeof(u64) * size_t(W), sizeof(u64),
                             size_t(H) + 1, cudaMemcpyDeviceToHost, s));
    DTV_CK(cudaStreamSynchronize(s));
    const u64* ro = r->h_rowoff;
    uint64_t largest = 0;
    int y0 = 0;
    while (y0 < H) {
        if (ro[y0 + 1] - ro[y0] > cap)
            throw DtvError(DTV_ERR_BUDGET, "pixel row " + std::to_string(y0) + " alone needs " +
                                               std::to_string(ro[y0 + 1] - ro[y0]) +
                                               " fragments, over the budget of " + std::to_string(cap));
        int y1 = y0 + 1;
        while (y1 < H && ro[y1 + 1] - ro[y0] <= cap) ++y1;
        r->bands.emplace_back(y0, y1);
        largest = std::max<uint64_t>(largest, ro[y1] - ro[y0]);
        y0 = y1;
    }
    return largest;
}

// Builds the sorted lists of rows [y0, y1) into the records buffer (band-local
// offsets): scan of the band's counts, fill (faces in the render's fill_order),
// per-pixel sort.  The band's counts must hold the rasterised counts; the fill
// leaves them zero.
void build_band_lists(dtv_renderer* r, const dtv_mesh* mesh, int W, int H, int y0, int y1, cudaStream_t s) {
    const uint64_t p0 = uint64_t(y0) * W, pb = uint64_t(y1 - y0) * W;
    dtv::launch_scan(r->counts.ptr + p0, pb, r->offsets.ptr + p0, r->scan_scratch.ptr, s);
    check_launch("band scan");
    dtv::launch_raster_fill(mesh->d_faces, uint32_t(mesh->host.num_faces), r->vproj.ptr, r->vfix.ptr, W, H,
                            r->counts.ptr, r->offsets.ptr, r->records.ptr, s, y0, y1, r->fill_order.ptr,
                            r->wide_list.ptr);
    check_launch("band fill");
    dtv::launch_sort(r->offsets.ptr + p0, r->records.ptr, uint32_t(pb), r->long_list.ptr, s, nullptr,
                     r->tuning.sort_surrogate_classes, r->tuning.sort_bucket_classes);
    check_launch("band sort");
}

// Composite of rows [y0, y1) with the stored lists: per-vertex colours
// (d_colors f32[4V]) or per-cell colours (f32[4T]).
void composite_rows(dtv_renderer* r, const dtv_mesh* mesh, const float* d_colors, const dtv::CamDev& cam,
                    const dtv::ShadeDev& sh, float* d_image, int y0, int y1, cudaStream_t s) {
    if (r->cells)
        dtv::launch_composite_cells(r->offsets.ptr, r->records.ptr, mesh->d_faces, mesh->d_face_to_tet, r->vgeo.ptr,
                                    reinterpret_cast<const float4*>(d_colors), cam.W, cam.H, sh,
                                    reinterpret_cast<float4*>(d_image), r->tfinal.ptr, r->term.ptr, s, y0, y1);
    else
        dtv::launch_composite(r->offsets.ptr, r->records.ptr, mesh->d_faces, r->vgeo.ptr,
                              reinterpret_cast<const float4*>(d_colors), cam.W, cam.H, sh,
                              reinterpret_cast<float4*>(d_image), r->tfinal.ptr, r->term.ptr, s, y0, y1,
                              r->tuning.composite_tile);
}

// Adjoint of rows [y0, y1) into the gradient rows (per-cell: the cell colour
// gradients go straight into d_grad_colors f32[4T]).
void adjoint_rows(dtv_renderer* r, const dtv_mesh* mesh, const float* d_colors, const float* d_image_adjoint,
                  const dtv::ShadeDev& sh, int y0, int y1, float* d_grad_colors, cudaStream_t s) {
    if (r->cells)
        dtv::launch_adjoint_cells_rows(r->offsets.ptr, r->records.ptr, mesh->d_faces, mesh->d_face_to_tet,
                                       r->vgeo.ptr, reinterpret_cast<const float4*>(d_colors), r->cam, sh,
                                       reinterpret_cast<const float4*>(d_image_adjoint), r->tfinal.ptr, r->term.ptr,
                                       y0, y1, r->grad_rows.ptr, reinterpret_cast<float4*>(d_grad_colors), s);
    else
        dtv::launch_adjoint_rows(r->offsets.ptr, r->records.ptr, mesh->d_faces, r->vgeo.ptr,
                                 reinterpret_cast<const float4*>(d_colors), r->cam, sh,
                                 reinterpret_cast<const float4*>(d_image_adjoint), r->tfinal.ptr, r->term.ptr, y0, y1,
                                 r->grad_rows.ptr, s, r->tuning.adjoint_tile);
}

// The list adjoint (launch_adjoint_rows) leaves screen-space position rows
// unless absolute gradients were asked for.
void scatter_rows(dtv_renderer* r, const dtv::ShadeDev& sh, float* d_grad_positions, float* d_grad_colors,
                  cudaStream_t s) {
    if (r->cells)
        dtv::launch_scatter_positions(r->grad_rows.ptr, uint32_t(r->V), d_grad_positions, s,
                                      sh.use_abs_grad ? nullptr : r->vgeo.ptr, &r->cam);
    else
        dtv::launch_scatter_grads(r->grad_rows.ptr, uint32_t(r->V), d_grad_positions,
                                  reinterpret_cast<float4*>(d_grad_colors), s,
                                  sh.use_abs_grad ? nullptr : r->vgeo.ptr, &r->cam);
}

// Forward in row bands (fragment lists over the budget): after the full count
// and scan, each band's lists are built and composited in turn, so at most
// `cap` records are held at once.  Counts of all rows come from the full count
// pass; each band's fill consumes its rows' counts.
void render_banded(dtv_renderer* r, const dtv_mesh* mesh, const float* d_colors, const dtv::CamDev& cam,
                   const dtv::ShadeDev& sh, float* d_image, uint64_t cap, cudaStream_t s) {
    const int W = cam.W, H = cam.H;
    uint64_t largest = 0;
    try {
        largest = plan_bands(r, W, H, cap, s);
        r->records.ensure(largest ? largest : 1, s, false, 1.0);
    } catch (...) {
        r->bands.clear();
        cudaMemsetAsync(r->counts.ptr, 0, uint64_t(W) * H * sizeof(uint32_t), s);
        throw;
    }
    rec_event(r, 3, s);
    for (const auto& b : r->bands) {
        build_band_lists(r, mesh, W, H, b.first, b.second, s);
        composite_rows(r, mesh, d_colors, cam, sh, d_image, b.first, b.second, s);
        check_launch("band composite");
    }
    rec_event(r, 4, s);
    rec_event(r, 5, s);
    rec_event(r, 6, s);
}

// Adjoint of a banded render: per band, the lists are rebuilt (count, scan,
// fill, sort of the band's rows, from the projection kept by the render) and
// the band's adjoint accumulates into the shared gradient rows.
void adjoint_banded(dtv_renderer* r, const dtv_mesh* mesh, const float* d_colors, const float* d_image_adjoint,
                    const dtv::ShadeDev& sh, float* d_grad_positions, float* d_grad_colors, cudaStream_t s) {
    const int W = r->cam.W, H = r->cam.H;
    DTV_CK(cudaMemsetAsync(r->grad_rows.ptr, 0, sizeof(float4) * 2 * size_t(r->V ? r->V : 1), s));
    r->wide_list.ensure(size_t(mesh->host.num_faces) + 1, s);
    for (const auto& b : r->bands) {
        dtv::launch_raster_count(mesh->d_faces, uint32_t(mesh->host.num_faces), r->vproj.ptr, r->vfix.ptr, W, H,
                                 r->counts.ptr, s, b.first, b.second, r->wide_list.ptr);
        check_launch("band count");
        build_band_lists(r, mesh, W, H, b.first, b.second, s);
        adjoint_rows(r, mesh, d_colors, d_image_adjoint, sh, b.first, b.second, d_grad_colors, s);
        check_launch("band adjoint");
    }
    scatter_rows(r, sh, d_grad_positions, d_grad_colors, s);
    check_launch("scatter gradients");
}

}  // namespace

extern "C" {

int32_t dtv_version(void) { return 100; }

const char* dtv_last_error_string(void) { return g_last_error.c_str(); }

int32_t dtv_build_hex_mesh(const float* aabb_min3, const float* aabb_max3, uint32_t xs, uint32_t ys, uint32_t zs,
                           uint32_t* h_cells, float* h_positions) {
    return guarded([&] {
        require(aabb_min3 && aabb_max3 && h_cells && h_positions, "null pointer");
        require(xs >= 2 && ys >= 2 && zs >= 2, "xs, ys, zs must be >= 2 (vertex counts per axis)");
        require(uint64_t(xs) * ys * zs < (1ull << 32), "grid too large for u32 vertex indices");
        dtv_build_hex_mesh_impl(aabb_min3, aabb_max3, xs, ys, zs, h_cells, h_positions);
    });
}

int32_t dtv_mesh_build_faces_host(const uint32_t* h_cells, uint64_t num_cells, uint64_t num_vertices,
                                  uint32_t* h_tri, uint32_t* h_fb, uint32_t* h_f2t, uint32_t* h_vb,
                                  uint64_t* num_faces) {
    return guarded([&] {
        require(h_cells != nullptr || num_cells == 0, "cells is null");
        require(h_tri && h_fb && h_f2t && h_vb && num_faces, "null output pointer");
        dtv::MeshHost mh;
        dtv::build_faces(h_cells, num_cells, num_vertices, mh);
        std::memcpy(h_tri, mh.tri.data(), sizeof(uint32_t) * mh.tri.size());
        std::memcpy(h_fb, mh.face_boundary.data(), sizeof(uint32_t) * mh.face_boundary.size());
        std::memcpy(h_f2t, mh.face_to_tet.data(), sizeof(uint32_t) * mh.face_to_tet.size());
        std::memcpy(h_vb, mh.vertex_boundary.data(), sizeof(uint32_t) * mh.vertex_boundary.size());
        *num_faces = mh.num_faces;
    });
}

int32_t dtv_mesh_create(const uint32_t* h_cells, uint64_t num_cells, uint64_t num_vertices, dtv_mesh** out) {
    return guarded([&] {
        require(out != nullptr, "out is null");
        require(h_cells != nullptr || num_cells == 0, "cells is null");
        require(num_vertices < (1ull << 32), "too many vertices");
        require(num_cells < (1ull << 28), "too many cells (face index must fit in 30 bits)");
        *out = nullptr;
        auto* m = new dtv_mesh();
        try {
            dtv::build_faces(h_cells, num_cells, num_vertices, m->host);
            const uint64_t F = m->host.num_faces;
            std::vector<uint4> faces(F);
            for (uint64_t f = 0; f < F; ++f)
                faces[f] = make_uint4(m->host.tri[3 * f], m->host.tri[3 * f + 1], m->host.tri[3 * f + 2],
                                      m->host.face_boundary[f]);
            DTV_CK(cudaMalloc(&m->d_faces, sizeof(uint4) * (F ? F : 1)));
            DTV_CK(cudaMalloc(&m->d_vertex_boundary, sizeof(uint32_t) * (num_vertices ? num_vertices : 1)));
            DTV_CK(cudaMalloc(&m->d_face_to_tet, sizeof(uint32_t) * (2 * F ? 2 * F : 1)));
            DTV_CK(cudaMalloc(&m->d_cells, sizeof(uint32_t) * (4 * num_cells ? 4 * num_cells : 1)));
            std::vector<uint4> bfaces;
            for (uint64_t f = 0; f < F; ++f)
                if (m->host.face_boundary[f]) {
                    m->bf_global.push_back(uint32_t(f));
                    bfaces.push_back(faces[f]);
                }
            const uint64_t Nb = m->bf_global.size();
            DTV_CK(cudaMalloc(&m->d_tet_faces, sizeof(uint32_t) * (4 * num_cells ? 4 * num_cells : 1)));
            DTV_CK(cudaMalloc(&m->d_tet_flip, num_cells ? num_cells : 1));
            DTV_CK(cudaMalloc(&m->d_bfaces, sizeof(uint4) * (Nb ? Nb : 1)));
            DTV_CK(cudaMalloc(&m->d_bf_global, sizeof(uint32_t) * (Nb ? Nb : 1)));
            if (Nb) {
                DTV_CK(cudaMemcpy(m->d_bfaces, bfaces.data(), sizeof(uint4) * Nb, cudaMemcpyHostToDevice));
                DTV_CK(cudaMemcpy(m->d_bf_global, m->bf_global.data(), sizeof(uint32_t) * Nb,
                                  cudaMemcpyHostToDevice));
            }
            if (num_cells) {
                DTV_CK(cudaMemcpy(m->d_tet_faces, m->host.tet_faces.data(), sizeof(uint32_t) * 4 * num_cells,
                                  cudaMemcpyHostToDevice));
                DTV_CK(cudaMemcpy(m->d_tet_flip, m->host.tet_flip.data(), num_cells, cudaMemcpyHostToDevice));
            }
            if (F) {
                DTV_CK(cudaMemcpy(m->d_faces, faces.data(), sizeof(uint4) * F, cudaMemcpyHostToDevice));
                DTV_CK(cudaMemcpy(m->d_face_to_tet, m->host.face_to_tet.data(), sizeof(uint32_t) * 2 * F,
                                  cudaMemcpyHostToDevice));
            }
            if (num_vertices)
                DTV_CK(cudaMemcpy(m->d_vertex_boundary, m->host.vertex_boundary.data(),
                                  sizeof(uint32_t) * num_vertices, cudaMemcpyHostToDevice));
            if (num_cells)
                DTV_CK(cudaMemcpy(m->d_cells, h_cells, sizeof(uint32_t) * 4 * num_cells, cudaMemcpyHostToDevice));
        } catch (...) {
            dtv_mesh_destroy(m);
            throw;
        }
        *out = m;
    });
}

int32_t dtv_mesh_destroy(dtv_mesh* m) {
    if (!m) return DTV_OK;
    cudaFree(m->d_faces);
    cudaFree(m->d_vertex_boundary);
    cudaFree(m->d_face_to_tet);
    cudaFree(m->d_cells);
    cudaFree(m->d_tet_faces);
    cudaFree(m->d_tet_flip);
    cudaFree(m->d_bfaces);
    cudaFree(m->d_bf_global);
    delete m;
    return DTV_OK;
}

int32_t dtv_mesh_get_info(const dtv_mesh* m, uint64_t* nc, uint64_t* nv, uint64_t* nfaces) {
    return guarded([&] {
        require(m != nullptr, "mesh is null");
        if (nc) *nc = m->host.num_cells;
        if (nv) *nv = m->host.num_vertices;
        if (nfaces) *nfaces = m->host.num_faces;
    });
}

int32_t dtv_mesh_copy_faces(const dtv_mesh* m, uint32_t* tri, uint32_t* fb, uint32_t* f2t, uint32_t* vb) {
    return guarded([&] {
        require(m != nullptr, "mesh is null");
        const auto& h = m->host;
        if (tri) std::memcpy(tri, h.tri.data(), sizeof(uint32_t) * h.tri.size());
        if (fb) std::memcpy(fb, h.face_boundary.data(), sizeof(uint32_t) * h.face_boundary.size());
        if (f2t) std::memcpy(f2t, h.face_to_tet.data(), sizeof(uint32_t) * h.face_to_tet.size());
        if (vb) std::memcpy(vb, h.vertex_boundary.data(), sizeof(uint32_t) * h.vertex_boundary.size());
    });
}

int32_t dtv_mesh_vertex_boundary_device(const dtv_mesh* m, const uint32_t** d_vb) {
    return guarded([&] {
        require(m != nullptr && d_vb != nullptr, "null pointer");
        *d_vb = m->d_vertex_boundary;
    });
}

int32_t dtv_renderer_create(int32_t type, dtv_renderer** out) {
    return guarded([&] {
        require(out != nullptr, "out is null");
        require(type == DTV_RENDERER_PPLL || type == DTV_RENDERER_INTERSECTION,
                "renderer type not provided by this library (PPLL = 0 and INTERSECTION = 2 are available)");
        *out = nullptr;
        auto* r = new dtv_renderer();
        r->type = type;
        try {
            DTV_CK(cudaMallocHost(&r->h_nf, sizeof(u64)));
            for (auto& e : r->ev) DTV_CK(cudaEventCreate(&e));
        } catch (...) {
            dtv_renderer_destroy(r);
            throw;
        }
        *out = r;
    });
}

int32_t dtv_renderer_destroy(dtv_renderer* r) {
    if (!r) return DTV_OK;
    cudaDeviceSynchronize();
    r->vproj.release();
    r->vfix.release();
    r->vgeo.release();
    r->counts.release();
    r->offsets.release();
    r->records.release();
    r->scan_scratch.release();
    r->tfinal.release();
    r->term.release();
    r->long_list.release();
    r->grad_rows.release();
    r->wstate.release();
    r->fill_order.release();
    r->band_scratch.release();
    r->wide_list.release();
    if (r->h_nf) cudaFreeHost(r->h_nf);
    if (r->h_rowoff) cudaFreeHost(r->h_rowoff);
    for (auto& e : r->ev)
        if (e) cudaEventDestroy(e);
    delete r;
    return DTV_OK;
}

}  // extern "C"

namespace {

// Forward render shared by dtv_renderer_render (per-vertex colours f32[4V])
// and dtv_renderer_render_cells (per-cell colours f32[4T]).
int32_t render_common(dtv_renderer* r, const dtv_mesh* mesh, const float* d_positions, const float* d_colors,
                      const dtv_camera* camera, const dtv_render_params* params, float* d_image, dtv_stream stream,
                      bool cells) {
    return guarded([&] {
        require(r && mesh && camera && params, "null handle or struct");
        require(!cells || r->type == DTV_RENDERER_PPLL,
                "per-cell colours are provided by the PPLL renderer only");
        require(d_positions && d_colors && d_image, "null device pointer");
        require((reinterpret_cast<uintptr_t>(d_colors) & 15u) == 0, "colors must be 16-byte aligned");
        require((reinterpret_cast<uintptr_t>(d_image) & 15u) == 0, "image must be 16-byte aligned");
        require(camera->width > 0 && camera->height > 0 && camera->width <= 16384 && camera->height <= 16384,
                "viewport size must be in [1, 16384]");
        require(camera->znear > 0.f && camera->zfar > camera->znear, "need 0 < znear < zfar");
        require(camera->fovy > 0.f && camera->fovy < 3.14159f, "fovy must be in (0, pi)");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        r->have_render = false;
        r->cells = cells;
        const bool raytet = r->type == DTV_RENDERER_INTERSECTION;
        const uint64_t V = mesh->host.num_vertices;
        // The ray-tet path rasterises only the boundary faces (interval entries and exits).
        const uint64_t F = raytet ? mesh->bf_global.size() : mesh->host.num_faces;
        const uint4* rfaces = raytet ? mesh->d_bfaces : mesh->d_faces;
        const int W = camera->width, H = camera->height;
        const uint64_t P = uint64_t(W) * H;
        dtv::CamDev cam = make_cam(*camera);
        dtv::ShadeDev sh = make_shade(*params);

        r->vproj.ensure(V ? V : 1, s);
        r->vfix.ensure(V ? V : 1, s);
        r->vgeo.ensure(V ? V : 1, s);
        r->counts.ensure(P, s, /*zero_new=*/true);
        r->offsets.ensure(P + 1, s);
        r->scan_scratch.ensure(dtv::scan_scratch_elems(P), s);
        r->tfinal.ensure(P, s);
        if (raytet)
            r->wstate.ensure(P, s);
        else
            r->term.ensure(P, s);
        r->long_list.ensure(dtv::sort_scratch_elems(P), s);

        rec_event(r, 0, s);
        dtv::launch_project(d_positions, uint32_t(V), cam, r->vproj.ptr, r->vfix.ptr, r->vgeo.ptr, s);
        check_launch("project");
        rec_event(r, 1, s);
        r->wide_list.ensure(size_t(F) + 1, s);
        dtv::launch_raster_count(rfaces, uint32_t(F), r->vproj.ptr, r->vfix.ptr, W, H, r->counts.ptr, s, 0, -1,
                                 r->wide_list.ptr);
        check_launch("raster count");
        rec_event(r, 2, s);
        dtv::launch_scan(r->counts.ptr, P, r->offsets.ptr, r->scan_scratch.ptr, s);
        check_launch("scan");
        DTV_CK(cudaMemcpyAsync(r->h_nf, r->offsets.ptr + P, sizeof(u64), cudaMemcpyDeviceToHost, s));
        DTV_CK(cudaStreamSynchronize(s));
        const uint64_t nf = *r->h_nf;
        const uint64_t budget = params->fragment_budget_bytes;
        r->bands.clear();
        if (budget && nf * sizeof(u64) > budget) {
            if (params->over_budget != DTV_OVER_BUDGET_RECOMPUTE || raytet) {
                // Leave counts zeroed for the next render.
                DTV_CK(cudaMemsetAsync(r->counts.ptr, 0, P * sizeof(uint32_t), s));
                throw DtvError(DTV_ERR_BUDGET, "render needs " + std::to_string(nf) + " fragments (" +
                                                   std::to_string(nf * sizeof(u64)) +
                                                   " bytes), over the budget of " + std::to_string(budget) +
                                                   " bytes");
            }
            r->fill_order.ensure(size_t(F), s);
            r->band_scratch.ensure(2 * dtv::kFillBands, s);
            dtv::launch_fill_order(rfaces, uint32_t(F), r->vfix.ptr, H, nf, r->fill_order.ptr, r->band_scratch.ptr,
                                   s);
            render_banded(r, mesh, d_colors, cam, sh, d_image, budget / sizeof(u64), s);
            r->adjoint_timed = false;
            r->have_render = true;
            r->mesh = mesh;
            r->cam = cam;
            r->sh = sh;
            r->P = P;
            r->V = V;
            r->nf = nf;
            return;
        }
        try {
            r->records.ensure(nf ? nf : 1, s, false, 1.25);
        } catch (...) {
            cudaMemsetAsync(r->counts.ptr, 0, P * sizeof(uint32_t), s);
            throw;
        }
        rec_event(r, 3, s);
        r->fill_order.ensure(size_t(F), s);
        r->band_scratch.ensure(2 * dtv::kFillBands, s);
        dtv::launch_fill_order(rfaces, uint32_t(F), r->vfix.ptr, H, nf, r->fill_order.ptr, r->band_scratch.ptr, s);
        dtv::launch_raster_fill(rfaces, uint32_t(F), r->vproj.ptr, r->vfix.ptr, W, H, r->counts.ptr,
                                r->offsets.ptr, r->records.ptr, s, 0, -1, r->fill_order.ptr, r->wide_list.ptr);
        check_launch("raster fill");
        rec_event(r, 4, s);
        dtv::launch_sort(r->offsets.ptr, r->records.ptr, uint32_t(P), r->long_list.ptr, s, nullptr,
                         r->tuning.sort_surrogate_classes, r->tuning.sort_bucket_classes);
        check_launch("sort");
        rec_event(r, 5, s);
        if (raytet) {
            dtv::launch_walk_composite(r->offsets.ptr, r->records.ptr, mesh->d_bf_global, mesh->d_faces,
                                       mesh->d_face_to_tet, mesh->d_tet_faces, mesh->d_cells, mesh->d_tet_flip,
                                       uint32_t(mesh->host.num_cells),
                                       r->vfix.ptr, r->vgeo.ptr, reinterpret_cast<const float4*>(d_colors), cam, sh,
                                       reinterpret_cast<float4*>(d_image), r->tfinal.ptr, r->wstate.ptr, s);
            check_launch("ray-tet walk");
        } else {
            composite_rows(r, mesh, d_colors, cam, sh, d_image, 0, H, s);
            check_launch("composite");
        }
        rec_event(r, 6, s);
        r->adjoint_timed = false;
        r->have_render = true;
        r->mesh = mesh;
        r->cam = cam;
        r->sh = sh;
        r->P = P;
        r->V = V;
        r->nf = nf;
    });
}

int32_t adjoint_common(dtv_renderer* r, const dtv_mesh* mesh, const float* d_positions, const float* d_colors,
                       const float* d_image_adjoint, int32_t use_abs_grad, float* d_grad_positions,
                       float* d_grad_colors, dtv_stream stream, bool cells) {
    return guarded([&] {
        require(r && mesh, "null handle");
        require(d_positions && d_colors && d_image_adjoint && d_grad_positions && d_grad_colors,
                "null device pointer");
        require((reinterpret_cast<uintptr_t>(d_colors) & 15u) == 0, "colors must be 16-byte aligned");
        require((reinterpret_cast<uintptr_t>(d_grad_colors) & 15u) == 0, "grad colors must be 16-byte aligned");
        require((reinterpret_cast<uintptr_t>(d_image_adjoint) & 15u) == 0,
                "image adjoint must be 16-byte aligned");
        if (!r->have_render) throw DtvError(DTV_ERR_STATE, "render_adjoint called before render");
        if (r->mesh != mesh) throw DtvError(DTV_ERR_STATE, "render_adjoint called with a different mesh");
        if (r->cells != cells)
            throw DtvError(DTV_ERR_STATE, cells ? "dtv_renderer_render_adjoint_cells after a per-vertex render"
                                                : "dtv_renderer_render_adjoint after a per-cell render");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        dtv::ShadeDev sh = r->sh;
        sh.use_abs_grad = use_abs_grad ? 1 : 0;
        r->grad_rows.ensure(2 * (r->V ? r->V : 1), s);
        rec_event(r, 7, s);
        if (!r->bands.empty()) {
            adjoint_banded(r, mesh, d_colors, d_image_adjoint, sh, d_grad_positions, d_grad_colors, s);
        } else if (r->type == DTV_RENDERER_INTERSECTION) {
            dtv::launch_walk_adjoint(r->offsets.ptr, r->records.ptr, mesh->d_bf_global, mesh->d_faces,
                                     mesh->d_face_to_tet, mesh->d_tet_faces, mesh->d_cells, mesh->d_tet_flip,
                                     uint32_t(mesh->host.num_cells),
                                     r->vfix.ptr, r->vgeo.ptr, reinterpret_cast<const float4*>(d_colors), r->cam, sh,
                                     reinterpret_cast<const float4*>(d_image_adjoint), r->tfinal.ptr,
                                     r->wstate.ptr, uint32_t(r->V), r->grad_rows.ptr, d_grad_positions,
                                     reinterpret_cast<float4*>(d_grad_colors), s);
            check_launch("ray-tet adjoint walk");
        } else {
            DTV_CK(cudaMemsetAsync(r->grad_rows.ptr, 0, sizeof(float4) * 2 * size_t(r->V ? r->V : 1), s));
            adjoint_rows(r, mesh, d_colors, d_image_adjoint, sh, 0, r->cam.H, d_grad_colors, s);
            check_launch("adjoint");
            scatter_rows(r, sh, d_grad_positions, d_grad_colors, s);
            check_launch("scatter gradients");
        }
        rec_event(r, 8, s);
        r->adjoint_timed = true;
    });
}

}  // namespace

extern "C" {

int32_t dtv_renderer_render(dtv_renderer* r, const dtv_mesh* mesh, const float* d_positions, const float* d_colors,
                            const dtv_camera* camera, const dtv_render_params* params, float* d_image,
                            dtv_stream stream) {
    return render_common(r, mesh, d_positions, d_colors, camera, params, d_image, stream, false);
}

int32_t dtv_renderer_render_cells(dtv_renderer* r, const dtv_mesh* mesh, const float* d_positions,
                                  const float* d_cell_colors, const dtv_camera* camera,
                                  const dtv_render_params* params, float* d_image, dtv_stream stream) {
    return render_common(r, mesh, d_positions, d_cell_colors, camera, params, d_image, stream, true);
}

int32_t dtv_renderer_render_adjoint(dtv_renderer* r, const dtv_mesh* mesh, const float* d_positions,
                                    const float* d_colors, const float* d_image_adjoint, int32_t use_abs_grad,
                                    float* d_grad_positions, float* d_grad_colors, dtv_stream stream) {
    return adjoint_common(r, mesh, d_positions, d_colors, d_image_adjoint, use_abs_grad, d_grad_positions,
                          d_grad_colors, stream, false);
}

int32_t dtv_renderer_render_adjoint_cells(dtv_renderer* r, const dtv_mesh* mesh, const float* d_positions,
                                          const float* d_cell_colors, const float* d_image_adjoint,
                                          int32_t use_abs_grad, float* d_grad_positions,
                                          float* d_grad_cell_colors, dtv_stream stream) {
    return adjoint_common(r, mesh, d_positions, d_cell_colors, d_image_adjoint, use_abs_grad, d_grad_positions,
                          d_grad_cell_colors, stream, true);
}

int32_t dtv_renderer_get_num_fragments(const dtv_renderer* r, uint64_t* nf) {
    return guarded([&] {
        require(r && nf, "null pointer");
        *nf = r->have_render ? r->nf : 0;
    });
}

int32_t dtv_renderer_set_tuning(dtv_renderer* r, const dtv_tuning* t) {
    return guarded([&] {
        require(r && t, "null pointer");
        require(t->composite_tile >= 0 && t->composite_tile <= 2 && t->adjoint_tile >= 0 && t->adjoint_tile <= 2,
                "tile index must be 0, 1 or 2");
        require((t->sort_surrogate_classes & ~0x1eu) == 0 && (t->sort_bucket_classes & ~0x3eu) == 0,
                "sort class masks: surrogate bits 1..4, bucket bits 1..5");
        r->tuning = *t;
    });
}

int32_t dtv_renderer_get_tuning(const dtv_renderer* r, dtv_tuning* t) {
    return guarded([&] {
        require(r && t, "null pointer");
        *t = r->tuning;
    });
}

int32_t dtv_renderer_get_num_bands(const dtv_renderer* r, int32_t* num_bands) {
    return guarded([&] {
        require(r && num_bands, "null pointer");
        *num_bands = r->have_render ? int32_t(r->bands.size()) : 0;
    });
}

int32_t dtv_renderer_copy_fragments(const dtv_renderer* r, uint64_t* h_offsets, uint64_t* h_records,
                                    uint64_t cap, dtv_stream stream) {
    return guarded([&] {
        require(r != nullptr, "renderer is null");
        if (!r->have_render) throw DtvError(DTV_ERR_STATE, "no render to copy from");
        if (!r->bands.empty())
            throw DtvError(DTV_ERR_STATE, "the last render ran in " + std::to_string(r->bands.size()) +
                                              " row bands under the fragment budget; its lists were not stored");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (h_offsets)
            DTV_CK(cudaMemcpyAsync(h_offsets, r->offsets.ptr, sizeof(u64) * (r->P + 1), cudaMemcpyDeviceToHost, s));
        if (h_records) {
            require(cap >= r->nf, "records capacity too small");
            if (r->nf)
                DTV_CK(cudaMemcpyAsync(h_records, r->records.ptr, sizeof(u64) * r->nf, cudaMemcpyDeviceToHost, s));
        }
        DTV_CK(cudaStreamSynchronize(s));
        if (h_records && r->type == DTV_RENDERER_INTERSECTION) {
            // Boundary-list records name faces of the boundary subset; report global face ids.
            const auto& bg = r->mesh->bf_global;
            for (uint64_t i = 0; i < r->nf; ++i) {
                const uint32_t lo = uint32_t(h_records[i]);
                const uint32_t g = bg[lo >> 2];
                h_records[i] = (h_records[i] & 0xffffffff00000000ull) | (uint64_t(g) << 2) | (lo & 3u);
            }
        }
    });
}

int32_t dtv_renderer_copy_pixel_state(const dtv_renderer* r, float* h_t, uint32_t* h_term, dtv_stream stream) {
    return guarded([&] {
        require(r != nullptr, "renderer is null");
        if (!r->have_render) throw DtvError(DTV_ERR_STATE, "no render to copy from");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (h_t) DTV_CK(cudaMemcpyAsync(h_t, r->tfinal.ptr, sizeof(float) * r->P, cudaMemcpyDeviceToHost, s));
        std::vector<uint4> ws;
        if (h_term && r->type == DTV_RENDERER_INTERSECTION) {
            // Ray-tet path: the per-pixel value is the number of tet segments composited.
            ws.resize(r->P);
            DTV_CK(cudaMemcpyAsync(ws.data(), r->wstate.ptr, sizeof(uint4) * r->P, cudaMemcpyDeviceToHost, s));
        } else if (h_term) {
            DTV_CK(cudaMemcpyAsync(h_term, r->term.ptr, sizeof(uint32_t) * r->P, cudaMemcpyDeviceToHost, s));
        }
        DTV_CK(cudaStreamSynchronize(s));
        for (uint64_t p = 0; p < ws.size(); ++p) h_term[p] = ws[p].w;
    });
}

int32_t dtv_renderer_set_timing(dtv_renderer* r, int32_t enable) {
    return guarded([&] {
        require(r != nullptr, "renderer is null");
        r->timing = enable != 0;
    });
}

int32_t dtv_renderer_stage_times(const dtv_renderer* r, float* h_ms, int32_t n) {
    return guarded([&] {
        require(r && h_ms, "null pointer");
        if (!r->timing || !r->have_render) throw DtvError(DTV_ERR_STATE, "timing not enabled or no render");
        const int stages = r->adjoint_timed ? 7 : 6;
        for (int i = 0; i < n && i < kNumStages; ++i) {
            h_ms[i] = 0.f;
            if (i < stages) {
                const int a = i < 6 ? i : 7;
                DTV_CK(cudaEventSynchronize(r->ev[a + 1]));
                DTV_CK(cudaEventElapsedTime(&h_ms[i], r->ev[a], r->ev[a + 1]));
            }
        }
    });
}

int32_t dtv_loss_l2(const float* d_image, const float* d_target, uint64_t n, float scale, float* d_adjoint,
                    float* d_loss, dtv_stream stream) {
    return guarded([&] {
        require(d_image && d_target, "null device pointer");
        dtv::launch_loss_l2(d_image, d_target, n, scale, d_adjoint, d_loss, static_cast<cudaStream_t>(stream));
        check_launch("loss");
    });
}

int32_t dtv_adam_step(float* d_param, const float* d_grad, float* d_m, float* d_v, uint64_t n, float lr,
                      float beta1, float beta2, float eps, int32_t step, int32_t clamp_mode,
                      const uint32_t* d_fixed_mask, int32_t fixed_mode, int32_t stride, dtv_stream stream) {
    return guarded([&] {
        require(d_param && d_grad && d_m && d_v, "null device pointer");
        require(step >= 1, "step must be >= 1");
        require(clamp_mode >= 0 && clamp_mode <= 2, "clamp_mode must be 0, 1 or 2");
        require(fixed_mode >= 0 && fixed_mode <= 2, "fixed_mode must be 0, 1 or 2");
        require(stride >= 1, "stride must be >= 1");
        require(clamp_mode != 2 || stride == 4 || n % 4 == 0, "clamp_mode 2 needs RGBA groups");
        const double bc1 = 1.0 - std::pow(double(beta1), double(step));
        const double bc2 = 1.0 - std::pow(double(beta2), double(step));
        dtv::launch_adam(d_param, d_grad, d_m, d_v, n, lr, beta1, beta2, eps, float(bc1), float(bc2), clamp_mode,
                         d_fixed_mask, fixed_mode, stride, static_cast<cudaStream_t>(stream));
        check_launch("adam");
    });
}

}  // extern "C"

// Helpers for the allocation-free entry point (dtv_noalloc.cu).
namespace dtv {
MeshView mesh_view(const dtv_mesh* m) { return MeshView{m->d_faces, m->host.num_faces, m->host.num_vertices}; }
uint64_t mesh_num_cells(const dtv_mesh* m) { return m->host.num_cells; }
const uint32_t* mesh_cells_device(const dtv_mesh* m) { return m->d_cells; }
CamDev camera_constants(const dtv_camera& c) { return make_cam(c); }
ShadeDev shade_constants(const dtv_render_params& p) { return make_shade(p); }
}  // namespace dtv

void dtv_set_last_error(const std::string& msg) { g_last_error = msg; }
