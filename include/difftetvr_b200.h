/*
 * difftetvr_b200 — C ABI of the B200-native differentiable tetrahedral
 * volume-rendering path.
 *
 * Plain pointers and sizes only.  Device pointers ("d_") are CUDA device
 * memory on the current device; host pointers ("h_") are host memory.  Every
 * function returns a status code (DTV_OK on success); the message of the last
 * failure on the calling thread is returned by dtv_last_error_string().
 *
 * Each entry point names the reference interface it replaces (paths inside
 * chrismile/DiffTetVR).  The Python module difftetvr_b200 binds this ABI with
 * ctypes and mirrors the reference module `difftetvr` (src/Module/Module.cpp).
 */
#ifndef DIFFTETVR_B200_H
#define DIFFTETVR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DTV_OK 0
#define DTV_ERR_ARG 1      /* invalid argument (bad pointer, size, alignment, enum) */
#define DTV_ERR_BUDGET 2   /* fragment storage exceeds the configured memory budget or a fixed limit */
#define DTV_ERR_CUDA 3     /* CUDA runtime error */
#define DTV_ERR_TIMEOUT 4  /* a bounded device-side wait gave up */
#define DTV_ERR_STATE 5    /* call out of order (e.g. adjoint before render) */

/* Renderer types, numbered as RendererType in src/Renderer/TetMeshRendererType.hpp:32-37. */
#define DTV_RENDERER_PPLL 0
#define DTV_RENDERER_PROJECTION 1   /* not provided; dtv_renderer_create returns DTV_ERR_ARG */
#define DTV_RENDERER_INTERSECTION 2 /* ray-tet: one segment per (pixel, tet), found by walking face adjacency */

typedef struct dtv_mesh dtv_mesh;
typedef struct dtv_renderer dtv_renderer;
typedef void* dtv_stream; /* cudaStream_t; NULL = legacy default stream */

/* Camera: Renderer.set_view_matrix (16 floats, column-major, Module.cpp:904-911),
 * Renderer.set_camera_fovy (radians, Module.cpp:900-903), near/far clip
 * (Module.cpp:458-460 defaults 0.01 / 100) and the viewport size
 * (Renderer.set_viewport_size, Module.cpp:874-887). */
typedef struct dtv_camera {
    float view[16];
    float fovy;
    float znear;
    float zfar;
    int32_t width;
    int32_t height;
} dtv_camera;

/* Per-render settings: Renderer.set_attenuation (Module.cpp:866),
 * set_use_early_ray_termination / set_early_ray_out_thresh (:868-870),
 * set_clear_color (:871-873); use_abs_grad is render_adjoint's flag (:922).
 * fragment_budget_bytes bounds the fragment records held at once (0 = no
 * bound).  When a render's records exceed it, over_budget selects what happens:
 * DTV_OVER_BUDGET_ERROR fails the render with DTV_ERR_BUDGET;
 * DTV_OVER_BUDGET_RECOMPUTE renders in row bands whose records each fit the
 * budget (the lists are then not stored: dtv_renderer_render_adjoint rebuilds
 * each band's lists before its adjoint, and dtv_renderer_copy_fragments fails
 * with DTV_ERR_STATE).  A single pixel row over the budget is DTV_ERR_BUDGET
 * in both modes. */
#define DTV_OVER_BUDGET_ERROR 0
#define DTV_OVER_BUDGET_RECOMPUTE 1
typedef struct dtv_render_params {
    float attenuation;
    int32_t use_early_ray_termination;
    float early_ray_out_thresh;
    float clear_color[4];
    int32_t use_abs_grad;
    int32_t over_budget;
    uint64_t fragment_budget_bytes;
} dtv_render_params;

/* Library version (major*10000 + minor*100 + patch). */
int32_t dtv_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char* dtv_last_error_string(void);

/* Tetrahedralised hex grid: replaces TetMesh::setHexMeshConst
 * (src/Tet/TetMesh.cpp:1882-1936; HEX_TO_TET_TABLE :104-117).  xs, ys, zs are
 * vertex counts per axis (>= 2).  h_cells receives 24*(xs-1)(ys-1)(zs-1) u32,
 * h_positions 3*xs*ys*zs floats. */
int32_t dtv_build_hex_mesh(const float* aabb_min3, const float* aabb_max3, uint32_t xs, uint32_t ys, uint32_t zs,
                           uint32_t* h_cells, float* h_positions);

/* Topology upload: replaces TetMesh::setTetMeshData (src/Tet/TetMesh.hpp:93-95)
 * with buildFacesSlim (TetMesh.cpp:1218-1268) and uploadDataToDevice
 * (TetMesh.cpp:560-778) for the face arrays.  Positions and colours stay
 * caller-owned device memory passed to each render. */
/* Host-only face build (same arrays and face order as dtv_mesh_create, no
 * device work): replaces buildFacesSlim (TetMesh.cpp:1218-1268).  h_tri needs
 * room for 3*4T entries, h_face_boundary 4T, h_face_to_tet 2*4T, h_vertex_boundary V;
 * *num_faces receives F. */
int32_t dtv_mesh_build_faces_host(const uint32_t* h_cells, uint64_t num_cells, uint64_t num_vertices,
                                  uint32_t* h_tri, uint32_t* h_face_boundary, uint32_t* h_face_to_tet,
                                  uint32_t* h_vertex_boundary, uint64_t* num_faces);
int32_t dtv_mesh_create(const uint32_t* h_cells, uint64_t num_cells, uint64_t num_vertices, dtv_mesh** out);
int32_t dtv_mesh_destroy(dtv_mesh* mesh);
/* TetMesh::getNumCells / getNumVertices (Module.cpp get_num_cells/get_num_vertices) and the face count. */
int32_t dtv_mesh_get_info(const dtv_mesh* mesh, uint64_t* num_cells, uint64_t* num_vertices, uint64_t* num_faces);
/* Host copies of the face arrays (triangleIndices u32[3F], faceBoundaryBit u32[F],
 * faceToTetMap u32[2F], vertexBoundaryBit u32[V]); any pointer may be NULL. */
int32_t dtv_mesh_copy_faces(const dtv_mesh* mesh, uint32_t* h_tri, uint32_t* h_face_boundary,
                            uint32_t* h_face_to_tet, uint32_t* h_vertex_boundary);
/* Device pointer of the per-vertex boundary bits (TetMesh::getVertexBoundaryBitTensor). */
int32_t dtv_mesh_vertex_boundary_device(const dtv_mesh* mesh, const uint32_t** d_vertex_boundary);

/* Renderer object: replaces the TetMeshVolumeRenderer subclasses
 * (TetMeshRendererPPLL.hpp:61-178, TetMeshRendererIntersection.hpp:41-135);
 * it owns the per-view fragment storage (the reference's fragment / start
 * offset buffers, TetMeshRendererPPLL.cpp:518-654). */
int32_t dtv_renderer_create(int32_t renderer_type, dtv_renderer** out);
int32_t dtv_renderer_destroy(dtv_renderer* r);

/* Forward render: replaces TetMeshRendererPPLL::render (TetMeshRendererPPLL.cpp:671-716)
 * / TetMeshRendererIntersection::render (:603-707) plus copyOutputImageToBuffer.
 * d_positions f32[3V], d_colors f32[4V] (16-byte aligned), d_image f32[H*W*4]
 * premultiplied RGBA over the clear colour.  Keeps the state the adjoint needs. */
int32_t dtv_renderer_render(dtv_renderer* r, const dtv_mesh* mesh, const float* d_positions,
                            const float* d_colors, const dtv_camera* camera, const dtv_render_params* params,
                            float* d_image, dtv_stream stream);

/* Adjoint: replaces TetMeshRendererPPLL::renderAdjoint (TetMeshRendererPPLL.cpp:718-724)
 * behind Renderer.render_adjoint (Module.cpp:922-959).  Gradients are ADDED to
 * d_grad_positions f32[3V] and d_grad_colors f32[4V] (16-byte aligned), as
 * the reference adds into the aliased .grad buffers.  Uses the camera and
 * parameters of the last dtv_renderer_render on this renderer (same mesh,
 * positions and colours).  use_abs_grad overrides params.use_abs_grad. */
int32_t dtv_renderer_render_adjoint(dtv_renderer* r, const dtv_mesh* mesh, const float* d_positions,
                                    const float* d_colors, const float* d_image_adjoint, int32_t use_abs_grad,
                                    float* d_grad_positions, float* d_grad_colors, dtv_stream stream);

/* Per-cell colours (ColorStorage::PER_CELL, Module.cpp:769-771): the same
 * render / adjoint with one RGBA per tet, d_cell_colors f32[4T] (16-byte
 * aligned).  Consecutive fragments bound a segment of the tet both faces
 * belong to (tetIdUnion, LinkedListResolve.glsl:85-94) with that cell's
 * constant colour and density (Forward.glsl:213-246, Backward.glsl:283-329);
 * the termination index counts fragments.  The adjoint ADDS into
 * d_grad_positions f32[3V] and d_grad_cell_colors f32[4T].  PPLL renderers
 * only; an adjoint must use the same colour storage as the render. */
int32_t dtv_renderer_render_cells(dtv_renderer* r, const dtv_mesh* mesh, const float* d_positions,
                                  const float* d_cell_colors, const dtv_camera* camera,
                                  const dtv_render_params* params, float* d_image, dtv_stream stream);
int32_t dtv_renderer_render_adjoint_cells(dtv_renderer* r, const dtv_mesh* mesh, const float* d_positions,
                                          const float* d_cell_colors, const float* d_image_adjoint,
                                          int32_t use_abs_grad, float* d_grad_positions,
                                          float* d_grad_cell_colors, dtv_stream stream);

/* Kernel configuration of a renderer (or batch): the pixel tile of the
 * composite blocks (0: 16 x 16, 1: 32 x 8, 2: 8 x 32 pixels), of the adjoint
 * blocks (0: 16 x 8, 1: 32 x 4, 2: 8 x 16) and,
 * per list-length class c (bit c; 1..4 = lists of up to 64, 128, 256, 512
 * records, 5 = up to 1024), the per-pixel sort method: distribution into
 * depth buckets plus an exact fix-up (bit c of sort_bucket_classes, c = 1..5),
 * else 32-bit surrogate keys through a bitonic network (bit c of
 * sort_surrogate_classes, c = 1..4), else the 64-bit bitonic network.  Every setting gives the same lists, images and
 * gradients; they differ in speed only.  An autotuner (difftetvr_b200.autotune)
 * times them on the caller's workload.  Batches use only the sort fields. */
typedef struct dtv_tuning {
    int32_t composite_tile;
    int32_t adjoint_tile;
    uint32_t sort_surrogate_classes;
    uint32_t sort_bucket_classes;
} dtv_tuning;
int32_t dtv_renderer_set_tuning(dtv_renderer* r, const dtv_tuning* tuning);
int32_t dtv_renderer_get_tuning(const dtv_renderer* r, dtv_tuning* tuning);

/* Total fragments of the last render (exact, from the scan). */
int32_t dtv_renderer_get_num_fragments(const dtv_renderer* r, uint64_t* num_fragments);

/* Row bands of the last render: 0 when its fragment lists were stored whole,
 * else the number of bands rendered (and recomputed by the adjoint) under
 * fragment_budget_bytes with DTV_OVER_BUDGET_RECOMPUTE.  No counterpart in the
 * reference, whose fragment buffer has a fixed size. */
int32_t dtv_renderer_get_num_bands(const dtv_renderer* r, int32_t* num_bands);

/* Sorted fragment lists of the last render: replaces get_fragment_buffer /
 * get_start_offset_buffer (Module.cpp:960-981) with an offsets + records
 * layout: h_offsets u64[H*W+1], h_records u64[Nf] where
 * record = (fp32 view-depth bits << 32) | (faceIndex << 2) | (boundary << 1) | frontFacing.
 * Either pointer may be NULL; records_capacity is the element count of h_records.
 * For an INTERSECTION renderer the lists hold the boundary faces only (the
 * interval entries and exits of each pixel ray); faceIndex is the global face id. */
int32_t dtv_renderer_copy_fragments(const dtv_renderer* r, uint64_t* h_offsets, uint64_t* h_records,
                                    uint64_t records_capacity, dtv_stream stream);

/* Per-pixel state of the last render: final transmittance f32[H*W] and the
 * termination index u32[H*W] (terminationIndexImage, Forward.glsl:256-259);
 * for an INTERSECTION renderer the second array is the number of tet segments
 * composited per pixel. */
int32_t dtv_renderer_copy_pixel_state(const dtv_renderer* r, float* h_transmittance, uint32_t* h_termination,
                                      dtv_stream stream);

/* Device time of each stage of the last render / adjoint, in ms:
 * [project, count, scan, fill, sort, composite, adjoint].  Stage timing is
 * recorded only after dtv_renderer_set_timing(r, 1).  A banded render reports
 * its whole band loop (scan, fill, sort, composite per band) as fill; a banded
 * adjoint includes the list rebuild. */
int32_t dtv_renderer_set_timing(dtv_renderer* r, int32_t enable);
int32_t dtv_renderer_stage_times(const dtv_renderer* r, float* h_ms, int32_t n);

/* Coarse-to-fine refinement: replaces TetMesh::subdivideVertices /
 * subdivideAtVertex (src/Tet/TetMesh.cpp:1374-1600, 1757-1784) behind
 * TetMesh.split_by_largest_gradient_magnitudes (Module.cpp:820-832).  For each
 * vertex of h_split_vertices in order, every incident edge gets a new vertex
 * at p_v + t (p_w - p_v) and every incident tet becomes the tet at v plus a
 * prism cut into three tets (diagonals through the smallest vertex index of
 * each quadrilateral: conforming); orientation and cell colour are inherited.
 * Host memory; colour arrays nullable.  The result (cells u32[4T'], positions
 * f32[3V'], vertex colours f32[4V'] / cell colours f32[4T'] when given) is
 * read with dtv_split_result_sizes / _copy and freed with _destroy. */
typedef struct dtv_split_result dtv_split_result;
int32_t dtv_mesh_subdivide_vertices(const uint32_t* h_cells, uint64_t num_cells, const float* h_positions,
                                    uint64_t num_vertices, const float* h_vertex_colors, const float* h_cell_colors,
                                    const uint32_t* h_split_vertices, uint64_t num_split, float t,
                                    dtv_split_result** out);
int32_t dtv_split_result_sizes(const dtv_split_result* r, uint64_t* num_cells, uint64_t* num_vertices);
int32_t dtv_split_result_copy(const dtv_split_result* r, uint32_t* h_cells, float* h_positions,
                              float* h_vertex_colors, float* h_cell_colors);
int32_t dtv_split_result_destroy(dtv_split_result* r);

/* .bintet mesh files: replaces BinTetLoader::loadFromFile / peekSizes and
 * BinTetWriter::saveToFile (src/Tet/Loaders/BinTetLoader.cpp:37-138) behind
 * TetMesh.load_from_file / save_to_file (Module.cpp:787-788).  Layout: u32
 * version (1, or 2 with cell colours), then u32-count-prefixed arrays of cell
 * indices (u32, count 4T), positions (3 f32 each), vertex colours (4 f32 each)
 * and, in version 2, cell colours (4 f32 each).  Host memory only.  Invalid
 * or truncated files fail with DTV_ERR_ARG.  dtv_bintet_read fills the arrays
 * sized by dtv_bintet_peek (colour pointers may be NULL to skip). */
int32_t dtv_bintet_peek(const char* path, uint32_t* version, uint64_t* num_cells, uint64_t* num_vertices,
                        uint64_t* num_vertex_colors, uint64_t* num_cell_colors);
int32_t dtv_bintet_read(const char* path, uint32_t* h_cells, float* h_positions, float* h_vertex_colors,
                        float* h_cell_colors);
/* Writes version 2 when num_cell_colors > 0, else version 1. */
int32_t dtv_bintet_write(const char* path, const uint32_t* h_cells, uint64_t num_cells, const float* h_positions,
                         uint64_t num_vertices, const float* h_vertex_colors, uint64_t num_vertex_colors,
                         const float* h_cell_colors, uint64_t num_cell_colors);

/* Tet-quality regularizer: replaces TetRegularizer.compute_grad (Module.cpp:663-695,
 * 983-995; TetRegularizerPass.cpp:94; Data/Shaders/Optimizer/TetRegularizer.glsl:108-166).
 * Per tet, the Parthasarathy quality q = 6 sqrt(2) V / l_rms^3 is penalised by
 * the mirrored softplus (lambda / beta) log(1 + exp(-beta q)); its gradient is
 * ADDED to d_grad_positions f32[3V].  d_loss (nullable, f32[1]) accumulates the
 * penalty summed over tets (the reference does not compute the value).
 * d_positions f32[3V] are the mesh's current vertex positions. */
int32_t dtv_tet_regularizer_grad(const dtv_mesh* mesh, const float* d_positions, float lambda, float beta,
                                 float* d_grad_positions, float* d_loss, dtv_stream stream);

/* Allocation-free forward render.  No counterpart in the reference: it is for
 * callers that cannot allocate device memory while rendering (a host
 * framework that owns the device heap, or a serving loop that must not call
 * cudaMalloc/cudaFree, which synchronise the device).  Same kernels and output
 * as dtv_renderer_render, with all scratch in one fixed file-scope device
 * array (about 39 MiB, held by every GPU that loads the library until exit).
 * Limits: <= 65,536 vertices, <= 65,536 pixels, <= 4,194,304 fragments; larger
 * requests return DTV_ERR_ARG / DTV_ERR_BUDGET.  The first call on a device
 * looks up the array's address (make it before any stream capture).  Calls
 * share the array, so calls that overlap on the GPU race; serialise them.
 * The call synchronises `stream` (it reads the exact fragment count). */
int32_t dtv_render_noalloc(const dtv_mesh* mesh, const float* d_positions, const float* d_colors,
                           const dtv_camera* camera, const dtv_render_params* params, float* d_image,
                           dtv_stream stream);

/* ---- Batched views (many cameras, several meshes, one launch per stage) ----
 * The reference renders one view per call; the batch renders and
 * differentiates many views of meshes of uneven size together.  A batch
 * holds a mesh table (dtv_batch_set_meshes); each view names its mesh. */
typedef struct dtv_batch dtv_batch;

typedef struct dtv_batch_view {
    int32_t mesh;              /* index into the batch's mesh table */
    int32_t grad_slot;         /* dtv_batch_render_adjoint: slot receiving this view's gradient, -1 = none */
    dtv_camera camera;         /* view matrix, fovy, clip planes, viewport size (may differ per view) */
    float* d_image;            /* out: f32[H*W*4], 16-byte aligned */
    const float* d_target;     /* dtv_batch_train_step: target image f32[H*W*4] */
    float* d_image_adjoint;    /* render_adjoint: dL/dimage (in); train step: written (NULL = internal) */
} dtv_batch_view;

typedef struct dtv_batch_grad_slot {
    int32_t mesh;              /* mesh of the views mapped to this slot */
    float* d_grad_positions;   /* f32[V*3]: gradients are ADDED */
    float* d_grad_colors;      /* f32[V*4], 16-byte aligned: gradients are ADDED */
} dtv_batch_grad_slot;

/* Adam of dtv_batch_train_step (torch.optim.Adam semantics, pytests/train.py:310-318,
 * 349-356): clamp_colors 0 none / 1 max(0) / 2 rgb in [0,1] alpha >= 0;
 * fixed_boundary 0 none / 1 zero boundary position gradients / 2 skip them. */
typedef struct dtv_batch_optim {
    float lr_positions;
    float lr_colors;
    float beta1;
    float beta2;
    float eps;
    int32_t clamp_colors;
    int32_t fixed_boundary;
} dtv_batch_optim;

int32_t dtv_batch_create(dtv_batch** out);
int32_t dtv_batch_destroy(dtv_batch* batch);
/* Sizes the batch's device scratch for up to max_views views, max_vertices
 * projected vertices (sum over views of the view's mesh size), max_pixels
 * pixels, max_fragments fragment records and max_grad_vertices gradient rows,
 * so later batches within these bounds allocate nothing (device allocation
 * synchronises the device, which a serving loop with several slots avoids). */
/* Forward render of a batch without a host synchronisation (for serving
 * loops): the record capacity already allocated (dtv_batch_reserve) bounds the
 * batch, and the kernels after the count and scan do nothing when the records
 * would not fit.  Once the stream has passed this render, dtv_batch_render_status
 * reports whether it fit and the fragment count; a batch that did not fit must
 * be rendered again with dtv_batch_render.  A dtv_batch_render_adjoint after
 * it is skipped on the device likewise. */
int32_t dtv_batch_render_async(dtv_batch* batch, int32_t num_views, const dtv_batch_view* views,
                               const dtv_render_params* params, dtv_stream stream);
int32_t dtv_batch_render_status(const dtv_batch* batch, int32_t* fits, uint64_t* num_fragments);
int32_t dtv_batch_set_tuning(dtv_batch* batch, const dtv_tuning* tuning);
int32_t dtv_batch_get_tuning(const dtv_batch* batch, dtv_tuning* tuning);
int32_t dtv_batch_reserve(dtv_batch* batch, uint64_t max_views, uint64_t max_vertices, uint64_t max_pixels,
                          uint64_t max_fragments, uint64_t max_grad_vertices, dtv_stream stream);
/* Mesh table: topology handles plus device positions f32[V*3] and colours f32[V*4]
 * (updated in place by dtv_batch_train_step). */
int32_t dtv_batch_set_meshes(dtv_batch* batch, int32_t num_meshes, const dtv_mesh* const* meshes,
                             float* const* d_positions, float* const* d_colors);
/* Forward render of all views (one synchronisation for the exact fragment count). */
int32_t dtv_batch_render(dtv_batch* batch, int32_t num_views, const dtv_batch_view* views,
                         const dtv_render_params* params, dtv_stream stream);
/* Adjoint of the last dtv_batch_render (same views, in the same order): each
 * view with grad_slot >= 0 reads its d_image_adjoint and adds its vertex
 * gradients into that slot. */
int32_t dtv_batch_render_adjoint(dtv_batch* batch, int32_t num_views, const dtv_batch_view* views,
                                 int32_t num_slots, const dtv_batch_grad_slot* slots, int32_t use_abs_grad,
                                 dtv_stream stream);
/* One training step over all views: render, L2 loss against each view's target
 * (torch.nn.MSELoss per view, summed into *d_loss), adjoint, Adam of every mesh. */
int32_t dtv_batch_train_step(dtv_batch* batch, int32_t num_views, const dtv_batch_view* views,
                             const dtv_render_params* params, const dtv_batch_optim* optim, float* d_loss,
                             dtv_stream stream);
/* Capture dtv_batch_train_step in a CUDA graph and replay it (1) or run eagerly (0). */
int32_t dtv_batch_set_graph(dtv_batch* batch, int32_t enable);
/* Fragments of the last step, record capacity, steps rerun after an overflow, graph in use. */
int32_t dtv_batch_get_info(const dtv_batch* batch, uint64_t* num_fragments, uint64_t* capacity,
                           uint64_t* steps_rerun, int32_t* graph_active);

/* L2 loss: replaces Loss.glsl:242-248 / torch.nn.MSELoss (pytests/train.py:321-326).
 * d_adjoint[i] = 2*scale*(d_image[i]-d_target[i]) (may be NULL);
 * *d_loss += scale * sum (d_image-d_target)^2 (may be NULL). */
int32_t dtv_loss_l2(const float* d_image, const float* d_target, uint64_t n, float scale, float* d_adjoint,
                    float* d_loss, dtv_stream stream);

/* Adam step: replaces Optimizer.glsl Compute.Adam (:88-169) and the
 * torch.optim.Adam step of pytests/train.py:318,351.  step >= 1 is the
 * 1-based time step.  clamp_mode: 0 none, 1 max(p,0) (train.py:352-356),
 * 2 rgb in [0,1] / alpha >= 0 (Optimizer.glsl:161-167).  d_fixed_mask (u32
 * per group of `stride` values, may be NULL) with fixed_mode 1 = zero the
 * gradient (train.py:349-350), 2 = skip the update (Optimizer.glsl:141-145). */
int32_t dtv_adam_step(float* d_param, const float* d_grad, float* d_m, float* d_v, uint64_t n, float lr,
                      float beta1, float beta2, float eps, int32_t step, int32_t clamp_mode,
                      const uint32_t* d_fixed_mask, int32_t fixed_mode, int32_t stride, dtv_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* DIFFTETVR_B200_H */
