/*
 * difftetvr_b200 — C++ classes over the C ABI (difftetvr_b200.h), with the
 * method names of the reference's C++ renderer interface so that code written
 * against TetMesh / TetMeshVolumeRenderer can switch to this library:
 *
 *   TetMesh   — src/Tet/TetMesh.hpp:86-140 (setTetMeshData, setTetMeshDataCell,
 *               setHexMeshConst, loadFromFile / saveToFile, onZeroGrad,
 *               getNumCells / getNumVertices, vertex / colour accessors)
 *   Renderer  — src/Renderer/TetMeshVolumeRenderer.hpp:84-165 (setTetMeshData,
 *               recreateSwapchain / setViewportSize, render, renderAdjoint,
 *               getImageTensor -> getImageDevice, copyAdjointBufferToImage,
 *               attenuation / clear colour / early-ray-termination setters)
 *
 * Header only; needs the CUDA runtime (device buffers) and libdifftetvr_b200.
 * Every failing call throws difftetvr_b200::Error carrying the DTV_ERR_* code
 * and the library's message (the reference throws through sgl::Logfile).
 * The vertex data live in device memory owned by the TetMesh; gradients are
 * accumulated into device buffers of the mesh (the reference's .grad buffers),
 * cleared by onZeroGrad().
 */
#ifndef DIFFTETVR_B200_HPP
#define DIFFTETVR_B200_HPP

#include <cuda_runtime_api.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "difftetvr_b200.h"

namespace difftetvr_b200 {

// TetMeshRendererType (src/Renderer/TetMeshRendererType.hpp:32-37).
enum class TetMeshRendererType : int32_t { PPLL = DTV_RENDERER_PPLL, PROJECTION = DTV_RENDERER_PROJECTION,
                                           INTERSECTION = DTV_RENDERER_INTERSECTION };
// ColorStorage (src/Tet/TetMesh.hpp, Module.cpp:769-771).
enum class ColorStorage : int32_t { PER_VERTEX = 0, PER_CELL = 1 };

class Error : public std::runtime_error {
public:
    Error(int32_t code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
    int32_t code() const { return code_; }

private:
    int32_t code_;
};

inline void check(int32_t rc) {
    if (rc != DTV_OK) throw Error(rc, dtv_last_error_string());
}

inline void checkCuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(DTV_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Owned device array of T.
template <class T>
class DeviceArray {
public:
    DeviceArray() = default;
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    DeviceArray(DeviceArray&& o) noexcept : ptr_(o.ptr_), n_(o.n_) { o.ptr_ = nullptr; o.n_ = 0; }
    DeviceArray& operator=(DeviceArray&& o) noexcept {
        if (this != &o) {
            release();
            std::swap(ptr_, o.ptr_);
            std::swap(n_, o.n_);
        }
        return *this;
    }
    ~DeviceArray() { release(); }

    void resize(size_t n) {
        if (n == n_) return;
        release();
        if (n) checkCuda(cudaMalloc(reinterpret_cast<void**>(&ptr_), n * sizeof(T)), "cudaMalloc");
        n_ = n;
    }
    void upload(const T* h, size_t n) {
        resize(n);
        if (n) checkCuda(cudaMemcpy(ptr_, h, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    }
    std::vector<T> download() const {
        std::vector<T> h(n_);
        if (n_) checkCuda(cudaMemcpy(h.data(), ptr_, n_ * sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
        return h;
    }
    void zero(cudaStream_t s = nullptr) {
        if (n_) checkCuda(cudaMemsetAsync(ptr_, 0, n_ * sizeof(T), s), "cudaMemsetAsync");
    }
    T* data() { return ptr_; }
    const T* data() const { return ptr_; }
    size_t size() const { return n_; }
    void release() {
        if (ptr_) cudaFree(ptr_);
        ptr_ = nullptr;
        n_ = 0;
    }

private:
    T* ptr_ = nullptr;
    size_t n_ = 0;
};

class TetMesh {
public:
    TetMesh() = default;
    TetMesh(const TetMesh&) = delete;
    TetMesh& operator=(const TetMesh&) = delete;
    ~TetMesh() { destroyHandle(); }

    // TetMesh::setTetMeshData (TetMesh.hpp:93-95): cells u32[4T], positions
    // f32[3V] (vec3), vertex colours f32[4V] (vec4).
    void setTetMeshData(const std::vector<uint32_t>& cellIndices, const std::vector<float>& vertexPositions,
                        const std::vector<float>& vertexColors) {
        validate(cellIndices, vertexPositions);
        if (vertexColors.size() != vertexPositions.size() / 3 * 4)
            throw Error(DTV_ERR_ARG, "setTetMeshData: need 4 colour values per vertex");
        upload(cellIndices, vertexPositions, vertexColors, ColorStorage::PER_VERTEX);
    }
    // TetMesh::setTetMeshDataCell (TetMesh.hpp:96-98): one RGBA per tet.
    void setTetMeshDataCell(const std::vector<uint32_t>& cellIndices, const std::vector<float>& vertexPositions,
                            const std::vector<float>& cellColors) {
        validate(cellIndices, vertexPositions);
        if (cellColors.size() != cellIndices.size())
            throw Error(DTV_ERR_ARG, "setTetMeshDataCell: need 4 colour values per cell");
        upload(cellIndices, vertexPositions, cellColors, ColorStorage::PER_CELL);
    }
    // TetMesh::setHexMeshConst (TetMesh.cpp:1882-1936): xs, ys, zs vertex counts per axis.
    void setHexMeshConst(const float aabbMin[3], const float aabbMax[3], uint32_t xs, uint32_t ys, uint32_t zs,
                         const float constColor[4], ColorStorage storage = ColorStorage::PER_VERTEX) {
        if (xs < 2 || ys < 2 || zs < 2) throw Error(DTV_ERR_ARG, "setHexMeshConst: xs, ys, zs must be >= 2");
        const size_t V = size_t(xs) * ys * zs, T = 6 * size_t(xs - 1) * (ys - 1) * (zs - 1);
        std::vector<uint32_t> cells(4 * T);
        std::vector<float> pos(3 * V);
        check(dtv_build_hex_mesh(aabbMin, aabbMax, xs, ys, zs, cells.data(), pos.data()));
        std::vector<float> col(4 * (storage == ColorStorage::PER_VERTEX ? V : T));
        for (size_t i = 0; i < col.size(); ++i) col[i] = constColor[i % 4];
        upload(cells, pos, col, storage);
    }
    // TetMesh::loadFromFile / saveToFile for .bintet (BinTetLoader.cpp:37-138).
    bool loadFromFile(const std::string& path) {
        uint32_t version = 0;
        uint64_t nc = 0, nv = 0, nvc = 0, ncc = 0;
        if (dtv_bintet_peek(path.c_str(), &version, &nc, &nv, &nvc, &ncc) != DTV_OK) return false;
        std::vector<uint32_t> cells(4 * nc);
        std::vector<float> pos(3 * nv), vcol(4 * nvc), ccol(4 * ncc);
        if (dtv_bintet_read(path.c_str(), cells.data(), pos.data(), nvc ? vcol.data() : nullptr,
                            ncc ? ccol.data() : nullptr) != DTV_OK)
            return false;
        if (ncc && !nvc)
            setTetMeshDataCell(cells, pos, ccol);
        else
            setTetMeshData(cells, pos, vcol);
        return true;
    }
    bool saveToFile(const std::string& path) const {
        const std::vector<float> pos = positions_.download(), col = colors_.download();
        const bool cellStorage = storage_ == ColorStorage::PER_CELL;
        return dtv_bintet_write(path.c_str(), cells_.data(), numCells_, pos.data(), numVertices_,
                                cellStorage ? nullptr : col.data(), cellStorage ? 0 : numVertices_,
                                cellStorage ? col.data() : nullptr, cellStorage ? numCells_ : 0) == DTV_OK;
    }

    // TetMesh::setUseGradients / onZeroGrad (Module.cpp:785, 792-793): the
    // gradient buffers start (and are reset) at zero.
    void setUseGradients(bool useGradients) {
        useGradients_ = useGradients;
        if (useGradients) {
            gradPositions_.resize(positions_.size());
            gradColors_.resize(colors_.size());
            onZeroGrad();
        }
    }
    bool getUseGradients() const { return useGradients_; }
    void onZeroGrad() {
        gradPositions_.zero();
        gradColors_.zero();
    }

    uint64_t getNumCells() const { return numCells_; }
    uint64_t getNumVertices() const { return numVertices_; }
    ColorStorage getColorStorage() const { return storage_; }
    bool getIsEmpty() const { return handle_ == nullptr; }
    const std::vector<uint32_t>& getCellIndices() const { return cells_; }
    // Host copies of the current device data.
    std::vector<float> getVertexPositions() const { return positions_.download(); }
    std::vector<float> getColors() const { return colors_.download(); }
    std::vector<float> getVertexPositionGradients() const { return gradPositions_.download(); }
    std::vector<float> getColorGradients() const { return gradColors_.download(); }
    // Device buffers (f32[3V] positions, f32[4V] or f32[4T] colours and their gradients).
    float* getVertexPositionsDevice() { return positions_.data(); }
    float* getColorsDevice() { return colors_.data(); }
    float* getVertexPositionGradientsDevice() { return gradPositions_.data(); }
    float* getColorGradientsDevice() { return gradColors_.data(); }
    const dtv_mesh* handle() const { return handle_; }

private:
    static void validate(const std::vector<uint32_t>& cells, const std::vector<float>& pos) {
        if (cells.empty() || cells.size() % 4 != 0) throw Error(DTV_ERR_ARG, "setTetMeshData: need 4 indices per cell");
        if (pos.empty() || pos.size() % 3 != 0)
            throw Error(DTV_ERR_ARG, "setTetMeshData: need 3 position values per vertex");
        const uint64_t V = pos.size() / 3;
        for (uint32_t c : cells)
            if (c >= V) throw Error(DTV_ERR_ARG, "setTetMeshData: cell index out of range");
    }
    void upload(const std::vector<uint32_t>& cells, const std::vector<float>& pos, const std::vector<float>& col,
                ColorStorage storage) {
        destroyHandle();
        numCells_ = cells.size() / 4;
        numVertices_ = pos.size() / 3;
        check(dtv_mesh_create(cells.data(), numCells_, numVertices_, &handle_));
        cells_ = cells;
        storage_ = storage;
        positions_.upload(pos.data(), pos.size());
        colors_.upload(col.data(), col.size());
        if (useGradients_) setUseGradients(true);
    }
    void destroyHandle() {
        if (handle_) dtv_mesh_destroy(handle_);
        handle_ = nullptr;
    }

    dtv_mesh* handle_ = nullptr;
    uint64_t numCells_ = 0, numVertices_ = 0;
    ColorStorage storage_ = ColorStorage::PER_VERTEX;
    bool useGradients_ = false;
    std::vector<uint32_t> cells_;
    DeviceArray<float> positions_, colors_, gradPositions_, gradColors_;
};

class Renderer {
public:
    explicit Renderer(TetMeshRendererType type = TetMeshRendererType::PPLL) : type_(type) {
        check(dtv_renderer_create(int32_t(type), &handle_));
        // Defaults of the reference (TetMeshVolumeRenderer.hpp:237-244, Module.cpp:458-463).
        const float view[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, -0.8f, 1};
        std::memcpy(camera_.view, view, sizeof(view));
        camera_.fovy = 2.0f * 0.4636476f;  // 2 atan(1/2)
        camera_.znear = 0.01f;
        camera_.zfar = 100.0f;
        camera_.width = camera_.height = 1;
        params_.attenuation = 100.0f;
        params_.use_early_ray_termination = 1;
        params_.early_ray_out_thresh = 1e-4f;
        params_.over_budget = DTV_OVER_BUDGET_RECOMPUTE;
    }
    Renderer(const Renderer&) = delete;
    Renderer& operator=(const Renderer&) = delete;
    ~Renderer() {
        if (handle_) dtv_renderer_destroy(handle_);
    }

    TetMeshRendererType getRendererType() const { return type_; }
    // TetMeshVolumeRenderer::setTetMeshData (hpp:95).
    void setTetMeshData(TetMesh& mesh) { mesh_ = &mesh; }
    TetMesh* getTetMeshData() const { return mesh_; }
    // recreateSwapchain / setViewportSize (hpp:93, 121): the image size.
    void recreateSwapchain(uint32_t width, uint32_t height) { setViewportSize(width, height); }
    void setViewportSize(uint32_t width, uint32_t height) {
        if (width == 0 || height == 0) throw Error(DTV_ERR_ARG, "setViewportSize: size must be positive");
        camera_.width = int32_t(width);
        camera_.height = int32_t(height);
    }
    float getAttenuationCoefficient() const { return params_.attenuation; }
    void setAttenuationCoefficient(float a) { params_.attenuation = a; }
    void setClearColor(float r, float g, float b, float a) {
        params_.clear_color[0] = r;
        params_.clear_color[1] = g;
        params_.clear_color[2] = b;
        params_.clear_color[3] = a;
    }
    void setUseAbsGrad(bool useAbsGrad) { useAbsGrad_ = useAbsGrad; }
    void setUseEarlyRayTermination(bool use) { useErt_ = use; }
    void setEarlyRayOutThresh(float thresh) { params_.early_ray_out_thresh = thresh; }
    void setEarlyRayOutAlpha(float alpha) { params_.early_ray_out_thresh = 1.0f - alpha; }
    // Camera (sgl::Camera in the reference; Module.cpp:900-911): column-major
    // view matrix, vertical field of view in radians, clip planes.
    void setViewMatrix(const float view[16]) { std::memcpy(camera_.view, view, sizeof(camera_.view)); }
    void setCameraFovy(float fovy) { camera_.fovy = fovy; }
    void setCameraClip(float znear, float zfar) {
        camera_.znear = znear;
        camera_.zfar = zfar;
    }
    // Fragment-storage bound (bytes, 0 = none); over it the render runs in
    // row bands (recompute = true) or fails with DTV_ERR_BUDGET.
    void setFragmentBudget(uint64_t bytes, bool recompute = true) {
        params_.fragment_budget_bytes = bytes;
        params_.over_budget = recompute ? DTV_OVER_BUDGET_RECOMPUTE : DTV_OVER_BUDGET_ERROR;
    }
    void setStream(cudaStream_t stream) { stream_ = stream; }

    // TetMeshVolumeRenderer::render (hpp:116): premultiplied RGBA f32[H][W][4]
    // into the renderer's image buffer (getImageDevice).
    void render() {
        TetMesh& m = requireMesh("render");
        image_.resize(size_t(camera_.width) * camera_.height * 4);
        dtv_render_params p = params_;
        // Early ray termination only with gradients on (TetMeshVolumeRenderer.cpp:417-419).
        p.use_early_ray_termination = (useErt_ && m.getUseGradients()) ? 1 : 0;
        if (m.getColorStorage() == ColorStorage::PER_CELL)
            check(dtv_renderer_render_cells(handle_, m.handle(), m.getVertexPositionsDevice(), m.getColorsDevice(),
                                            &camera_, &p, image_.data(), stream_));
        else
            check(dtv_renderer_render(handle_, m.handle(), m.getVertexPositionsDevice(), m.getColorsDevice(),
                                      &camera_, &p, image_.data(), stream_));
        rendered_ = true;
    }
    // copyAdjointBufferToImage (hpp:125): dL/dimage f32[H][W][4] from device memory.
    void copyAdjointBufferToImage(const float* d_imageAdjoint) {
        imageAdjoint_.resize(size_t(camera_.width) * camera_.height * 4);
        checkCuda(cudaMemcpyAsync(imageAdjoint_.data(), d_imageAdjoint, imageAdjoint_.size() * sizeof(float),
                                  cudaMemcpyDeviceToDevice, stream_),
                  "copyAdjointBufferToImage");
    }
    // TetMeshVolumeRenderer::renderAdjoint (hpp:117): adds the gradients of the
    // last render into the mesh's gradient buffers (setUseGradients(true)).
    void renderAdjoint() {
        TetMesh& m = requireMesh("renderAdjoint");
        if (!rendered_) throw Error(DTV_ERR_STATE, "renderAdjoint called before render");
        if (!m.getUseGradients()) throw Error(DTV_ERR_STATE, "renderAdjoint: the mesh does not use gradients");
        if (imageAdjoint_.size() != size_t(camera_.width) * camera_.height * 4)
            throw Error(DTV_ERR_STATE, "renderAdjoint: no adjoint image (copyAdjointBufferToImage)");
        if (m.getColorStorage() == ColorStorage::PER_CELL)
            check(dtv_renderer_render_adjoint_cells(handle_, m.handle(), m.getVertexPositionsDevice(),
                                                    m.getColorsDevice(), imageAdjoint_.data(), useAbsGrad_ ? 1 : 0,
                                                    m.getVertexPositionGradientsDevice(),
                                                    m.getColorGradientsDevice(), stream_));
        else
            check(dtv_renderer_render_adjoint(handle_, m.handle(), m.getVertexPositionsDevice(), m.getColorsDevice(),
                                              imageAdjoint_.data(), useAbsGrad_ ? 1 : 0,
                                              m.getVertexPositionGradientsDevice(), m.getColorGradientsDevice(),
                                              stream_));
    }
    // getImageTensor (hpp:122): the image of the last render in device memory.
    const float* getImageDevice() const { return image_.data(); }
    std::vector<float> getImage() const {
        checkCuda(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
        return image_.download();
    }
    uint64_t getNumFragments() const {
        uint64_t n = 0;
        check(dtv_renderer_get_num_fragments(handle_, &n));
        return n;
    }
    dtv_renderer* handle() const { return handle_; }

private:
    TetMesh& requireMesh(const char* what) const {
        if (!mesh_ || mesh_->getIsEmpty()) throw Error(DTV_ERR_STATE, std::string("Missing valid tet mesh in ") + what);
        return *mesh_;
    }

    TetMeshRendererType type_;
    dtv_renderer* handle_ = nullptr;
    TetMesh* mesh_ = nullptr;
    dtv_camera camera_{};
    dtv_render_params params_{};
    bool useErt_ = true, useAbsGrad_ = false, rendered_ = false;
    cudaStream_t stream_ = nullptr;
    DeviceArray<float> image_, imageAdjoint_;
};

}  // namespace difftetvr_b200

#endif  // DIFFTETVR_B200_HPP
