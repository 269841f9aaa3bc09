// Check program for the C++ classes of include/difftetvr_b200.hpp, compiled
// against the public headers and libdifftetvr_b200.so only (tests/cpp/build.py).
//
//   cabi_classes errors            error paths that need no GPU
//   cabi_classes render DIR RES    one render + adjoint of the arrays in DIR
//                                  (cells.u32, pos.f32, col.f32, view.f32,
//                                  adj.f32), written back as image.f32,
//                                  gpos.f32, gcol.f32
// Prints "OK <mode>" and exits 0 on success.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "difftetvr_b200.hpp"

namespace dtv = difftetvr_b200;

template <class T>
static std::vector<T> read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error("cannot open " + path);
    const std::streamsize n = f.tellg();
    f.seekg(0);
    std::vector<T> v(size_t(n) / sizeof(T));
    f.read(reinterpret_cast<char*>(v.data()), n);
    return v;
}

template <class T>
static void write_file(const std::string& path, const std::vector<T>& v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(T)));
}

template <class F>
static bool throws_code(F&& fn, int32_t code) {
    try {
        fn();
    } catch (const dtv::Error& e) {
        return e.code() == code;
    }
    return false;
}

static int run_errors() {
    int bad = 0;
    auto expect = [&](bool ok, const char* what) {
        if (!ok) {
            std::printf("FAIL %s\n", what);
            ++bad;
        }
    };
    // The projection renderer is not provided (checked before any device work).
    expect(throws_code([] { dtv::Renderer r(dtv::TetMeshRendererType::PROJECTION); }, DTV_ERR_ARG),
           "PROJECTION renderer rejected");
    dtv::TetMesh mesh;
    expect(throws_code([&] { mesh.setTetMeshData({0, 1, 2}, {0, 0, 0, 1, 0, 0, 0, 1, 0}, {}); }, DTV_ERR_ARG),
           "cells not a multiple of 4");
    expect(throws_code([&] { mesh.setTetMeshData({0, 1, 2, 7}, std::vector<float>(12, 0.f), std::vector<float>(16)); },
                       DTV_ERR_ARG),
           "cell index out of range");
    expect(throws_code([&] { mesh.setTetMeshData({0, 1, 2, 3}, std::vector<float>(12, 0.f), std::vector<float>(8)); },
                       DTV_ERR_ARG),
           "colour count");
    expect(throws_code([&] { mesh.setTetMeshDataCell({0, 1, 2, 3}, std::vector<float>(12, 0.f), {}); }, DTV_ERR_ARG),
           "cell colour count");
    const float lo[3] = {-1, -1, -1}, hi[3] = {1, 1, 1}, c[4] = {1, 1, 1, 1};
    expect(throws_code([&] { mesh.setHexMeshConst(lo, hi, 1, 2, 2, c); }, DTV_ERR_ARG), "hex grid size");
    expect(!mesh.loadFromFile("/nonexistent/mesh.bintet"), "missing .bintet file");
    expect(mesh.getIsEmpty(), "mesh stays empty after failures");
    // The C ABI's messages reach the exception.
    try {
        dtv::check(dtv_build_hex_mesh(lo, hi, 1, 1, 1, nullptr, nullptr));
        expect(false, "dtv_build_hex_mesh with null output");
    } catch (const dtv::Error& e) {
        expect(e.code() == DTV_ERR_ARG && std::string(e.what()).size() > 0, "error message carried");
    }
    if (bad) return 1;
    std::printf("OK errors\n");
    return 0;
}

static int run_render(const std::string& dir, int res) {
    const auto cells = read_file<uint32_t>(dir + "/cells.u32");
    const auto pos = read_file<float>(dir + "/pos.f32");
    const auto col = read_file<float>(dir + "/col.f32");
    const auto view = read_file<float>(dir + "/view.f32");
    const auto adj = read_file<float>(dir + "/adj.f32");
    dtv::TetMesh mesh;
    mesh.setUseGradients(true);
    mesh.setTetMeshData(cells, pos, col);
    dtv::Renderer renderer(dtv::TetMeshRendererType::PPLL);
    renderer.setTetMeshData(mesh);
    renderer.setViewportSize(uint32_t(res), uint32_t(res));
    renderer.setCameraFovy(float(45.0 * M_PI / 180.0));
    renderer.setViewMatrix(view.data());
    renderer.setAttenuationCoefficient(1.0f);
    renderer.setUseEarlyRayTermination(false);
    renderer.setClearColor(0, 0, 0, 0);
    renderer.render();
    // renderAdjoint before an adjoint image is set is an ordering error.
    if (!throws_code([&] { renderer.renderAdjoint(); }, DTV_ERR_STATE)) {
        std::printf("FAIL renderAdjoint without adjoint image\n");
        return 1;
    }
    dtv::DeviceArray<float> d_adj;
    d_adj.upload(adj.data(), adj.size());
    renderer.copyAdjointBufferToImage(d_adj.data());
    renderer.renderAdjoint();
    write_file(dir + "/image.f32", renderer.getImage());
    write_file(dir + "/gpos.f32", mesh.getVertexPositionGradients());
    write_file(dir + "/gcol.f32", mesh.getColorGradients());
    std::printf("OK render fragments=%llu\n", static_cast<unsigned long long>(renderer.getNumFragments()));
    return 0;
}

int main(int argc, char** argv) {
    try {
        const std::string mode = argc > 1 ? argv[1] : "";
        if (mode == "errors") return run_errors();
        if (mode == "render" && argc > 3) return run_render(argv[2], std::atoi(argv[3]));
        std::fprintf(stderr, "usage: %s errors | render DIR RES\n", argv[0]);
        return 2;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
