// .bintet mesh files: the reference's BinTetLoader / BinTetWriter
// (src/Tet/Loaders/BinTetLoader.cpp:37-138).  Little-endian layout:
//   u32 version (1 or 2)
//   array cell indices      (u32 count = 4 T, then count x u32)
//   array vertex positions  (u32 count = V, then count x 3 f32)
//   array vertex colours    (u32 count, then count x 4 f32)
//   [version 2] array cell colours (u32 count = T, then count x 4 f32)
// Each array is written as a u32 element count followed by the raw elements,
// the layout of the length-prefixed arrays of sgl::BinaryWriteStream that the
// reference uses (peekSizes, BinTetLoader.cpp:72-93, reads it the same way).
// Version 1 files carry vertex colours, version 2 files also cell colours
// (the writer picks 2 whenever cell colours are given, :117-129).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "difftetvr_b200.h"
#include "dtv_host.h"

namespace {

using namespace dtv_host;

struct BinTetHeader {
    uint32_t version = 0;
    uint64_t n_cell_indices = 0, n_positions = 0, n_vertex_colors = 0, n_cell_colors = 0;
    long off_cells = 0, off_positions = 0, off_vertex_colors = 0, off_cell_colors = 0;
};

struct File {
    FILE* f = nullptr;
    explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

long file_size(FILE* f) {
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    return n;
}

// Reads the array headers and checks every array lies inside the file.
BinTetHeader read_header(FILE* f, const std::string& path) {
    BinTetHeader h;
    const long size = file_size(f);
    long pos = 0;
    auto read_u32 = [&](uint32_t& v) {
        if (pos + 4 > size || std::fread(&v, 4, 1, f) != 1)
            throw DtvError(DTV_ERR_ARG, "truncated .bintet file \"" + path + "\"");
        pos += 4;
    };
    auto array = [&](uint64_t& count, long& off, size_t elem) {
        uint32_t n = 0;
        read_u32(n);
        count = n;
        off = pos;
        const long bytes = long(elem * n);
        if (pos + bytes > size) throw DtvError(DTV_ERR_ARG, "truncated .bintet file \"" + path + "\"");
        pos += bytes;
        std::fseek(f, pos, SEEK_SET);
    };
    read_u32(h.version);
    if (h.version != 1u && h.version != 2u)
        throw DtvError(DTV_ERR_ARG, "invalid version number " + std::to_string(h.version) + " in .bintet file \"" +
                                        path + "\"");
    array(h.n_cell_indices, h.off_cells, 4);
    array(h.n_positions, h.off_positions, 12);
    array(h.n_vertex_colors, h.off_vertex_colors, 16);
    if (h.version == 2u) array(h.n_cell_colors, h.off_cell_colors, 16);
    if (h.n_cell_indices % 4 != 0)
        throw DtvError(DTV_ERR_ARG, "cell index count is not a multiple of 4 in \"" + path + "\"");
    return h;
}

void read_at(FILE* f, long off, void* dst, size_t bytes) {
    if (!bytes) return;
    std::fseek(f, off, SEEK_SET);
    if (std::fread(dst, 1, bytes, f) != bytes) throw DtvError(DTV_ERR_ARG, "read error");
}

}  // namespace

extern "C" {

int32_t dtv_bintet_peek(const char* path, uint32_t* version, uint64_t* num_cells, uint64_t* num_vertices,
                        uint64_t* num_vertex_colors, uint64_t* num_cell_colors) {
    return guarded([&] {
        require(path != nullptr, "path is null");
        File file(path, "rb");
        if (!file.f) throw DtvError(DTV_ERR_ARG, std::string("cannot open \"") + path + "\" for reading");
        const BinTetHeader h = read_header(file.f, path);
        if (version) *version = h.version;
        if (num_cells) *num_cells = h.n_cell_indices / 4;
        if (num_vertices) *num_vertices = h.n_positions;
        if (num_vertex_colors) *num_vertex_colors = h.n_vertex_colors;
        if (num_cell_colors) *num_cell_colors = h.n_cell_colors;
    });
}

int32_t dtv_bintet_read(const char* path, uint32_t* h_cells, float* h_positions, float* h_vertex_colors,
                        float* h_cell_colors) {
    return guarded([&] {
        require(path != nullptr, "path is null");
        File file(path, "rb");
        if (!file.f) throw DtvError(DTV_ERR_ARG, std::string("cannot open \"") + path + "\" for reading");
        const BinTetHeader h = read_header(file.f, path);
        require(h_cells || h.n_cell_indices == 0, "cells buffer is null");
        require(h_positions || h.n_positions == 0, "positions buffer is null");
        read_at(file.f, h.off_cells, h_cells, 4 * h.n_cell_indices);
        read_at(file.f, h.off_positions, h_positions, 12 * h.n_positions);
        if (h_vertex_colors) read_at(file.f, h.off_vertex_colors, h_vertex_colors, 16 * h.n_vertex_colors);
        if (h_cell_colors) read_at(file.f, h.off_cell_colors, h_cell_colors, 16 * h.n_cell_colors);
    });
}

int32_t dtv_bintet_write(const char* path, const uint32_t* h_cells, uint64_t num_cells, const float* h_positions,
                         uint64_t num_vertices, const float* h_vertex_colors, uint64_t num_vertex_colors,
                         const float* h_cell_colors, uint64_t num_cell_colors) {
    return guarded([&] {
        require(path != nullptr, "path is null");
        require(4 * num_cells < (1ull << 32) && num_vertices < (1ull << 32) && num_vertex_colors < (1ull << 32) &&
                    num_cell_colors < (1ull << 32),
                "array too large for the .bintet u32 counts");
        require((h_cells || num_cells == 0) && (h_positions || num_vertices == 0) &&
                    (h_vertex_colors || num_vertex_colors == 0) && (h_cell_colors || num_cell_colors == 0),
                "null buffer");
        File file(path, "wb");
        if (!file.f) throw DtvError(DTV_ERR_ARG, std::string("cannot open \"") + path + "\" for writing");
        const uint32_t version = num_cell_colors ? 2u : 1u;
        auto put = [&](const void* p, size_t bytes) {
            if (bytes && std::fwrite(p, 1, bytes, file.f) != bytes) throw DtvError(DTV_ERR_ARG, "write error");
        };
        auto array = [&](const void* p, uint64_t count, size_t elem) {
            const uint32_t n = uint32_t(count);
            put(&n, 4);
            put(p, elem * count);
        };
        put(&version, 4);
        array(h_cells, 4 * num_cells, 4);
        array(h_positions, num_vertices, 12);
        array(h_vertex_colors, num_vertex_colors, 16);
        if (version == 2u) array(h_cell_colors, num_cell_colors, 16);
        if (std::fflush(file.f) != 0) throw DtvError(DTV_ERR_ARG, "write error");
    });
}

}  // extern "C"
