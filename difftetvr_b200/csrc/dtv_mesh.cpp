// Host-side mesh preparation: tetrahedralised hex grid and unique-face build.
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "dtv_internal.h"

namespace dtv {

// Outward-wound faces of a tet (src/Tet/TetMesh.cpp:1175-1181).
static const int kTetFaceTable[4][3] = {{0, 1, 2}, {1, 0, 3}, {0, 2, 3}, {2, 1, 3}};

// Unique faces of a tet mesh: every tet contributes four faces; faces are
// identified by their sorted vertex triple, ordered by (triple, faceId), and
// each unique face keeps the winding of its lowest-faceId copy.  A face seen
// once is a boundary face.  Same result and face order as buildFacesSlim
// (TetMesh.cpp:1218-1268); implemented as a counting sort on the smallest
// vertex index followed by small per-bucket sorts, so 10^7-tet meshes prepare
// in about a second.
void build_faces(const uint32_t* cells, uint64_t T, uint64_t V, MeshHost& out) {
    const uint64_t NF4 = 4 * T;
    struct Rec {
        uint32_t v1, v2, fid;
    };
    std::vector<uint32_t> v0(NF4);
    std::vector<Rec> recs(NF4);
    for (uint64_t c = 0; c < T; ++c) {
        for (int j = 0; j < 4; ++j) {
            uint32_t a = cells[4 * c + kTetFaceTable[j][0]];
            uint32_t b = cells[4 * c + kTetFaceTable[j][1]];
            uint32_t d = cells[4 * c + kTetFaceTable[j][2]];
            if (a >= V || b >= V || d >= V) throw std::invalid_argument("cell vertex index out of range");
            uint32_t s[3] = {a, b, d};
            std::sort(s, s + 3);
            const uint64_t fid = 4 * c + j;
            v0[fid] = s[0];
            recs[fid] = Rec{s[1], s[2], uint32_t(fid)};
        }
    }
    // Counting sort by v0 (stable in fid order).
    std::vector<uint64_t> start(V + 1, 0);
    for (uint64_t i = 0; i < NF4; ++i) start[v0[i] + 1]++;
    for (uint64_t i = 0; i < V; ++i) start[i + 1] += start[i];
    std::vector<Rec> sorted(NF4);
    {
        std::vector<uint64_t> cur(start.begin(), start.end() - 1);
        for (uint64_t i = 0; i < NF4; ++i) sorted[cur[v0[i]]++] = recs[i];
    }
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t b = 0; b < int64_t(V); ++b) {
        std::sort(sorted.begin() + start[b], sorted.begin() + start[b + 1], [](const Rec& x, const Rec& y) {
            if (x.v1 != y.v1) return x.v1 < y.v1;
            if (x.v2 != y.v2) return x.v2 < y.v2;
            return x.fid < y.fid;
        });
    }
    out.tri.clear();
    out.face_boundary.clear();
    out.face_to_tet.clear();
    out.tri.reserve(3 * (NF4 / 2 + 16));
    out.face_boundary.reserve(NF4 / 2 + 16);
    out.face_to_tet.reserve(2 * (NF4 / 2 + 16));
    out.tet_faces.assign(NF4, 0u);
    for (uint64_t b = 0; b < V; ++b) {
        for (uint64_t i = start[b]; i < start[b + 1]; ++i) {
            const Rec& r = sorted[i];
            const bool same = (i > start[b]) && sorted[i - 1].v1 == r.v1 && sorted[i - 1].v2 == r.v2;
            const uint32_t tet = r.fid / 4;
            out.tet_faces[r.fid] = uint32_t(out.face_boundary.size() - (same ? 1 : 0));
            if (!same) {
                const int j = int(r.fid % 4);
                for (int k = 0; k < 3; ++k) out.tri.push_back(cells[4 * uint64_t(tet) + kTetFaceTable[j][k]]);
                out.face_boundary.push_back(1u);
                out.face_to_tet.push_back(tet);
                out.face_to_tet.push_back(0xffffffffu);
            } else {
                out.face_boundary.back() = 0u;
                out.face_to_tet.back() = tet;
            }
        }
    }
    out.num_faces = out.face_boundary.size();
    out.num_cells = T;
    out.num_vertices = V;
    out.vertex_boundary.assign(V, 0u);
    for (uint64_t f = 0; f < out.num_faces; ++f)
        if (out.face_boundary[f])
            for (int k = 0; k < 3; ++k) out.vertex_boundary[out.tri[3 * f + k]] = 1u;
    out.cells.assign(cells, cells + 4 * T);
    // Per tet and face j: is face j camera-facing for tet c when c's own
    // vertex order (kTetFaceTable) winds clockwise on screen?  The ray-tet walk
    // classifies faces by the stored winding of the unique face and whether c
    // owns it (owner: same order; other tet: the stored order read reversed);
    // k_j = !(odd_j ^ owner_j), odd_j = the stored order is an odd permutation
    // of c's order, turns that rule into one on c's own order.
    out.tet_flip.assign(T, 0u);
    for (uint64_t c = 0; c < T; ++c) {
        uint8_t mask = 0;
        for (int j = 0; j < 4; ++j) {
            const uint32_t f = out.tet_faces[4 * c + uint64_t(j)];
            const bool owner = out.face_to_tet[2 * uint64_t(f)] == uint32_t(c);
            const uint32_t a = cells[4 * c + kTetFaceTable[j][0]], b = cells[4 * c + kTetFaceTable[j][1]],
                           d = cells[4 * c + kTetFaceTable[j][2]];
            const uint32_t* s = &out.tri[3 * uint64_t(f)];
            const bool even = (s[0] == a && s[1] == b && s[2] == d) || (s[0] == b && s[1] == d && s[2] == a) ||
                              (s[0] == d && s[1] == a && s[2] == b);
            const bool odd = !even;
            if (!(odd ^ owner)) mask |= uint8_t(1u << j);
        }
        out.tet_flip[c] = mask;
    }
}

}  // namespace dtv

extern "C" {

// Kuhn / Freudenthal split of every hex of a regular vertex grid into six
// tets around the diagonal 0-6 (TetMesh::setHexMeshConst, TetMesh.cpp:1882-1936,
// with HEX_TO_TET_TABLE :104-117).  Vertex index = z*xs*ys + y*xs + x.
int32_t dtv_build_hex_mesh_impl(const float* mn, const float* mx, uint32_t xs, uint32_t ys, uint32_t zs,
                                uint32_t* cells, float* positions) {
    static const int kHexToTet[6][4] = {{0, 4, 7, 6}, {0, 4, 6, 5}, {0, 3, 6, 7},
                                        {0, 3, 2, 6}, {0, 1, 5, 6}, {0, 1, 6, 2}};
    uint64_t v = 0;
    for (uint32_t iz = 0; iz < zs; ++iz)
        for (uint32_t iy = 0; iy < ys; ++iy)
            for (uint32_t ix = 0; ix < xs; ++ix) {
                positions[3 * v + 0] = mn[0] + (float(ix) / float(xs - 1)) * (mx[0] - mn[0]);
                positions[3 * v + 1] = mn[1] + (float(iy) / float(ys - 1)) * (mx[1] - mn[1]);
                positions[3 * v + 2] = mn[2] + (float(iz) / float(zs - 1)) * (mx[2] - mn[2]);
                ++v;
            }
    const uint64_t dy = xs, dz = uint64_t(xs) * ys;
    uint64_t c = 0;
    for (uint32_t iz = 0; iz + 1 < zs; ++iz)
        for (uint32_t iy = 0; iy + 1 < ys; ++iy)
            for (uint32_t ix = 0; ix + 1 < xs; ++ix) {
                const uint64_t b = iz * dz + iy * dy + ix;
                uint32_t hex[8];
                hex[0] = uint32_t(b);
                hex[1] = uint32_t(b + 1);
                hex[2] = uint32_t(b + 1 + dy);
                hex[3] = uint32_t(b + dy);
                hex[4] = uint32_t(b + dz);
                hex[5] = uint32_t(b + 1 + dz);
                hex[6] = uint32_t(b + 1 + dy + dz);
                hex[7] = uint32_t(b + dy + dz);
                for (int t = 0; t < 6; ++t)
                    for (int k = 0; k < 4; ++k) cells[c++] = hex[kHexToTet[t][k]];
            }
    return 0;
}

}  // extern "C"
