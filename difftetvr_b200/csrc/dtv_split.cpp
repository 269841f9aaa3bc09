// Coarse-to-fine refinement: subdivision of the tets around chosen vertices.
//
// Reference: TetMesh::subdivideVertices / subdivideAtVertex
// (src/Tet/TetMesh.cpp:1374-1600, 1757-1784), called by
// split_by_largest_gradient_magnitudes (Module.cpp:820-832, TetMesh.cpp:1786-1881)
// for the vertices with the largest gradient magnitudes, in descending order.
// Splitting at vertex v: every edge (v, w) gets a new vertex at
// p_v + t (p_w - p_v) (vertex colour interpolated the same way); every tet of
// v's star becomes the tet (v, m_a, m_b, m_c) at v plus the prism between the
// triangle (m_a, m_b, m_c) and the opposite face (a, b, c), cut into three
// tets; new tets keep the cell colour of the tet they came from.
//
// The prisms are cut with the rule of Dompierre et al. (1999, "How to
// subdivide pyramids, prisms and hexahedra into tetrahedra"): each quadrilateral
// face is divided along the diagonal through its vertex of smallest index.  Two
// prisms sharing a quadrilateral therefore cut it the same way, and the three
// diagonals of a prism never form a cycle, so every prism has a valid 3-tet
// decomposition (the reference solves a constraint problem for the same
// purpose, TetMesh.cpp:1510-1518).  Every new tet is oriented like the tet it
// replaces (two vertices swapped where needed).
//
// Cell order: surviving tets keep their relative order, new tets follow in
// creation order (the compaction of the reference's mesh garbage collection);
// new vertices are appended, one per split edge, edges in increasing order of
// the far vertex.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>
#include "difftetvr_b200.h"
#include "dtv_host.h"

struct dtv_split_result {
    std::vector<uint32_t> cells;          // 4T
    std::vector<float> positions;         // 3V
    std::vector<float> vertex_colors;     // 4V or empty
    std::vector<float> cell_colors;       // 4T or empty
};

namespace {

using namespace dtv_host;

double signed_det(const float* P, const uint32_t* c) {
    const float* p0 = P + 3 * size_t(c[0]);
    double e[3][3];
    for (int j = 1; j < 4; ++j)
        for (int k = 0; k < 3; ++k) e[j - 1][k] = double(P[3 * size_t(c[j]) + k]) - double(p0[k]);
    return e[0][0] * (e[1][1] * e[2][2] - e[1][2] * e[2][1]) - e[0][1] * (e[1][0] * e[2][2] - e[1][2] * e[2][0]) +
           e[0][2] * (e[1][0] * e[2][1] - e[1][1] * e[2][0]);
}

struct Mesh {
    std::vector<uint32_t> cells;
    std::vector<char> alive;
    std::vector<float> pos, vcol, ccol;
    std::vector<std::vector<uint32_t>> vert_cells;  // vertex -> incident cells (alive or not)
    bool has_vcol = false, has_ccol = false;

    uint32_t add_cell(const std::array<uint32_t, 4>& c, const float* colour) {
        const uint32_t id = uint32_t(alive.size());
        cells.insert(cells.end(), c.begin(), c.end());
        alive.push_back(1);
        if (has_ccol) ccol.insert(ccol.end(), colour, colour + 4);
        for (uint32_t v : c) vert_cells[v].push_back(id);
        return id;
    }

    // Adds cell c with the orientation sign `want` of the tet it replaces.
    void add_oriented(std::array<uint32_t, 4> c, double want, const float* colour) {
        if ((signed_det(pos.data(), c.data()) < 0) != (want < 0)) std::swap(c[2], c[3]);
        add_cell(c, colour);
    }

    void subdivide(uint32_t v, float t) {
        std::vector<uint32_t> star;
        for (uint32_t c : vert_cells[v])
            if (alive[c]) star.push_back(c);
        if (star.empty()) return;
        // New vertex per incident edge, in increasing order of the far vertex.
        std::map<uint32_t, uint32_t> mid;
        for (uint32_t c : star)
            for (int j = 0; j < 4; ++j)
                if (cells[4 * size_t(c) + j] != v) mid[cells[4 * size_t(c) + j]] = 0;
        for (auto& kv : mid) {
            const uint32_t w = kv.first, m = uint32_t(pos.size() / 3);
            for (int k = 0; k < 3; ++k)
                pos.push_back(pos[3 * size_t(v) + k] + t * (pos[3 * size_t(w) + k] - pos[3 * size_t(v) + k]));
            if (has_vcol)
                for (int k = 0; k < 4; ++k)
                    vcol.push_back(vcol[4 * size_t(v) + k] + t * (vcol[4 * size_t(w) + k] - vcol[4 * size_t(v) + k]));
            vert_cells.emplace_back();
            kv.second = m;
        }
        for (uint32_t c : star) {
            alive[c] = 0;
            std::array<uint32_t, 4> old;
            std::memcpy(old.data(), &cells[4 * size_t(c)], sizeof(old));
            const double sign = signed_det(pos.data(), old.data());
            float colour[4] = {0, 0, 0, 0};
            if (has_ccol) std::memcpy(colour, &ccol[4 * size_t(c)], sizeof(colour));
            // Tet at v: the other three vertices moved to their edge vertices.
            std::array<uint32_t, 4> top = old;
            for (auto& x : top)
                if (x != v) x = mid[x];
            add_cell(top, colour);
            // Prism: bottom (a, b, c) = face opposite v, top (m_a, m_b, m_c).
            uint32_t a[3];
            int n = 0;
            for (uint32_t x : old)
                if (x != v) a[n++] = x;
            uint32_t P[6] = {a[0], a[1], a[2], mid[a[0]], mid[a[1]], mid[a[2]]};
            // Rotate / reflect the prism so that P[0] holds its smallest index.
            int imin = 0;
            for (int i = 1; i < 6; ++i)
                if (P[i] < P[imin]) imin = i;
            static const int kRot[6][6] = {{0, 1, 2, 3, 4, 5}, {1, 2, 0, 4, 5, 3}, {2, 0, 1, 5, 3, 4},
                                           {3, 5, 4, 0, 2, 1}, {4, 3, 5, 1, 0, 2}, {5, 4, 3, 2, 1, 0}};
            uint32_t Q[6];
            for (int i = 0; i < 6; ++i) Q[i] = P[kRot[imin][i]];
            // Q0 < all: the quads at Q0 are cut along Q0-Q4 and Q0-Q5; the
            // quad (Q1, Q2, Q5, Q4) along the diagonal through its smallest vertex.
            if (std::min(Q[1], Q[5]) < std::min(Q[2], Q[4])) {
                add_oriented({Q[0], Q[1], Q[2], Q[5]}, sign, colour);
                add_oriented({Q[0], Q[1], Q[5], Q[4]}, sign, colour);
            } else {
                add_oriented({Q[0], Q[1], Q[2], Q[4]}, sign, colour);
                add_oriented({Q[0], Q[4], Q[2], Q[5]}, sign, colour);
            }
            add_oriented({Q[0], Q[4], Q[5], Q[3]}, sign, colour);
        }
    }
};

}  // namespace

extern "C" {

int32_t dtv_mesh_subdivide_vertices(const uint32_t* h_cells, uint64_t num_cells, const float* h_positions,
                                    uint64_t num_vertices, const float* h_vertex_colors, const float* h_cell_colors,
                                    const uint32_t* h_split_vertices, uint64_t num_split, float t,
                                    dtv_split_result** out) {
    return guarded([&] {
        require(out != nullptr, "out is null");
        require((h_cells || num_cells == 0) && (h_positions || num_vertices == 0), "null mesh array");
        require(h_split_vertices || num_split == 0, "null split vertex list");
        require(t > 0.f && t < 1.f, "t must be in (0, 1)");
        *out = nullptr;
        Mesh m;
        m.has_vcol = h_vertex_colors != nullptr;
        m.has_ccol = h_cell_colors != nullptr;
        m.cells.assign(h_cells, h_cells + 4 * num_cells);
        m.alive.assign(num_cells, 1);
        m.pos.assign(h_positions, h_positions + 3 * num_vertices);
        if (m.has_vcol) m.vcol.assign(h_vertex_colors, h_vertex_colors + 4 * num_vertices);
        if (m.has_ccol) m.ccol.assign(h_cell_colors, h_cell_colors + 4 * num_cells);
        m.vert_cells.resize(num_vertices);
        for (uint64_t c = 0; c < num_cells; ++c)
            for (int j = 0; j < 4; ++j) {
                const uint32_t v = h_cells[4 * c + j];
                require(v < num_vertices, "cell index out of range");
                m.vert_cells[v].push_back(uint32_t(c));
            }
        for (uint64_t i = 0; i < num_split; ++i) {
            require(h_split_vertices[i] < num_vertices, "split vertex out of range");
            m.subdivide(h_split_vertices[i], t);
        }
        auto* r = new dtv_split_result();
        const size_t nc = m.alive.size();
        for (size_t c = 0; c < nc; ++c) {
            if (!m.alive[c]) continue;
            r->cells.insert(r->cells.end(), &m.cells[4 * c], &m.cells[4 * c] + 4);
            if (m.has_ccol) r->cell_colors.insert(r->cell_colors.end(), &m.ccol[4 * c], &m.ccol[4 * c] + 4);
        }
        r->positions = std::move(m.pos);
        r->vertex_colors = std::move(m.vcol);
        *out = r;
    });
}

int32_t dtv_split_result_sizes(const dtv_split_result* r, uint64_t* num_cells, uint64_t* num_vertices) {
    return guarded([&] {
        require(r != nullptr, "result is null");
        if (num_cells) *num_cells = r->cells.size() / 4;
        if (num_vertices) *num_vertices = r->positions.size() / 3;
    });
}

int32_t dtv_split_result_copy(const dtv_split_result* r, uint32_t* h_cells, float* h_positions,
                              float* h_vertex_colors, float* h_cell_colors) {
    return guarded([&] {
        require(r != nullptr, "result is null");
        if (h_cells) std::memcpy(h_cells, r->cells.data(), sizeof(uint32_t) * r->cells.size());
        if (h_positions) std::memcpy(h_positions, r->positions.data(), sizeof(float) * r->positions.size());
        if (h_vertex_colors && !r->vertex_colors.empty())
            std::memcpy(h_vertex_colors, r->vertex_colors.data(), sizeof(float) * r->vertex_colors.size());
        if (h_cell_colors && !r->cell_colors.empty())
            std::memcpy(h_cell_colors, r->cell_colors.data(), sizeof(float) * r->cell_colors.size());
    });
}

int32_t dtv_split_result_destroy(dtv_split_result* r) {
    delete r;
    return DTV_OK;
}

}  // extern "C"
