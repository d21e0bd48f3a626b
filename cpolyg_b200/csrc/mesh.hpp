// Host polygonal mesh: Voronoi construction, vertex deduplication, edge
// neighbours (p2p), bounding boxes and the sub-triangulation used by the
// volume quadrature.  Replaces PolyMesh (src/PolyMesh.h:13-55) of the
// reference; stays on the host.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace cpg {

struct Mesh {
    int n = 0;
    double width = 1, height = 1;
    bool periodic = false;
    int side_code[4] = {-1, -1, -1, -1};  // bottom, right, top, left

    std::vector<int> cell_ptr;      // n+1
    std::vector<double> vxy;        // 2 per cell-vertex, cell frame coords
    std::vector<int> vid;           // canonical vertex id per cell-vertex
    std::vector<double> verts;      // 2 per canonical vertex
    std::vector<int> nbr;           // per cell-edge: neighbour or code < 0
    std::vector<double> shift;      // 2 per cell-edge
    std::vector<double> bb;         // 4 per cell: x0, y0, w, h
    std::vector<int> tri_ptr;       // n+1
    std::vector<double> tri;        // 6 per sub-triangle
};

// std::mt19937_64(seed); x = (g() >> 11) * 2^-53 * width, then y.
void uniform_seeds(uint64_t seed, int n, double width, double height,
                   double *xy);

// Voronoi cells of the seeds.  Returns false and sets err on failure.
bool build_voronoi(const double *xy, int n, double width, double height,
                   bool periodic, const int *side_codes, Mesh &out,
                   std::string &err);

// Mesh from explicit polygons (cell-frame coordinates).
bool build_from_polygons(int n, const int *cell_ptr, const double *poly_xy,
                         double width, double height, bool periodic,
                         const int *side_codes, Mesh &out, std::string &err);

// Jacobian block pattern (Jacobian ctor, src/Jacobian.cpp:7-47): row i holds
// the diagonal block, then one block per edge with a neighbour, edge order.
void jacobian_pattern(const Mesh &m, std::vector<int> &rowptr,
                      std::vector<int> &colidx);

// ILU(0) level schedule of a block pattern: lower level of row j is
// 1 + max lower level of its neighbours i < j (0 if none); upper level of
// row i is 1 + max upper level of its neighbours j > i.  Rows are listed
// by level, ascending within a level.
void level_sets(int n, const std::vector<int> &rowptr,
                const std::vector<int> &col, std::vector<int> &lptr,
                std::vector<int> &lrows, std::vector<int> &uptr,
                std::vector<int> &urows);

}  // namespace cpg
