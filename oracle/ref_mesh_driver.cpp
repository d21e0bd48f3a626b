// ORACLE -- test infrastructure only.
//
// Calls the reference's own vendored Voro++ 2D and Triangle libraries
// (compiled unmodified from the reference tree into oracle/_ref by
// oracle/build_oracle.py) the way the reference does, so the tests can pin
// this project's host mesh against the reference's:
//   ref_voronoi     -- PolyMesh::PolyMesh(pts, width, height)
//                      (src/PolyMesh.cpp:162-218): a non-periodic
//                      container_2d with a 1x1 block grid, compute_cell per
//                      particle, vertices at pt + 0.5*pts, deduplicated by
//                      PolyMesh::findVertex (|dx|+|dy| < 1e-10, first match)
//   ref_triangulate -- Triangulation::doTriangulation
//                      (src/Triangulation.cpp:11-101): Triangle with "zQq"
//                      on the polygon's vertices.
#include <array>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "voro++_2d.hh"
extern "C" {
#include "triangle.h"
}

using namespace voro;

namespace {
const double kEPS = 1e-10;

int find_vertex(const std::vector<std::array<double, 2>> &v, double x, double y) {
    for (size_t i = 0; i < v.size(); i++)
        if (std::fabs(x - v[i][0]) + std::fabs(y - v[i][1]) < kEPS) return (int)i;
    return -1;
}
}  // namespace

extern "C" {

// Returns the number of polygon vertices written, or -1 when a cell could
// not be computed or the capacity is too small.
int ref_voronoi(int n, const double *xy, double width, double height, int *cell_ptr, double *poly_xy, int cap) {
    container_2d con(0, width + kEPS, 0, height + kEPS, 1, 1, false, false, 8);
    voronoicell_2d cell;
    for (int i = 0; i < n; i++) con.put(i, xy[2 * i], xy[2 * i + 1]);
    std::vector<std::array<double, 2>> v;
    int out = 0;
    cell_ptr[0] = 0;
    for (int i = 0; i < n; i++) {
        if (!con.compute_cell(cell, 0, i)) return -1;
        std::vector<int> polygon;
        int k = 0;
        do {
            const double x = xy[2 * i] + 0.5 * cell.pts[2 * k];
            const double y = xy[2 * i + 1] + 0.5 * cell.pts[2 * k + 1];
            int vi = find_vertex(v, x, y);
            if (vi < 0) {
                v.push_back({x, y});
                vi = (int)v.size() - 1;
            }
            bool seen = false;
            for (int q : polygon) seen |= (q == vi);
            if (!seen) polygon.push_back(vi);
            k = cell.ed[2 * k];
        } while (k != 0);
        for (int q : polygon) {
            if (out >= cap) return -1;
            poly_xy[2 * out] = v[q][0];
            poly_xy[2 * out + 1] = v[q][1];
            out++;
        }
        cell_ptr[i + 1] = out;
    }
    return out;
}

// Triangle "zQq" of a point set; writes triangles as (x1,y1,x2,y2,x3,y3).
// Returns the number of triangles, or -1 if the capacity is too small.
int ref_triangulate(int nv, const double *pts, double *tri_xy, int cap) {
    struct triangulateio in, out;
    char switches[] = "zQq";
    in.numberofpointattributes = 0;
    in.pointattributelist = NULL;
    in.pointmarkerlist = NULL;
    in.numberofpoints = nv;
    in.pointlist = (double *)malloc(sizeof(double) * 2 * nv);
    for (int j = 0; j < 2 * nv; j++) in.pointlist[j] = pts[j];
    in.trianglelist = NULL;
    in.triangleattributelist = NULL;
    in.trianglearealist = NULL;
    in.neighborlist = NULL;
    in.numberoftriangles = 0;
    in.numberofcorners = 0;
    in.numberoftriangleattributes = 0;
    in.segmentlist = NULL;
    in.segmentmarkerlist = NULL;
    in.numberofsegments = 0;
    in.holelist = NULL;
    in.numberofholes = 0;
    in.regionlist = NULL;
    in.numberofregions = 0;
    in.edgelist = NULL;
    in.edgemarkerlist = NULL;
    in.normlist = NULL;
    out.pointlist = NULL;
    out.pointattributelist = NULL;
    out.pointmarkerlist = NULL;
    out.trianglelist = NULL;
    out.neighborlist = NULL;
    out.triangleattributelist = NULL;
    out.segmentlist = NULL;
    out.segmentmarkerlist = NULL;
    out.edgelist = NULL;
    out.edgemarkerlist = NULL;
    triangulate(switches, &in, &out, NULL);
    free(in.pointlist);
    int nt = out.numberoftriangles;
    if (nt > cap) nt = -1;
    for (int i = 0; i < nt; i++)
        for (int c = 0; c < 3; c++) {
            const int p = out.trianglelist[out.numberofcorners * i + c];
            tri_xy[6 * i + 2 * c] = out.pointlist[2 * p];
            tri_xy[6 * i + 2 * c + 1] = out.pointlist[2 * p + 1];
        }
    free(out.pointlist);
    free(out.trianglelist);
    free(out.pointmarkerlist);
    free(out.segmentlist);
    free(out.segmentmarkerlist);
    return nt;
}

}  // extern "C"
