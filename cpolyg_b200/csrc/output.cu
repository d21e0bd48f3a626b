// Text output in the reference's gnuplot formats, for visual cross-checks:
//   PolyMesh::gnuplot  (src/PolyMesh.cpp:221-241)  polygon outlines;
//   MeshFn::gnuplot    (src/MeshFn.cpp:161-207)    field values at the
//                      3-point (degree-2) rule of every sub-triangle;
//   BlockMatrix::spy   (src/BlockMatrix.cpp:318-349) nonzero entries.
// Numbers are printed as a default-formatted C++ stream prints them (six
// significant digits) and field values with twenty, as the reference does.
// The field is evaluated on the device; only the formatting runs on the host.
#include <cmath>
#include <cstdio>
#include <vector>

#include "internal.hpp"
#include "quadrature.hpp"

using namespace cpg;

namespace {

constexpr double kSpyEps = 1e-10;  // entries at or below this are not written (kEPS, PolyMesh.h:11)

// value of every component of the field at physical points (x, y) of cells
template <int P, int NC>
__global__ void k_eval_points(int npts, const int *__restrict__ cell, const double *__restrict__ px,
                              const double *__restrict__ py, const double4 *__restrict__ bb,
                              const double *__restrict__ u, double *__restrict__ out) {
    constexpr int NB = nbasis<P>();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npts) return;
    const int i = cell[q];
    const double4 b = bb[i];
    double psi[NB];
    basis<P>(2.0 * (px[q] - b.x) / b.z - 1.0, 2.0 * (py[q] - b.y) / b.w - 1.0, psi);
    const double *uc = u + (size_t)i * NB * NC;
#pragma unroll
    for (int c = 0; c < NC; c++) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < NB; k++) v += uc[c * NB + k] * psi[k];
        out[(size_t)q * NC + c] = v;
    }
}

struct File {
    FILE *f;
    explicit File(const char *path) : f(path ? std::fopen(path, "w") : nullptr) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

}  // namespace

extern "C" {

cpg_status cpg_mesh_write_gnuplot(const cpg_mesh *mm, const char *path) {
    if (!mm || !path) return CPG_ERR_INVALID_ARG;
    const Mesh &m = cpg_mesh_ref(mm);
    File out(path);
    if (!out.f) return CPG_ERR_INVALID_ARG;
    // the cell's own frame: periodic cells are not cut at the domain edge
    for (int i = 0; i < m.n; i++) {
        std::fprintf(out.f, "# polygon number %d\n", i);
        const int s = m.cell_ptr[i], nv = m.cell_ptr[i + 1] - s;
        for (int j = 0; j <= nv; j++) {
            const int k = s + j % nv;
            std::fprintf(out.f, "%g\t%g\n", m.vxy[2 * k], m.vxy[2 * k + 1]);
        }
        std::fprintf(out.f, "\n");
    }
    return std::ferror(out.f) ? CPG_ERR_INVALID_ARG : CPG_OK;
}

cpg_status cpg_field_write_gnuplot(cpg_ctx *ctx, const cpg_equation *eq, const cpg_mesh *mm, const double *u,
                                   const char *path) {
    if (!ctx || !eq || !mm || !u || !path) return CPG_ERR_INVALID_ARG;
    const Mesh &m = cpg_mesh_ref(mm);
    if (m.n != eq->n) return fail(ctx, CPG_ERR_INVALID_ARG, "the mesh is not the equation's");
    // points: the degree-2 (3-point) triangle rule on every sub-triangle
    const auto &qr = quad::kTri3;
    std::vector<int> cell;
    std::vector<double> px, py;
    cell.reserve(3 * (size_t)m.tri_ptr[m.n]);
    for (int i = 0; i < m.n; i++)
        for (int t = m.tri_ptr[i]; t < m.tri_ptr[i + 1]; t++) {
            const double *T = &m.tri[6 * (size_t)t];
            for (int k = 0; k < 3; k++) {
                const double a = qr[k][0], b = qr[k][1];
                cell.push_back(i);
                px.push_back(T[0] * (1 - a - b) + T[2] * a + T[4] * b);
                py.push_back(T[1] * (1 - a - b) + T[3] * a + T[5] * b);
            }
        }
    const int npts = (int)cell.size(), nc = eq->nc;
    int *d_cell = nullptr;
    double *d_px = nullptr, *d_py = nullptr, *d_out = nullptr;
    cpg_status st = upload(ctx, &d_cell, cell);
    if (st == CPG_OK) st = upload(ctx, &d_px, px);
    if (st == CPG_OK) st = upload(ctx, &d_py, py);
    if (st == CPG_OK) st = dmalloc(ctx, &d_out, (size_t)npts * nc);
    std::vector<double> vals((size_t)npts * nc);
    if (st == CPG_OK) {
        const int T = 256, grid = (npts + T - 1) / T;
        auto launch = [&](auto pc) {
            constexpr int P = decltype(pc)::value;
            if (nc == 4) k_eval_points<P, 4><<<grid, T, 0, ctx->stream>>>(npts, d_cell, d_px, d_py, eq->bb, u, d_out);
            else k_eval_points<P, 1><<<grid, T, 0, ctx->stream>>>(npts, d_cell, d_px, d_py, eq->bb, u, d_out);
        };
        if (eq->degree == 1) launch(std::integral_constant<int, 1>{});
        else if (eq->degree == 2) launch(std::integral_constant<int, 2>{});
        else launch(std::integral_constant<int, 3>{});
        st = launched(ctx, "point evaluation kernel");
    }
    if (st == CPG_OK) {
        cudaError_t e = cudaMemcpyAsync(vals.data(), d_out, vals.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                        ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = cuda_fail(ctx, e, "field values to host");
    }
    dfree(d_cell);
    dfree(d_px);
    dfree(d_py);
    dfree(d_out);
    if (st != CPG_OK) return st;
    File out(path);
    if (!out.f) return fail(ctx, CPG_ERR_INVALID_ARG, "cannot open the output file");
    for (int q = 0; q < npts; q++) {
        std::fprintf(out.f, "%g\t%g", px[q], py[q]);
        for (int c = 0; c < nc; c++) std::fprintf(out.f, "\t%.20g", vals[(size_t)q * nc + c]);
        std::fprintf(out.f, "\n");
    }
    return std::ferror(out.f) ? fail(ctx, CPG_ERR_INVALID_ARG, "write error") : CPG_OK;
}

cpg_status cpg_bsr_write_spy(cpg_ctx *ctx, const cpg_bsr *A, const char *path) {
    if (!ctx || !A || !path) return CPG_ERR_INVALID_ARG;
    const size_t b2 = (size_t)A->bl * A->bl;
    std::vector<double> v(A->nnzb * b2);
    CPG_TRY(cpg_bsr_export(ctx, A, nullptr, nullptr, v.data()));
    File out(path);
    if (!out.f) return fail(ctx, CPG_ERR_INVALID_ARG, "cannot open the output file");
    const int bl = A->bl;
    for (int i = 0; i < A->n_rows; i++)
        for (int k = A->rowptr[i]; k < A->rowptr[i + 1]; k++) {
            const int j = A->colidx[k];
            for (int ii = 0; ii < bl; ii++)
                for (int jj = 0; jj < bl; jj++) {
                    const double x = v[(size_t)k * b2 + (size_t)jj * bl + ii];  // blocks are column-major
                    if (std::fabs(x) > kSpyEps)
                        std::fprintf(out.f, "%d\t%d\t%g\n", i * bl + ii, j * bl + jj, x);
                }
        }
    return std::ferror(out.f) ? fail(ctx, CPG_ERR_INVALID_ARG, "write error") : CPG_OK;
}

}  // extern "C"
