// Context, error handling and the host-mesh part of the C ABI.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <utility>

#include "common.cuh"
#include "internal.hpp"
#include "mesh.hpp"

struct cpg_mesh {
    cpg::Mesh m;
};

namespace cpg {

cpg_status fail(cpg_ctx *ctx, cpg_status s, const std::string &msg) {
    if (ctx) ctx->err = msg;
    return s;
}

cpg_status cuda_fail(cpg_ctx *ctx, cudaError_t e, const char *where) {
    (void)cudaGetLastError();
    return fail(ctx, e == cudaErrorMemoryAllocation ? CPG_ERR_OOM : CPG_ERR_CUDA,
                std::string(where) + ": " + cudaGetErrorString(e));
}

cpg_status scratch(cpg_ctx *ctx, size_t n, double **out) {
    if (n > ctx->scratch_cap) {
        if (ctx->scratch) {
            CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            cudaFree(ctx->scratch);
            ctx->scratch = nullptr;
            ctx->scratch_cap = 0;
        }
        size_t cap = n < 65536 ? 65536 : n;
        CPG_TRY(dmalloc(ctx, &ctx->scratch, cap));
        ctx->scratch_cap = cap;
    }
    *out = ctx->scratch;
    return CPG_OK;
}

cpg_status pinned(cpg_ctx *ctx, size_t n, double **out) {
    if (n > ctx->pinned_cap) {
        if (ctx->pinned) {
            CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            cudaFreeHost(ctx->pinned);
            ctx->pinned = nullptr;
            ctx->pinned_cap = 0;
        }
        size_t cap = n < 4096 ? 4096 : n;
        CPG_CUDA(ctx, cudaMallocHost((void **)&ctx->pinned, cap * sizeof(double)));
        ctx->pinned_cap = cap;
    }
    *out = ctx->pinned;
    return CPG_OK;
}

cpg_status launched(cpg_ctx *ctx, const char *what) {
    ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, what);
    return CPG_OK;
}

cpg_status smem_limit_once(cpg_ctx *ctx, const void *kernel, int bytes) {
    if (bytes <= 48 * 1024) return CPG_OK;
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> done;
    std::lock_guard<std::mutex> lk(mu);
    int &have = done[{kernel, ctx->device}];
    if (have >= bytes) return CPG_OK;
    if (have > 0)  // a second, larger value would race with launches in flight
        return fail(ctx, CPG_ERR_UNSUPPORTED, "kernel shared-memory limit raised twice");
    const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaFuncSetAttribute(MaxDynamicSharedMemorySize)");
    have = bytes;
    return CPG_OK;
}

cpg_status check_state(cpg_ctx *ctx, const std::string &where) {
    double *hp;
    CPG_TRY(pinned(ctx, 1, &hp));
    int *flag = (int *)hp;
    CPG_CUDA(ctx, cudaMemcpyAsync(flag, ctx->flag_dev + FLAG_NONPHYS, sizeof(int), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const int v = *flag;
    if (v == 0) return CPG_OK;
    CPG_CUDA(ctx, cudaMemsetAsync(ctx->flag_dev + FLAG_NONPHYS, 0, sizeof(int), ctx->stream));
    return fail(ctx, CPG_ERR_NONPHYSICAL,
                "non-physical state (density or pressure <= 0, or not finite) in cell " + std::to_string(v - 1) +
                    " (" + where + ")");
}

}  // namespace cpg

using namespace cpg;

extern "C" {

const char *cpg_version(void) { return "cpolyg_b200 0.1 sm_100a"; }

cpg_status cpg_ctx_create(int device, void *stream, cpg_ctx **out) {
    if (!out) return CPG_ERR_INVALID_ARG;
    *out = nullptr;
    cpg_ctx *ctx = new (std::nothrow) cpg_ctx();
    if (!ctx) return CPG_ERR_OOM;
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        delete ctx;
        return CPG_ERR_CUDA;
    }
    ctx->stream = (cudaStream_t)stream;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
        ctx->num_sms = sms;
    if (cudaMalloc((void **)&ctx->flag_dev, 64 * sizeof(int)) != cudaSuccess) {
        (void)cudaGetLastError();
        delete ctx;
        return CPG_ERR_OOM;
    }
    cudaMemset(ctx->flag_dev, 0, 64 * sizeof(int));
    *out = ctx;
    return CPG_OK;
}

void cpg_ctx_destroy(cpg_ctx *ctx) {
    if (!ctx) return;
    cudaStreamSynchronize(ctx->stream);
    dfree(ctx->scratch);
    dfree(ctx->kws);
    dfree(ctx->flag_dev);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    delete ctx;
}

const char *cpg_last_error(const cpg_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

cpg_status cpg_ctx_sync(cpg_ctx *ctx) {
    if (!ctx) return CPG_ERR_INVALID_ARG;
    CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    CPG_TRY(check_sweep_error(ctx, CPG_OK));
    return check_state(ctx, "a residual since the last check");
}

cpg_status cpg_ctx_set_deferred_checks(cpg_ctx *ctx, int on) {
    if (!ctx) return CPG_ERR_INVALID_ARG;
    ctx->deferred_checks = on != 0;
    return CPG_OK;
}

uint64_t cpg_ctx_launch_count(const cpg_ctx *ctx) { return ctx ? ctx->launches : 0; }

// ------------------------------------------------------------------- mesh
cpg_status cpg_seeds_uniform(uint64_t seed, int n, double width, double height, double *xy_host) {
    if (n < 0 || !xy_host) return CPG_ERR_INVALID_ARG;
    uniform_seeds(seed, n, width, height, xy_host);
    return CPG_OK;
}

cpg_status cpg_mesh_voronoi(const double *xy_host, int n, double width, double height, int periodic,
                            const int *side_codes, cpg_mesh **out) {
    if (!xy_host || !out || n <= 0) return CPG_ERR_INVALID_ARG;
    *out = nullptr;
    cpg_mesh *m = new (std::nothrow) cpg_mesh();
    if (!m) return CPG_ERR_OOM;
    std::string err;
    if (!build_voronoi(xy_host, n, width, height, periodic != 0, side_codes, m->m, err)) {
        fprintf(stderr, "cpolyg_b200: %s\n", err.c_str());
        delete m;
        return CPG_ERR_MESH;
    }
    *out = m;
    return CPG_OK;
}

cpg_status cpg_mesh_from_polygons(int n, const int *cell_ptr, const double *poly_xy, double width,
                                  double height, int periodic, const int *side_codes, cpg_mesh **out) {
    if (!cell_ptr || !poly_xy || !out || n <= 0) return CPG_ERR_INVALID_ARG;
    *out = nullptr;
    cpg_mesh *m = new (std::nothrow) cpg_mesh();
    if (!m) return CPG_ERR_OOM;
    std::string err;
    if (!build_from_polygons(n, cell_ptr, poly_xy, width, height, periodic != 0, side_codes, m->m, err)) {
        fprintf(stderr, "cpolyg_b200: %s\n", err.c_str());
        delete m;
        return CPG_ERR_MESH;
    }
    *out = m;
    return CPG_OK;
}

cpg_status cpg_mesh_set_subtriangles(cpg_mesh *mm, const int *tri_ptr, const double *tri_xy) {
    if (!mm || !tri_ptr || !tri_xy) return CPG_ERR_INVALID_ARG;
    Mesh &m = mm->m;
    if (tri_ptr[0] != 0) return CPG_ERR_INVALID_ARG;
    for (int i = 0; i < m.n; i++)
        if (tri_ptr[i + 1] <= tri_ptr[i]) return CPG_ERR_INVALID_ARG;  // every cell needs a triangle
    // the triangles of a cell must tile its polygon: same total area, and
    // every vertex inside the cell's bounding box (cell-frame coordinates)
    for (int i = 0; i < m.n; i++) {
        const int s = m.cell_ptr[i], e = m.cell_ptr[i + 1];
        double poly = 0.0;
        for (int k = s; k < e; k++) {
            const int k1 = k + 1 < e ? k + 1 : s;
            poly += m.vxy[2 * k] * m.vxy[2 * k1 + 1] - m.vxy[2 * k1] * m.vxy[2 * k + 1];
        }
        poly *= 0.5;
        double area = 0.0;
        const double x0 = m.bb[4 * i], y0 = m.bb[4 * i + 1], w = m.bb[4 * i + 2], h = m.bb[4 * i + 3];
        const double tol = 1e-9 * std::max(w, h);
        for (int t = tri_ptr[i]; t < tri_ptr[i + 1]; t++) {
            const double *T = tri_xy + 6 * (size_t)t;
            for (int v = 0; v < 3; v++)
                if (T[2 * v] < x0 - tol || T[2 * v] > x0 + w + tol || T[2 * v + 1] < y0 - tol ||
                    T[2 * v + 1] > y0 + h + tol)
                    return CPG_ERR_MESH;
            area += 0.5 * std::fabs((T[2] - T[0]) * (T[5] - T[1]) - (T[4] - T[0]) * (T[3] - T[1]));
        }
        if (std::fabs(area - poly) > 1e-9 * std::fabs(poly)) return CPG_ERR_MESH;
    }
    m.tri_ptr.assign(tri_ptr, tri_ptr + m.n + 1);
    m.tri.assign(tri_xy, tri_xy + 6 * (size_t)tri_ptr[m.n]);
    return CPG_OK;
}

void cpg_mesh_destroy(cpg_mesh *m) { delete m; }

cpg_status cpg_mesh_get_info(const cpg_mesh *mm, cpg_mesh_info *info) {
    if (!mm || !info) return CPG_ERR_INVALID_ARG;
    const Mesh &m = mm->m;
    info->n_cells = m.n;
    info->n_verts = (int)(m.verts.size() / 2);
    info->n_edges = m.cell_ptr[m.n];
    info->n_tris = m.tri_ptr[m.n];
    info->periodic = m.periodic ? 1 : 0;
    info->width = m.width;
    info->height = m.height;
    return CPG_OK;
}

cpg_status cpg_mesh_export(const cpg_mesh *mm, int *cell_ptr, double *poly_xy, int *vert_id, int *edge_nbr,
                           double *edge_shift, double *bb, int *tri_ptr, double *tri_xy) {
    if (!mm) return CPG_ERR_INVALID_ARG;
    const Mesh &m = mm->m;
    auto cp = [](void *dst, const void *src, size_t bytes) {
        if (dst && bytes) std::memcpy(dst, src, bytes);
    };
    cp(cell_ptr, m.cell_ptr.data(), m.cell_ptr.size() * sizeof(int));
    cp(poly_xy, m.vxy.data(), m.vxy.size() * sizeof(double));
    cp(vert_id, m.vid.data(), m.vid.size() * sizeof(int));
    cp(edge_nbr, m.nbr.data(), m.nbr.size() * sizeof(int));
    cp(edge_shift, m.shift.data(), m.shift.size() * sizeof(double));
    cp(bb, m.bb.data(), m.bb.size() * sizeof(double));
    cp(tri_ptr, m.tri_ptr.data(), m.tri_ptr.size() * sizeof(int));
    cp(tri_xy, m.tri.data(), m.tri.size() * sizeof(double));
    return CPG_OK;
}

cpg_status cpg_mesh_pattern(const cpg_mesh *mm, int *rowptr, int *colidx, int64_t *nnzb) {
    if (!mm) return CPG_ERR_INVALID_ARG;
    std::vector<int> rp, cl;
    jacobian_pattern(mm->m, rp, cl);
    if (nnzb) *nnzb = (int64_t)cl.size();
    if (rowptr) std::memcpy(rowptr, rp.data(), sizeof(int) * rp.size());
    if (colidx) std::memcpy(colidx, cl.data(), sizeof(int) * cl.size());
    return CPG_OK;
}

cpg_status cpg_pattern_levels(int n, const int *rowptr, const int *colidx, int *n_lower, int *lower_ptr,
                              int *lower_rows, int *n_upper, int *upper_ptr, int *upper_rows) {
    if (n <= 0 || !rowptr || !colidx) return CPG_ERR_INVALID_ARG;
    std::vector<int> rp(rowptr, rowptr + n + 1), cl(colidx, colidx + rowptr[n]);
    std::vector<int> lp, lr, up, ur;
    level_sets(n, rp, cl, lp, lr, up, ur);
    if (n_lower) *n_lower = (int)lp.size() - 1;
    if (n_upper) *n_upper = (int)up.size() - 1;
    if (lower_ptr) std::memcpy(lower_ptr, lp.data(), sizeof(int) * lp.size());
    if (lower_rows) std::memcpy(lower_rows, lr.data(), sizeof(int) * lr.size());
    if (upper_ptr) std::memcpy(upper_ptr, up.data(), sizeof(int) * up.size());
    if (upper_rows) std::memcpy(upper_rows, ur.data(), sizeof(int) * ur.size());
    return CPG_OK;
}

}  // extern "C"

// accessor for the other translation units
const cpg::Mesh &cpg_mesh_ref(const cpg_mesh *m) { return m->m; }
