// Host mesh construction.  See mesh.hpp.
//
// Voronoi cells are built by clipping a start box with the bisectors of
// nearby seeds, found through a uniform bucket grid (O(N) overall, versus the
// reference's O(N^2) Voro++ container with a 1x1 block grid,
// src/PolyMesh.cpp:169-184).  Vertex deduplication follows
// PolyMesh::addVertex/findVertex (src/PolyMesh.cpp:129-160): a vertex equal
// to an existing one within |dx|+|dy| < 1e-10 takes the existing (first
// inserted) id, and a polygon never lists an id twice.  Edge neighbours follow
// PolyMesh::computep2p (src/PolyMesh.cpp:12-67): edge (a,b) of cell i is
// matched with edge (a,b) or (b,a) of another cell; unmatched edges are
// exterior.  Periodic meshes match edges through canonical (wrapped) vertex
// ids and record the lattice shift between the two cells' frames.
#include "mesh.hpp"

#include <algorithm>
#include <cmath>
#include <random>
#include <unordered_map>

namespace cpg {

static const double kEPS = 1e-10;  // PolyMesh.h:11

void uniform_seeds(uint64_t seed, int n, double width, double height,
                   double *xy) {
    std::mt19937_64 g(seed);
    const double s = 1.0 / 9007199254740992.0;  // 2^-53
    for (int i = 0; i < n; i++) {
        double x = (double)(g() >> 11) * s;
        double y = (double)(g() >> 11) * s;
        xy[2 * i] = x * width;
        xy[2 * i + 1] = y * height;
    }
}

namespace {

struct Pt {
    double x, y;
};

// Keep the part of convex polygon P on the seed side of the bisector of s, q.
void clip(std::vector<Pt> &P, std::vector<Pt> &out, std::vector<double> &f,
          Pt s, Pt q, double tol) {
    const double dx = q.x - s.x, dy = q.y - s.y;
    const double mx = 0.5 * (s.x + q.x), my = 0.5 * (s.y + q.y);
    const double eps = tol * std::sqrt(dx * dx + dy * dy);
    const size_t n = P.size();
    f.resize(n);
    bool any_out = false;
    for (size_t k = 0; k < n; k++) {
        f[k] = (P[k].x - mx) * dx + (P[k].y - my) * dy;
        if (f[k] > eps) any_out = true;
    }
    if (!any_out) return;
    out.clear();
    for (size_t k = 0; k < n; k++) {
        const size_t k1 = (k + 1) % n;
        const bool in0 = f[k] <= eps, in1 = f[k1] <= eps;
        const bool on0 = std::fabs(f[k]) <= eps, on1 = std::fabs(f[k1]) <= eps;
        if (in0) out.push_back(P[k]);
        if ((in0 && !on0 && !in1) || (!in0 && in1 && !on1)) {
            const double t = f[k] / (f[k] - f[k1]);
            out.push_back({P[k].x + t * (P[k1].x - P[k].x),
                           P[k].y + t * (P[k1].y - P[k].y)});
        }
    }
    P.swap(out);
}

// Bucket hash of canonical vertices with the findVertex tolerance.
struct VertexTable {
    double W, H;
    bool periodic;
    double h;          // bucket size
    int64_t nbx = 0, nby = 0;
    std::unordered_map<int64_t, std::vector<int>> buckets;
    std::vector<double> xy;

    VertexTable(double w, double hh, bool per) : W(w), H(hh), periodic(per) {
        h = 1e-6 * std::max(1.0, std::max(w, hh));
        if (periodic) {
            nbx = std::max<int64_t>(1, (int64_t)std::floor(W / h));
            nby = std::max<int64_t>(1, (int64_t)std::floor(H / h));
        }
    }
    void canon(double &x, double &y) const {
        if (!periodic) return;
        x -= W * std::floor(x / W);
        y -= H * std::floor(y / H);
        if (x >= W) x -= W;
        if (y >= H) y -= H;
    }
    int64_t bx(double x) const {
        return periodic ? std::min(nbx - 1, (int64_t)(x / (W / nbx)))
                        : (int64_t)std::floor(x / h);
    }
    int64_t by(double y) const {
        return periodic ? std::min(nby - 1, (int64_t)(y / (H / nby)))
                        : (int64_t)std::floor(y / h);
    }
    int64_t key(int64_t ix, int64_t iy) const {
        if (periodic) {
            ix = ((ix % nbx) + nbx) % nbx;
            iy = ((iy % nby) + nby) % nby;
        }
        const int64_t off = (int64_t)1 << 30;
        return (ix + off) * ((int64_t)1 << 32) + (iy + off);
    }
    double ddx(double a, double b) const {
        double d = a - b;
        if (periodic) d -= W * std::round(d / W);
        return d;
    }
    double ddy(double a, double b) const {
        double d = a - b;
        if (periodic) d -= H * std::round(d / H);
        return d;
    }
    // returns canonical id (existing within tolerance or new)
    int add(double x, double y) {
        canon(x, y);
        const int64_t ix = bx(x), iy = by(y);
        int best = -1;
        for (int64_t a = -1; a <= 1; a++)
            for (int64_t b = -1; b <= 1; b++) {
                auto it = buckets.find(key(ix + a, iy + b));
                if (it == buckets.end()) continue;
                for (int id : it->second) {
                    if (std::fabs(ddx(x, xy[2 * id])) +
                            std::fabs(ddy(y, xy[2 * id + 1])) < kEPS) {
                        if (best < 0 || id < best) best = id;
                    }
                }
            }
        if (best >= 0) return best;
        const int id = (int)(xy.size() / 2);
        xy.push_back(x);
        xy.push_back(y);
        buckets[key(ix, iy)].push_back(id);
        return id;
    }
};

}  // namespace

bool build_from_polygons(int n, const int *cell_ptr, const double *poly_xy,
                         double width, double height, bool periodic,
                         const int *side_codes, Mesh &m, std::string &err) {
    m = Mesh();
    m.n = n;
    m.width = width;
    m.height = height;
    m.periodic = periodic;
    if (side_codes)
        for (int s = 0; s < 4; s++) m.side_code[s] = side_codes[s];
    if (n <= 0 || !(width > 0) || !(height > 0)) {
        err = "mesh: need n > 0 and a positive domain";
        return false;
    }
    VertexTable vt(width, height, periodic);

    // 1. deduplicate vertices, drop repeated ids within a polygon
    m.cell_ptr.assign(1, 0);
    for (int i = 0; i < n; i++) {
        std::vector<int> ids;
        std::vector<double> fr;
        for (int k = cell_ptr[i]; k < cell_ptr[i + 1]; k++) {
            const double x = poly_xy[2 * k], y = poly_xy[2 * k + 1];
            const int id = vt.add(x, y);
            if (std::find(ids.begin(), ids.end(), id) != ids.end()) continue;
            ids.push_back(id);
            // frame coordinate = canonical + lattice offset of this cell
            double fx = vt.xy[2 * id], fy = vt.xy[2 * id + 1];
            if (periodic) {
                fx += width * std::round((x - fx) / width);
                fy += height * std::round((y - fy) / height);
            }
            fr.push_back(fx);
            fr.push_back(fy);
        }
        if (ids.size() < 3) {
            err = "mesh: cell " + std::to_string(i) + " has fewer than 3 vertices";
            return false;
        }
        for (size_t k = 0; k < ids.size(); k++) {
            m.vid.push_back(ids[k]);
            m.vxy.push_back(fr[2 * k]);
            m.vxy.push_back(fr[2 * k + 1]);
        }
        m.cell_ptr.push_back((int)m.vid.size());
    }
    m.verts = vt.xy;
    const int E = m.cell_ptr[n];

    // 2. edge neighbours
    std::unordered_map<int64_t, std::vector<int>> emap;
    emap.reserve((size_t)E);
    auto ekey = [](int a, int b) {
        if (a > b) std::swap(a, b);
        return (int64_t)a * 2147483648LL + b;
    };
    std::vector<int> edge_cell(E);
    for (int i = 0; i < n; i++) {
        const int s = m.cell_ptr[i], nv = m.cell_ptr[i + 1] - s;
        for (int j = 0; j < nv; j++) {
            edge_cell[s + j] = i;
            emap[ekey(m.vid[s + j], m.vid[s + (j + 1) % nv])].push_back(s + j);
        }
    }
    m.nbr.assign(E, 0);
    m.shift.assign(2 * (size_t)E, 0.0);
    const double tolb = 1e-9 * std::max(width, height);
    for (int i = 0; i < n; i++) {
        const int s = m.cell_ptr[i], nv = m.cell_ptr[i + 1] - s;
        for (int j = 0; j < nv; j++) {
            const int e = s + j;
            const int a = m.vid[e], b = m.vid[s + (j + 1) % nv];
            const auto &lst = emap[ekey(a, b)];
            int match = -1;
            for (int e2 : lst) {
                if (e2 == e) continue;
                if (match < 0 || edge_cell[e2] < edge_cell[match]) match = e2;
            }
            if (lst.size() > 2) {
                err = "mesh: edge shared by more than two cells near cell " +
                      std::to_string(i);
                return false;
            }
            if (match < 0) {
                if (periodic) {
                    err = "mesh: unmatched edge in a periodic mesh at cell " +
                          std::to_string(i);
                    return false;
                }
                const double mx = 0.5 * (m.vxy[2 * e] + m.vxy[2 * (s + (j + 1) % nv)]);
                const double my = 0.5 * (m.vxy[2 * e + 1] + m.vxy[2 * (s + (j + 1) % nv) + 1]);
                int code = -1;
                if (std::fabs(my) < tolb) code = m.side_code[0];
                else if (std::fabs(mx - width) < tolb) code = m.side_code[1];
                else if (std::fabs(my - height) < tolb) code = m.side_code[2];
                else if (std::fabs(mx) < tolb) code = m.side_code[3];
                else {
                    err = "mesh: unmatched interior edge at cell " + std::to_string(i);
                    return false;
                }
                m.nbr[e] = code;
                continue;
            }
            const int k = edge_cell[match];
            if (k == i) {
                err = "mesh: cell " + std::to_string(i) +
                      " neighbours itself; mesh too coarse for periodicity";
                return false;
            }
            m.nbr[e] = k;
            if (periodic) {
                // vertex a in cell k's frame
                const int sk = m.cell_ptr[k], nk = m.cell_ptr[k + 1] - sk;
                double ax = 0, ay = 0, bxk = 0, byk = 0;
                bool fa = false, fb = false;
                for (int l = 0; l < nk; l++) {
                    if (m.vid[sk + l] == a) { ax = m.vxy[2 * (sk + l)]; ay = m.vxy[2 * (sk + l) + 1]; fa = true; }
                    if (m.vid[sk + l] == b) { bxk = m.vxy[2 * (sk + l)]; byk = m.vxy[2 * (sk + l) + 1]; fb = true; }
                }
                const int eb = s + (j + 1) % nv;
                if (!fa || !fb) {
                    err = "mesh: inconsistent periodic edge at cell " + std::to_string(i);
                    return false;
                }
                const double sx = width * std::round((ax - m.vxy[2 * e]) / width);
                const double sy = height * std::round((ay - m.vxy[2 * e + 1]) / height);
                const double sx2 = width * std::round((bxk - m.vxy[2 * eb]) / width);
                const double sy2 = height * std::round((byk - m.vxy[2 * eb + 1]) / height);
                if (sx != sx2 || sy != sy2) {
                    err = "mesh: periodic edge endpoints disagree on the shift at cell " +
                          std::to_string(i);
                    return false;
                }
                m.shift[2 * e] = sx;
                m.shift[2 * e + 1] = sy;
            }
        }
        // a neighbour reached through two edges would give two blocks with
        // the same column in one BSR row
        for (int j = 0; j < nv; j++)
            for (int l = j + 1; l < nv; l++)
                if (m.nbr[s + j] >= 0 && m.nbr[s + j] == m.nbr[s + l]) {
                    err = "mesh: cell " + std::to_string(i) + " meets cell " +
                          std::to_string(m.nbr[s + j]) +
                          " through two edges; mesh too coarse";
                    return false;
                }
    }

    // 3. bounding boxes (PolyMesh::computebb, src/PolyMesh.cpp:70-104)
    m.bb.resize(4 * (size_t)n);
    for (int i = 0; i < n; i++) {
        const int s = m.cell_ptr[i], e = m.cell_ptr[i + 1];
        double x0 = m.vxy[2 * s], y0 = m.vxy[2 * s + 1], x1 = x0, y1 = y0;
        for (int k = s; k < e; k++) {
            x0 = std::min(x0, m.vxy[2 * k]);
            y0 = std::min(y0, m.vxy[2 * k + 1]);
            x1 = std::max(x1, m.vxy[2 * k]);
            y1 = std::max(y1, m.vxy[2 * k + 1]);
        }
        m.bb[4 * i] = x0;
        m.bb[4 * i + 1] = y0;
        m.bb[4 * i + 2] = x1 - x0;
        m.bb[4 * i + 3] = y1 - y0;
    }

    // 4. sub-triangulation: fan from the vertex centroid (cells are convex)
    m.tri_ptr.assign(1, 0);
    for (int i = 0; i < n; i++) {
        const int s = m.cell_ptr[i], nv = m.cell_ptr[i + 1] - s;
        double cx = 0, cy = 0;
        for (int k = 0; k < nv; k++) {
            cx += m.vxy[2 * (s + k)];
            cy += m.vxy[2 * (s + k) + 1];
        }
        cx /= nv;
        cy /= nv;
        for (int k = 0; k < nv; k++) {
            const int a = s + k, b = s + (k + 1) % nv;
            const double t[6] = {cx, cy, m.vxy[2 * a], m.vxy[2 * a + 1],
                                 m.vxy[2 * b], m.vxy[2 * b + 1]};
            m.tri.insert(m.tri.end(), t, t + 6);
        }
        m.tri_ptr.push_back((int)(m.tri.size() / 6));
    }
    return true;
}

void jacobian_pattern(const Mesh &m, std::vector<int> &rowptr, std::vector<int> &colidx) {
    rowptr.assign(1, 0);
    colidx.clear();
    for (int i = 0; i < m.n; i++) {
        colidx.push_back(i);
        for (int e = m.cell_ptr[i]; e < m.cell_ptr[i + 1]; e++)
            if (m.nbr[e] >= 0) colidx.push_back(m.nbr[e]);
        rowptr.push_back((int)colidx.size());
    }
}

void level_sets(int n, const std::vector<int> &rowptr, const std::vector<int> &col, std::vector<int> &lptr,
                std::vector<int> &lrows, std::vector<int> &uptr, std::vector<int> &urows) {
    std::vector<int> lv(n, 0), uv(n, 0);
    int nl = 0, nu = 0;
    for (int j = 0; j < n; j++) {
        int l = 0;
        for (int k = rowptr[j]; k < rowptr[j + 1]; k++)
            if (col[k] < j) l = std::max(l, lv[col[k]] + 1);
        lv[j] = l;
        nl = std::max(nl, l + 1);
    }
    for (int i = n - 1; i >= 0; i--) {
        int l = 0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; k++)
            if (col[k] > i) l = std::max(l, uv[col[k]] + 1);
        uv[i] = l;
        nu = std::max(nu, l + 1);
    }
    auto bucket = [&](const std::vector<int> &lvv, int nlev, std::vector<int> &ptr, std::vector<int> &rows) {
        ptr.assign(nlev + 1, 0);
        for (int i = 0; i < n; i++) ptr[lvv[i] + 1]++;
        for (int l = 0; l < nlev; l++) ptr[l + 1] += ptr[l];
        rows.assign(n, 0);
        std::vector<int> fill(ptr.begin(), ptr.end() - 1);
        for (int i = 0; i < n; i++) rows[fill[lvv[i]]++] = i;
    };
    bucket(lv, nl, lptr, lrows);
    bucket(uv, nu, uptr, urows);
}

bool build_voronoi(const double *xy, int n, double W, double H, bool periodic,
                   const int *side_codes, Mesh &out, std::string &err) {
    if (n <= 0 || !(W > 0) || !(H > 0)) {
        err = "voronoi: need n > 0 and a positive domain";
        return false;
    }
    for (int i = 0; i < n; i++) {
        const double x = xy[2 * i], y = xy[2 * i + 1];
        if (!(x >= 0 && x <= W && y >= 0 && y <= H)) {
            err = "voronoi: seed " + std::to_string(i) + " outside the domain";
            return false;
        }
    }
    const int nbx = std::max(1, (int)std::floor(std::sqrt((double)n * W / H)));
    const int nby = std::max(1, (int)std::floor(std::sqrt((double)n * H / W)));
    const double bw = W / nbx, bh = H / nby, bmin = std::min(bw, bh);
    std::vector<int> bstart((size_t)nbx * nby + 1, 0), bseed(n);
    std::vector<int> sb(n);
    for (int i = 0; i < n; i++) {
        const int ix = std::min(nbx - 1, (int)(xy[2 * i] / bw));
        const int iy = std::min(nby - 1, (int)(xy[2 * i + 1] / bh));
        sb[i] = iy * nbx + ix;
        bstart[sb[i] + 1]++;
    }
    for (size_t b = 0; b < (size_t)nbx * nby; b++) bstart[b + 1] += bstart[b];
    {
        std::vector<int> fill(bstart.begin(), bstart.end() - 1);
        for (int i = 0; i < n; i++) bseed[fill[sb[i]]++] = i;
    }
    const double tol = 1e-12 * std::max(W, H);

    std::vector<int> cptr(1, 0);
    std::vector<double> pxy;
    pxy.reserve((size_t)n * 14);
    std::vector<Pt> P, tmp;
    std::vector<double> f;
    struct Cand {
        double d2;
        double x, y;
    };
    std::vector<Cand> cand;
    for (int i = 0; i < n; i++) {
        const Pt s{xy[2 * i], xy[2 * i + 1]};
        P.clear();
        if (periodic) {
            P = {{s.x - W, s.y - H}, {s.x + W, s.y - H}, {s.x + W, s.y + H}, {s.x - W, s.y + H}};
        } else {
            P = {{0, 0}, {W, 0}, {W, H}, {0, H}};
        }
        const int bx = sb[i] % nbx, by = sb[i] / nbx;
        for (int r = 0;; r++) {
            cand.clear();
            bool any_bucket = false;
            for (int dy = -r; dy <= r; dy++)
                for (int dx = -r; dx <= r; dx++) {
                    if (std::max(std::abs(dx), std::abs(dy)) != r) continue;
                    int ix = bx + dx, iy = by + dy;
                    double ox = 0, oy = 0;
                    if (periodic) {
                        const int qx = (int)std::floor((double)ix / nbx);
                        const int qy = (int)std::floor((double)iy / nby);
                        ox = qx * W;
                        oy = qy * H;
                        ix -= qx * nbx;
                        iy -= qy * nby;
                    } else if (ix < 0 || iy < 0 || ix >= nbx || iy >= nby) {
                        continue;
                    }
                    any_bucket = true;
                    const int b = iy * nbx + ix;
                    for (int t = bstart[b]; t < bstart[b + 1]; t++) {
                        const int j = bseed[t];
                        if (j == i && ox == 0 && oy == 0) continue;
                        const double qx = xy[2 * j] + ox, qy = xy[2 * j + 1] + oy;
                        const double d2 = (qx - s.x) * (qx - s.x) + (qy - s.y) * (qy - s.y);
                        cand.push_back({d2, qx, qy});
                    }
                }
            std::sort(cand.begin(), cand.end(),
                      [](const Cand &a, const Cand &b) { return a.d2 < b.d2; });
            for (const Cand &c : cand) {
                if (c.d2 == 0) {
                    err = "voronoi: coincident seeds at seed " + std::to_string(i);
                    return false;
                }
                clip(P, tmp, f, s, {c.x, c.y}, tol);
            }
            double R2 = 0;
            for (const Pt &p : P)
                R2 = std::max(R2, (p.x - s.x) * (p.x - s.x) + (p.y - s.y) * (p.y - s.y));
            const double reach = r * bmin;
            if (reach * reach >= 4 * R2) break;
            if (!periodic && !any_bucket) break;
            if (r > 4 * (nbx + nby) + 8) break;
        }
        for (const Pt &p : P) {
            pxy.push_back(p.x);
            pxy.push_back(p.y);
        }
        cptr.push_back((int)(pxy.size() / 2));
    }
    return build_from_polygons(n, cptr.data(), pxy.data(), W, H, periodic,
                               side_codes, out, err);
}

}  // namespace cpg
