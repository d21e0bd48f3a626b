// ORACLE -- test infrastructure only.
//
// CPU restatement of the cpolyg reference's DG path, used as the checker for
// the CUDA implementation (tests/, __graft_entry__.smoke, and bench.py's CPU
// baseline leg only; the product never links or calls this file).
//
// Each routine follows the reference file:line cited beside it, in FP64, with
// the reference's loop structure (including its per-test-function
// recomputation in assemble/jacobian).  Third-party arithmetic of the
// reference is restated here:
//   gsl_sf_legendre_Pl             -> explicit P0..P3, Bonnet recurrence above
//   gsl_integration_glfixed nodes  -> Newton iteration on P_m
//   arma::inv / LAPACK dgetrf/getrs -> partial-pivot LU (dgetf2 algorithm)
//   arma::solve (overdetermined)   -> Householder QR least squares
//   dgemv / dnrm2 / dtpsv          -> plain loops
// Reference defects handled explicitly:
//   D1 periodic trace degree: periodic faces are ordinary neighbours with a
//      coordinate shift, evaluated with the full basis;
//   D2 MassMatrix::solve offset: uses i*bl;
//   D3 vortex pressure: a parameterised standard isentropic vortex;
//   D4 Euler off-diagonal Jacobian: replicated as in the reference.
// Parity pins: no reference output exists (the reference needs Armadillo,
// GSL and BLAS, absent here); the restatement is pinned by known-answer
// tests in tests/test_oracle_kat.py and by the reference's own Triangle and
// Voro++ sources compiled into oracle/_ref (tests/test_ref_pins.py).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

using std::vector;
static const double kEPS = 1e-10;  // src/PolyMesh.h:11

// ------------------------------------------------------------------------
// Legendre (src/Legendre.h:51-68, src/Legendre.cpp:34-124)
// ------------------------------------------------------------------------
static inline double legendre_Pl(int l, double x) {
    // gsl_sf_legendre_Pl restated: closed forms for l <= 3, then upward
    // Bonnet recurrence (l) P_l = (2l-1) x P_{l-1} - (l-1) P_{l-2}
    if (l == 0) return 1.0;
    if (l == 1) return x;
    if (l == 2) return 0.5 * (3.0 * x * x - 1.0);
    if (l == 3) return 0.5 * x * (5.0 * x * x - 3.0);
    double pm2 = 0.5 * (3.0 * x * x - 1.0), pm1 = 0.5 * x * (5.0 * x * x - 3.0), p = 0;
    for (int k = 4; k <= l; k++) {
        p = ((2 * k - 1) * x * pm1 - (k - 1) * pm2) / k;
        pm2 = pm1;
        pm1 = p;
    }
    return p;
}

// Leg2D (Legendre.h:51-68): sum_{i<m} sum_{j<m-i} c_k P_i(x) P_j(y)
static inline double Leg2D(double x, double y, int m, const double *c) {
    double val = 0;
    int k = 0;
    for (int i = 0; i < m; i++)
        for (int j = 0; j < m - i; j++) {
            val += c[k] * legendre_Pl(i, x) * legendre_Pl(j, y);
            k++;
        }
    return val;
}

// LegDerX (Legendre.cpp:34-74)
static vector<double> LegDerX(int m, const vector<double> &a_c) {
    vector<double> c = a_c, cp(m * (m + 1) / 2, 0.0);
    for (int i = m - 1; i > 2; i--)
        for (int j = 0; j < m - i; j++) {
            cp[-(i - 1) * (i - 2 * (1 + m)) / 2 + j] = (2 * i - 1) * c[-i * (i - 1 - 2 * m) / 2 + j];
            c[-(i - 2) * (i - 3 - 2 * m) / 2 + j] += c[-i * (i - 1 - 2 * m) / 2 + j];
        }
    if (m > 2)
        for (int j = 0; j < m - 2; j++) cp[m + j] = 3 * c[2 * m - 1 + j];
    for (int j = 0; j < m - 1; j++) cp[j] = c[m + j];
    return cp;
}

// LegDerY (Legendre.cpp:84-124)
static vector<double> LegDerY(int m, const vector<double> &a_c) {
    vector<double> c = a_c, cp(m * (m + 1) / 2, 0.0);
    for (int j = m - 1; j > 2; j--)
        for (int i = 0; i < m - j; i++) {
            cp[-i * (i - 1 - 2 * m) / 2 + j - 1] = (2 * j - 1) * c[-i * (i - 1 - 2 * m) / 2 + j];
            c[-i * (i - 1 - 2 * m) / 2 + j - 2] += c[-i * (i - 1 - 2 * m) / 2 + j];
        }
    if (m > 2)
        for (int i = 0; i < m - 2; i++)
            cp[-i * (i - 1 - 2 * m) / 2 + 1] = 3 * c[-i * (i - 1 - 2 * m) / 2 + 2];
    for (int i = 0; i < m - 1; i++) cp[-i * (i - 1 - 2 * m) / 2] = c[-i * (i - 1 - 2 * m) / 2 + 1];
    return cp;
}

// ------------------------------------------------------------------------
// Quadrature rules (src/Quadrature.cpp:103-171): Gauss-Legendre on [-1,1]
// (point, weight) and symmetric triangle rules (a, b, w), weights sum to 1.
// ------------------------------------------------------------------------
static const double lin2[][2] = {{-0.5773502691896257, 1.0}, {0.5773502691896257, 1.0}};
static const double lin4[][2] = {{-0.3399810435848563, 0.6521451548625461},
                                 {0.3399810435848563, 0.6521451548625461},
                                 {-0.8611363115940526, 0.3478548451374538},
                                 {0.8611363115940526, 0.3478548451374538}};
static const double lin6[][2] = {{0.6612093864662645, 0.3607615730481386},
                                 {-0.6612093864662645, 0.3607615730481386},
                                 {-0.2386191860831969, 0.4679139345726910},
                                 {0.2386191860831969, 0.4679139345726910},
                                 {-0.9324695142031521, 0.1713244923791704},
                                 {0.9324695142031521, 0.1713244923791704}};
static const double lin10[][2] = {{0.1488743389816312, 0.2955242247147529},
                                  {-0.1488743389816312, 0.2955242247147529},
                                  {-0.4333953941292472, 0.2692667193099963},
                                  {0.4333953941292472, 0.2692667193099963},
                                  {-0.6794095682990244, 0.2190863625159820},
                                  {0.6794095682990244, 0.2190863625159820},
                                  {-0.8650633666889845, 0.1494513491505806},
                                  {0.8650633666889845, 0.1494513491505806},
                                  {-0.9739065285171717, 0.0666713443086881},
                                  {0.9739065285171717, 0.0666713443086881}};
static const double tri2[][3] = {{0.16666666666667, 0.16666666666667, 0.33333333333333},
                                 {0.16666666666667, 0.66666666666667, 0.33333333333333},
                                 {0.66666666666667, 0.16666666666667, 0.33333333333333}};
static const double tri4[][3] = {{0.44594849091597, 0.44594849091597, 0.22338158967801},
                                 {0.44594849091597, 0.10810301816807, 0.22338158967801},
                                 {0.10810301816807, 0.44594849091597, 0.22338158967801},
                                 {0.09157621350977, 0.09157621350977, 0.10995174365532},
                                 {0.09157621350977, 0.81684757298046, 0.10995174365532},
                                 {0.81684757298046, 0.09157621350977, 0.10995174365532}};
static const double tri6[][3] = {{0.24928674517091, 0.24928674517091, 0.11678627572638},
                                 {0.24928674517091, 0.50142650965818, 0.11678627572638},
                                 {0.50142650965818, 0.24928674517091, 0.11678627572638},
                                 {0.06308901449150, 0.06308901449150, 0.05084490637021},
                                 {0.06308901449150, 0.87382197101700, 0.05084490637021},
                                 {0.87382197101700, 0.06308901449150, 0.05084490637021},
                                 {0.31035245103378, 0.63650249912140, 0.08285107561837},
                                 {0.63650249912140, 0.05314504984482, 0.08285107561837},
                                 {0.05314504984482, 0.31035245103378, 0.08285107561837},
                                 {0.63650249912140, 0.31035245103378, 0.08285107561837},
                                 {0.31035245103378, 0.05314504984482, 0.08285107561837},
                                 {0.05314504984482, 0.63650249912140, 0.08285107561837}};
static const double tri10[][3] = {{0.33333333333333, 0.33333333333333, 0.09081799038275},
                                  {0.48557763338366, 0.48557763338366, 0.03672595775647},
                                  {0.48557763338366, 0.02884473323269, 0.03672595775647},
                                  {0.02884473323269, 0.48557763338366, 0.03672595775647},
                                  {0.10948157548504, 0.10948157548504, 0.04532105943553},
                                  {0.10948157548504, 0.78103684902993, 0.04532105943553},
                                  {0.78103684902993, 0.10948157548504, 0.04532105943553},
                                  {0.30793983876412, 0.55035294182100, 0.07275791684542},
                                  {0.55035294182100, 0.14170721941488, 0.07275791684542},
                                  {0.14170721941488, 0.30793983876412, 0.07275791684542},
                                  {0.55035294182100, 0.30793983876412, 0.07275791684542},
                                  {0.30793983876412, 0.14170721941488, 0.07275791684542},
                                  {0.14170721941488, 0.55035294182100, 0.07275791684542},
                                  {0.24667256063990, 0.72832390459741, 0.02832724253106},
                                  {0.72832390459741, 0.02500353476269, 0.02832724253106},
                                  {0.02500353476269, 0.24667256063990, 0.02832724253106},
                                  {0.72832390459741, 0.24667256063990, 0.02832724253106},
                                  {0.24667256063990, 0.02500353476269, 0.02832724253106},
                                  {0.02500353476269, 0.72832390459741, 0.02832724253106},
                                  {0.06680325101220, 0.92365593358750, 0.00942166696373},
                                  {0.92365593358750, 0.00954081540030, 0.00942166696373},
                                  {0.00954081540030, 0.06680325101220, 0.00942166696373},
                                  {0.92365593358750, 0.06680325101220, 0.00942166696373},
                                  {0.06680325101220, 0.00954081540030, 0.00942166696373},
                                  {0.00954081540030, 0.92365593358750, 0.00942166696373}};

struct Rule {
    const double *d;
    int n, stride;
};
// Quadrature.cpp:20-27
static Rule tri_rule(int deg) {
    if (deg <= 2) return {&tri2[0][0], 3, 3};
    if (deg <= 4) return {&tri4[0][0], 6, 3};
    if (deg <= 6) return {&tri6[0][0], 12, 3};
    return {&tri10[0][0], 25, 3};
}
// Quadrature.cpp:74-81
static Rule lin_rule(int deg) {
    if (deg <= 2) return {&lin2[0][0], 2, 2};
    if (deg <= 4) return {&lin4[0][0], 4, 2};
    if (deg <= 6) return {&lin6[0][0], 6, 2};
    return {&lin10[0][0], 10, 2};
}

// ------------------------------------------------------------------------
// Mesh (PolyMesh, src/PolyMesh.h:13-55).  Cells carry their vertex
// coordinates in their own frame; periodic neighbours carry a shift.
// ------------------------------------------------------------------------
struct Mesh {
    int np = 0;
    double W = 1, H = 1;
    bool periodic = false;
    int side_code[4] = {-1, -1, -1, -1};
    vector<vector<int>> p;                 // canonical vertex ids
    vector<vector<std::array<double, 2>>> pv;  // frame coordinates
    vector<std::array<double, 2>> v;       // canonical vertices
    vector<vector<int>> p2p;               // neighbour or boundary code
    vector<vector<std::array<double, 2>>> shift;
    vector<std::array<double, 4>> bb;
    vector<vector<std::array<double, 6>>> tri;

    void getLocalCoordinates(int pi, double x, double y, double &xo, double &yo) const {
        // PolyMesh.h:44-49
        xo = 2.0 * (x - bb[pi][0]) / bb[pi][2] - 1;
        yo = 2.0 * (y - bb[pi][1]) / bb[pi][3] - 1;
    }
    // PolyMesh::getOutwardNormal (PolyMesh.cpp:248-273), cell i, edge e
    void getOutwardNormal(int i, int e, double &nx, double &ny) const {
        double cx = 0, cy = 0;
        const int nv = (int)pv[i].size();
        for (int j = 0; j < nv; j++) {
            cx += pv[i][j][0];
            cy += pv[i][j][1];
        }
        cx /= nv;
        cy /= nv;
        const auto &a = pv[i][e], &b = pv[i][(e + 1) % nv];
        const double dx = a[0] - b[0], dy = a[1] - b[1];
        const double length = std::sqrt(dx * dx + dy * dy);
        const double sv = -dy * (a[0] - cx) + dx * (a[1] - cy);
        const int s = (0.0 < sv) - (sv < 0.0);
        nx = -s * dy / length;
        ny = s * dx / length;
    }
};

// findVertex/addVertex (PolyMesh.cpp:129-160) with a bucket grid and the
// periodic wrap; first inserted vertex within |dx|+|dy| < kEPS wins.
struct VTab {
    double W, H;
    bool per;
    double h;
    std::unordered_map<int64_t, vector<int>> b;
    vector<std::array<double, 2>> v;
    int64_t key(int64_t ix, int64_t iy) const {
        return (ix + (1LL << 30)) * (1LL << 32) + (iy + (1LL << 30));
    }
    void wrap(double &x, double &y) const {
        if (!per) return;
        x -= W * std::floor(x / W);
        y -= H * std::floor(y / H);
        if (x >= W) x -= W;
        if (y >= H) y -= H;
    }
    int add(double x, double y) {
        wrap(x, y);
        const int64_t nbx = per ? std::max<int64_t>(1, (int64_t)std::floor(W / h)) : 0;
        const int64_t nby = per ? std::max<int64_t>(1, (int64_t)std::floor(H / h)) : 0;
        auto bi = [&](double c, double L, int64_t nb) {
            return per ? std::min(nb - 1, (int64_t)(c / (L / nb))) : (int64_t)std::floor(c / h);
        };
        const int64_t ix = bi(x, W, nbx), iy = bi(y, H, nby);
        int best = -1;
        for (int a = -1; a <= 1; a++)
            for (int c = -1; c <= 1; c++) {
                int64_t jx = ix + a, jy = iy + c;
                if (per) {
                    jx = ((jx % nbx) + nbx) % nbx;
                    jy = ((jy % nby) + nby) % nby;
                }
                auto it = b.find(key(jx, jy));
                if (it == b.end()) continue;
                for (int id : it->second) {
                    double dx = x - v[id][0], dy = y - v[id][1];
                    if (per) {
                        dx -= W * std::round(dx / W);
                        dy -= H * std::round(dy / H);
                    }
                    if (std::fabs(dx) + std::fabs(dy) < kEPS && (best < 0 || id < best)) best = id;
                }
            }
        if (best >= 0) return best;
        v.push_back({x, y});
        b[key(ix, iy)].push_back((int)v.size() - 1);
        return (int)v.size() - 1;
    }
};

static std::string g_err;

static bool build_mesh(Mesh &m, int n, const int *cell_ptr, const double *xy, double W,
                       double H, int periodic, const int *codes, const int *tri_ptr,
                       const double *tri_xy) {
    m = Mesh();
    m.np = n;
    m.W = W;
    m.H = H;
    m.periodic = periodic != 0;
    if (codes)
        for (int s = 0; s < 4; s++) m.side_code[s] = codes[s];
    VTab vt{W, H, m.periodic, 1e-6 * std::max(1.0, std::max(W, H)), {}, {}};
    m.p.resize(n);
    m.pv.resize(n);
    for (int i = 0; i < n; i++) {
        for (int k = cell_ptr[i]; k < cell_ptr[i + 1]; k++) {
            const double x = xy[2 * k], y = xy[2 * k + 1];
            const int id = vt.add(x, y);
            if (std::find(m.p[i].begin(), m.p[i].end(), id) != m.p[i].end()) continue;
            m.p[i].push_back(id);
            double fx = vt.v[id][0], fy = vt.v[id][1];
            if (m.periodic) {
                fx += W * std::round((x - fx) / W);
                fy += H * std::round((y - fy) / H);
            }
            m.pv[i].push_back({fx, fy});
        }
    }
    m.v = vt.v;
    // computep2p (PolyMesh.cpp:12-67): first other cell (lowest index) with a
    // matching edge; hashed instead of the O(N^2) scan.
    std::unordered_map<int64_t, vector<std::pair<int, int>>> em;
    auto ek = [](int a, int b) {
        if (a > b) std::swap(a, b);
        return (int64_t)a * 2147483648LL + b;
    };
    for (int i = 0; i < n; i++) {
        const int nv = (int)m.p[i].size();
        for (int j = 0; j < nv; j++) em[ek(m.p[i][j], m.p[i][(j + 1) % nv])].push_back({i, j});
    }
    m.p2p.resize(n);
    m.shift.resize(n);
    const double tolb = 1e-9 * std::max(W, H);
    for (int i = 0; i < n; i++) {
        const int nv = (int)m.p[i].size();
        m.p2p[i].assign(nv, 0);
        m.shift[i].assign(nv, {0.0, 0.0});
        for (int j = 0; j < nv; j++) {
            const int a = m.p[i][j], bvid = m.p[i][(j + 1) % nv];
            int k = -1;
            for (auto &pr : em[ek(a, bvid)])
                if (pr.first != i && (k < 0 || pr.first < k)) k = pr.first;
            if (k < 0) {
                const auto &A = m.pv[i][j], &B = m.pv[i][(j + 1) % nv];
                const double mx = 0.5 * (A[0] + B[0]), my = 0.5 * (A[1] + B[1]);
                int code = -1;
                if (std::fabs(my) < tolb) code = m.side_code[0];
                else if (std::fabs(mx - W) < tolb) code = m.side_code[1];
                else if (std::fabs(my - H) < tolb) code = m.side_code[2];
                else if (std::fabs(mx) < tolb) code = m.side_code[3];
                m.p2p[i][j] = code;
                continue;
            }
            m.p2p[i][j] = k;
            if (m.periodic) {
                for (size_t l = 0; l < m.p[k].size(); l++)
                    if (m.p[k][l] == a) {
                        m.shift[i][j] = {W * std::round((m.pv[k][l][0] - m.pv[i][j][0]) / W),
                                         H * std::round((m.pv[k][l][1] - m.pv[i][j][1]) / H)};
                    }
            }
        }
    }
    // computebb (PolyMesh.cpp:70-104)
    m.bb.resize(n);
    for (int i = 0; i < n; i++) {
        double x0 = m.pv[i][0][0], y0 = m.pv[i][0][1], x1 = x0, y1 = y0;
        for (auto &q : m.pv[i]) {
            if (q[0] < x0) x0 = q[0];
            if (q[1] < y0) y0 = q[1];
            if (q[0] > x1) x1 = q[0];
            if (q[1] > y1) y1 = q[1];
        }
        m.bb[i] = {x0, y0, x1 - x0, y1 - y0};
    }
    // sub-triangulation (input, as the reference's Triangle output)
    m.tri.resize(n);
    for (int i = 0; i < n; i++)
        for (int t = tri_ptr[i]; t < tri_ptr[i + 1]; t++) {
            std::array<double, 6> T;
            for (int q = 0; q < 6; q++) T[q] = tri_xy[6 * t + q];
            m.tri[i].push_back(T);
        }
    return true;
}

// Seeds of the synthetic meshes: std::mt19937_64(seed), x = (g()>>11) 2^-53
// scaled to the domain, then y (the same generator the library's host code
// uses, so both read identical points).
static void seeds_uniform(uint64_t seed, int n, double W, double H, double *xy) {
    std::mt19937_64 g(seed);
    for (int i = 0; i < n; i++) {
        const double x = (double)(g() >> 11) * 0x1.0p-53, y = (double)(g() >> 11) * 0x1.0p-53;
        xy[2 * i] = x * W;
        xy[2 * i + 1] = y * H;
    }
}

// Voronoi cells by brute force, independent of the library's bucket-grid
// mesher: cell i is the domain box (periodic: the box of side 2W x 2H around
// the seed) cut by the bisector half-plane of every other seed and, when
// periodic, of its 8 lattice images, nearest first.  O(n^2); used for the
// CPU-baseline sample meshes and as a check of the library's cells.  The
// polygon is counter-clockwise in the frame of seed i; its volume quadrature
// runs on the fan of triangles from the vertex centroid (the reference uses
// Triangle's "zQq" sub-triangles, Triangulation.cpp:11-101; both are exact
// for polynomial integrands).
static void voronoi_polys(const double *xy, int n, double W, double H, bool periodic, vector<int> &cptr,
                          vector<double> &pxy, vector<int> &tptr, vector<double> &txy) {
    cptr.assign(1, 0);
    pxy.clear();
    tptr.assign(1, 0);
    txy.clear();
    vector<std::array<double, 3>> cand;
    vector<std::array<double, 2>> P, Q;
    for (int i = 0; i < n; i++) {
        const double sx = xy[2 * i], sy = xy[2 * i + 1];
        cand.clear();
        const int img = periodic ? 1 : 0;
        for (int j = 0; j < n; j++)
            for (int a = -img; a <= img; a++)
                for (int b = -img; b <= img; b++) {
                    if (j == i && a == 0 && b == 0) continue;
                    const double qx = xy[2 * j] + a * W, qy = xy[2 * j + 1] + b * H;
                    cand.push_back({(qx - sx) * (qx - sx) + (qy - sy) * (qy - sy), qx, qy});
                }
        std::sort(cand.begin(), cand.end(), [](const std::array<double, 3> &u, const std::array<double, 3> &v) {
            return u[0] < v[0];
        });
        if (periodic) P = {{sx - W, sy - H}, {sx + W, sy - H}, {sx + W, sy + H}, {sx - W, sy + H}};
        else P = {{0, 0}, {W, 0}, {W, H}, {0, H}};
        for (const auto &c : cand) {
            // a candidate farther than twice the cell's radius cannot cut it
            double R2 = 0;
            for (const auto &p : P) R2 = std::max(R2, (p[0] - sx) * (p[0] - sx) + (p[1] - sy) * (p[1] - sy));
            if (c[0] > 4 * R2) break;
            const double dx = c[1] - sx, dy = c[2] - sy, mx = 0.5 * (c[1] + sx), my = 0.5 * (c[2] + sy);
            Q.clear();
            const size_t m = P.size();
            for (size_t k = 0; k < m; k++) {
                const auto &A = P[k], &B = P[(k + 1) % m];
                const double fa = (A[0] - mx) * dx + (A[1] - my) * dy, fb = (B[0] - mx) * dx + (B[1] - my) * dy;
                if (fa <= 0) Q.push_back(A);
                if ((fa < 0 && fb > 0) || (fa > 0 && fb < 0)) {
                    const double t = fa / (fa - fb);
                    Q.push_back({A[0] + t * (B[0] - A[0]), A[1] + t * (B[1] - A[1])});
                }
            }
            P.swap(Q);
        }
        double cx = 0, cy = 0;
        for (const auto &p : P) {
            pxy.push_back(p[0]);
            pxy.push_back(p[1]);
            cx += p[0];
            cy += p[1];
        }
        cx /= (double)P.size();
        cy /= (double)P.size();
        for (size_t k = 0; k < P.size(); k++) {
            const auto &A = P[k], &B = P[(k + 1) % P.size()];
            const double T[6] = {cx, cy, A[0], A[1], B[0], B[1]};
            txy.insert(txy.end(), T, T + 6);
        }
        cptr.push_back((int)(pxy.size() / 2));
        tptr.push_back((int)(txy.size() / 6));
    }
}

// polygonIntegral (Quadrature.cpp:13-57), integrand f(x, y, out[nout])
template <class F>
static void polygonIntegral(const Mesh &m, int pi, int deg, int nout, F &&f, double *integ) {
    Rule qr = tri_rule(deg);
    double z[64], val[64];
    for (int o = 0; o < nout; o++) integ[o] = 0;
    for (const auto &T : m.tri[pi]) {
        const double x1 = T[0], y1 = T[1], x2 = T[2], y2 = T[3], x3 = T[4], y3 = T[5];
        const double area = 0.5 * std::fabs(x1 * y2 + x2 * y3 + x3 * y1 - x1 * y3 - x3 * y2 - x2 * y1);
        for (int o = 0; o < nout; o++) z[o] = 0;
        for (int k = 0; k < qr.n; k++) {
            const double a = qr.d[k * 3], b = qr.d[k * 3 + 1], w = qr.d[k * 3 + 2];
            const double x = x1 * (1 - a - b) + x2 * a + x3 * b;
            const double y = y1 * (1 - a - b) + y2 * a + y3 * b;
            f(x, y, val);
            for (int o = 0; o < nout; o++) z[o] += val[o] * w;
        }
        for (int o = 0; o < nout; o++) integ[o] += z[o] * area;
    }
}

// lineIntegral (Quadrature.cpp:67-101) over edge e of cell i
template <class F>
static void lineIntegral(const Mesh &m, int i, int e, int deg, int nout, F &&f, double *integ) {
    Rule qr = lin_rule(deg);
    const int nv = (int)m.pv[i].size();
    const double x1 = m.pv[i][e][0], y1 = m.pv[i][e][1];
    const double x2 = m.pv[i][(e + 1) % nv][0], y2 = m.pv[i][(e + 1) % nv][1];
    const double length = std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
    double val[64];
    for (int o = 0; o < nout; o++) integ[o] = 0;
    for (int k = 0; k < qr.n; k++) {
        const double xi = qr.d[k * 2], w = qr.d[k * 2 + 1];
        const double x = x1 + 0.5 * (xi + 1) * (x2 - x1);
        const double y = y1 + 0.5 * (xi + 1) * (y2 - y1);
        f(x, y, val);
        for (int o = 0; o < nout; o++) integ[o] += w * val[o];
    }
    for (int o = 0; o < nout; o++) integ[o] = integ[o] * 0.5 * length;
}

// ------------------------------------------------------------------------
// Analytic fields (initial data, Dirichlet states)
// ------------------------------------------------------------------------
enum { INIT_CONSTANT = 0, INIT_GAUSSIAN = 1, INIT_VORTEX = 2, INIT_BUMP = 3 };

static void field_eval(int kind, const double *P, int nc, double x, double y, double t,
                       double *out) {
    if (kind == INIT_CONSTANT) {
        for (int c = 0; c < nc; c++) out[c] = P[c];
    } else if (kind == INIT_GAUSSIAN) {
        // centre (x0, y0) + (bx, by) t, nearest periodic image when Lx, Ly > 0
        double dx = x - (P[1] + P[3] * t), dy = y - (P[2] + P[4] * t);
        if (P[5] > 0) dx -= P[5] * std::round(dx / P[5]);
        if (P[6] > 0) dy -= P[6] * std::round(dy / P[6]);
        out[0] = std::exp(-P[0] * (dx * dx + dy * dy));
        for (int c = 1; c < nc; c++) out[c] = 0;
    } else if (kind == INIT_VORTEX) {
        // standard isentropic vortex of strength beta (Shu's formulation),
        // centred at (x0, y0) + (uinf, vinf) t, nearest periodic image
        const double beta = P[0], x0 = P[1], y0 = P[2], ui = P[3], vi = P[4], g = P[5];
        const double Lx = P[6], Ly = P[7];
        double dx = x - (x0 + ui * t), dy = y - (y0 + vi * t);
        if (Lx > 0) dx -= Lx * std::round(dx / Lx);
        if (Ly > 0) dy -= Ly * std::round(dy / Ly);
        const double r2 = dx * dx + dy * dy;
        const double e = std::exp(0.5 * (1.0 - r2));
        const double du = -beta / (2.0 * M_PI) * dy * e;
        const double dv = beta / (2.0 * M_PI) * dx * e;
        const double T = 1.0 - (g - 1.0) * beta * beta / (8.0 * g * M_PI * M_PI) * e * e;
        const double rho = std::pow(T, 1.0 / (g - 1.0));
        const double p = std::pow(rho, g);
        const double u = ui + du, v = vi + dv;
        out[0] = rho;
        out[1] = rho * u;
        out[2] = rho * v;
        out[3] = p / (g - 1.0) + 0.5 * rho * (u * u + v * v);
    } else if (kind == INIT_BUMP) {
        // rho = 1 + A exp(-r^2/w^2), u = mach (c = 1 at rho = 1), v = 0, p = 1/gamma
        const double A = P[0], w = P[1], x0 = P[2], y0 = P[3], mach = P[4], g = P[5];
        const double dx = x - x0, dy = y - y0;
        const double rho = 1.0 + A * std::exp(-(dx * dx + dy * dy) / (w * w));
        const double p = 1.0 / g, u = mach;
        out[0] = rho;
        out[1] = rho * u;
        out[2] = 0.0;
        out[3] = p / (g - 1.0) + 0.5 * rho * u * u;
    }
}

// ------------------------------------------------------------------------
// Equation (src/Equation.h:8-67) with the physics of eqns/
// ------------------------------------------------------------------------
enum { PHYS_ADV_CONST = 0, PHYS_ADV_ROT = 1, PHYS_EULER = 2 };
enum { BC_DIRICHLET = -1, BC_WALL = -2, BC_OUTFLOW = -3, BC_INFLOW = -4 };

struct Equation {
    const Mesh *msh;
    int phys, nc, deg, nb, bl;
    double gamma, bx, by;
    // false: neighbour blocks as the reference (A and alpha' of the own
    // state, Euler.cpp:168-179); true: exact derivative w.r.t. the neighbour
    bool exact_nbr = false;
    int dkind;
    double dparams[8];
    double inflow[4];

    double betaX(double x, double y) const { return phys == PHYS_ADV_CONST ? bx : 2 * y - 1; }
    double betaY(double x, double y) const { return phys == PHYS_ADV_CONST ? by : -2 * x + 1; }

    // Euler::flux (eqns/Euler.cpp:7-33)
    void eflux(const double *U, double *fx, double *fy, double &c, double &u, double &v) const {
        const double rho = U[0], rhoU = U[1], rhoV = U[2], rhoE = U[3];
        u = rhoU / rho;
        v = rhoV / rho;
        const double P = (gamma - 1) * (rhoE - 0.5 * (rhoU * rhoU + rhoV * rhoV) / rho);
        fx[0] = rhoU;
        fx[1] = rhoU * u + P;
        fx[2] = rhoU * v;
        fx[3] = (rhoE + P) * u;
        fy[0] = rhoV;
        fy[1] = rhoU * v;
        fy[2] = rhoV * v + P;
        fy[3] = (rhoE + P) * v;
        c = std::sqrt(gamma * P / rho);
    }
    // fluxFunction: F[c][0..1]
    void fluxFunction(const double *U, double x, double y, double F[][2]) const {
        if (phys != PHYS_EULER) {  // Advection.cpp:18-22
            F[0][0] = betaX(x, y) * U[0];
            F[0][1] = betaY(x, y) * U[0];
            return;
        }
        double fx[4], fy[4], c, u, v;
        eflux(U, fx, fy, c, u, v);
        for (int k = 0; k < 4; k++) {
            F[k][0] = fx[k];
            F[k][1] = fy[k];
        }
    }
    // numericalFluxFunction (Advection.cpp:24-38, Euler.cpp:113-132)
    void numericalFlux(const double *Um, const double *Up, double x, double y, double nx,
                       double ny, double *out) const {
        if (phys != PHYS_EULER) {
            const double bn = betaX(x, y) * nx + betaY(x, y) * ny;
            out[0] = bn > 0 ? Um[0] * bn : Up[0] * bn;
            return;
        }
        double fxm[4], fym[4], fxp[4], fyp[4], cm, um, vm, cp, up, vp;
        eflux(Um, fxm, fym, cm, um, vm);
        eflux(Up, fxp, fyp, cp, up, vp);
        const double vnm = um * nx + vm * ny, vnp = up * nx + vp * ny;
        const double alpha = std::max({std::fabs(vnm - cm), std::fabs(vnm), std::fabs(vnm + cm),
                                       std::fabs(vnp - cp), std::fabs(vnp), std::fabs(vnp + cp)});
        for (int k = 0; k < 4; k++)
            out[k] = 0.5 * ((fxp[k] + fxm[k]) * nx + (fyp[k] + fym[k]) * ny + alpha * (Um[k] - Up[k]));
    }
    // fluxJacobian (Advection.cpp:40-48, Euler.cpp:134-166): A[d][r][c]
    void fluxJacobian(const double *U, double x, double y, double A[2][4][4]) const {
        if (phys != PHYS_EULER) {
            A[0][0][0] = betaX(x, y);
            A[1][0][0] = betaY(x, y);
            return;
        }
        const double g = gamma, rho = U[0];
        const double u = U[1] / rho, v = U[2] / rho, E = U[3] / rho;
        const double usq = u * u + v * v, e = E - 0.5 * usq, P = (g - 1) * rho * e, Hh = E + P / rho;
        const double a0[4][4] = {{0, 1, 0, 0},
                                 {-u * u + 0.5 * (g - 1) * usq, (3 - g) * u, -(g - 1) * v, g - 1},
                                 {-u * v, v, u, 0},
                                 {u * (0.5 * (g - 1) * usq - Hh), Hh - (g - 1) * usq, -(g - 1) * u * v, g * u}};
        const double a1[4][4] = {{0, 0, 1, 0},
                                 {-u * v, v, u, 0},
                                 {-v * v + 0.5 * (g - 1) * usq, -(g - 1) * u, (3 - g) * v, g - 1},
                                 {v * (0.5 * (g - 1) * usq - Hh), -(g - 1) * u * v, Hh - (g - 1) * v * v, g * v}};
        std::memcpy(A[0], a0, sizeof(a0));
        std::memcpy(A[1], a1, sizeof(a1));
        // the reference's entry (3,1) of A_x reads H - (g-1)(u^2+v^2); the
        // derivative of (rhoE + p) u with respect to rho u is H - (g-1) u^2
        if (exact_nbr) A[0][3][1] = Hh - (g - 1) * u * u;
    }
    // Euler::alphaDerivative (Euler.cpp:35-98)
    void alphaDerivative(const double *v1s, const double *v2s, double nx, double ny,
                         double *der, double &alpha) const {
        const double g = gamma;
        for (int k = 0; k < 4; k++) der[k] = 0;
        const double u1 = v1s[1] / v1s[0], v1 = v1s[2] / v1s[0];
        const double u2 = v2s[1] / v2s[0], v2 = v2s[2] / v2s[0];
        const double P1 = (g - 1) * (v1s[3] - 0.5 * (v1s[1] * v1s[1] + v1s[2] * v1s[2]) / v1s[0]);
        const double c1 = std::sqrt(g * P1 / v1s[0]);
        const double P2 = (g - 1) * (v2s[3] - 0.5 * (v2s[1] * v2s[1] + v2s[2] * v2s[2]) / v2s[0]);
        const double c2 = std::sqrt(g * P2 / v2s[0]);
        const double vn1 = u1 * nx + v1 * ny, vn2 = u2 * nx + v2 * ny;
        const double eigs[6] = {vn1 - c1, vn1, vn1 + c1, vn2 - c2, vn2, vn2 + c2};
        int idx = 0;
        alpha = std::fabs(eigs[0]);
        for (int k = 1; k < 6; k++)
            if (std::fabs(eigs[k]) > alpha) {
                alpha = std::fabs(eigs[k]);
                idx = k;
            }
        if (idx <= 2) {
            const double rho = v1s[0], E = v1s[3] / rho;
            der[0] = -u1 / rho * nx - v1 / rho * ny;
            der[1] = 1 / rho * nx;
            der[2] = 1 / rho * ny;
            const double usq = u1 * u1 + v1 * v1;
            const double a = std::sqrt(g * g - g), b = rho * std::sqrt(4 * E - 2 * usq);
            if (idx == 0) {
                der[0] -= a * (usq - E) / b;
                der[1] -= -a * u1 / b;
                der[2] -= -a * v1 / b;
                der[3] -= a / b;
            } else if (idx == 2) {
                der[0] += a * (usq - E) / b;
                der[1] += -a * u1 / b;
                der[2] += -a * v1 / b;
                der[3] += a / b;
            }
            if (eigs[idx] < 0)
                for (int k = 0; k < 4; k++) der[k] *= -1;
        }
    }
    // numericalFluxJacobian (Advection.cpp:50-66, Euler.cpp:168-179): J[r][c]
    void numericalFluxJacobian(const double *U, const double *U2, double x, double y,
                               double nx, double ny, int sgn, double J[4][4]) const {
        if (phys != PHYS_EULER) {
            const double bn = nx * betaX(x, y) + ny * betaY(x, y);
            J[0][0] = (sgn * bn > 0) ? bn : 0.0;
            return;
        }
        double A[2][4][4], ap[4], alpha;
        if (sgn < 0 && exact_nbr) {
            // exact derivative with respect to the neighbour state U2:
            // 0.5 [A(U2) n - alpha I + (U - U2) (d alpha / d U2)^T]
            fluxJacobian(U2, x, y, A);
            alphaDerivative(U2, U, nx, ny, ap, alpha);
        } else {
            fluxJacobian(U, x, y, A);
            alphaDerivative(U, U2, nx, ny, ap, alpha);
        }
        for (int r = 0; r < 4; r++)
            for (int c = 0; c < 4; c++)
                J[r][c] = 0.5 * (A[0][r][c] * nx + A[1][r][c] * ny + (r == c ? sgn * alpha : 0.0) +
                                 (U[r] - U2[r]) * ap[c]);
    }

    // computeVariables (Equation.cpp:8-18); coeffs column-major nb x nc
    void vars(const double *coeffs, double xx, double yy, double *out) const {
        for (int c = 0; c < nc; c++) out[c] = Leg2D(xx, yy, deg + 1, coeffs + c * nb);
    }
    // exterior state u+ for boundary code b (BoundaryConditions.cpp:7-37,
    // extended with wall / outflow / inflow)
    void boundaryValue(int b, const double *Um, double x, double y, double t, double nx,
                       double ny, double *out) const {
        if (b == BC_WALL && phys == PHYS_EULER) {
            const double mn = Um[1] * nx + Um[2] * ny;
            out[0] = Um[0];
            out[1] = Um[1] - 2 * mn * nx;
            out[2] = Um[2] - 2 * mn * ny;
            out[3] = Um[3];
        } else if (b == BC_OUTFLOW || b == BC_WALL) {
            for (int c = 0; c < nc; c++) out[c] = Um[c];
        } else if (b == BC_INFLOW) {
            for (int c = 0; c < nc; c++) out[c] = inflow[c];
        } else {
            field_eval(dkind, dparams, nc, x, y, t, out);
        }
    }
    // d u+ / d u- for boundary code b
    void boundaryDerivative(int b, double nx, double ny, double R[4][4], bool &dep) const {
        for (int r = 0; r < 4; r++)
            for (int c = 0; c < 4; c++) R[r][c] = (r == c) ? 1.0 : 0.0;
        dep = (b == BC_WALL || b == BC_OUTFLOW);
        if (b == BC_WALL && phys == PHYS_EULER) {
            R[1][1] = 1 - 2 * nx * nx;
            R[1][2] = -2 * nx * ny;
            R[2][1] = -2 * nx * ny;
            R[2][2] = 1 - 2 * ny * ny;
        }
    }
};

// MeshFn storage: a[k + nb*c + bl*i]

// Equation::assemble (Equation.cpp:152-191 with computeVolumeTerm :20-33,
// computeBoundaryTerm :35-57, boundaryIntegral :114-145)
static void assemble(const Equation &eq, const double *u, double t, double *b) {
    const Mesh &msh = *eq.msh;
    const int nb = eq.nb, nc = eq.nc, bl = eq.bl, deg = eq.deg, m = deg + 1;
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < msh.np; i++) {
        const double w = msh.bb[i][2], h = msh.bb[i][3];
        const double *UMinus = u + (size_t)bl * i;
        vector<double> psi(nb, 0.0);
        for (int j = 0; j < nb; j++) {
            psi[j] = 1.0;
            vector<double> psi_x = LegDerX(deg + 1, psi), psi_y = LegDerY(deg + 1, psi);
            for (auto &q : psi_x) q *= 2.0 / w;
            for (auto &q : psi_y) q *= 2.0 / h;
            double vol[4], bnd[4] = {0, 0, 0, 0};
            // volumeIntegral (Equation.cpp:147-150)
            polygonIntegral(msh, i, deg * 2, nc, [&](double x, double y, double *out) {
                double xx, yy, vars[4], F[4][2];
                msh.getLocalCoordinates(i, x, y, xx, yy);
                eq.vars(UMinus, xx, yy, vars);
                eq.fluxFunction(vars, x, y, F);
                const double dx = Leg2D(xx, yy, m, psi_x.data()), dy = Leg2D(xx, yy, m, psi_y.data());
                for (int c = 0; c < nc; c++) out[c] = F[c][0] * dx + F[c][1] * dy;
            }, vol);
            // boundaryIntegral
            const int nv1 = (int)msh.pv[i].size();
            for (int e = 0; e < nv1; e++) {
                double nx, ny;
                msh.getOutwardNormal(i, e, nx, ny);
                const int iPlus = msh.p2p[i][e];
                const double sx = msh.shift[i][e][0], sy = msh.shift[i][e][1];
                const double *UPlus = iPlus >= 0 ? u + (size_t)bl * iPlus : nullptr;
                double li[4];
                lineIntegral(msh, i, e, deg * 2, nc, [&](double x, double y, double *out) {
                    double xm, ym, vm[4], vp[4], F[4];
                    msh.getLocalCoordinates(i, x, y, xm, ym);
                    const double psiVal = Leg2D(xm, ym, m, psi.data());
                    eq.vars(UMinus, xm, ym, vm);
                    if (iPlus < 0) {
                        eq.boundaryValue(iPlus, vm, x, y, t, nx, ny, vp);
                    } else {
                        double xp, yp;
                        msh.getLocalCoordinates(iPlus, x + sx, y + sy, xp, yp);
                        eq.vars(UPlus, xp, yp, vp);
                    }
                    eq.numericalFlux(vm, vp, x, y, nx, ny, F);
                    for (int c = 0; c < nc; c++) out[c] = psiVal * F[c];
                }, li);
                for (int c = 0; c < nc; c++) bnd[c] += li[c];
            }
            for (int c = 0; c < nc; c++) {
                double r = vol[c];
                r -= bnd[c];
                b[(size_t)bl * i + nb * c + j] = r;
            }
            psi[j] = 0.0;
        }
    }
}

// BSR (BlockMatrix, src/BlockMatrix.h:10-77): blocks contiguous, col-major
struct BSR {
    int n_rows = 0, bl = 0, nb = 0;
    vector<double> blocks;  // nb * bl * bl
    vector<int> colIndices, rowBlock;
    double *blk(int k) { return blocks.data() + (size_t)k * bl * bl; }
    const double *blk(int k) const { return blocks.data() + (size_t)k * bl * bl; }
};

// Jacobian ctor pattern (Jacobian.cpp:7-47)
static void jacobian_pattern(const Mesh &msh, int bl, BSR &J) {
    J.n_rows = msh.np;
    J.bl = bl;
    J.rowBlock.clear();
    J.colIndices.clear();
    int numBlocks = 0;
    for (int i = 0; i < msh.np; i++) {
        J.colIndices.push_back(i);
        J.rowBlock.push_back(numBlocks);
        numBlocks++;
        for (size_t j = 0; j < msh.p2p[i].size(); j++)
            if (msh.p2p[i][j] >= 0) {
                J.colIndices.push_back(msh.p2p[i][j]);
                numBlocks++;
            }
    }
    J.rowBlock.push_back(numBlocks);
    J.nb = numBlocks;
    J.blocks.assign((size_t)numBlocks * bl * bl, 0.0);
}

// Equation::jacobian (Equation.cpp:193-279 with computeVolumeJacobian :59-73,
// computeBoundaryJacobian :75-112)
static void jacobian(const Equation &eq, const double *f, double t, BSR &J) {
    const Mesh &msh = *eq.msh;
    const int nb = eq.nb, nc = eq.nc, bl = eq.bl, deg = eq.deg, m = deg + 1;
    jacobian_pattern(msh, bl, J);
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < msh.np; i++) {
        const double w = msh.bb[i][2], h = msh.bb[i][3];
        const int diagonalBlock = J.rowBlock[i];
        const double *U = f + (size_t)bl * i;
        vector<double> phi(nb, 0.0), psi(nb, 0.0);
        for (int j = 0; j < nb; j++) {
            phi[j] = 1;
            for (int k = 0; k < nb; k++) {
                psi[k] = 1;
                vector<double> psi_x = LegDerX(deg + 1, psi), psi_y = LegDerY(deg + 1, psi);
                for (auto &q : psi_x) q *= 2.0 / w;
                for (auto &q : psi_y) q *= 2.0 / h;
                auto addto = [&](int blockIdx, const double *integ, double sgn) {
                    double *B = J.blk(blockIdx);
                    for (int c = 0; c < nc; c++)
                        for (int c2 = 0; c2 < nc; c2++)
                            B[(size_t)(c2 * nb + j) * bl + (c * nb + k)] += sgn * integ[c * nc + c2];
                };
                double integ[16];
                polygonIntegral(msh, i, deg * 2, nc * nc, [&](double x, double y, double *out) {
                    double xx, yy, vars[4], A[2][4][4];
                    msh.getLocalCoordinates(i, x, y, xx, yy);
                    eq.vars(U, xx, yy, vars);
                    eq.fluxJacobian(vars, x, y, A);
                    const double ph = Leg2D(xx, yy, m, phi.data());
                    const double px = Leg2D(xx, yy, m, psi_x.data()), py = Leg2D(xx, yy, m, psi_y.data());
                    for (int c = 0; c < nc; c++)
                        for (int c2 = 0; c2 < nc; c2++)
                            out[c * nc + c2] = ph * (A[0][c][c2] * px + A[1][c][c2] * py);
                }, integ);
                addto(diagonalBlock, integ, 1.0);
                const int nv1 = (int)msh.pv[i].size();
                int blockIdx = diagonalBlock + 1;
                for (int e = 0; e < nv1; e++) {
                    double nx, ny;
                    msh.getOutwardNormal(i, e, nx, ny);
                    const int neighbor = msh.p2p[i][e];
                    const double sx = msh.shift[i][e][0], sy = msh.shift[i][e][1];
                    const double *UN = neighbor >= 0 ? f + (size_t)bl * neighbor : nullptr;
                    auto bj = [&](int iPhi, double *out_integ) {
                        lineIntegral(msh, i, e, deg * 2, nc * nc, [&](double x, double y, double *out) {
                            double xp, yp, vars[4], vars2[4], Jm[4][4];
                            msh.getLocalCoordinates(i, x, y, xp, yp);
                            const double psiVal = Leg2D(xp, yp, m, psi.data());
                            eq.vars(U, xp, yp, vars);
                            double phiVal;
                            if (iPhi >= 0 && iPhi != i) {
                                double xq, yq;
                                msh.getLocalCoordinates(iPhi, x + sx, y + sy, xq, yq);
                                phiVal = Leg2D(xq, yq, m, phi.data());
                            } else {
                                phiVal = Leg2D(xp, yp, m, phi.data());
                            }
                            if (neighbor >= 0) {
                                double xn, yn;
                                msh.getLocalCoordinates(neighbor, x + sx, y + sy, xn, yn);
                                eq.vars(UN, xn, yn, vars2);
                            } else {
                                eq.boundaryValue(neighbor, vars, x, y, t, nx, ny, vars2);
                            }
                            const int sgn = (iPhi == i) ? 1 : -1;
                            eq.numericalFluxJacobian(vars, vars2, x, y, nx, ny, sgn, Jm);
                            if (neighbor < 0 && iPhi == i) {
                                // chain rule through a state-dependent exterior
                                // value (wall, outflow); Dirichlet adds nothing
                                double R[4][4];
                                bool dep;
                                eq.boundaryDerivative(neighbor, nx, ny, R, dep);
                                if (dep) {
                                    double Jp[4][4];
                                    eq.numericalFluxJacobian(vars, vars2, x, y, nx, ny, -1, Jp);
                                    for (int r = 0; r < nc; r++)
                                        for (int c = 0; c < nc; c++) {
                                            double s = 0;
                                            for (int q = 0; q < nc; q++) s += Jp[r][q] * R[q][c];
                                            Jm[r][c] += s;
                                        }
                                }
                            }
                            for (int r = 0; r < nc; r++)
                                for (int c = 0; c < nc; c++) out[r * nc + c] = phiVal * psiVal * Jm[r][c];
                        }, out_integ);
                    };
                    if (neighbor >= 0) {
                        bj(neighbor, integ);
                        addto(blockIdx, integ, -1.0);
                        blockIdx++;
                    }
                    bj(i, integ);
                    addto(diagonalBlock, integ, -1.0);
                }
                psi[k] = 0;
            }
            phi[j] = 0;
        }
    }
}

// ------------------------------------------------------------------------
// dense LU (LAPACK dgetf2/dgetrs algorithm), column-major n x n
// ------------------------------------------------------------------------
static bool getrf(int n, double *A, int *ipiv) {
    bool ok = true;
    for (int j = 0; j < n; j++) {
        int p = j;
        double amax = std::fabs(A[(size_t)j * n + j]);
        for (int i = j + 1; i < n; i++)
            if (std::fabs(A[(size_t)j * n + i]) > amax) {
                amax = std::fabs(A[(size_t)j * n + i]);
                p = i;
            }
        ipiv[j] = p;
        if (A[(size_t)j * n + p] != 0.0) {
            if (p != j)
                for (int k = 0; k < n; k++) std::swap(A[(size_t)k * n + j], A[(size_t)k * n + p]);
            const double r = 1.0 / A[(size_t)j * n + j];
            for (int i = j + 1; i < n; i++) A[(size_t)j * n + i] *= r;
        } else {
            ok = false;
        }
        for (int k = j + 1; k < n; k++) {
            const double akj = A[(size_t)k * n + j];
            for (int i = j + 1; i < n; i++) A[(size_t)k * n + i] -= A[(size_t)j * n + i] * akj;
        }
    }
    return ok;
}
static void getrs(int n, const double *LU, const int *ipiv, double *b) {
    for (int i = 0; i < n; i++)
        if (ipiv[i] != i) std::swap(b[i], b[ipiv[i]]);
    for (int j = 0; j < n; j++)
        for (int i = j + 1; i < n; i++) b[i] -= LU[(size_t)j * n + i] * b[j];
    for (int j = n - 1; j >= 0; j--) {
        b[j] /= LU[(size_t)j * n + j];
        for (int i = 0; i < j; i++) b[i] -= LU[(size_t)j * n + i] * b[j];
    }
}
// arma::inv
static bool inv(int n, const double *A, double *Ainv) {
    vector<double> LU(A, A + (size_t)n * n);
    vector<int> piv(n);
    const bool ok = getrf(n, LU.data(), piv.data());
    for (int c = 0; c < n; c++) {
        double *col = Ainv + (size_t)c * n;
        for (int r = 0; r < n; r++) col[r] = (r == c) ? 1.0 : 0.0;
        getrs(n, LU.data(), piv.data(), col);
    }
    return ok;
}
// C = A * B (col-major)
static void gemm(int n, const double *A, const double *B, double *C) {
    for (int j = 0; j < n; j++) {
        double *c = C + (size_t)j * n;
        for (int i = 0; i < n; i++) c[i] = 0;
        for (int k = 0; k < n; k++) {
            const double b = B[(size_t)j * n + k];
            const double *a = A + (size_t)k * n;
            for (int i = 0; i < n; i++) c[i] += a[i] * b;
        }
    }
}
// y += alpha * A x  (dgemv 'N', col-major)
static void gemv(int n, double alpha, const double *A, const double *x, double *y) {
    for (int c = 0; c < n; c++) {
        const double t = alpha * x[c];
        const double *a = A + (size_t)c * n;
        for (int r = 0; r < n; r++) y[r] += t * a[r];
    }
}

// ------------------------------------------------------------------------
// MassMatrix (src/MassMatrix.cpp:30-135)
// ------------------------------------------------------------------------
struct Mass {
    int np, nb, nc, bl;
    vector<double> blocks;  // np * bl * bl (nc replicated diagonal copies)
    vector<double> LU;
    vector<int> ipvt;
};

static void mass_build(const Equation &eq, Mass &M) {
    const Mesh &msh = *eq.msh;
    const int nb = eq.nb, nc = eq.nc, bl = eq.bl, deg = eq.deg, m = deg + 1;
    M.np = msh.np;
    M.nb = nb;
    M.nc = nc;
    M.bl = bl;
    M.blocks.assign((size_t)msh.np * bl * bl, 0.0);
    M.LU.assign((size_t)msh.np * bl * bl, 0.0);
    M.ipvt.assign((size_t)msh.np * bl, 0);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < msh.np; i++) {
        vector<double> phi(nb, 0.0), psi(nb, 0.0);
        double *block = M.blocks.data() + (size_t)i * bl * bl;
        for (int j = 0; j < nb; j++) {
            phi[j] = 1.0;
            for (int k = 0; k <= j; k++) {
                psi[k] = 1.0;
                double integ;
                polygonIntegral(msh, i, deg * 2, 1, [&](double x, double y, double *out) {
                    double xx, yy;
                    msh.getLocalCoordinates(i, x, y, xx, yy);
                    out[0] = Leg2D(xx, yy, m, phi.data()) * Leg2D(xx, yy, m, psi.data());
                }, &integ);
                for (int c = 0; c < nc; c++) {
                    block[(size_t)(k + c * nb) * bl + (j + c * nb)] = integ;
                    block[(size_t)(j + c * nb) * bl + (k + c * nb)] = integ;
                }
                psi[k] = 0.0;
            }
            phi[j] = 0.0;
        }
        std::memcpy(M.LU.data() + (size_t)i * bl * bl, block, sizeof(double) * bl * bl);
        getrf(bl, M.LU.data() + (size_t)i * bl * bl, M.ipvt.data() + (size_t)i * bl);
    }
}
// MassMatrix::solve with the offset defect D2 fixed (i*bl)
static void mass_solve(const Mass &M, const double *x, double *y) {
    std::memcpy(y, x, sizeof(double) * (size_t)M.np * M.bl);
    for (int i = 0; i < M.np; i++)
        getrs(M.bl, M.LU.data() + (size_t)i * M.bl * M.bl, M.ipvt.data() + (size_t)i * M.bl,
              y + (size_t)i * M.bl);
}
// MassMatrix::matvec -> BlockMatrix::matvec over block-diagonal blocks
static void mass_matvec(const Mass &M, const double *x, double *y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < M.np; i++) {
        double *yi = y + (size_t)i * M.bl;
        for (int r = 0; r < M.bl; r++) yi[r] = 0;
        gemv(M.bl, 1.0, M.blocks.data() + (size_t)i * M.bl * M.bl, x + (size_t)i * M.bl, yi);
    }
}

// MeshFn::L2Norm (MeshFn.cpp:299-312)
static void l2norm(const Equation &eq, const double *u, double *out) {
    const Mesh &msh = *eq.msh;
    const int nc = eq.nc, bl = eq.bl, nb = eq.nb, m = eq.deg + 1;
    vector<double> l2(nc, 0.0);
    for (int i = 0; i < msh.np; i++) {
        double integ[4];
        polygonIntegral(msh, i, eq.deg * 2, nc, [&](double x, double y, double *o) {
            double xx, yy;
            msh.getLocalCoordinates(i, x, y, xx, yy);
            for (int c = 0; c < nc; c++) o[c] = std::pow(Leg2D(xx, yy, m, u + (size_t)bl * i + c * nb), 2);
        }, integ);
        for (int c = 0; c < nc; c++) l2[c] += integ[c];
    }
    for (int c = 0; c < nc; c++) out[c] = std::sqrt(l2[c]);
}

// MeshFn::L2Error (MeshFn.cpp:283-296 with L2Difference :249-261): per
// component sqrt(sum_K int_K (u_h - exact)^2) with the rule of degree 2p
static void l2error(const Equation &eq, const double *u, int kind, const double *P, double t, double *out) {
    const Mesh &msh = *eq.msh;
    const int nc = eq.nc, bl = eq.bl, nb = eq.nb, m = eq.deg + 1;
    vector<double> err(nc, 0.0);
    for (int i = 0; i < msh.np; i++) {
        double integ[4];
        polygonIntegral(msh, i, eq.deg * 2, nc, [&](double x, double y, double *o) {
            double xx, yy, ex[4];
            msh.getLocalCoordinates(i, x, y, xx, yy);
            field_eval(kind, P, nc, x, y, t, ex);
            for (int c = 0; c < nc; c++)
                o[c] = std::pow(Leg2D(xx, yy, m, u + (size_t)bl * i + c * nb) - ex[c], 2);
        }, integ);
        for (int c = 0; c < nc; c++) err[c] += integ[c];
    }
    for (int c = 0; c < nc; c++) out[c] = std::sqrt(err[c]);
}

// Gauss-Legendre nodes of order m (gsl glfixed restated), ascending
static vector<double> gl_nodes(int m) {
    vector<double> x(m);
    for (int i = 0; i < m; i++) {
        double z = std::cos(M_PI * (i + 0.75) / (m + 0.5));
        for (int it = 0; it < 100; it++) {
            double p0 = 1, p1 = z;
            for (int k = 2; k <= m; k++) {
                double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            if (m == 1) { p1 = z; p0 = 1; }
            const double dp = m * (z * p1 - p0) / (z * z - 1);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        x[m - 1 - i] = z;
    }
    if (m % 2 == 1) x[m / 2] = 0.0;
    for (int i = 0; i < m / 2; i++) {  // exact symmetry as in MeshFn.cpp:83-99
        const double a = 0.5 * (x[m - 1 - i] - x[i]);
        x[m - 1 - i] = a;
        x[i] = -a;
    }
    return x;
}

// least squares x = argmin |G x - v| by Householder QR; G is r x c col-major
static void lsq_pinv(int r, int c, const vector<double> &G, vector<double> &pinv) {
    // pinv (c x r) column j = solution for unit vector e_j
    pinv.assign((size_t)c * r, 0.0);
    vector<double> A = G;
    vector<double> beta(c);
    vector<vector<double>> vs(c);
    for (int k = 0; k < c; k++) {
        double nrm = 0;
        for (int i = k; i < r; i++) nrm += A[(size_t)k * r + i] * A[(size_t)k * r + i];
        nrm = std::sqrt(nrm);
        const double alpha = A[(size_t)k * r + k] > 0 ? -nrm : nrm;
        vector<double> v(r, 0.0);
        for (int i = k; i < r; i++) v[i] = A[(size_t)k * r + i];
        v[k] -= alpha;
        double vn = 0;
        for (int i = k; i < r; i++) vn += v[i] * v[i];
        beta[k] = vn > 0 ? 2.0 / vn : 0.0;
        for (int j = k; j < c; j++) {
            double s = 0;
            for (int i = k; i < r; i++) s += v[i] * A[(size_t)j * r + i];
            s *= beta[k];
            for (int i = k; i < r; i++) A[(size_t)j * r + i] -= s * v[i];
        }
        vs[k] = v;
    }
    for (int e = 0; e < r; e++) {
        vector<double> b(r, 0.0);
        b[e] = 1.0;
        for (int k = 0; k < c; k++) {
            double s = 0;
            for (int i = k; i < r; i++) s += vs[k][i] * b[i];
            s *= beta[k];
            for (int i = k; i < r; i++) b[i] -= s * vs[k][i];
        }
        for (int k = c - 1; k >= 0; k--) {
            double s = b[k];
            for (int j = k + 1; j < c; j++) s -= A[(size_t)j * r + k] * b[j];
            b[k] = s / A[(size_t)k * r + k];
        }
        for (int k = 0; k < c; k++) pinv[(size_t)e * c + k] = b[k];
    }
}

// MeshFn::interp (MeshFn.cpp:56-145) of an analytic field into all components
static void interp(const Equation &eq, int kind, const double *params, double t, double *u) {
    const Mesh &msh = *eq.msh;
    const int deg = eq.deg, nb = eq.nb, nc = eq.nc, bl = eq.bl, m = deg + 1;
    const vector<double> q = gl_nodes(m);
    const int nq = m * m;
    vector<double> G((size_t)nq * nb), c(nb, 0.0), pinv;
    for (int k = 0; k < nb; k++) {
        c[k] = 1.0;
        for (int i = 0; i < m; i++)
            for (int j = 0; j < m; j++) G[(size_t)k * nq + i * m + j] = Leg2D(q[i], q[j], m, c.data());
        c[k] = 0.0;
    }
    lsq_pinv(nq, nb, G, pinv);
#pragma omp parallel for schedule(static)
    for (int p = 0; p < msh.np; p++) {
        const double ax = msh.bb[p][0], by = msh.bb[p][1], w = msh.bb[p][2], h = msh.bb[p][3];
        vector<double> vals((size_t)nq * nc);
        for (int i = 0; i < m; i++)
            for (int j = 0; j < m; j++) {
                double o[4];
                field_eval(kind, params, nc, (q[i] + 1) * w / 2.0 + ax, (q[j] + 1) * h / 2.0 + by, t, o);
                for (int cc = 0; cc < nc; cc++) vals[(size_t)cc * nq + i * m + j] = o[cc];
            }
        for (int cc = 0; cc < nc; cc++)
            for (int k = 0; k < nb; k++) {
                double s = 0;
                for (int e = 0; e < nq; e++) s += pinv[(size_t)e * nb + k] * vals[(size_t)cc * nq + e];
                u[(size_t)bl * p + nb * cc + k] = s;
            }
    }
}

// ------------------------------------------------------------------------
// BlockMatrix operations (src/BlockMatrix.cpp)
// ------------------------------------------------------------------------
// matvec (BlockMatrix.cpp:28-49), out of place
static void bsr_matvec(const BSR &A, const double *x, double *y) {
    const int bl = A.bl;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < A.n_rows; i++) {
        double *yi = y + (size_t)i * bl;
        for (int r = 0; r < bl; r++) yi[r] = 0;
        for (int k = A.rowBlock[i]; k < A.rowBlock[i + 1]; k++)
            gemv(bl, 1.0, A.blk(k), x + (size_t)A.colIndices[k] * bl, yi);
    }
}

struct Precond {
    virtual void solve(double *x) const = 0;
    virtual ~Precond() {}
};
struct NoPC : Precond {
    void solve(double *) const override {}
};
// BlockJacobi (Preconditioners.cpp:8-47)
struct BlockJacobiPC : Precond {
    int n, bl;
    vector<double> F;
    vector<int> piv;
    explicit BlockJacobiPC(const BSR &M) : n(M.n_rows), bl(M.bl) {
        F.assign((size_t)n * bl * bl, 0.0);
        piv.assign((size_t)n * bl, 0);
        for (int i = 0; i < n; i++)
            for (int k = M.rowBlock[i]; k < M.rowBlock[i + 1]; k++)
                if (M.colIndices[k] == i) {
                    std::memcpy(F.data() + (size_t)i * bl * bl, M.blk(k), sizeof(double) * bl * bl);
                    getrf(bl, F.data() + (size_t)i * bl * bl, piv.data() + (size_t)i * bl);
                    break;
                }
    }
    void solve(double *x) const override {
        for (int i = 0; i < n; i++)
            getrs(bl, F.data() + (size_t)i * bl * bl, piv.data() + (size_t)i * bl, x + (size_t)i * bl);
    }
};
// BlockILU0 (Preconditioners.cpp:49-158)
struct BlockILU0PC : Precond {
    int n, bl;
    BSR DD, L, DU;
    bool singular = false;
    int singular_row = -1;
    explicit BlockILU0PC(const BSR &A) : n(A.n_rows), bl(A.bl) {
        const size_t b2 = (size_t)bl * bl;
        // AD = diag(A), AO = offDiag(A) (BlockMatrix.cpp:166-294)
        vector<double> AD((size_t)n * b2);
        BSR AO;
        AO.n_rows = n;
        AO.bl = bl;
        AO.rowBlock.assign(1, 0);
        for (int i = 0; i < n; i++) {
            for (int k = A.rowBlock[i]; k < A.rowBlock[i + 1]; k++) {
                if (A.colIndices[k] == i) {
                    std::memcpy(AD.data() + i * b2, A.blk(k), sizeof(double) * b2);
                } else {
                    AO.colIndices.push_back(A.colIndices[k]);
                    AO.blocks.insert(AO.blocks.end(), A.blk(k), A.blk(k) + b2);
                }
            }
            AO.rowBlock.push_back((int)AO.colIndices.size());
        }
        AO.nb = (int)AO.colIndices.size();
        DD.n_rows = n;
        DD.bl = bl;
        DD.blocks.assign((size_t)n * b2, 0.0);
        vector<double> tmp(b2), tmp2(b2);
        for (int i = 0; i < n; i++) {
            double *D = DD.blk(i);
            if (!inv(bl, AD.data() + i * b2, D) && !singular) {
                singular = true;
                singular_row = i;
            }
            for (int k = AO.rowBlock[i]; k < AO.rowBlock[i + 1]; k++) {
                const int j = AO.colIndices[k];
                if (j > i) {
                    for (int k2 = AO.rowBlock[j]; k2 < AO.rowBlock[j + 1]; k2++) {
                        if (AO.colIndices[k2] == i) {
                            gemm(bl, AO.blk(k2), D, tmp.data());
                            std::memcpy(AO.blk(k2), tmp.data(), sizeof(double) * b2);
                            gemm(bl, AO.blk(k2), AO.blk(k), tmp2.data());
                            double *ADj = AD.data() + (size_t)j * b2;
                            for (size_t q = 0; q < b2; q++) ADj[q] = ADj[q] - tmp2[q];
                            gemm(bl, D, AO.blk(k), tmp.data());
                            std::memcpy(AO.blk(k), tmp.data(), sizeof(double) * b2);
                            break;
                        }
                    }
                }
            }
        }
        L.n_rows = DU.n_rows = n;
        L.bl = DU.bl = bl;
        L.rowBlock.assign(1, 0);
        DU.rowBlock.assign(1, 0);
        for (int i = 0; i < n; i++) {
            for (int k = AO.rowBlock[i]; k < AO.rowBlock[i + 1]; k++) {
                const int j = AO.colIndices[k];
                if (j < i) {
                    L.colIndices.push_back(j);
                    L.blocks.insert(L.blocks.end(), AO.blk(k), AO.blk(k) + b2);
                } else if (j > i) {
                    DU.colIndices.push_back(j);
                    DU.blocks.insert(DU.blocks.end(), AO.blk(k), AO.blk(k) + b2);
                }
            }
            L.rowBlock.push_back((int)L.colIndices.size());
            DU.rowBlock.push_back((int)DU.colIndices.size());
        }
        L.nb = (int)L.colIndices.size();
        DU.nb = (int)DU.colIndices.size();
    }
    void solve(double *x) const override {
        for (int i = 0; i < n; i++)
            for (int k = L.rowBlock[i]; k < L.rowBlock[i + 1]; k++)
                gemv(bl, -1.0, L.blk(k), x + (size_t)bl * L.colIndices[k], x + (size_t)bl * i);
        // DD.matvec(x) (in place, via a copy)
        vector<double> tmp(bl);
        for (int i = 0; i < n; i++) {
            for (int r = 0; r < bl; r++) tmp[r] = 0;
            gemv(bl, 1.0, DD.blk(i), x + (size_t)bl * i, tmp.data());
            std::memcpy(x + (size_t)bl * i, tmp.data(), sizeof(double) * bl);
        }
        for (int i = n - 1; i >= 0; i--)
            for (int k = DU.rowBlock[i]; k < DU.rowBlock[i + 1]; k++)
                gemv(bl, -1.0, DU.blk(k), x + (size_t)bl * DU.colIndices[k], x + (size_t)bl * i);
    }
};

// matrix-free operator interface for GMRES
struct Op {
    virtual void apply(double *x) const = 0;  // in place, as BlockMatrix::matvec(double*)
    virtual size_t size() const = 0;
    virtual ~Op() {}
};
struct BSROp : Op {
    const BSR &A;
    explicit BSROp(const BSR &a) : A(a) {}
    void apply(double *x) const override {
        vector<double> y((size_t)A.n_rows * A.bl);
        bsr_matvec(A, x, y.data());
        std::memcpy(x, y.data(), sizeof(double) * y.size());
    }
    size_t size() const override { return (size_t)A.n_rows * A.bl; }
};

static double dnrm2(size_t n, const double *x) {
    // scaled 2-norm (reference BLAS dnrm2 algorithm)
    double scale = 0, ssq = 1;
    for (size_t i = 0; i < n; i++) {
        if (x[i] != 0) {
            const double a = std::fabs(x[i]);
            if (scale < a) {
                ssq = 1 + ssq * (scale / a) * (scale / a);
                scale = a;
            } else {
                ssq += (a / scale) * (a / scale);
            }
        }
    }
    return scale * std::sqrt(ssq);
}

// BlockMatrix::gmres (BlockMatrix.cpp:79-163)
static void gmres(const Op &A, const double *b, double *x, int m, double &tol, int &maxit,
                  const Precond &pc) {
    const size_t n = A.size();
    vector<double> v(n * (m + 1)), h(m * (m + 1) / 2 + 1), r(n), y(m + 1), c(m), s(m);
    double beta, hnew, rd, dd, nrm2b;
    int i = 0, j, uki, u0i;
    std::memcpy(r.data(), b, sizeof(double) * n);
    pc.solve(r.data());
    nrm2b = dnrm2(n, r.data());
    if (maxit % m > 0) maxit = (maxit / m + 1) * m;
    for (j = 0; j < maxit / m; j++) {
        std::memcpy(r.data(), x, sizeof(double) * n);
        A.apply(r.data());
        for (size_t q = 0; q < n; q++) r[q] += -1.0 * b[q];
        pc.solve(r.data());
        beta = dnrm2(n, r.data());
        for (size_t q = 0; q < n; q++) v[q] = r[q] * (1. / beta);
        y[0] = beta;
        uki = 0;
        for (i = 0; i < m; i++) {
            if (std::fabs(y[i]) < tol * nrm2b) break;
            double *vi = v.data() + n * i, *vi1 = v.data() + n * (i + 1);
            u0i = uki;
            std::memcpy(vi1, vi, sizeof(double) * n);
            A.apply(vi1);
            pc.solve(vi1);
            // h = V^T w (dgemv 'T'), w -= V h (dgemv 'N')
            for (int l = 0; l <= i; l++) {
                double d = 0;
                const double *vl = v.data() + n * l;
                for (size_t q = 0; q < n; q++) d += vl[q] * vi1[q];
                h[u0i + l] = d;
            }
            for (int l = 0; l <= i; l++) {
                const double hl = -h[u0i + l];
                const double *vl = v.data() + n * l;
                for (size_t q = 0; q < n; q++) vi1[q] += hl * vl[q];
            }
            hnew = dnrm2(n, vi1);
            for (size_t q = 0; q < n; q++) vi1[q] *= 1. / hnew;
            for (int k = 0; k < i; ++k) {
                const double tmp = c[k] * h[uki] - s[k] * h[uki + 1];
                h[uki + 1] = s[k] * h[uki] + c[k] * h[uki + 1];
                h[uki] = tmp;
                ++uki;
            }
            rd = h[uki];
            dd = std::sqrt(rd * rd + hnew * hnew);
            c[i] = rd / dd;
            s[i] = -hnew / dd;
            h[uki] = dd;
            ++uki;
            y[i + 1] = s[i] * y[i];
            y[i] = c[i] * y[i];
        }
        // dtpsv('U','N','N', i, h, y): packed upper, column-major
        for (int col = i - 1; col >= 0; col--) {
            const int kk = col * (col + 1) / 2;  // start of packed column col
            y[col] /= h[kk + col];
            for (int row = 0; row < col; row++) y[row] -= y[col] * h[kk + row];
        }
        for (int l = 0; l < i; l++) {
            const double yl = -y[l];
            const double *vl = v.data() + n * l;
            for (size_t q = 0; q < n; q++) x[q] += yl * vl[q];
        }
        if (std::fabs(y[i]) < tol * nrm2b) break;
    }
    maxit = m * j + i;
    tol = std::fabs(y[i]) / nrm2b;
}

// BlockMatrix::jacobi (BlockMatrix.cpp:51-77)
static void jacobi(const Op &A, const double *b, double *x, double &tol, int &maxIt,
                   const Precond &pc) {
    const size_t n = A.size();
    vector<double> Dinvb(b, b + n), DinvAur(n), r(n);
    const double omega = 1.0;
    pc.solve(Dinvb.data());
    int m;
    for (m = 0; m < maxIt; m++) {
        std::memcpy(DinvAur.data(), x, sizeof(double) * n);
        A.apply(DinvAur.data());
        for (size_t q = 0; q < n; q++) r[q] = DinvAur[q] - b[q];
        double nr = 0;
        for (size_t q = 0; q < n; q++) nr += r[q] * r[q];
        if (std::sqrt(nr) < tol) break;
        pc.solve(DinvAur.data());
        for (size_t q = 0; q < n; q++) x[q] = omega * Dinvb[q] + x[q] - omega * DinvAur[q];
    }
    double nr = 0;
    for (size_t q = 0; q < n; q++) nr += r[q] * r[q];
    tol = std::sqrt(nr);
    maxIt = m;
}

// ------------------------------------------------------------------------
// time integration (src/TimeIntegration.cpp)
// ------------------------------------------------------------------------
enum {
    ST_FE = 0, ST_RK2 = 1, ST_RK4 = 2, ST_BE = 3, ST_DIRK3 = 4, ST_DIRK5 = 5,
    ST_IRK2 = 6, ST_IRK3 = 7, ST_IRK2_INV = 8, ST_IRK3_INV = 9, ST_SDIRK3 = 10
};
enum { PC_NONE = 0, PC_BJACOBI = 1, PC_ILU0 = 2, PC_BJACOBI_CELL = 3 };

struct Stepper {
    Equation *eq;
    Mass *M;
    int kind, pc;
    int gm;
    double gtol;
    int gmaxit;
    double ntol;
    int nmaxit;
    // stats
    int newton_its = 0, gmres_its = 0, solves = 0, converged = 1;
    double last_res = 0;
};

static size_t ndof(const Equation &eq) { return (size_t)eq.msh->np * eq.bl; }

static double maxnorm(const Equation &eq, const double *r) {
    double l2[4];
    l2norm(eq, r, l2);
    double mx = l2[0];
    for (int c = 1; c < eq.nc; c++) mx = std::max(mx, l2[c]);
    return mx;
}

// k = dt * M^{-1} assemble(u, t)
static void rk_stage(Stepper &S, const double *u, double t, double dt, double *k) {
    const size_t N = ndof(*S.eq);
    vector<double> b(N);
    assemble(*S.eq, u, t, b.data());
    mass_solve(*S.M, b.data(), k);
    for (size_t q = 0; q < N; q++) k[q] = dt * k[q];
}

// Alexander's L-stable 3-stage SDIRK of order 3 (R. Alexander, SIAM J. Numer.
// Anal. 14 (1977) 1006-1021): gamma is the root in (1/6, 1/2) of
// g^3 - 3g^2 + 3g/2 - 1/6 = 0, the last row of A is b (stiffly accurate).
// The reference's getDIRK(3) uses this gamma with Crouzeix's tableau
// instead, which is of order 2 and not A-stable (|R(-inf)| = 1.78).
static void getSDIRK3(vector<double> &A, vector<double> &b, vector<double> &c) {
    const double g = 0.435866521508459;
    const double t2 = (1 + g) / 2.0;
    const double b1 = -(6 * g * g - 16 * g + 1) / 4.0, b2 = (6 * g * g - 20 * g + 5) / 4.0;
    A = {g, 0, 0, t2 - g, g, 0, b1, b2, g};
    b = {b1, b2, g};
    c = {g, t2, 1.0};
}

static void getDIRK(int s, vector<double> &A, vector<double> &b, vector<double> &c) {
    // TimeIntegration.cpp:68-91
    const double alpha = 0.435866521508459;
    if (s == 3) {
        A = {(1 + alpha) / 2.0, 0, 0, -alpha / 2.0, (1 + alpha) / 2.0, 0, 1 + alpha, -(1 + 2 * alpha),
             (1 + alpha) / 2.0};
        b = {1.0 / 6.0 / (alpha * alpha), 1 - 1.0 / 3.0 / (alpha * alpha), 1.0 / 6.0 / (alpha * alpha)};
        c = {(1 + alpha) / 2.0, 1.0 / 2.0, (1 - alpha) / 2.0};
    } else {
        const double g = (6 - std::sqrt(6)) / 10.0, r6 = std::sqrt(6);
        A = {g, 0, 0, 0, 0,
             (-6 + 5 * r6) / 14.0, g, 0, 0, 0,
             (888 + 607 * r6) / 2850.0, (126 - 161 * r6) / 1425.0, g, 0, 0,
             (3153 - 3082 * r6) / 14250.0, (3213 + 1148 * r6) / 28500.0, (-267 + 88 * r6) / 500.0, g, 0,
             (-32583 + 14638 * r6) / 71250.0, (-17199 + 364 * r6) / 142500.0, (1329 - 544 * r6) / 2500.0,
             (-96 + 131 * r6) / 625.0, g};
        b = {0, 0, 1 / 9.0, (16 - r6) / 36.0, (16 + r6) / 36.0};
        c = {g, (6 + 9 * r6) / 35.0, 1, (4 - r6) / 10.0, (4 + r6) / 10.0};
    }
}

static void getIRK(int s, vector<double> &A, vector<double> &Ainv, vector<double> &b,
                   vector<double> &c) {
    // TimeIntegration.cpp:153-186
    const double r6 = std::sqrt(6);
    if (s == 2) {
        A = {5 / 12.0, -1 / 12.0, 3 / 4.0, 1 / 4.0};
        Ainv = {3 / 2.0, 1 / 2.0, -9 / 2.0, 5 / 2.0};
        b = {3 / 4.0, 1 / 4.0};
        c = {1 / 3.0, 1};
    } else {
        A = {(88 - 7 * r6) / 360.0, (296 - 169 * r6) / 1800.0, (-2 + 3 * r6) / 225.0,
             (296 + 169 * r6) / 1800.0, (88 + 7 * r6) / 360.0, (-2 - 3 * r6) / 225.0,
             (16 - r6) / 36.0, (16 + r6) / 36.0, 1 / 9.0};
        Ainv = {60 * (1 / 30.0 + 1.0 / (20 * r6)), 60 * (-1 / 50.0 + 29.0 / (300 * r6)),
                60 * (1 / 150.0 - std::sqrt(2 / 3.0) / 75.0),
                60 * (-1 / 50.0 - 29.0 / (300 * r6)), 60 * (1 / 30.0 - 1.0 / (20 * r6)),
                60.0 * (1 / 150.0 + std::sqrt(2 / 3.0) / 75.0),
                60 * (-1 / 60.0 + (2 * std::sqrt(2 / 3.0)) / 15.0),
                60 * (-1 / 60.0 - (2 * std::sqrt(2 / 3.0)) / 15.0), 5};
        b = {(16 - r6) / 36.0, (16 + r6) / 36.0, 1 / 9.0};
        c = {(4 - r6) / 10.0, (4 + r6) / 10.0, 1};
    }
}

// B = jacobian(u); B *= scale; B += M  (BlockMatrix.cpp:297-308, Jacobian.cpp:99-110)
static void newton_matrix(Stepper &S, const double *u, double t, double scale, BSR &B) {
    jacobian(*S.eq, u, t, B);
    for (auto &q : B.blocks) q *= scale;
    const size_t b2 = (size_t)B.bl * B.bl;
    for (int i = 0; i < B.n_rows; i++) {
        double *d = B.blk(B.rowBlock[i]);
        const double *mb = S.M->blocks.data() + i * b2;
        for (size_t q = 0; q < b2; q++) d[q] += mb[q];
    }
}

static Precond *make_pc(int kind, const BSR &B) {
    if (kind == PC_ILU0) return new BlockILU0PC(B);
    if (kind == PC_BJACOBI) return new BlockJacobiPC(B);
    return new NoPC();
}

// Jacobian::solve (Jacobian.cpp:68-97) with parameters
static void linear_solve(Stepper &S, const Op &A, const Precond &pc, const double *r, double *x) {
    const size_t N = A.size();
    std::fill(x, x + N, 0.0);
    double tol = S.gtol;
    int maxit = S.gmaxit;
    gmres(A, r, x, S.gm, tol, maxit, pc);
    S.gmres_its += maxit;
    S.solves++;
}

static void dirk_advance(Stepper &S, double *u, double dt, double t) {
    // DIRK::advance (TimeIntegration.cpp:93-151); BackwardEuler is the
    // one-stage case with A = 1, b = 1, c = 1 (TimeIntegration.cpp:31-66)
    vector<double> A, b, c;
    int s;
    if (S.kind == ST_BE) {
        s = 1;
        A = {1.0};
        b = {1.0};
        c = {1.0};
    } else if (S.kind == ST_SDIRK3) {
        s = 3;
        getSDIRK3(A, b, c);
    } else {
        s = S.kind == ST_DIRK3 ? 3 : 5;
        getDIRK(s, A, b, c);
    }
    const size_t N = ndof(*S.eq);
    vector<vector<double>> k(s, vector<double>(N, 0.0));
    vector<double> cu(N), rhs(N), r(N), dk(N);
    for (int stage = 0; stage < s; stage++) {
        int iter;
        for (iter = 0; iter < S.nmaxit; iter++) {
            for (size_t q = 0; q < N; q++) cu[q] = u[q];
            for (int j = 0; j <= stage; j++)
                for (size_t q = 0; q < N; q++) cu[q] += A[stage * s + j] * k[j][q];
            assemble(*S.eq, cu.data(), t + dt * c[stage], rhs.data());
            mass_matvec(*S.M, k[stage].data(), r.data());
            for (size_t q = 0; q < N; q++) r[q] = r[q] - dt * rhs[q];
            S.last_res = maxnorm(*S.eq, r.data());
            if (std::getenv("ORC_VERBOSE"))
                std::fprintf(stderr, "  stage %d newton %d residual %.3e gmres_total %d\n", stage, iter,
                             S.last_res, S.gmres_its);
            if (S.last_res < S.ntol) break;
            S.newton_its++;
            BSR B;
            newton_matrix(S, cu.data(), t + dt * c[stage], -dt * A[stage * s + stage], B);
            Precond *pc = make_pc(S.pc, B);
            BSROp op(B);
            linear_solve(S, op, *pc, r.data(), dk.data());
            delete pc;
            for (size_t q = 0; q < N; q++) k[stage][q] -= dk[q];
        }
        if (iter == S.nmaxit) S.converged = 0;
    }
    for (int i = 0; i < s; i++)
        for (size_t q = 0; q < N; q++) u[q] += b[i] * k[i][q];
}

// stage-major coupled operator of IRK::advance: y_i = sum_j Blk(i,j) x_j with
// Blk(i,j) = -dt A(i,j) J_i (i != j), M - dt A(i,i) J_i (i == j)
// (BlockMatrix::blockBlockMatrix, BlockMatrix.cpp:228-258)
static void block_block(const vector<BSR> &Js, const Mass &M, const vector<double> &A, int s,
                        double dt, bool inverted, const vector<double> &Ainv, BSR &full) {
    const int n = Js[0].n_rows, bl = Js[0].bl;
    const size_t b2 = (size_t)bl * bl;
    full = BSR();
    full.n_rows = n * s;
    full.bl = bl;
    full.rowBlock.assign(1, 0);
    for (int i = 0; i < s; i++)
        for (int r = 0; r < n; r++) {
            for (int j = 0; j < s; j++) {
                if (!inverted) {
                    for (int k = Js[i].rowBlock[r]; k < Js[i].rowBlock[r + 1]; k++) {
                        const double sc = -dt * A[i * s + j];
                        const double *src = Js[i].blk(k);
                        const size_t off = full.blocks.size();
                        full.blocks.resize(off + b2);
                        for (size_t q = 0; q < b2; q++) full.blocks[off + q] = src[q] * sc;
                        if (i == j && Js[i].colIndices[k] == r)
                            for (size_t q = 0; q < b2; q++) full.blocks[off + q] += M.blocks[r * b2 + q];
                        full.colIndices.push_back(j * n + Js[i].colIndices[k]);
                    }
                } else {
                    if (i == j) {
                        for (int k = Js[i].rowBlock[r]; k < Js[i].rowBlock[r + 1]; k++) {
                            const double *src = Js[i].blk(k);
                            const size_t off = full.blocks.size();
                            full.blocks.resize(off + b2);
                            for (size_t q = 0; q < b2; q++) full.blocks[off + q] = src[q] * -dt;
                            if (Js[i].colIndices[k] == r)
                                for (size_t q = 0; q < b2; q++)
                                    full.blocks[off + q] += M.blocks[r * b2 + q] * Ainv[i * s + i];
                            full.colIndices.push_back(j * n + Js[i].colIndices[k]);
                        }
                    } else {
                        const size_t off = full.blocks.size();
                        full.blocks.resize(off + b2);
                        for (size_t q = 0; q < b2; q++)
                            full.blocks[off + q] = M.blocks[r * b2 + q] * Ainv[i * s + j];
                        full.colIndices.push_back(j * n + r);
                    }
                }
            }
            full.rowBlock.push_back((int)full.colIndices.size());
        }
    full.nb = (int)full.colIndices.size();
}

// cell-coupled block Jacobi for the stage system: per cell the (s*bl)^2
// matrix of the stage-major diagonal blocks, applied to the stage-major vector
struct CellCoupledPC : Precond {
    int n, bl, s;
    vector<double> F;
    vector<int> piv;
    CellCoupledPC(const BSR &full, int nstages) : n(full.n_rows / nstages), bl(full.bl), s(nstages) {
        const int S = s * bl;
        F.assign((size_t)n * S * S, 0.0);
        piv.assign((size_t)n * S, 0);
        for (int cell = 0; cell < n; cell++) {
            double *Fc = F.data() + (size_t)cell * S * S;
            for (int i = 0; i < s; i++) {
                const int row = i * n + cell;
                for (int k = full.rowBlock[row]; k < full.rowBlock[row + 1]; k++) {
                    const int col = full.colIndices[k];
                    if (col % n != cell) continue;
                    const int j = col / n;
                    const double *B = full.blk(k);
                    for (int cc = 0; cc < bl; cc++)
                        for (int rr = 0; rr < bl; rr++)
                            Fc[(size_t)(j * bl + cc) * S + (i * bl + rr)] = B[(size_t)cc * bl + rr];
                }
            }
            getrf(S, Fc, piv.data() + (size_t)cell * S);
        }
    }
    void solve(double *x) const override {
        const int S = s * bl;
        vector<double> t(S);
        for (int cell = 0; cell < n; cell++) {
            for (int i = 0; i < s; i++)
                for (int r = 0; r < bl; r++) t[i * bl + r] = x[((size_t)i * n + cell) * bl + r];
            getrs(S, F.data() + (size_t)cell * S * S, piv.data() + (size_t)cell * S, t.data());
            for (int i = 0; i < s; i++)
                for (int r = 0; r < bl; r++) x[((size_t)i * n + cell) * bl + r] = t[i * bl + r];
        }
    }
};

static Precond *make_stage_pc(int kind, const BSR &full, int s) {
    if (kind == PC_BJACOBI_CELL) return new CellCoupledPC(full, s);
    return make_pc(kind, full);
}

// IRK::advance (TimeIntegration.cpp:188-281)
static void irk_advance(Stepper &S, double *u, double dt, double t) {
    const int s = (S.kind == ST_IRK2) ? 2 : 3;
    vector<double> A, Ainv, b, c;
    getIRK(s, A, Ainv, b, c);
    const size_t N = ndof(*S.eq);
    vector<vector<double>> k(s, vector<double>(N, 0.0)), r(s, vector<double>(N)), w(s, vector<double>(N));
    vector<double> rhs(N), bigR(N * s), bigK(N * s), tmp(N);
    vector<BSR> Js(s);
    int iter;
    for (iter = 0; iter < S.nmaxit; iter++) {
        double rNorm = 0;
        for (int st = 0; st < s; st++) {
            for (size_t q = 0; q < N; q++) w[st][q] = u[q];
            for (int j = 0; j < s; j++)
                for (size_t q = 0; q < N; q++) w[st][q] += A[st * s + j] * k[j][q];
            assemble(*S.eq, w[st].data(), t + dt * c[st], rhs.data());
            mass_matvec(*S.M, k[st].data(), r[st].data());
            for (size_t q = 0; q < N; q++) r[st][q] = r[st][q] - dt * rhs[q];
            rNorm += std::pow(maxnorm(*S.eq, r[st].data()), 2);
        }
        rNorm = std::sqrt(rNorm);
        S.last_res = rNorm;
        if (rNorm < S.ntol) break;
        S.newton_its++;
        for (int st = 0; st < s; st++) jacobian(*S.eq, w[st].data(), t + dt * c[st], Js[st]);
        BSR full;
        block_block(Js, *S.M, A, s, dt, false, Ainv, full);
        for (int st = 0; st < s; st++) std::memcpy(bigR.data() + st * N, r[st].data(), sizeof(double) * N);
        Precond *pc = make_stage_pc(S.pc, full, s);
        BSROp op(full);
        // the reference keeps bigK from the previous Newton iteration as the
        // initial guess (TimeIntegration.cpp:202,258-260)
        double tol = S.gtol;
        int maxit = S.gmaxit;
        gmres(op, bigR.data(), bigK.data(), S.gm, tol, maxit, *pc);
        S.gmres_its += maxit;
        S.solves++;
        delete pc;
        for (int st = 0; st < s; st++)
            for (size_t q = 0; q < N; q++) k[st][q] -= bigK[st * N + q];
    }
    if (iter == S.nmaxit) S.converged = 0;
    for (int i = 0; i < s; i++)
        for (size_t q = 0; q < N; q++) u[q] += b[i] * k[i][q];
}

// IRK::newAdvance (TimeIntegration.cpp:283-395)
static void irk_new_advance(Stepper &S, double *u, double dt, double t) {
    const int s = (S.kind == ST_IRK2_INV) ? 2 : 3;
    vector<double> A, Ainv, b, c;
    getIRK(s, A, Ainv, b, c);
    const size_t N = ndof(*S.eq);
    vector<vector<double>> k(s, vector<double>(N, 0.0)), r(s, vector<double>(N, 0.0)),
        w(s, vector<double>(N, 0.0));
    vector<double> rhs(N), bigR(N * s), bigU(N * s, 0.0), uw(N);
    vector<BSR> Js(s);
    int iter;
    for (iter = 0; iter < S.nmaxit; iter++) {
        for (int i = 0; i < s; i++) {
            std::fill(k[i].begin(), k[i].end(), 0.0);
            for (int j = 0; j < s; j++)
                for (size_t q = 0; q < N; q++) k[i][q] += Ainv[i * s + j] * w[j][q];
        }
        double rNorm = 0;
        for (int st = 0; st < s; st++) {
            for (size_t q = 0; q < N; q++) uw[q] = u[q] + w[st][q];
            assemble(*S.eq, uw.data(), t + dt * c[st], rhs.data());
            mass_matvec(*S.M, k[st].data(), r[st].data());
            for (size_t q = 0; q < N; q++) r[st][q] = r[st][q] - dt * rhs[q];
            rNorm += std::pow(maxnorm(*S.eq, r[st].data()), 2);
        }
        rNorm = std::sqrt(rNorm);
        S.last_res = rNorm;
        if (rNorm < S.ntol) break;
        S.newton_its++;
        for (int st = 0; st < s; st++) {
            for (size_t q = 0; q < N; q++) uw[q] = u[q] + w[st][q];
            jacobian(*S.eq, uw.data(), t + dt * c[st], Js[st]);
        }
        BSR full, fullPC;
        block_block(Js, *S.M, A, s, dt, true, Ainv, full);
        // preconditioner on the stage-diagonal part only (:345-365)
        {
            const int n = Js[0].n_rows, bl = Js[0].bl;
            const size_t b2 = (size_t)bl * bl;
            fullPC.n_rows = n * s;
            fullPC.bl = bl;
            fullPC.rowBlock.assign(1, 0);
            for (int i = 0; i < s; i++)
                for (int rr = 0; rr < n; rr++) {
                    for (int kk = Js[i].rowBlock[rr]; kk < Js[i].rowBlock[rr + 1]; kk++) {
                        const size_t off = fullPC.blocks.size();
                        fullPC.blocks.resize(off + b2);
                        const double *src = Js[i].blk(kk);
                        for (size_t q = 0; q < b2; q++) fullPC.blocks[off + q] = src[q] * -dt;
                        if (Js[i].colIndices[kk] == rr)
                            for (size_t q = 0; q < b2; q++)
                                fullPC.blocks[off + q] += S.M->blocks[rr * b2 + q] * Ainv[i * s + i];
                        fullPC.colIndices.push_back(i * n + Js[i].colIndices[kk]);
                    }
                    fullPC.rowBlock.push_back((int)fullPC.colIndices.size());
                }
            fullPC.nb = (int)fullPC.colIndices.size();
        }
        for (int st = 0; st < s; st++) std::memcpy(bigR.data() + st * N, r[st].data(), sizeof(double) * N);
        Precond *pc = make_stage_pc(S.pc, fullPC, s);
        BSROp op(full);
        double tol = S.gtol;
        int maxit = S.gmaxit;
        gmres(op, bigR.data(), bigU.data(), S.gm, tol, maxit, *pc);
        S.gmres_its += maxit;
        S.solves++;
        delete pc;
        for (int st = 0; st < s; st++)
            for (size_t q = 0; q < N; q++) w[st][q] -= bigU[st * N + q];
    }
    if (iter == S.nmaxit) S.converged = 0;
    // btAinv = b^T Ainv
    for (int i = 0; i < s; i++) {
        double bt = 0;
        for (int j = 0; j < s; j++) bt += b[j] * Ainv[j * s + i];
        for (size_t q = 0; q < N; q++) u[q] += bt * w[i][q];
    }
}

static void advance(Stepper &S, double *u, double dt, double t) {
    const size_t N = ndof(*S.eq);
    if (S.kind == ST_FE) {  // TimeIntegration.cpp:10-12
        vector<double> k(N);
        rk_stage(S, u, t, dt, k.data());
        for (size_t q = 0; q < N; q++) u[q] = u[q] + k[q];
    } else if (S.kind == ST_RK2) {  // :24-29
        vector<double> k1(N), k2(N), tmp(N);
        rk_stage(S, u, t, dt, k1.data());
        for (size_t q = 0; q < N; q++) tmp[q] = u[q] + 0.5 * k1[q];
        rk_stage(S, tmp.data(), t + 0.5 * dt, dt, k2.data());
        for (size_t q = 0; q < N; q++) u[q] = u[q] + 0.5 * (k1[q] + k2[q]);
    } else if (S.kind == ST_RK4) {  // :14-22
        vector<double> k1(N), k2(N), k3(N), k4(N), tmp(N);
        rk_stage(S, u, t, dt, k1.data());
        for (size_t q = 0; q < N; q++) tmp[q] = u[q] + 0.5 * k1[q];
        rk_stage(S, tmp.data(), t + 0.5 * dt, dt, k2.data());
        for (size_t q = 0; q < N; q++) tmp[q] = u[q] + 0.5 * k2[q];
        rk_stage(S, tmp.data(), t + 0.5 * dt, dt, k3.data());
        for (size_t q = 0; q < N; q++) tmp[q] = u[q] + k3[q];
        rk_stage(S, tmp.data(), t + dt, dt, k4.data());
        for (size_t q = 0; q < N; q++)
            u[q] = u[q] + (((k1[q] + 2 * k2[q]) + 2 * k3[q]) + k4[q]) * (1.0 / 6.0);
    } else if (S.kind == ST_BE || S.kind == ST_DIRK3 || S.kind == ST_DIRK5 || S.kind == ST_SDIRK3) {
        dirk_advance(S, u, dt, t);
    } else if (S.kind == ST_IRK2 || S.kind == ST_IRK3) {
        irk_advance(S, u, dt, t);
    } else {
        irk_new_advance(S, u, dt, t);
    }
}

// ILU(0) level schedule of a BSR pattern (pull formulation): lower level of
// row j = 1 + max over lower neighbours i < j; upper level of row i =
// 1 + max over upper neighbours j > i.  Rows listed by level, ascending.
static void levels(int n, const int *rowptr, const int *col, vector<int> &lptr, vector<int> &lrows,
                   vector<int> &uptr, vector<int> &urows) {
    vector<int> lv(n, 0), uv(n, 0);
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
    auto bucket = [&](const vector<int> &lvv, int nlev, vector<int> &ptr, vector<int> &rows) {
        ptr.assign(nlev + 1, 0);
        for (int i = 0; i < n; i++) ptr[lvv[i] + 1]++;
        for (int l = 0; l < nlev; l++) ptr[l + 1] += ptr[l];
        rows.assign(n, 0);
        vector<int> fill(ptr.begin(), ptr.end() - 1);
        for (int i = 0; i < n; i++) rows[fill[lvv[i]]++] = i;
    };
    bucket(lv, nl, lptr, lrows);
    bucket(uv, nu, uptr, urows);
}

}  // namespace orc

// ==========================================================================
// extern "C" interface for the tests (ctypes) and the CPU baseline
// ==========================================================================
using namespace orc;

struct orc_mesh { Mesh m; };
struct orc_eq { Equation e; Mass M; orc_mesh *mesh; };
struct orc_stepper { Stepper s; };

extern "C" {

const char *orc_last_error() { return g_err.c_str(); }

void orc_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
#else
    (void)n;
#endif
}
int orc_get_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

orc_mesh *orc_mesh_create(int n, const int *cell_ptr, const double *poly_xy, double W, double H,
                          int periodic, const int *codes, const int *tri_ptr, const double *tri_xy) {
    orc_mesh *h = new orc_mesh();
    build_mesh(h->m, n, cell_ptr, poly_xy, W, H, periodic, codes, tri_ptr, tri_xy);
    return h;
}
// seeds (std::mt19937_64 spec) and a brute-force Voronoi mesh of them
void orc_seeds_uniform(uint64_t seed, int n, double W, double H, double *xy) { seeds_uniform(seed, n, W, H, xy); }
orc_mesh *orc_mesh_voronoi(const double *xy, int n, double W, double H, int periodic, const int *codes) {
    vector<int> cptr, tptr;
    vector<double> pxy, txy;
    voronoi_polys(xy, n, W, H, periodic != 0, cptr, pxy, tptr, txy);
    orc_mesh *h = new orc_mesh();
    build_mesh(h->m, n, cptr.data(), pxy.data(), W, H, periodic, codes, tptr.data(), txy.data());
    return h;
}
// cell-frame polygons of an oracle mesh (after vertex deduplication)
void orc_mesh_polys(orc_mesh *h, int *cell_ptr, double *poly_xy) {
    const Mesh &m = h->m;
    int e = 0;
    cell_ptr[0] = 0;
    for (int i = 0; i < m.np; i++) {
        for (const auto &q : m.pv[i]) {
            poly_xy[2 * e] = q[0];
            poly_xy[2 * e + 1] = q[1];
            e++;
        }
        cell_ptr[i + 1] = e;
    }
}
// Jacobian block pattern (Jacobian ctor, Jacobian.cpp:7-47) without values
int orc_mesh_nnzb(orc_mesh *h) {
    int nnzb = h->m.np;
    for (const auto &q : h->m.p2p)
        for (int k : q) nnzb += k >= 0;
    return nnzb;
}
void orc_mesh_pattern(orc_mesh *h, int *rowptr, int *col) {
    const Mesh &m = h->m;
    int k = 0;
    for (int i = 0; i < m.np; i++) {
        rowptr[i] = k;
        col[k++] = i;
        for (int j : m.p2p[i])
            if (j >= 0) col[k++] = j;
    }
    rowptr[m.np] = k;
}
void orc_mesh_destroy(orc_mesh *h) { delete h; }
int orc_mesh_nedges(orc_mesh *h) {
    int E = 0;
    for (auto &q : h->m.p) E += (int)q.size();
    return E;
}
// edge neighbours, shifts, bb, normals in the oracle's own derivation
void orc_mesh_export(orc_mesh *h, int *cell_ptr, int *nbr, double *shift, double *bb, double *normals) {
    const Mesh &m = h->m;
    int e = 0;
    if (cell_ptr) cell_ptr[0] = 0;
    for (int i = 0; i < m.np; i++) {
        for (size_t j = 0; j < m.p[i].size(); j++, e++) {
            if (nbr) nbr[e] = m.p2p[i][j];
            if (shift) {
                shift[2 * e] = m.shift[i][j][0];
                shift[2 * e + 1] = m.shift[i][j][1];
            }
            if (normals) m.getOutwardNormal(i, (int)j, normals[2 * e], normals[2 * e + 1]);
        }
        if (cell_ptr) cell_ptr[i + 1] = e;
        if (bb)
            for (int q = 0; q < 4; q++) bb[4 * i + q] = m.bb[i][q];
    }
}

orc_eq *orc_eq_create(orc_mesh *mh, int phys, int degree, double gamma, double bx, double by,
                      int dkind, const double *dparams, const double *inflow) {
    orc_eq *h = new orc_eq();
    Equation &e = h->e;
    h->mesh = mh;
    e.msh = &mh->m;
    e.phys = phys;
    e.nc = phys == PHYS_EULER ? 4 : 1;
    e.deg = degree;
    e.nb = (degree + 1) * (degree + 2) / 2;
    e.bl = e.nb * e.nc;
    e.gamma = gamma;
    e.bx = bx;
    e.by = by;
    e.dkind = dkind;
    for (int q = 0; q < 8; q++) e.dparams[q] = dparams ? dparams[q] : 0.0;
    for (int q = 0; q < 4; q++) e.inflow[q] = inflow ? inflow[q] : 0.0;
    mass_build(e, h->M);
    return h;
}
void orc_eq_destroy(orc_eq *h) { delete h; }
void orc_eq_set_exact_jacobian(orc_eq *h, int exact) { h->e.exact_nbr = exact != 0; }
int orc_eq_nnzb(orc_eq *h) {
    int nnzb = h->e.msh->np;
    for (auto &q : h->e.msh->p2p)
        for (int v : q)
            if (v >= 0) nnzb++;
    return nnzb;
}
void orc_assemble(orc_eq *h, const double *u, double t, double *b) { assemble(h->e, u, t, b); }
void orc_jacobian(orc_eq *h, const double *u, double t, int *rowptr, int *col, double *blocks) {
    BSR J;
    jacobian(h->e, u, t, J);
    if (rowptr) std::memcpy(rowptr, J.rowBlock.data(), sizeof(int) * J.rowBlock.size());
    if (col) std::memcpy(col, J.colIndices.data(), sizeof(int) * J.colIndices.size());
    if (blocks) std::memcpy(blocks, J.blocks.data(), sizeof(double) * J.blocks.size());
}
void orc_mass_blocks(orc_eq *h, double *out) {
    std::memcpy(out, h->M.blocks.data(), sizeof(double) * h->M.blocks.size());
}
void orc_mass_solve(orc_eq *h, const double *x, double *y) { mass_solve(h->M, x, y); }
void orc_mass_matvec(orc_eq *h, const double *x, double *y) { mass_matvec(h->M, x, y); }
void orc_l2norm(orc_eq *h, const double *u, double *out) { l2norm(h->e, u, out); }
void orc_l2error(orc_eq *h, const double *u, int kind, const double *params, double t, double *out) {
    l2error(h->e, u, kind, params, t, out);
}
void orc_interp(orc_eq *h, int kind, const double *params, double t, double *u) {
    interp(h->e, kind, params, t, u);
}

static BSR make_bsr(int n, int bl, const int *rowptr, const int *col, const double *blocks) {
    BSR A;
    A.n_rows = n;
    A.bl = bl;
    A.rowBlock.assign(rowptr, rowptr + n + 1);
    A.nb = rowptr[n];
    A.colIndices.assign(col, col + A.nb);
    A.blocks.assign(blocks, blocks + (size_t)A.nb * bl * bl);
    return A;
}
void orc_bsr_matvec(int n, int bl, const int *rowptr, const int *col, const double *blocks,
                    const double *x, double *y) {
    BSR A = make_bsr(n, bl, rowptr, col, blocks);
    bsr_matvec(A, x, y);
}
// ILU(0): dd[n*bl*bl], L/DU pattern and blocks (capacity nnzb each)
int orc_ilu0(int n, int bl, const int *rowptr, const int *col, const double *blocks, double *dd,
             int *lrow, int *lcol, double *lblk, int *urow, int *ucol, double *ublk) {
    BSR A = make_bsr(n, bl, rowptr, col, blocks);
    BlockILU0PC P(A);
    std::memcpy(dd, P.DD.blocks.data(), sizeof(double) * P.DD.blocks.size());
    std::memcpy(lrow, P.L.rowBlock.data(), sizeof(int) * (n + 1));
    std::memcpy(urow, P.DU.rowBlock.data(), sizeof(int) * (n + 1));
    if (P.L.nb) {
        std::memcpy(lcol, P.L.colIndices.data(), sizeof(int) * P.L.nb);
        std::memcpy(lblk, P.L.blocks.data(), sizeof(double) * P.L.blocks.size());
    }
    if (P.DU.nb) {
        std::memcpy(ucol, P.DU.colIndices.data(), sizeof(int) * P.DU.nb);
        std::memcpy(ublk, P.DU.blocks.data(), sizeof(double) * P.DU.blocks.size());
    }
    return P.singular ? P.singular_row : -1;
}
void orc_precond_apply(int kind, int n, int bl, const int *rowptr, const int *col,
                       const double *blocks, double *x) {
    BSR A = make_bsr(n, bl, rowptr, col, blocks);
    Precond *P = make_pc(kind, A);
    P->solve(x);
    delete P;
}
void orc_gmres(int pc_kind, int n, int bl, const int *rowptr, const int *col, const double *blocks,
               const double *b, double *x, int m, double *tol, int *maxit) {
    BSR A = make_bsr(n, bl, rowptr, col, blocks);
    Precond *P = make_pc(pc_kind, A);
    BSROp op(A);
    gmres(op, b, x, m, *tol, *maxit, *P);
    delete P;
}
void orc_jacobi(int n, int bl, const int *rowptr, const int *col, const double *blocks,
                const double *b, double *x, double *tol, int *maxit) {
    BSR A = make_bsr(n, bl, rowptr, col, blocks);
    BlockJacobiPC P(A);
    BSROp op(A);
    jacobi(op, b, x, *tol, *maxit, P);
}
int orc_levels(int n, const int *rowptr, const int *col, int *lptr, int *lrows, int *uptr,
               int *urows, int *nlev) {
    vector<int> a, b, c, d;
    levels(n, rowptr, col, a, b, c, d);
    nlev[0] = (int)a.size() - 1;
    nlev[1] = (int)c.size() - 1;
    if (lptr) std::memcpy(lptr, a.data(), sizeof(int) * a.size());
    if (lrows) std::memcpy(lrows, b.data(), sizeof(int) * n);
    if (uptr) std::memcpy(uptr, c.data(), sizeof(int) * c.size());
    if (urows) std::memcpy(urows, d.data(), sizeof(int) * n);
    return 0;
}

orc_stepper *orc_stepper_create(orc_eq *h, int kind, int pc, int gm, double gtol, int gmaxit,
                                double ntol, int nmaxit) {
    orc_stepper *s = new orc_stepper();
    s->s.eq = &h->e;
    s->s.M = &h->M;
    s->s.kind = kind;
    s->s.pc = pc;
    s->s.gm = gm;
    s->s.gtol = gtol;
    s->s.gmaxit = gmaxit;
    s->s.ntol = ntol;
    s->s.nmaxit = nmaxit;
    return s;
}
void orc_stepper_destroy(orc_stepper *s) { delete s; }
// stats: newton its, gmres its, solves, converged; last residual in *res
void orc_step(orc_stepper *s, double *u, double dt, double t, int *stats, double *res) {
    s->s.newton_its = s->s.gmres_its = s->s.solves = 0;
    s->s.converged = 1;
    advance(s->s, u, dt, t);
    if (stats) {
        stats[0] = s->s.newton_its;
        stats[1] = s->s.gmres_its;
        stats[2] = s->s.solves;
        stats[3] = s->s.converged;
    }
    if (res) *res = s->s.last_res;
}

// Leg2D / LegDerX / LegDerY / quadrature exposed for known-answer tests
double orc_leg2d(double x, double y, int m, const double *c) { return Leg2D(x, y, m, c); }
void orc_legder(int m, const double *c, double *dx, double *dy) {
    vector<double> cc(c, c + m * (m + 1) / 2);
    vector<double> a = LegDerX(m, cc), b = LegDerY(m, cc);
    std::memcpy(dx, a.data(), sizeof(double) * a.size());
    std::memcpy(dy, b.data(), sizeof(double) * b.size());
}
// integral of x^a y^b over a triangle with the rule for degree deg
double orc_tri_integral(const double *T, int deg, int a, int b) {
    Mesh m;
    m.np = 1;
    m.tri.resize(1);
    std::array<double, 6> t6;
    for (int q = 0; q < 6; q++) t6[q] = T[q];
    m.tri[0].push_back(t6);
    double r;
    polygonIntegral(m, 0, deg, 1, [&](double x, double y, double *o) { o[0] = std::pow(x, a) * std::pow(y, b); }, &r);
    return r;
}
double orc_line_integral(double x1, double y1, double x2, double y2, int deg, int a, int b) {
    Mesh m;
    m.np = 1;
    m.pv.resize(1);
    m.pv[0] = {{x1, y1}, {x2, y2}};
    double r;
    lineIntegral(m, 0, 0, deg, 1, [&](double x, double y, double *o) { o[0] = std::pow(x, a) * std::pow(y, b); }, &r);
    return r;
}
void orc_gl_nodes(int m, double *out) {
    vector<double> x = gl_nodes(m);
    std::memcpy(out, x.data(), sizeof(double) * m);
}

}  // extern "C"
