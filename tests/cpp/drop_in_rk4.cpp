// Drop-in use of the C++ interface (include/cpolyg.hpp), written the way the
// reference's drivers use PolyMesh / Equation / TimeStepper
// (examples/ExpAdv.cpp): periodic Voronoi mesh, constant advection (1,1),
// p=2, Gaussian initial data, RK4 steps.  Prints the final L2 norm and the
// first coefficients so a test can compare with the Python path.
#include <cstdio>
#include <random>
#include <vector>

#include "cpolyg.hpp"

int main(int argc, char **argv) {
    const int n = argc > 1 ? std::atoi(argv[1]) : 1000;
    const int steps = argc > 2 ? std::atoi(argv[2]) : 10;
    std::vector<double> xy(2 * n);
    cpolyg::check(cpg_seeds_uniform(1, n, 1.0, 1.0, xy.data()));
    std::vector<std::array<double, 2>> pts(n);
    for (int i = 0; i < n; i++) pts[i] = {xy[2 * i], xy[2 * i + 1]};
    cpolyg::Context ctx(0);
    cpolyg::PolyMesh msh(pts, 1.0, 1.0, true);
    cpolyg::ConstantAdvection eqn(ctx, msh, 2, 1.0, 1.0);
    cpolyg::MeshFn u = eqn.interp(CPG_INIT_GAUSSIAN, {100.0, 0.5, 0.5});
    cpolyg::RK4 ti(eqn);
    double t = 0, dt = 1e-4;
    for (int k = 0; k < steps; k++, t += dt) u = ti.advance(u, dt, t);
    std::vector<double> h = u.download();
    std::printf("l2 %.17g\n", eqn.L2Norm(u)[0]);
    for (int i = 0; i < 6; i++) std::printf("u %d %.17g\n", i, h[i]);
    return 0;
}
