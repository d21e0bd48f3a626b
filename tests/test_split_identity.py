"""The algebra behind the split form of the left-preconditioned operator,
checked on the CPU with the oracle's own block ILU(0) (the reference's
BlockILU0: only the pivot blocks are modified).

With DD = D^{-1}, L = L_A D^{-1} and DU = D^{-1} U_A, the preconditioner is
P^{-1} = (I + DU)^{-1} DD (I + L)^{-1}, and A = (I + L) D + U_A + E with
E_i = A_ii - D_i.  Then

    P^{-1} A v = (I + DU)^{-1} [v + DD (I + L)^{-1} (U_A + E) v],

which the library evaluates with one product over A's upper blocks and E,
the usual forward sweep, and a backward sweep that adds v to every row."""
import numpy as np

import cpolyg_b200 as cp
import oracle
from cases import mesh


def stage_matrix(n=60, degree=1, gamma=0.435866521508459):
    """M - gamma dt J of the periodic Euler vortex at the benchmark's CFL, from
    the oracle (its Lax-Friedrichs flux couples each face both ways, so the
    pivot blocks are modified: E != 0)."""
    width = 10.0
    _, _, om = mesh(n, True, width)
    vortex = [5.0, 5.0, 5.0, 1.0, 1.0, 1.4, width, width]
    oe = oracle.Equation(om, cp.EULER, degree, dkind=cp.INIT_VORTEX, dparams=vortex, exact_jacobian=True)
    u = oe.interp(cp.INIT_VORTEX, vortex)
    rp, cl, jb = oe.jacobian(u)
    mass = oe.mass_blocks()  # [cell][j][k] = M(k, j)
    nb = mass.shape[-1]
    nc = jb.shape[-1] // nb
    dt = 0.05 * (100000 / n) ** 0.5
    blocks = -dt * gamma * jb
    for i in range(len(rp) - 1):
        for k in range(rp[i], rp[i + 1]):
            if cl[k] == i:
                for c in range(nc):  # the mass matrix on every component (column-major blocks)
                    blocks[k][c * nb:(c + 1) * nb, c * nb:(c + 1) * nb] += mass[i]
    return rp, cl, blocks


def test_split_form_equals_the_preconditioned_product():
    rp, cl, blocks = stage_matrix()
    n, bl = len(rp) - 1, blocks.shape[-1]
    mat = [b.T for b in blocks]  # BSR blocks are column-major
    v = np.random.default_rng(3).standard_normal((n, bl))

    # the layout assumption, against the oracle's own matvec
    av = np.array([sum(mat[k] @ v[cl[k]] for k in range(rp[i], rp[i + 1])) for i in range(n)])
    assert np.allclose(oracle.bsr_matvec(rp, cl, blocks, v.ravel()), av.ravel(), rtol=0, atol=1e-13)

    # plain: P^{-1} (A v), as the reference's GMRES step computes it
    plain = oracle.precond_apply(cp.PC_ILU0, rp, cl, blocks, av.ravel()).reshape(n, bl)

    dd, (lr, lc, lb), (ur, uc, ub), singular = oracle.ilu0(rp, cl, blocks)
    assert singular < 0
    diag = {i: next(k for k in range(rp[i], rp[i + 1]) if cl[k] == i) for i in range(n)}
    E = [mat[diag[i]] - np.linalg.inv(dd[i].T) for i in range(n)]
    # (U_A + E) v
    r = np.array([E[i] @ v[i] + sum(mat[k] @ v[cl[k]] for k in range(rp[i], rp[i + 1]) if cl[k] > i)
                  for i in range(n)])
    # forward sweep (I + L)^{-1}
    y = r.copy()
    for i in range(n):
        for k in range(lr[i], lr[i + 1]):
            y[i] -= lb[k].T @ y[lc[k]]
    # backward sweep (I + DU)^{-1} of v + DD y
    z = v + np.array([dd[i].T @ y[i] for i in range(n)])
    for i in reversed(range(n)):
        for k in range(ur[i], ur[i + 1]):
            z[i] -= ub[k].T @ z[uc[k]]

    cond = max(np.linalg.norm(mat[diag[i]] - E[i], np.inf) * np.linalg.norm(dd[i].T, np.inf) for i in range(n))
    err = np.abs(z - plain).max() / np.abs(plain).max()
    # the split form's rounding is of order eps * cond(D_i)
    assert err < 0.25 * np.finfo(float).eps * cond + 1e-14, (err, cond)
    # and the plain form differs from the identity by rounding only: drop E and it fails
    r_bad = r - np.array([E[i] @ v[i] for i in range(n)])
    y = r_bad.copy()
    for i in range(n):
        for k in range(lr[i], lr[i + 1]):
            y[i] -= lb[k].T @ y[lc[k]]
    z_bad = v + np.array([dd[i].T @ y[i] for i in range(n)])
    for i in reversed(range(n)):
        for k in range(ur[i], ur[i + 1]):
            z_bad[i] -= ub[k].T @ z_bad[uc[k]]
    assert np.abs(z_bad - plain).max() / np.abs(plain).max() > 1e-6
