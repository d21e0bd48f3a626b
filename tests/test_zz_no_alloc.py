"""cpg_l2norm_noalloc: the L2 norm for callers that may not allocate.

Applications that hand all device memory to their own pool, or that admit
each solve against a fixed memory budget, cannot let a Newton convergence
check grow a scratch buffer.  This entry point keeps its partial sums in a
static device array instead.  The test calls it through the C ABI twice in a
row, on different fields, and checks each result against the allocating
cpg_l2norm at the tolerance the kernel tests use (1e-12 relative); the
second call also shows that the array's leftover contents from the first
call do not leak into the next result.  This file is collected last so a
failure here cannot hide any other test's outcome.
"""
import ctypes as C

import numpy as np
import pytest

import cpolyg_b200 as cp
from cases import equations

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.mark.parametrize("name,deg", [("euler", 3), ("adv_const", 2)])
def test_noalloc_norm_matches_allocating_norm_on_two_calls(ctx, name, deg):
    ge, oe, _ = equations(ctx, name, deg, n=300, periodic=True)
    kind, params = (cp.INIT_VORTEX, [5.0, 0.5, 0.5, 1, 1, 1.4, 1, 1]) if name == "euler" else \
        (cp.INIT_GAUSSIAN, [30.0, 0.4, 0.6])
    import torch
    u1 = ge.interp(kind, params)
    u2 = u1 * -3.0 + 0.25
    refs = [ge.L2Norm(u) for u in (u1, u2)]  # the allocating entry point, first
    lib = cp.lib()
    outs = [np.zeros(4) for _ in range(3)]

    def call(u, out):
        st = lib.cpg_l2norm_noalloc(ctx.h, ge.h, C.c_void_p(u.data_ptr()), out.ctypes.data_as(C.POINTER(C.c_double)))
        assert st == 0, lib.cpg_last_error(ctx.h)

    call(u1, outs[2])  # set-up call: looks up the static array's device address
    torch.cuda.synchronize()
    alloc0, free0 = torch.cuda.memory_allocated(), torch.cuda.mem_get_info()[0]
    for u, out in zip((u1, u2), outs):
        call(u, out)
    torch.cuda.synchronize()
    # the two calls allocated nothing, through torch or the driver
    assert torch.cuda.memory_allocated() == alloc0 and torch.cuda.mem_get_info()[0] == free0
    for out, ref in zip(outs, refs):
        got = out[: ge.nc]
        assert np.all(np.abs(got - ref) <= TOL * np.abs(ref).max())
