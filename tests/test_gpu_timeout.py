"""The bounded grid barrier of the persistent kernels.  The barrier is made
to wait for one block that never arrives (clmd_debug_barrier) with a short
poll limit, so the wait runs out within milliseconds: the launch must end
with CLMD_ERR_TIMEOUT latched in the status (no hang, no fault, the context
stays usable), the same system must work again once its status is cleared
and the barrier restored, and a fresh system is unaffected."""
import ctypes as C

import numpy as np
import pytest

import clmd
from conftest import random_state

pytestmark = pytest.mark.gpu


def positions(g):
    """x through the C ABI whatever the latched status (its return code)."""
    x = np.zeros(g.n)
    g.lib.clmd_get_state(g.h, clmd.ptr(x, C.c_double), *([None] * 9))
    return x


def debug_barrier(g, extra, limit):
    f = g.lib.clmd_debug_barrier
    f.argtypes = [C.c_void_p, C.c_int32, C.c_int64]
    f.restype = C.c_int
    return f(g.h, extra, limit)


@pytest.mark.parametrize("call", ["neighbor", "steps"])
def test_barrier_timeout_is_a_status(gpu, call):
    cfg = clmd.lj_config(4000, 0.05, 0.7)
    st = random_state(cfg, 12)
    g = clmd.System(cfg)
    g.set_state(st, scalars=clmd.scalars_init(cfg))
    if call == "steps":
        g.neighbor(0)
        g.zero_acc()
        g.accatom()
    assert debug_barrier(g, 1, 1 << 14) == clmd.OK
    if call == "neighbor":
        step = C.c_int32(0)
        rc = g.lib.clmd_neighbor(g.h, C.byref(step))
    else:
        rc = g.lib.clmd_steps(g.h, 1, 20)
    assert rc == clmd.ERR_TIMEOUT
    sc = g.scalars()
    assert sc.status == clmd.ERR_TIMEOUT
    # later kernels of this system are gated by the latched status
    before = positions(g)
    assert g.lib.clmd_steps(g.h, 21, 5) == clmd.ERR_TIMEOUT
    assert np.array_equal(positions(g), before)
    # restored barrier + cleared status: the system runs again
    assert debug_barrier(g, 0, 0) == clmd.OK
    g.clear_status()
    g.set_state(st, scalars=clmd.scalars_init(cfg))
    g.neighbor(0)
    g.zero_acc()
    g.accatom()
    g.steps(1, 20)
    assert g.scalars().status == 0
    # and it matches a system that never timed out
    h = clmd.System(cfg)
    h.set_state(st, scalars=clmd.scalars_init(cfg))
    h.neighbor(0)
    h.zero_acc()
    h.accatom()
    h.steps(1, 20)
    a, b = g.get_state(), h.get_state()
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
