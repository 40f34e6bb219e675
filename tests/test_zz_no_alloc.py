"""clmd_stoddard_noalloc: the Stillinger analysis for callers that cannot let
the library allocate device memory (they pass only buffers they own).

Checked through the C ABI against the library's regular entry point
(clmd_stoddard on a system handle) on the same positions and half list, for
two calls in a row: labels, sizes and the size histogram must be identical
(integer outputs; csi[0] accumulates across calls in both, as in the
reference).  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import clmd
import orc
from conftest import random_state, start_pair

pytestmark = pytest.mark.gpu


def test_noalloc_matches_stoddard_two_calls(gpu):
    import torch

    cfg = clmd.lj_config(6000, 0.25, 0.7)
    st = random_state(cfg, 99)
    g = clmd.System(cfg)
    o = orc.Oracle(cfg)
    start_pair(g, o, cfg, st)
    g.steps(1, 40)  # clusters form; positions leave [0, L) between rebuilds

    state = g.get_state()
    lst, idx = g.halflist()
    sc = g.scalars()
    n = cfg.natom
    api = np.ones(n, dtype=np.int32)

    dev = torch.device("cuda")
    tx, ty, tz = (torch.from_numpy(a).to(dev) for a in (state.x, state.y, state.z))
    tapi = torch.from_numpy(api).to(dev)
    tl = torch.from_numpy(lst.astype(np.int32)).to(dev)
    ti = torch.from_numpy(idx.astype(np.int32)).to(dev)
    cl = torch.zeros(n, dtype=torch.int32, device=dev)
    cs = torch.zeros(n, dtype=torch.int32, device=dev)
    csi = torch.zeros(n + 1, dtype=torch.int32, device=dev)

    lib = clmd.load()
    f = lib.clmd_stoddard_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int32] + [C.c_void_p] * 6 + [C.c_int64] * 0
    f.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_int64, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    stream = torch.cuda.current_stream().cuda_stream

    for call in range(2):
        rc = f(n, tx.data_ptr(), ty.data_ptr(), tz.data_ptr(), tapi.data_ptr(), tl.data_ptr(),
               len(lst), ti.data_ptr(), cfg.boxx, cfg.boxy, cfg.boxz, sc.atrskin,
               cfg.apsig[0], cfg.atskin, cl.data_ptr(), cs.data_ptr(), csi.data_ptr(), stream)
        assert rc == clmd.OK
        torch.cuda.synchronize()
        g.stoddard(100 + call)
        ref = g.clusters()
        assert np.array_equal(cl.cpu().numpy(), ref["cl"]), f"labels, call {call}"
        assert np.array_equal(cs.cpu().numpy(), ref["cs"]), f"sizes, call {call}"
        assert np.array_equal(csi.cpu().numpy(), ref["csi"]), f"histogram, call {call}"
    # clusters exist, so the test exercises more than monomers
    assert ref["cs"].max() > 2


def test_noalloc_rejects_sizes_beyond_the_array(gpu):
    lib = clmd.load()
    f = lib.clmd_stoddard_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_int64, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    big = (1 << 20) + 1
    dummy = C.c_void_p(1)
    rc = f(big, dummy, dummy, dummy, dummy, dummy, big + 1, dummy, 10.0, 10.0, 10.0, 3.0, 1.0,
           1.5, dummy, dummy, dummy, dummy, None)
    assert rc == clmd.ERR_ARG
