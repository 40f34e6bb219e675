"""clmd_stoddard_noalloc: the Stillinger analysis for callers that cannot
let the library allocate device memory (they pass only buffers they own,
from their own pool or a fixed budget).

Checked through the C ABI, for two calls in a row, against the library's
regular entry point (clmd_stoddard on a system handle) and against the
oracle (stoddard-pbc-n-m.f), on the same positions and half list of a
two-species system: every 7th atom is species 2, so rows that end at a
species-2 neighbour (stoddard-pbc-n-m.f:85) and species-2 atoms left as
their own clusters both occur.  Labels, sizes and the size histogram must
be identical (integer outputs; csi[0] accumulates across calls in all three,
as in the reference).  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import clmd
import orc
from conftest import random_state

pytestmark = pytest.mark.gpu

ARGTYPES = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
            C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
            C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]


def noalloc():
    f = clmd.load().clmd_stoddard_noalloc
    f.restype = C.c_int
    f.argtypes = ARGTYPES
    return f


def test_noalloc_matches_stoddard_and_oracle_two_calls(gpu):
    import torch

    n = 6000
    api = np.ones(n, dtype=np.int32)
    api[::7] = 2
    cfg = clmd.lj_config(n, 0.25, 0.7, species=dict(n=int((api == 2).sum()), sigma=1.0,
                                                    eps=1.0, mass=1.0))
    st = random_state(cfg, 99)
    g = clmd.System(cfg)
    g.set_state(st, api=api, scalars=clmd.scalars_init(cfg))
    g.stopdead(-1)
    g.neighbor(0)
    g.zero_acc()
    g.accatom()
    g.steps(1, 40)  # clusters form; positions leave [0, L) between rebuilds
    # a list rebuilt on the current positions, by the engine and the oracle
    pre, sc0 = g.get_state(), g.scalars()
    g.neighbor(41)
    o = orc.Oracle(cfg)
    o.set_state(pre, api=api, scalars=sc0)
    o.neighbor(41)
    state = g.get_state()
    lst, idx = g.halflist()
    lo, io = o.halflist()
    assert np.array_equal(lst, lo) and np.array_equal(idx, io)
    sc = g.scalars()
    # rows that a species-2 neighbour ends: the case the test is built for
    rows_cut = 0
    for i in range(n - 1):
        k = idx[i]
        while k < len(lst) and lst[k] > 0:
            if api[lst[k] - 1] == 2 and api[i] == 1:
                rows_cut += 1
                break
            k += 1
    assert rows_cut > 100

    dev = torch.device("cuda")
    tx, ty, tz = (torch.from_numpy(a).to(dev) for a in (state.x, state.y, state.z))
    tapi = torch.from_numpy(api).to(dev)
    tl = torch.from_numpy(lst.astype(np.int32)).to(dev)
    ti = torch.from_numpy(idx.astype(np.int32)).to(dev)
    cl = torch.zeros(n, dtype=torch.int32, device=dev)
    cs = torch.zeros(n, dtype=torch.int32, device=dev)
    csi = torch.zeros(n + 1, dtype=torch.int32, device=dev)
    f = noalloc()
    stream = torch.cuda.current_stream().cuda_stream

    for call in range(2):
        rc = f(n, tx.data_ptr(), ty.data_ptr(), tz.data_ptr(), tapi.data_ptr(), tl.data_ptr(),
               len(lst), ti.data_ptr(), cfg.boxx, cfg.boxy, cfg.boxz, sc.atrskin,
               cfg.apsig[0], cfg.atskin, cl.data_ptr(), cs.data_ptr(), csi.data_ptr(), stream)
        assert rc == clmd.OK
        torch.cuda.synchronize()
        g.stoddard(100 + call)
        o.stoddard(100 + call)
        ref, oref = g.clusters(), o.clusters()
        got = {"cl": cl.cpu().numpy(), "cs": cs.cpu().numpy(), "csi": csi.cpu().numpy()}
        for k in ("cl", "cs", "csi"):
            assert np.array_equal(got[k], ref[k]), f"{k} vs clmd_stoddard, call {call}"
            assert np.array_equal(got[k], oref[k]), f"{k} vs the oracle, call {call}"
    # clusters exist, and species-2 atoms stay alone
    assert ref["cs"].max() > 2
    two = np.nonzero(api == 2)[0]
    assert np.array_equal(got["cl"][two], two + 1)


def test_noalloc_rejects_sizes_beyond_the_array(gpu):
    f = noalloc()
    big = (1 << 20) + 1
    dummy = C.c_void_p(1)
    rc = f(big, dummy, dummy, dummy, dummy, dummy, big + 1, dummy, 10.0, 10.0, 10.0, 3.0, 1.0,
           1.5, dummy, dummy, dummy, dummy, None)
    assert rc == clmd.ERR_ARG
