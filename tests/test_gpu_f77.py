"""The drop-in surface itself: the gfortran-mangled entry points over the
common blocks (include/clmd_f77.h), driven in main.f's order from a deck
read by the library's read-3d.f, against the oracle driven the same way.
Bars as the handle API's: velocity-Verlet trajectory and cluster labels
bit-exact, energies within 1e-12."""
import ctypes as C
import os

import numpy as np
import pytest

import clmd
import orc
from conftest import REPO
from test_deck import ATOMP, DMMPP, MXA

pytestmark = pytest.mark.gpu


class ATOMC(C.Structure):
    _fields_ = [(k, C.c_double * MXA) for k in
                ("x0", "y0", "z0", "x1", "y1", "z1", "x2", "y2", "z2",
                 "x3", "y3", "z3", "x4", "y4", "z4", "x5", "y5", "z5")]


class ENERG(C.Structure):
    _fields_ = [("ekin", C.c_double), ("sumv2", C.c_double), ("epot", C.c_double),
                ("ekinA", C.c_double * 10), ("H", C.c_double), ("ewall", C.c_double),
                ("ewallsum", C.c_double), ("fwall", C.c_double), ("fwallsum", C.c_double),
                ("ecltim", C.c_int32), ("ethst", C.c_char), ("eclth", C.c_char)]


class CVTPP(C.Structure):
    _fields_ = [("cek", C.c_double * MXA), ("cekf", C.c_double * (MXA + 1)),
                ("ceks", C.c_double * (MXA + 1)), ("ceksf", C.c_double * (MXA + 1)),
                ("mcts", C.c_double), ("omcts", C.c_double),
                ("cl", C.c_int32 * MXA), ("clf", C.c_int32 * MXA), ("cs", C.c_int32 * MXA),
                ("csf", C.c_int32 * (MXA + 1)), ("cc", C.c_int32 * MXA),
                ("ccf", C.c_int32 * MXA), ("csi", C.c_int32 * (MXA + 1)),
                ("csif", C.c_int32 * (MXA + 1)), ("cgs", C.c_int32 * MXA),
                ("cgsf", C.c_int32 * (MXA + 1)), ("cgsa", C.c_int32 * MXA),
                ("cgsfa", C.c_int32 * (MXA + 1)), ("cnum", C.c_int32), ("cnumf", C.c_int32),
                ("cfpt", C.c_int32 * MXA), ("cfptf", C.c_int32 * MXA), ("ccn", C.c_int32),
                ("cen", C.c_int32), ("ctrat", C.c_int32), ("cstep", C.c_int32),
                ("csover", C.c_int32), ("cbiggest", C.c_int32), ("cbiggestf", C.c_int32),
                ("clookfor", C.c_int32), ("clookforf", C.c_int32), ("clwait", C.c_int32),
                ("clbrkt", C.c_int32), ("clnuctrl", C.c_char)]


def test_f77_surface_matches_oracle(gpu, monkeypatch):
    monkeypatch.setenv("CLMD_TARGET", "SILENT")
    monkeypatch.setenv("CLMD_SYNC", "resident")
    deck = os.path.join(REPO, "tests", "golden", "nose_vapour.3d")
    lib = clmd.load()
    for name, args in (("clmd_f77_readdata", [C.c_char_p]), ("clmd_f77_reset", []),
                       ("clmd_f77_sync_to_host", [])):
        getattr(lib, name).argtypes = args
    i32 = C.POINTER(C.c_int32)
    for name in ("neighbor_", "integrator_", "stoddard_", "chk_nucleation_"):
        getattr(lib, name).argtypes = [i32]
    lib.accatom_.argtypes = []
    lib.clmd_f77_reset()
    assert lib.clmd_f77_readdata(deck.encode()) == 0
    P = ATOMP.in_dll(lib, "atomp_")
    X = ATOMC.in_dll(lib, "atomc_")
    E = ENERG.in_dll(lib, "energ_")
    V = CVTPP.in_dll(lib, "cvtpp_")
    # one species (argon) of the deck, velocity Verlet, Stillinger
    n = P.natom
    P.atsorts = 1
    P.apnum[0] = n
    P.apnum[1] = 0
    for i in range(n):
        P.api[i] = 1
    cfg, _, _ = orc.readdata(deck)
    cfg.atsorts = 1
    cfg.apnum[0] = n
    cfg.apnum[1] = 0
    cfg.integrator = clmd.INT_VERLET
    cfg.ethst = b"-"
    E.ethst = b"-"
    L = cfg.boxx
    arrs = clmd.init_random(n, (L, L, L), 0.9 * cfg.apsig[0],
                            clmd.CIKB * cfg.att / cfg.apmas[0], 23)
    z0 = np.zeros(n)
    o = orc.Oracle(cfg)
    o.set_state(clmd.State(*arrs, z0, z0, z0), scalars=orc.scalars_init(cfg))
    o.stopdead(-1)  # its state goes into the commons: stopdead's sums differ in order
    s0 = o.get_state()
    for k in ("x", "y", "z"):
        getattr(X, k + "0")[:n] = getattr(s0, k)
        getattr(X, k + "1")[:n] = getattr(s0, "v" + k)
        getattr(X, k + "2")[:n] = z0
    E.ekin = o.scalars().ekin
    step = C.c_int32(0)
    lib.neighbor_(C.byref(step))
    lib.accatom_()
    step = C.c_int32(-1)
    lib.stoddard_(C.byref(step))
    o.neighbor(0)
    o.zero_acc()
    o.accatom()
    o.stoddard(-1)
    ftcsi = cfg.ftcsi
    for i in range(0, 300):
        if i % ftcsi == 0:
            if V.cstep != i:  # wrt-csi.f:27
                s = C.c_int32(i)
                lib.stoddard_(C.byref(s))
            if o.scalars().cstep != i:
                o.stoddard(i)
        s = C.c_int32(i)
        lib.integrator_(C.byref(s))
        o.integrator(i)
    lib.clmd_f77_sync_to_host()
    r = o.get_state()
    for k in ("x", "y", "z"):
        assert np.array_equal(np.array(getattr(X, k + "0")[:n]), getattr(r, k)), k
        assert np.array_equal(np.array(getattr(X, k + "1")[:n]), getattr(r, "v" + k)), k
        assert np.array_equal(np.array(getattr(X, k + "2")[:n]), getattr(r, "a" + k)), k
    co = o.clusters()
    assert np.array_equal(np.array(V.cl[:n]), co["cl"])
    assert np.array_equal(np.array(V.csi[:n + 1])[1:], co["csi"][1:])
    q = o.scalars()
    assert abs(E.epot - q.epot) <= 1e-12 * abs(q.epot)
    assert abs(E.ekin - q.ekin) <= 1e-12 * abs(q.ekin)
    assert P.atrskin == q.atrskin and q.nrebuild > 3
    D = DMMPP.in_dll(lib, "dmmpp_")
    assert D.dmms == q.dmms and D.dmmst == q.dmmst
    lib.clmd_f77_reset()
