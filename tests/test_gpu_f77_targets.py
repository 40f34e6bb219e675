"""The drop-in surface for the other link targets and the restart path:

  * NOSE (int-verlet-nh-mav.f + scalev-nh-m.f): integrator_ through the
    gfortran-mangled entry point against the oracle, one call at a time
    from identical commons (mirror sync): positions and accelerations
    bit-exact, velocities and PSI within the rounding of the implicit
    solve's sums (1e-12);
  * FRENKEL (stoddard-pbc-n-m-fre.f): stoddard_ on a vapour with liquid
    droplets: Stillinger and ten Wolde-Frenkel labels, sizes, histograms and
    the liquid atoms bit-exact;
  * readRST -> neighbor(btim) (read-rst.f:37-65): a fresh program whose
    commons come from the deck plus the six restart records continues
    bit-identically to the oracle restarted the same way.
"""
import ctypes as C
import os

import numpy as np
import pytest

import clmd
import orc
from conftest import REPO, droplet_state
from test_deck import ATOMP, DMMPP, TIMEP
from test_gpu_f77 import ATOMC, CVTPP, ENERG

pytestmark = pytest.mark.gpu

DECK = os.path.join(REPO, "tests", "golden", "nose_vapour.3d")


def shim(monkeypatch, target, sync):
    monkeypatch.setenv("CLMD_TARGET", target)
    monkeypatch.setenv("CLMD_SYNC", sync)
    lib = clmd.load()
    for name, args in (("clmd_f77_readdata", [C.c_char_p]), ("clmd_f77_reset", []),
                       ("clmd_f77_sync_to_host", [])):
        getattr(lib, name).argtypes = args
    i32 = C.POINTER(C.c_int32)
    for name in ("neighbor_", "integrator_", "stoddard_", "chk_nucleation_", "thermostat_",
                 "stopdead_"):
        getattr(lib, name).argtypes = [i32]
    lib.accatom_.argtypes = []
    lib.clmd_f77_reset()
    assert lib.clmd_f77_readdata(DECK.encode()) == 0
    return lib


def one_species(lib, cfg):
    """Argon only (the NH solve of int-verlet-nh-mav.f uses apmas(1) for
    every atom)."""
    P = ATOMP.in_dll(lib, "atomp_")
    n = P.natom
    P.atsorts = 1
    P.apnum[0] = n
    P.apnum[1] = 0
    for i in range(n):
        P.api[i] = 1
    cfg.atsorts = 1
    cfg.apnum[0] = n
    cfg.apnum[1] = 0
    return n


def put_state(lib, n, st):
    X = ATOMC.in_dll(lib, "atomc_")
    for k in ("x", "y", "z"):
        getattr(X, k + "0")[:n] = getattr(st, k)
        getattr(X, k + "1")[:n] = getattr(st, "v" + k)
        getattr(X, k + "2")[:n] = getattr(st, "a" + k)


def get_state(lib, n):
    X = ATOMC.in_dll(lib, "atomc_")
    return {k: np.array(getattr(X, k)[:n]) for k in
            ("x0", "y0", "z0", "x1", "y1", "z1", "x2", "y2", "z2")}


def put_scalars(lib, q):
    P = ATOMP.in_dll(lib, "atomp_")
    E = ENERG.in_dll(lib, "energ_")
    D = DMMPP.in_dll(lib, "dmmpp_")
    E.ekin, E.epot, E.sumv2 = q.ekin, q.epot, q.sumv2
    P.psi, P.s, P.atrskin = q.psi, q.s, q.atrskin
    D.dmms, D.dmmsu, D.dmmst, D.dmmi = q.dmms, q.dmmsu, q.dmmst, q.dmmi
    D.dmmax, D.dmmav = q.dmmax, q.dmmav
    for k in range(256):
        D.dmmh[k] = q.dmmh[k]


def test_nose_target_integrator_per_call(gpu, monkeypatch):
    lib = shim(monkeypatch, "NOSE", "mirror")
    cfg, _, _ = orc.readdata(DECK)
    n = one_species(lib, cfg)
    cfg.integrator = clmd.INT_NOSE
    L = cfg.boxx
    arrs = clmd.init_random(n, (L, L, L), 0.9 * cfg.apsig[0],
                            clmd.CIKB * cfg.att / cfg.apmas[0], 31)
    z0 = np.zeros(n)
    o = orc.Oracle(cfg)
    o.set_state(clmd.State(*arrs, z0, z0, z0), scalars=orc.scalars_init(cfg))
    o.stopdead(-1)
    # the same list and accelerations on both sides: neighbor(0) + AccAtom
    # on the post-stopdead state (main.f's start)
    put_state(lib, n, o.get_state())
    put_scalars(lib, o.scalars())
    s = C.c_int32(0)
    lib.neighbor_(C.byref(s))
    lib.accatom_()
    o.neighbor(0)
    o.zero_acc()
    o.accatom()
    s0 = o.scalars()
    # main.f:96-101
    s0.psi = (cfg.apmas[0] * 2.0 * s0.ekin / cfg.apmas[0]
              - 3.0 * n * clmd.CIKB * cfg.att) / cfg.Q
    s0.s = 0.0
    o.set_scalars(s0)
    P = ATOMP.in_dll(lib, "atomp_")
    for step in range(1, 9):
        ref, q = o.get_state(), o.scalars()
        put_state(lib, n, ref)
        put_scalars(lib, q)
        s = C.c_int32(step)
        lib.integrator_(C.byref(s))
        o.integrator(step)
        got, r = get_state(lib, n), o.get_state()
        for k in ("x", "y", "z"):
            assert np.array_equal(got[k + "0"], getattr(r, k)), (step, k)
            assert np.array_equal(got[k + "2"], getattr(r, "a" + k)), (step, k)
            np.testing.assert_allclose(got[k + "1"], getattr(r, "v" + k), rtol=1e-12,
                                       atol=1e-15 * np.abs(getattr(r, "v" + k)).max())
        q = o.scalars()
        assert abs(P.psi - q.psi) <= 1e-11 * abs(q.psi)
    assert o.scalars().nrebuild >= 1


def test_frenkel_target_labels(gpu, monkeypatch):
    lib = shim(monkeypatch, "FRENKEL", "mirror")
    cfg, _, _ = orc.readdata(DECK)
    n = one_species(lib, cfg)
    cfg.clustering = clmd.CLU_FRENKEL
    sig = cfg.apsig[0]
    st = droplet_state(cfg, 8, 6, 4.0 * sig, spacing=1.1 * sig, rmin=0.9 * sig,
                       temp=clmd.CIKB * cfg.att / cfg.apmas[0])
    o = orc.Oracle(cfg)
    o.set_state(st, scalars=orc.scalars_init(cfg))
    o.neighbor(0)
    put_state(lib, n, st)
    put_scalars(lib, orc.scalars_init(cfg))
    s = C.c_int32(0)
    lib.neighbor_(C.byref(s))
    for step in (100, 200):
        s = C.c_int32(step)
        lib.stoddard_(C.byref(s))
        o.stoddard(step)
        V = CVTPP.in_dll(lib, "cvtpp_")
        co = o.clusters()
        liq = o.liquid().astype(bool)
        assert liq.sum() > 100
        assert np.array_equal(np.array(V.cl[:n]), co["cl"])
        assert np.array_equal(np.array(V.cs[:n]), co["cs"])
        assert np.array_equal(np.array(V.csi[:n + 1]), co["csi"])
        assert np.array_equal(np.array(V.csf[:n + 1]), co["csf"])
        assert np.array_equal(np.array(V.csif[:n + 1]), co["csif"])
        clf = np.array(V.clf[:n])
        assert np.array_equal(clf > 0, liq)
        assert np.array_equal(clf[liq], co["clf"][liq])
        q = o.scalars()
        assert (V.cnumf, V.cbiggest, V.cbiggestf, V.clookforf) == \
            (q.cnumf, q.cbiggest, q.cbiggestf, q.clookforf)
        assert np.array_equal(np.array(V.cfptf[:n]), co["cfptf"])


def test_restart_through_shim(gpu, monkeypatch):
    """SILENT run, then the restart: a fresh program reads the deck, takes
    x0..z5 and the energies from the six restart records (read-rst.f:
    39-48), btim from the deck, and calls neighbor(btim) (:61-65)."""
    lib = shim(monkeypatch, "SILENT", "resident")
    cfg, _, _ = orc.readdata(DECK)
    n = one_species(lib, cfg)
    cfg.integrator = clmd.INT_VERLET
    cfg.ethst = b"-"
    E = ENERG.in_dll(lib, "energ_")
    E.ethst = b"-"
    L = cfg.boxx
    arrs = clmd.init_random(n, (L, L, L), 0.9 * cfg.apsig[0],
                            clmd.CIKB * cfg.att / cfg.apmas[0], 41)
    z0 = np.zeros(n)
    o = orc.Oracle(cfg)
    o.set_state(clmd.State(*arrs, z0, z0, z0), scalars=orc.scalars_init(cfg))
    o.stopdead(-1)
    put_state(lib, n, o.get_state())
    E.ekin = o.scalars().ekin
    s = C.c_int32(0)
    lib.neighbor_(C.byref(s))
    lib.accatom_()
    for i in range(0, 120):
        s = C.c_int32(i)
        lib.integrator_(C.byref(s))
    lib.clmd_f77_sync_to_host()
    rst = get_state(lib, n)
    ek, ep = E.ekin, E.epot
    # the restarted program: commons from the deck, then readRST
    lib.clmd_f77_reset()
    assert lib.clmd_f77_readdata(DECK.encode()) == 0
    one_species(lib, cfg)
    E.ethst = b"-"
    T = TIMEP.in_dll(lib, "timep_")
    btim = 120
    T.btim = btim
    X = ATOMC.in_dll(lib, "atomc_")
    for k, v in rst.items():
        getattr(X, k)[:n] = v
    E.ekin, E.epot = ek, ep
    s = C.c_int32(btim)
    lib.neighbor_(C.byref(s))
    # the oracle restarted the same way
    cfg.btim = btim
    o2 = orc.Oracle(cfg)
    o2.set_state(clmd.State(rst["x0"], rst["y0"], rst["z0"], rst["x1"], rst["y1"], rst["z1"],
                            rst["x2"], rst["y2"], rst["z2"]), scalars=orc.scalars_init(cfg))
    sc = o2.scalars()
    sc.ekin, sc.epot = ek, ep
    o2.set_scalars(sc)
    o2.neighbor(btim)
    lg = get_state(lib, n)
    r = o2.get_state()
    for k in ("x", "y", "z"):
        assert np.array_equal(lg[k + "0"], getattr(r, k)), k  # wrapped alike
    for i in range(btim, btim + 150):
        s = C.c_int32(i)
        lib.integrator_(C.byref(s))
        o2.integrator(i)
    lib.clmd_f77_sync_to_host()
    got, r = get_state(lib, n), o2.get_state()
    for k in ("x", "y", "z"):
        assert np.array_equal(got[k + "0"], getattr(r, k)), k
        assert np.array_equal(got[k + "1"], getattr(r, "v" + k)), k
        assert np.array_equal(got[k + "2"], getattr(r, "a" + k)), k
    q = o2.scalars()
    P = ATOMP.in_dll(lib, "atomp_")
    assert P.atrskin == q.atrskin and q.nrebuild >= 2
    lib.clmd_f77_reset()
