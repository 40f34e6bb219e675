"""Restart files and analysis writers: the
reference's wrt-rst.f record layout, a restart that continues bit-identically,
and the wrt-csi.f / wrt-csi-fre.f / wrt-fpt.f text formats checked against an
independent Python restatement of their Fortran edit descriptors."""
import os
import struct
from pathlib import Path

import numpy as np
import pytest

import clmd
import orc
from conftest import random_state, start_pair

pytestmark = pytest.mark.gpu

GOLDEN = Path(os.path.dirname(os.path.abspath(__file__))) / "golden"


def read_records(path):
    """gfortran unformatted sequential: [int32 n][n bytes][int32 n]..."""
    data = open(path, "rb").read()
    recs, p = [], 0
    while p < len(data):
        (n,) = struct.unpack_from("<i", data, p)
        recs.append(data[p + 4:p + 4 + n])
        (m,) = struct.unpack_from("<i", data, p + 4 + n)
        assert m == n
        p += 8 + n
    return recs


def F(v, w, d):
    s = f"{v:.{d}f}"
    return "*" * w if len(s) > w else s.rjust(w)


def I(v, w):
    s = str(int(v))
    return "*" * w if len(s) > w else s.rjust(w)


def test_restart_layout_and_bit_identical_continuation(gpu, tmp_path):
    cfg = clmd.lj_config(3000, 0.05, 0.7, ftcsi=50)
    a = clmd.System(cfg)
    o = orc.Oracle(cfg)
    start_pair(a, o, cfg, random_state(cfg, 4))
    a.stoddard(-1)
    a.run(0, 200)
    path = tmp_path / "x.rst"
    a.write_rst(path, mxa=4096)
    # wrt-rst.f:35-44
    recs = read_records(path)
    assert len(recs) == 10
    assert struct.unpack("<i", recs[0])[0] == 4096
    sc = a.scalars()
    assert struct.unpack("<5d", recs[1]) == (sc.ekin, sc.epot, sc.ekin, sc.epot, sc.ekin)
    assert struct.unpack("<4d", recs[2]) == (0.0, 0.0, 0.0, 0.0)
    st = a.get_state()
    for k, names in enumerate((("x", "y", "z"), ("vx", "vy", "vz"), ("ax", "ay", "az"))):
        arr = np.frombuffer(recs[3 + k], dtype="<f8").reshape(3, 4096)
        for d, nm in enumerate(names):
            assert np.array_equal(arr[d, :3000], getattr(st, nm))
            assert not arr[d, 3000:].any()
    for k in range(6, 9):
        assert len(recs[k]) == 24 * 4096 and not np.frombuffer(recs[k], dtype="<f8").any()
    assert recs[9][:8] == b"CLMDSC01"
    # read-rst.f: restore, neighbor(btim); the run then continues as the
    # original does after the same neighbor() call
    b = clmd.System(cfg)
    assert b.read_rst(path) == cfg.btim
    step = cfg.btim
    a.neighbor(step)
    for s_ in (a, b):
        s_.run(200, 300)
    sa, sb = a.get_state(), b.get_state()
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"):
        assert np.array_equal(getattr(sa, k), getattr(sb, k)), k
    qa, qb = a.scalars(), b.scalars()
    assert (qa.atrskin, qa.nrebuild, qa.dmms) == (qb.atrskin, qb.nrebuild, qb.dmms)


def csi_lines(step, n, csi, ceks, cgsa=None):
    """wrt-csi.f:28-36 / wrt-csi-fre.f:46-50 restated."""
    out = [I(step, 15)]
    cikb = clmd.CIKB
    for i in range(1, n + 1):
        if csi[i] == 0:
            continue
        den = float(i * int(csi[i]))
        s = "   " + I(i, 7) + "   " + I(csi[i], 7)
        if cgsa is not None:
            s += "   " + F(float(np.float32(cgsa[i - 1]) / np.float32(csi[i])), 7, 3)
        s += "   " + F(ceks[i] / den, 17, 15) + "   " + F(ceks[i] / (den * 1.5 * cikb), 10, 5)
        out.append(s)
    return out


def fsi_lines(step, n, csif, ceksf, cgsfa):
    """wrt-csi-fre.f:33-56 restated (the tWF file)."""
    cikb = clmd.CIKB
    out = [I(step, 15)]
    head = "   " + I(0, 7) + "   " + I(csif[0], 7) + "   " + F(0.0, 7, 3) + "   "
    if csif[0] == 0:
        out.append(head + F(0.0, 17, 15) + "   " + F(0.0, 10, 5))
    else:
        out.append(head + F(ceksf[0] / float(csif[0]), 17, 15) + "   "
                   + F(ceksf[0] / (float(csif[0]) * 1.5 * cikb), 10, 5))
    f32 = np.float32
    for i in range(1, n + 1):
        if csif[i] == 0:
            continue
        ic = i * int(csif[i])
        out.append("   " + I(i, 7) + "   " + I(csif[i], 7) + "   "
                   + F(float(f32(cgsfa[i]) / f32(csif[i])), 7, 3) + "   "
                   + F(float(f32(ceksf[i]) / f32(ic)), 17, 15) + "   "
                   + F(float(f32(ceksf[i]) / f32(float(ic) * 1.5 * cikb)), 10, 5))
    return out


@pytest.mark.parametrize("clustering", [clmd.CLU_STILLINGER, clmd.CLU_FRENKEL])
def test_csi_writers_match_reference_formats(gpu, tmp_path, clustering):
    n = 4000
    cfg = clmd.lj_config(n, 0.3, 0.7, clustering=clustering, atnenum=3)
    g = clmd.System(cfg)
    o = orc.Oracle(cfg)
    start_pair(g, o, cfg, random_state(cfg, 5))
    g.stoddard(7)
    csi_p, fsi_p = tmp_path / "a.csi", tmp_path / "a.fsi"
    g.write_csi(7, csi_p, fsi_p)
    g.write_csi(7, csi_p, fsi_p)  # appends, as the open unit does
    c = g.clusters()
    fre = clustering == clmd.CLU_FRENKEL
    want = csi_lines(7, n, c["csi"], c["ceks"], c["cgsa"] if fre else None)
    got = open(csi_p).read().splitlines()
    assert got == want + want
    if fre:
        want_f = fsi_lines(7, n, c["csif"], c["ceksf"], c["cgsfa"])
        assert open(fsi_p).read().splitlines() == want_f + want_f
    else:
        assert not fsi_p.exists()
    # the columns come from cluster arrays that match the oracle's
    o.stoddard(7)
    co = o.clusters()
    assert np.array_equal(c["csi"], co["csi"])


def test_fpt_writers(gpu, tmp_path):
    n = 4000
    cfg = clmd.lj_config(n, 0.3, 0.7, clustering=clmd.CLU_FRENKEL, atnenum=3)
    g = clmd.System(cfg)
    o = orc.Oracle(cfg)
    start_pair(g, o, cfg, random_state(cfg, 6))
    g.stoddard(0)
    g.write_fpt(tmp_path / "a.fpt")
    c = g.clusters()
    dt = cfg.dt
    rdt = np.float32(dt * 1.0e6)
    want = []
    for i in range(1, n + 1):
        fp, ff = int(c["cfpt"][i - 1]), int(c["cfptf"][i - 1])
        if fp == -1:
            continue
        if ff == -1:
            ff = int(np.float32(ff) * rdt)
        want.append(I(i, 7) + "   " + F(float(np.float32(fp)) / (dt * 1.0e6), 12, 4) + "   "
                    + F(float(np.float32(ff) / rdt), 12, 4))
    assert open(tmp_path / "a.fpt").read().splitlines() == want
    assert len(want) > 0


def test_ensemble_replica_files(gpu, tmp_path):
    e = clmd.Ensemble(clmd.ens_config(4000, 4, ftcsi=20, threads=256))
    box = (1500 / 0.05) ** (1 / 3)
    arrs = clmd.init_random(1500, (box,) * 3, 0.9, 0.65, 9)
    s = e.add(1500, box, 0.65, *arrs, csover=10**6, budget=200)
    e.step(10)
    e.write_rst(s, tmp_path / "r.rst")
    recs = read_records(tmp_path / "r.rst")
    st, _ = e.state(s)
    x = np.frombuffer(recs[3], dtype="<f8").reshape(3, 1500)
    assert np.array_equal(x[0], st.x) and np.array_equal(x[2], st.z)
    assert recs[9][:8] == b"CLMDRP01"
    e.write_fpt(s, 0.005, tmp_path / "r.fpt")
    fpt = e.fpt(s, 128)
    rdt = np.float32(0.005 * 1.0e6)
    want = [I(i, 7) + "   " + F(float(np.float32(fpt[i - 1])) / (0.005 * 1.0e6), 12, 4) + "   "
            + F(float(np.float32(int(np.float32(-1) * rdt)) / rdt), 12, 4)
            for i in range(1, 129) if fpt[i - 1] != -1]
    assert open(tmp_path / "r.fpt").read().splitlines() == want


@pytest.mark.parametrize("ctrat", [1, 20])
def test_rates_match_oracle(gpu, tmp_path, ctrat):
    """rates.f on the device against the oracle's restatement, both driven in
    lockstep through main.f's order (rates(i), then the integrator) on the
    bit-identical FP64 velocity-Verlet trajectory: the unit-67 file and the
    size-change log agree line for line.  Real units from a deck (argon,
    Angstrom, K), at a density where the largest cluster changes."""
    cfg, _, _ = orc.readdata(str(GOLDEN / "nose_vapour.3d"))
    n = 3000
    sig = cfg.apsig[0]
    L = (n / 0.3) ** (1.0 / 3.0) * sig
    cfg.natom = n
    cfg.atsorts = 1  # argon only (the deck also has a carrier species)
    cfg.apnum[0] = n
    cfg.apnum[1] = 0
    cfg.boxx = cfg.boxy = cfg.boxz = L
    cfg.integrator = clmd.INT_VERLET
    cfg.ethst = b"-"
    cfg.clustering = clmd.CLU_STILLINGER
    kt_m = clmd.CIKB * cfg.att / cfg.apmas[0]
    arrs = clmd.init_random(n, (L, L, L), 0.9 * sig, kt_m, 12)
    z0 = np.zeros(n)
    st = clmd.State(*arrs, z0, z0, z0)
    g = clmd.System(cfg)
    o = orc.Oracle(cfg)
    start_pair(g, o, cfg, st)
    g.stoddard(-1)
    o.stoddard(-1)
    acc = clmd.RatesAcc()
    paths = {k: tmp_path / k for k in ("g.rat", "g.log", "o.rat", "o.log")}
    for i in range(120):
        g.rates(i, ctrat, acc, paths["g.rat"], paths["g.log"])
        o.rates(i, ctrat, str(paths["o.rat"]), str(paths["o.log"]))
        g.integrator(i)
        o.integrator(i)
    rg, ro = open(paths["g.rat"]).read(), open(paths["o.rat"]).read()
    assert rg == ro
    assert open(paths["g.log"]).read() == open(paths["o.log"]).read()
    assert len(rg.splitlines()) > 0
