"""The C oracle pinned on CPU: golden fixtures (tests/golden/, from an
independent Python restatement of the reference's arithmetic, bit for bit),
analytic known answers, the all-pairs vs cell-list list identity, and the
reference's quirks (species-2 row end, never-reset csi(0), chk_nucleation's
persistence rule)."""
import glob
import json
import math
import os

import numpy as np
import pytest

import clmd
import orc
from conftest import REPO, random_state

GOLDEN = sorted(glob.glob(os.path.join(REPO, "tests", "golden", "*.json")))


def fx(v):
    return np.array([float.fromhex(s) for s in v])


def config_of(d, rc=2.5):
    rskin = float.fromhex(d["rskin"])
    c = clmd.Config()
    n = d["n"]
    api = d["api"]
    L = float.fromhex(d["box"])
    c.natom = n
    c.boxx = c.boxy = c.boxz = L
    sig, eps, mas = fx(d["sig"]), fx(d["eps"]), fx(d["mas"])
    c.atsorts = max(api)
    for s in range(c.atsorts):
        c.apnum[s] = sum(1 for a in api if a == s + 1)
        c.apsig[s], c.apeps[s], c.apmas[s] = sig[s], eps[s], mas[s]
    c.att = 0.7 / clmd.CIKB
    c.atskin, c.atrcut, c.atrskin, c.dt, c.nbtim = 1.5, rc, rskin, 0.005, 10
    c.ethst = b"-"
    c.clnuctrl = b"-"
    c.atnenum = d.get("atnenum", 5)
    c.clustering = clmd.CLU_FRENKEL if "atnenum" in d else clmd.CLU_STILLINGER
    return c


def oracle_of(d, mode=0):
    c = config_of(d)
    o = orc.Oracle(c, neighbor_mode=mode)
    n = d["n"]
    z = np.zeros(n)
    st = clmd.State(fx(d["x0"]), fx(d["y0"]), fx(d["z0"]), fx(d["vx0"]), fx(d["vy0"]),
                    fx(d["vz0"]), z, z, z)
    o.set_state(st, api=np.array(d["api"], dtype=np.int32), scalars=orc.scalars_init(c))
    return o


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-5] for p in GOLDEN])
@pytest.mark.parametrize("mode", [0, 1], ids=["allpairs", "cells"])
def test_oracle_matches_golden(path, mode):
    d = json.load(open(path))
    o = oracle_of(d, mode)
    o.neighbor(0)
    o.zero_acc()
    o.accatom()
    lst, idx = o.halflist()
    assert lst.tolist() == d["atnlist"]
    assert idx.tolist() == d["atnidx"]
    st = o.get_state()
    for k, key in (("x", "xw"), ("y", "yw"), ("z", "zw"), ("ax", "ax"), ("ay", "ay"),
                   ("az", "az")):
        assert np.array_equal(getattr(st, k), fx(d[key])), k
    assert o.scalars().epot == float.fromhex(d["epot"])
    if "cl" in d:
        o.stoddard(0)
        c = o.clusters()
        assert c["cl"].tolist() == d["cl"]
        if "atnenum" not in d:
            assert c["cs"].tolist() == d["cs"]
            assert c["csi"].tolist() == d["csi"]
    if "clf" in d:
        c = o.clusters()
        liq = np.array(d["liquid"], dtype=bool)
        assert np.array_equal(c["clf"][liq], np.array(d["clf"])[liq])
        assert c["csif"][0] == int((~liq).sum())
    if "steps" in d:
        for i in range(1, d["steps"] + 1):
            o.integrator(i)
        st = o.get_state()
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(getattr(st, k), fx(d[k])), k
        s = o.scalars()
        assert s.nrebuild - 1 == d["nrebuild"] - 1
        assert s.atrskin == float.fromhex(d["atrskin"])
        assert s.ekin == float.fromhex(d["ekin"])


def test_lj_known_answers():
    """U(2^(1/6) sigma) = -eps with zero force; U(sigma) = 0; the cut-off and
    the list radius are inclusive (r^2 <= rc^2, neighbor-pbc-mav.f:89,
    for-a-lj-n-pbc-m.f:115)."""
    get = {os.path.basename(p)[:-5]: json.load(open(p)) for p in GOLDEN}
    d = get["pair_min"]
    assert math.isclose(float.fromhex(d["epot"]), -1.0, abs_tol=1e-15)
    assert abs(float.fromhex(d["ax"][0])) < 1e-13
    assert float.fromhex(get["pair_sigma"]["epot"]) == 0.0
    assert float.fromhex(get["pair_rc"]["epot"]) != 0.0        # r = rc counts
    assert float.fromhex(get["pair_beyond_rc"]["epot"]) == 0.0
    assert get["pair_rs"]["atnlist"] == [-1, 2, -2]             # r = rs listed
    assert get["pair_beyond_rs"]["atnlist"] == [-1, -2]


def test_species2_ends_stillinger_row():
    d = json.load(open(os.path.join(REPO, "tests", "golden", "species2_row_end.json")))
    # atoms 1 and 3 are 1.08 apart, but atom 2 (species 2) comes first in
    # atom 1's row and ends it (stoddard-pbc-n-m.f:85)
    assert d["cl"] == [1, 2, 3, 4]


@pytest.mark.parametrize("n,rho,seed", [(2000, 0.05, 1), (3000, 0.4, 2), (300, 0.8, 3),
                                        (500, 0.01, 4)])
def test_allpairs_equals_cells(n, rho, seed):
    cfg = clmd.lj_config(n, rho, 0.7)
    x, y, z, vx, vy, vz = clmd.init_random(n, (cfg.boxx,) * 3, 0.8 if rho > 0.3 else 0.9, 0.7,
                                           seed)
    # drift positions outside the box so the wrap is exercised
    x = x + cfg.boxx * np.where(np.arange(n) % 3 == 0, 1.0, -1.0)
    lists = []
    for mode in (0, 1):
        o = orc.Oracle(cfg, neighbor_mode=mode)
        st = clmd.State(x, y, z, vx, vy, vz, 0 * x, 0 * x, 0 * x)
        o.set_state(st, scalars=orc.scalars_init(cfg))
        o.neighbor(0)
        lists.append(o.halflist())
    assert np.array_equal(lists[0][0], lists[1][0])
    assert np.array_equal(lists[0][1], lists[1][1])


def test_csi0_accumulates_and_chk_nucleation_rule():
    """csi(0) is never reset (stoddard-pbc-n-m.f:60-68); chk_nucleation needs
    the cluster at a later call with tim - clbrkt >= clwait, and a miss
    resets clbrkt (chk-nucleation.f:33-56)."""
    d = json.load(open(os.path.join(REPO, "tests", "golden", "chain_pbc.json")))
    c = config_of(d)
    c.csover, c.clwait = 5, 100
    o = orc.Oracle(c)
    z = np.zeros(d["n"])
    o.set_state(clmd.State(fx(d["x0"]), fx(d["y0"]), fx(d["z0"]), z, z, z, z, z, z),
                api=np.array(d["api"], dtype=np.int32), scalars=orc.scalars_init(c))
    o.neighbor(0)
    o.stoddard(0)
    o.stoddard(1)
    assert o.clusters()["csi"][0] == 2 * d["csi"][0]
    assert o.chk_nucleation(0)[1] == 0 and o.scalars().clbrkt == 0   # step 0 never counts
    assert o.chk_nucleation(50)[1] == 50 and o.scalars().clbrkt == 50
    assert o.chk_nucleation(120)[1] == 120                          # 70 < clwait
    assert o.chk_nucleation(150)[1] == -150                         # aborted
    c2 = config_of(d)
    c2.csover, c2.clwait = 6, 0                                     # no cluster >= 6
    o2 = orc.Oracle(c2)
    o2.set_state(clmd.State(fx(d["x0"]), fx(d["y0"]), fx(d["z0"]), z, z, z, z, z, z),
                 api=np.array(d["api"], dtype=np.int32), scalars=orc.scalars_init(c2))
    o2.neighbor(0)
    o2.stoddard(0)
    assert o2.chk_nucleation(100)[1] == 100 and o2.scalars().clbrkt == 0


def test_velocity_verlet_energy_and_momentum():
    cfg = clmd.lj_config(800, 0.3, 0.7)
    x, y, z, vx, vy, vz = clmd.init_random(800, (cfg.boxx,) * 3, 0.9, 0.7, 9)
    o = orc.Oracle(cfg, neighbor_mode=1)
    o.set_state(clmd.State(x, y, z, vx, vy, vz, 0 * x, 0 * x, 0 * x),
                scalars=orc.scalars_init(cfg))
    o.stopdead(-1)
    st = o.get_state()
    assert abs(st.vx.sum()) < 1e-10 and abs(st.vz.sum()) < 1e-10
    s = o.scalars()
    assert math.isclose(2 * s.ekin / (3 * 800), 0.7, rel_tol=1e-12)
    o.neighbor(0)
    o.zero_acc()
    o.accatom()
    e0 = o.scalars().ekin + o.scalars().epot
    for i in range(1, 201):
        o.integrator(i)
    s = o.scalars()
    assert s.status == 0
    # truncated (unshifted) LJ: small drift from pairs crossing rc
    assert abs(s.ekin + s.epot - e0) / s.ekin < 1e-2


def test_nose_hoover_conserved_h():
    cfg = clmd.lj_config(600, 0.1, 0.75, integrator=clmd.INT_NOSE, ethst="N")
    x, y, z, vx, vy, vz = clmd.init_random(600, (cfg.boxx,) * 3, 0.9, 0.75, 11)
    o = orc.Oracle(cfg, neighbor_mode=1)
    o.set_state(clmd.State(x, y, z, vx, vy, vz, 0 * x, 0 * x, 0 * x),
                scalars=orc.scalars_init(cfg))
    o.stopdead(-1)
    o.neighbor(0)
    o.zero_acc()
    o.accatom()
    s = o.scalars()
    nkt = 3.0 * 600 * clmd.CIKB * cfg.att
    s.psi = (2.0 * s.ekin - nkt) / cfg.Q  # main.f:158-160
    o.set_scalars(s)

    def H(q):
        return q.ekin + q.epot + q.psi * q.psi * cfg.Q / 2 + 3 * 600 * clmd.CIKB * cfg.att * q.s

    h0 = H(o.scalars())
    for i in range(1, 201):
        o.integrator(i)
    s = o.scalars()
    assert s.status == 0 and 1 <= s.nh_iters < 50
    assert abs((H(s) - h0) / h0) < 1e-2


def test_errors_are_statuses_not_stops():
    cfg = clmd.lj_config(500, 0.3, 0.7, dt=0.5)  # absurd time step: skin exceeded
    x, y, z, vx, vy, vz = clmd.init_random(500, (cfg.boxx,) * 3, 0.9, 0.7, 3)
    o = orc.Oracle(cfg, neighbor_mode=1)
    o.set_state(clmd.State(x, y, z, vx, vy, vz, 0 * x, 0 * x, 0 * x),
                scalars=orc.scalars_init(cfg))
    o.neighbor(0)
    o.zero_acc()
    o.accatom()
    for i in range(1, 10):
        o.integrator(i)
    assert o.scalars().status == clmd.ERR_SKIN
    cfg2 = clmd.lj_config(500, 0.5, 0.7, nlist_cap=600)  # list capacity too small
    o2 = orc.Oracle(cfg2)
    x, y, z, vx, vy, vz = clmd.init_random(500, (cfg2.boxx,) * 3, 0.9, 0.7, 3)
    o2.set_state(clmd.State(x, y, z, vx, vy, vz, 0 * x, 0 * x, 0 * x),
                 scalars=orc.scalars_init(cfg2))
    assert o2.neighbor(0)[0] == clmd.ERR_LIST_OVERFLOW


def test_oracle_rates_warning_and_quiet_step(tmp_path):
    """rates.f:50-54: a step already analysed keeps the old lists (warning),
    so nothing condensed or evaporated and, with ctrat = 1, no line."""
    cfg = clmd.lj_config(400, 0.3, 0.7)
    st = random_state(cfg, 3)
    o = orc.Oracle(cfg)
    o.set_state(st, scalars=orc.scalars_init(cfg))
    o.neighbor(0)
    o.stoddard(5)
    out, log = tmp_path / "o.rat", tmp_path / "o.log"
    assert o.rates(5, 1, str(out), str(log)) == 0
    assert "No old Stoddard-list" in open(log).read()
    assert not out.exists()
    assert o.rates(6, 1, str(out), str(log)) == 0  # same positions: same clusters
    assert not out.exists()


@pytest.mark.parametrize("clustering", [clmd.CLU_STILLINGER, clmd.CLU_FRENKEL])
@pytest.mark.parametrize("n,rho,two", [(3000, 0.3, False), (6000, 0.12, False),
                                       (5000, 0.18, True), (8000, 0.2, False)])
def test_union_find_labels_equal_reference_sweeps(clustering, n, rho, two):
    """label_mode 1 (union-find, O(bonds)) gives the reference sweeps'
    labels, sizes, histograms, liquid atoms, counters and first-passage
    stamps bit for bit (cluster energies to rounding): the checker for the
    systems too large for the O(N^2) sweeps.  Two analyses in a row, so the
    never-reset csi(0) and the running cbiggest/clookfor take part."""
    sp = dict(n=n // 5, sigma=0.758, eps=0.085, mass=0.1) if two else None
    cfg = clmd.lj_config(n, rho, 0.7, clustering=clustering, atnenum=3, species=sp)
    st = random_state(cfg, 5)
    out = []
    for mode in (0, 1):
        o = orc.Oracle(cfg, neighbor_mode=1, label_mode=mode)
        o.set_state(st, scalars=orc.scalars_init(cfg))
        o.neighbor(0)
        o.stoddard(3)
        o.stoddard(4)
        out.append((o.clusters(), o.scalars(), o.liquid()))
        o.close()
    (ca, sa, la), (cb, sb, lb) = out
    for k in ca:
        if ca[k].dtype == np.int32:
            assert np.array_equal(ca[k], cb[k]), k
        else:
            np.testing.assert_allclose(ca[k], cb[k], rtol=1e-12, atol=1e-12, err_msg=k)
    assert np.array_equal(la, lb)
    if clustering == clmd.CLU_FRENKEL:
        assert la.sum() > 0
    for f in ("cnum", "cnumf", "cbiggest", "cbiggestf", "clookfor", "clookforf", "maxcs"):
        assert getattr(sa, f) == getattr(sb, f), f


def test_init_random_restatement_is_byte_identical():
    """The oracle's copy of the seeded start gives the engine's bytes, so a
    CPU-only process builds the same inputs without the engine library."""
    for n, rho, seed in [(1000, 0.01, 3), (5000, 0.3, 9), (200, 0.05, 1)]:
        L = (n / rho) ** (1.0 / 3.0)
        a = clmd.init_random(n, (L, L, L), 0.9, 0.7, seed)
        b = orc.init_random(n, (L, L, L), 0.9, 0.7, seed)
        for u, v in zip(a, b):
            assert np.array_equal(u, v)


def test_passage_time_known_answers():
    """helpers/passage-time.f:47-90 on a hand-made sizer record: sizes are
    stamped with the first analysis whose largest cluster reaches them; a
    jump stamps every size in between; a shrinking cluster stamps nothing;
    probab.largest counts analyses from `warmup` until (and including) the
    one that first reaches endsize."""
    ts = [0, 100, 200, 300, 400, 500, 600]
    cs = [1, 3, 2, 6, 5, 9, 12]
    pt, pb = orc.passage_time(ts, cs, startsize=2, endsize=8, warmup=100)
    assert pt.tolist() == [-1, -1, 100, 100, 300, 300, 300, 500, 500]
    # counted: 100(3), 200(2), 300(6), 400(5), 500(9 >= endsize: counted, then stop)
    assert pb.tolist() == [0, 0, 1, 1, 0, 1, 1, 0, 0]
    pt, _ = orc.passage_time(ts, cs, startsize=1, endsize=12)
    assert pt.tolist() == [-1, 0, 100, 100, 300, 300, 300, 500, 500, 500, 600, 600, 600]


def test_mpt_known_answers():
    """helpers/mpt.f:52-110: per size the mean of ts/500000 (nanoseconds at
    a 2 fs step), the standard error sqrt((<t^2> - <t>^2) / count), the
    count; an unreached size is 0/0 as in the reference."""
    ts = [500000, 1500000, 1000000, 250000]
    cs = [3, 3, 4, 3]
    m, sd, cnt = orc.mpt(ts, cs, 3, 5)
    assert cnt.tolist() == [3, 1, 0]
    t3 = np.array([1.0, 3.0, 0.5])
    assert m[0] == pytest.approx(t3.mean(), rel=1e-15)
    assert sd[0] == pytest.approx(math.sqrt(((t3 ** 2).mean() - t3.mean() ** 2) / 3), rel=1e-12)
    assert m[1] == 2.0 and sd[1] == 0.0
    assert math.isnan(m[2]) and math.isnan(sd[2])
