"""Parity at the sizes the workloads are quoted on, and energy drift over
10^4 steps against the oracle.

  * the FP64 drop-in at N = 262,144, rho* = 0.02, T* = 0.7 (velocity
    Verlet): neighbour list, 20 steps with adaptive rebuilds, a Stillinger
    analysis -- list, positions, velocities, accelerations, skin scalars,
    labels, sizes and histogram bit-exact; sums within 1e-12;
  * the mixed-precision NVT system at N = 2,097,152, rho* = 0.05, T* = 0.75
    (vapour with 300 liquid droplets, ten Wolde-Frenkel >= 5 neighbours
    within 1.5 sigma): forces within 1e-5 of the FP64 oracle (normwise, and
    per atom against max(|F_i|, max|F| / 10)), list and tWF labels
    bit-exact on identical positions;
  * 10^4 steps of the FP64 engine beside the oracle: velocity Verlet stays
    bit-identical (so does its conserved H); Nose-Hoover (whose implicit
    solve sums in another order) drifts like the oracle within the spread
    that two oracle twins started 1e-13 apart show (main.f:106,142 H).

The oracle checks the large systems with its cell-list neighbour mode and
its union-find labelling mode, both shown equal to the reference's own
O(N^2) loops on CPU (tests/test_oracle.py).
"""
import numpy as np
import pytest

import clmd
import orc
from conftest import droplet_state, random_state, start_pair

pytestmark = pytest.mark.gpu

RTOL_SUM = 1e-12


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def test_dropin_at_config_size_bit_exact(gpu):
    cfg = clmd.lj_config(262144, 0.02, 0.7)
    st = random_state(cfg, 1234)
    g = clmd.System(cfg)
    o = orc.Oracle(cfg, neighbor_mode=1, label_mode=1)
    start_pair(g, o, cfg, st)
    lg, ig = g.halflist()
    lo, io = o.halflist()
    assert np.array_equal(lg, lo) and np.array_equal(ig, io)
    for i in range(1, 21):
        g.integrator(i)
        o.integrator(i)
    sg, so = g.scalars(), o.scalars()
    assert sg.status == 0 and so.status == 0
    assert sg.nrebuild == so.nrebuild >= 3  # neighbor(0) + adaptive rebuilds
    assert (sg.atrskin, sg.dmms, sg.dmmsu, sg.dmmst) == (so.atrskin, so.dmms, so.dmmsu, so.dmmst)
    a, b = g.get_state(), o.get_state()
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert rel(sg.ekin, so.ekin) < RTOL_SUM and rel(sg.epot, so.epot) < RTOL_SUM
    lg, _ = g.halflist()
    lo, _ = o.halflist()
    assert np.array_equal(lg, lo)
    g.stoddard(20)
    o.stoddard(20)
    cg, co = g.clusters(), o.clusters()
    for k in ("cl", "cs", "csi", "cfpt"):
        assert np.array_equal(cg[k], co[k]), k
    for k in ("cek", "ceks"):
        np.testing.assert_allclose(cg[k], co[k], rtol=1e-12, atol=1e-12, err_msg=k)
    assert g.scalars().maxcs == o.scalars().maxcs >= 2


def test_mixed_nvt_at_config_size(gpu):
    n = 2097152
    cfg = clmd.lj_config(n, 0.05, 0.75, integrator=clmd.INT_NOSE, ethst="N",
                         clustering=clmd.CLU_FRENKEL, atnenum=5, ftcsi=50,
                         precision=clmd.PREC_MIXED)
    st = droplet_state(cfg, 3, 300, 5.0)
    g = clmd.System(cfg)
    g.set_state(st, scalars=clmd.scalars_init(cfg))
    g.neighbor(0)
    g.zero_acc()
    g.accatom()
    ocfg = clmd.lj_config(n, 0.05, 0.75, integrator=clmd.INT_NOSE, ethst="N",
                          clustering=clmd.CLU_FRENKEL, atnenum=5, ftcsi=50)
    o = orc.Oracle(ocfg, neighbor_mode=1, label_mode=1)
    o.set_state(st, scalars=orc.scalars_init(ocfg))
    o.neighbor(0)
    o.zero_acc()
    o.accatom()
    lg, ig = g.halflist()
    lo, io = o.halflist()
    assert np.array_equal(lg, lo) and np.array_equal(ig, io)
    a, b = g.get_state(), o.get_state()
    fa = np.stack([a.ax, a.ay, a.az], 1)
    fb = np.stack([b.ax, b.ay, b.az], 1)
    assert np.linalg.norm(fa - fb) / np.linalg.norm(fb) <= 1e-5
    # per atom: relative to the atom's force, or to a tenth of the largest
    # where the net force is a small difference of large pair forces (the
    # droplets' lattice atoms: six neighbours pulling against each other)
    mag = np.linalg.norm(fb, axis=1)
    scale = np.maximum(mag, 0.1 * mag.max())
    assert (np.linalg.norm(fa - fb, axis=1) / scale).max() <= 1e-5
    assert rel(g.scalars().epot, o.scalars().epot) < 1e-5
    # the cluster tests stay FP64 on identical positions: labels bit-exact
    g.stoddard(0)
    o.stoddard(0)
    cg, co = g.clusters(), o.clusters()
    liq = o.liquid().astype(bool)
    assert liq.sum() > 10000
    assert np.array_equal(cg["clf"] > 0, liq)
    assert np.array_equal(cg["clf"][liq], co["clf"][liq])
    for k in ("cl", "cs", "csi", "csf", "csif", "cgs", "cgsf", "cgsfa", "cfpt", "cfptf"):
        assert np.array_equal(cg[k], co[k]), k
    sg, so = g.scalars(), o.scalars()
    assert (sg.cnumf, sg.cbiggest, sg.cbiggestf) == (so.cnumf, so.cbiggest, so.cbiggestf)
    assert sg.cbiggestf > 100


def _h(s, cfg):
    # main.f:106,142
    return (s.ekin + s.epot + s.psi * s.psi * cfg.Q / 2
            + 3 * cfg.natom * clmd.CIKB * cfg.att * s.s)


def _run_h(sysx, cfg, nsteps, every):
    hs = [_h(sysx.scalars(), cfg)]
    for k in range(nsteps // every):
        sysx.run(k * every, every)
        hs.append(_h(sysx.scalars(), cfg))
    return np.array(hs)


@pytest.mark.parametrize("integ", [clmd.INT_VERLET, clmd.INT_NOSE])
def test_fp64_energy_drift_matches_oracle(gpu, integ):
    nh = integ == clmd.INT_NOSE
    cfg = clmd.lj_config(3000, 0.05, 0.75, integrator=integ, ethst="N" if nh else "-", ftcsi=0)
    st = random_state(cfg, 17)
    g = clmd.System(cfg)
    o = orc.Oracle(cfg, neighbor_mode=1)
    start_pair(g, o, cfg, st)
    if nh:  # main.f:96-101
        s0 = o.scalars()
        psi = (2.0 * s0.ekin - 3.0 * cfg.natom * clmd.CIKB * cfg.att) / cfg.Q
        for x in (g, o):
            s = x.scalars()
            s.psi, s.s = psi, 0.0
            x.set_scalars(s)
    nsteps, every = 10000, 1000
    hg = _run_h(g, cfg, nsteps, every)
    ho = _run_h(o, cfg, nsteps, every)
    assert g.scalars().status == 0 and o.scalars().status == 0
    dg = (hg[-1] - hg[0]) / abs(hg[0])
    do = (ho[-1] - ho[0]) / abs(ho[0])
    if not nh:
        # bit-identical trajectory: the same H up to the order of its sums
        a, b = g.get_state(), o.get_state()
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(getattr(a, k), getattr(b, k)), k
        np.testing.assert_allclose(hg, ho, rtol=1e-12)
        return
    # Nose-Hoover: chaos separates any two runs; the spread of two oracle
    # twins started 1e-13 apart bounds how far the engine may drift from it
    spread = 0.0
    for t in (1, 2):
        tw = orc.Oracle(cfg, neighbor_mode=1)
        s = st.copy()
        s.vx = s.vx.copy()
        s.vx[t] *= 1.0 + t * 1e-13
        tw.set_state(s, scalars=orc.scalars_init(cfg))
        tw.stopdead(-1)
        tw.neighbor(0)
        tw.zero_acc()
        tw.accatom()
        s0 = tw.scalars()
        s0.psi = (2.0 * s0.ekin - 3.0 * cfg.natom * clmd.CIKB * cfg.att) / cfg.Q
        s0.s = 0.0
        tw.set_scalars(s0)
        ht = _run_h(tw, cfg, nsteps, every)
        spread = max(spread, abs((ht[-1] - ht[0]) / abs(ht[0]) - do))
    assert abs(dg - do) <= 3.0 * spread + 1e-6, (dg, do, spread)
    # and step by step the two runs' H stay as close as the twins' do
    assert np.max(np.abs(hg - ho) / np.abs(ho)) <= 3.0 * spread + 1e-6
