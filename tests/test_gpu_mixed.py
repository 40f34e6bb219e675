"""Mixed precision in the single-system engine (CLMD_PREC_MIXED): FP32 pair
terms with Kahan-compensated FP32 sums; positions, velocities, the list and
cluster tests, Nose-Hoover and the energies stay FP64.

Bars: relative force error <= 1e-5 against the FP64 oracle on identical
positions (normwise, and per atom for atoms above 1% of the largest force);
list membership bit-exact (the list test is FP64); cluster labels bit-exact
on identical positions; the Nose-Hoover conserved quantity drifts by the
same amount as the FP64 engine's within 1e-4 of H per 1e4 steps.
"""
import numpy as np
import pytest

import clmd
import orc
from conftest import random_state

pytestmark = pytest.mark.gpu


def nvt_config(n, precision, **kw):
    return clmd.lj_config(n, 0.05, 0.75, integrator=clmd.INT_NOSE, ethst="N",
                          precision=precision, **kw)


def start(cfg, st):
    """main.f's start: stopdead(-1), neighbor(0), a = 0, AccAtom, PSI
    (main.f:156-160)."""
    g = clmd.System(cfg)
    g.set_state(st, scalars=clmd.scalars_init(cfg))
    g.stopdead(-1)
    g.neighbor(0)
    g.zero_acc()
    g.accatom()
    s = g.scalars()
    s.psi = (2.0 * s.ekin - 3.0 * cfg.natom * clmd.CIKB * cfg.att) / cfg.Q
    g.set_scalars(s)
    return g


@pytest.mark.parametrize("rho", [0.05, 0.3])
def test_mixed_forces_against_fp64_oracle(gpu, rho):
    n = 20000
    cfg = clmd.lj_config(n, rho, 0.75, precision=clmd.PREC_MIXED)
    st = random_state(cfg, 31)
    g = clmd.System(cfg)
    g.set_state(st, scalars=clmd.scalars_init(cfg))
    o = orc.Oracle(cfg, neighbor_mode=1)
    o.set_state(st, scalars=orc.scalars_init(cfg))
    for s_ in (g, o):
        s_.neighbor(0)
        s_.zero_acc()
        s_.accatom()
    lg, ig = g.halflist()
    lo, io = o.halflist()
    assert np.array_equal(lg, lo) and np.array_equal(ig, io)
    a, b = g.get_state(), o.get_state()
    fa = np.stack([a.ax, a.ay, a.az], 1)
    fb = np.stack([b.ax, b.ay, b.az], 1)
    assert np.linalg.norm(fa - fb) / np.linalg.norm(fb) <= 1e-5
    mag = np.linalg.norm(fb, axis=1)
    big = mag > 0.01 * mag.max()
    assert (np.linalg.norm(fa - fb, axis=1)[big] / mag[big]).max() <= 1e-5
    assert abs(g.scalars().epot - o.scalars().epot) <= 1e-6 * abs(o.scalars().epot)


def test_mixed_cluster_labels_exact_on_own_positions(gpu):
    n = 6000
    cfg = nvt_config(n, clmd.PREC_MIXED, clustering=clmd.CLU_FRENKEL, ftcsi=50)
    g = start(cfg, random_state(cfg, 8))
    g.stoddard(-1)
    g.run(0, 300)
    st = g.get_state()
    # both sides from the mixed engine's positions, fresh list radius
    h = clmd.System(cfg)
    o = orc.Oracle(cfg, neighbor_mode=1)
    h.set_state(st, scalars=clmd.scalars_init(cfg))
    o.set_state(st, scalars=orc.scalars_init(cfg))
    for s_ in (h, o):
        s_.neighbor(0)
        s_.stoddard(7)
    ch, co = h.clusters(), o.clusters()
    for k in ("cl", "cs", "csi", "csf", "csif"):
        assert np.array_equal(ch[k], co[k]), k


def nh_energy(g, cfg):
    q = g.scalars()
    nkt3 = 3.0 * cfg.natom * clmd.CIKB * cfg.att
    return q.ekin + q.epot + 0.5 * cfg.Q * q.psi ** 2 + nkt3 * q.s


def test_mixed_nose_hoover_step_against_oracle_sweeps(gpu):
    """The mixed engine solves the implicit Nose-Hoover velocity step in
    closed form (the fixed point of int-verlet-nh-mav.f:105-147); the oracle
    runs the reference's Newton sweeps to their 1e-10 test.  From identical
    injected states the positions agree exactly (the drift is FP64) and every
    gap after the step is what the FP32 pair terms explain: with da the
    accelerations' gap, v = (V + dth a) / (1 + dth PSI) moves by at most
    dth |da| (x1.5), PSI by 2 dth^2 |v| |da| / Q (x2), ekin by |v| |dv|, on
    top of 1e-10 (the sweeps' own test)."""
    from conftest import start_pair
    cfg = nvt_config(3000, clmd.PREC_MIXED)
    dth = 0.5 * cfg.dt
    st = random_state(cfg, 21)
    g = clmd.System(cfg)
    o = orc.Oracle(cfg)
    start_pair(g, o, cfg, st)
    s0 = o.scalars()
    psi = (2.0 * s0.ekin - 3.0 * cfg.natom * clmd.CIKB * cfg.att) / cfg.Q
    for sysx in (g, o):
        s = sysx.scalars()
        s.psi, s.s = psi, 0.0
        sysx.set_scalars(s)
    for step in range(1, 6):
        ref, so = o.get_state(), o.scalars()
        g.set_state(ref, scalars=so)
        g.integrator(step)
        o.integrator(step)
        a, b = g.get_state(), o.get_state()
        for k in ("x", "y", "z"):
            assert np.array_equal(getattr(a, k), getattr(b, k)), k
        aa = np.stack([a.ax, a.ay, a.az])
        ab = np.stack([b.ax, b.ay, b.az])
        da = np.linalg.norm(aa - ab)
        assert da <= 1e-5 * np.linalg.norm(ab)
        va = np.stack([a.vx, a.vy, a.vz])
        vb = np.stack([b.vx, b.vy, b.vz])
        nv = np.linalg.norm(vb)
        dv = np.linalg.norm(va - vb)
        assert dv <= 1.5 * dth * da + 1e-10 * nv, (dv, dth * da)
        sg, so = g.scalars(), o.scalars()
        assert sg.status == 0 and sg.nh_iters == 1 and so.nh_iters >= 2
        dpsi = abs(sg.psi - so.psi)
        assert dpsi <= 4.0 * dth * dth * nv * da / cfg.Q + 1e-10 * abs(so.psi), dpsi
        assert abs(sg.ekin - so.ekin) <= nv * dv + 1e-10 * so.ekin
    g.close()


def test_mixed_nose_hoover_launch_same_as_single_steps(gpu):
    """Inside one launch the mixed Nose-Hoover step scales v = W / (1 + dth
    PSI) in the same pass as the next step's drift; a launch's last step
    scales alone and the next launch drifts first.  Both orders evaluate the
    same expressions: 60 steps in one launch and 60 one-step launches give
    bit-identical states (rebuilds included)."""
    cfg = nvt_config(20000, clmd.PREC_MIXED, ftcsi=0)
    st = random_state(cfg, 5)
    out = []
    for per_step in (False, True):
        g = start(cfg, st.copy())
        if per_step:
            for step in range(1, 61):
                g.integrator(step)
        else:
            g.steps(1, 60)
        s = g.scalars()
        assert s.status == 0 and s.nrebuild >= 2
        out.append((g.get_state(), s))
        g.close()
    (a, sa), (b, sb) = out
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert (sa.psi, sa.s, sa.ekin, sa.atrskin) == (sb.psi, sb.s, sb.ekin, sb.atrskin)


def test_mixed_energy_drift_tracks_fp64(gpu):
    """H = ekin + epot + Q PSI^2 / 2 + 3 N kT s over 1e4 Nose-Hoover steps.
    The truncated (unshifted) LJ of the reference loses energy whenever a pair
    enters the cut-off, so H drifts in FP64 too (about -1.5% per 1e4 steps
    while the vapour condenses), and how much depends on the trajectory: two
    FP64 runs whose starts differ by 1e-13 in one velocity end ~2e-4 of H
    apart.  Mixed precision may add at most 1e-4 of H per 1e4 steps beyond
    that spread."""
    n, steps = 200000, 10000
    st = None
    drift = {}
    for name, prec, kick in (("fp64", clmd.PREC_FP64, 0.0), ("fp64'", clmd.PREC_FP64, 1e-13),
                             ("mixed", clmd.PREC_MIXED, 0.0)):
        cfg = nvt_config(n, prec, ftcsi=0)
        if st is None:
            st = random_state(cfg, 17)
        s0 = st.copy()
        s0.vx[0] += kick
        g = start(cfg, s0)
        h0 = nh_energy(g, cfg)
        g.run(0, steps)
        assert g.scalars().status == 0
        drift[name] = (nh_energy(g, cfg) - h0) / abs(h0)
        g.close()
    spread = abs(drift["fp64'"] - drift["fp64"])
    assert abs(drift["mixed"] - drift["fp64"]) <= 1e-4 + spread, drift
