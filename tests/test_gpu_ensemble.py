"""Ensembles (batched / served replicas) on the GPU against the FP64 oracle.

Bars (north_star): mixed precision relative force error <= 1e-5 against the
FP64 oracle on the same positions; FP64 ensemble forces within 1e-12;
cluster labels bit-exact on identical positions; a replica's result is the
same alone and in a mix (bit-identical: per-replica work never depends on the
other replicas).
"""
import numpy as np
import pytest

import clmd
import orc

pytestmark = pytest.mark.gpu


def replica_inputs(n, rho, temp, seed):
    box = (n / rho) ** (1.0 / 3.0)
    x, y, z, vx, vy, vz = clmd.init_random(n, (box, box, box), 0.9, temp, seed)
    return box, (x, y, z, vx, vy, vz)


def oracle_forces(n, box, st):
    """FP64 reference accelerations on the given positions (for-a-lj-n-pbc-m.f)."""
    cfg = clmd.lj_config(n, n / box ** 3, 0.7)
    o = orc.Oracle(cfg, neighbor_mode=1)
    z0 = np.zeros(n)
    o.set_state(clmd.State(st.x, st.y, st.z, z0, z0, z0, z0, z0, z0),
                scalars=orc.scalars_init(cfg))
    o.neighbor(0)
    o.zero_acc()
    o.accatom()
    return o


def force_errors(st, ref):
    a = np.stack([st.ax, st.ay, st.az], 1)
    b = np.stack([ref.ax, ref.ay, ref.az], 1)
    norm = np.linalg.norm(a - b) / np.linalg.norm(b)
    mag = np.linalg.norm(b, axis=1)
    big = mag > 0.01 * mag.max()
    per_atom = (np.linalg.norm(a - b, axis=1)[big] / mag[big]).max()
    return norm, per_atom


@pytest.mark.parametrize("precision,tol", [(clmd.PREC_MIXED, 1e-5), (clmd.PREC_FP64, 1e-12)])
def test_ensemble_forces_against_oracle(gpu, precision, tol):
    e = clmd.Ensemble(clmd.ens_config(20000, 8, precision=precision, ftcsi=50))
    slots = []
    for k, (n, rho) in enumerate([(1500, 0.05), (800, 0.02), (3000, 0.3)]):
        box, arrs = replica_inputs(n, rho, 0.75, 100 + k)
        slots.append((e.add(n, box, 0.75, *arrs), n, box))
    e.step(2)
    for slot, n, box in slots:
        st, _ = e.state(slot)
        o = oracle_forces(n, box, st)
        norm, per_atom = force_errors(st, o.get_state())
        assert norm <= tol, (n, norm)
        assert per_atom <= 10 * tol, (n, per_atom)
    res = e.results()
    assert all(r.status == 0 for r in res.values())


def test_ensemble_cluster_labels_exact(gpu):
    e = clmd.Ensemble(clmd.ens_config(10000, 4, ftcsi=20))
    n, rho = 4000, 0.3
    box, arrs = replica_inputs(n, rho, 0.7, 7)
    slot = e.add(n, box, 0.7, *arrs)
    e.step(1)
    st, _ = e.state(slot)  # positions at the next analysis step
    e.step(1)
    _, cl = e.state(slot)  # labels of that analysis
    cfg = clmd.lj_config(n, rho, 0.7)
    o = orc.Oracle(cfg, neighbor_mode=1)
    z0 = np.zeros(n)
    sc = orc.scalars_init(cfg)
    o.set_state(clmd.State(st.x, st.y, st.z, z0, z0, z0, z0, z0, z0), scalars=sc)
    o.neighbor(0)
    o.stoddard(0)
    assert np.array_equal(cl, o.clusters()["cl"])
    assert o.clusters()["cs"].max() > 2


def test_replica_same_alone_and_in_mix(gpu):
    n, rho, temp = 2000, 0.04, 0.7
    box, arrs = replica_inputs(n, rho, temp, 42)
    alone = clmd.Ensemble(clmd.ens_config(4000, 2, ftcsi=25, threads=256))
    sa = alone.add(n, box, temp, *arrs, csover=51, budget=400)
    alone.step(4)
    mix = clmd.Ensemble(clmd.ens_config(60000, 40, ftcsi=25, threads=256))
    others = []
    rng = np.random.default_rng(0)
    for k in range(20):
        m = int(rng.integers(200, 3000))
        b2, a2 = replica_inputs(m, float(rng.uniform(0.01, 0.05)), 0.75, 1000 + k)
        others.append(mix.add(m, b2, 0.75, *a2, csover=51, budget=400))
    sm = mix.add(n, box, temp, *arrs, csover=51, budget=400)
    mix.step(4)
    a, ca = alone.state(sa)
    b, cb = mix.state(sm)
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert np.array_equal(ca, cb)
    ra, rb = alone.results()[sa], mix.results()[sm]
    assert (ra.step, ra.maxcs, ra.clbrkt, ra.psi) == (rb.step, rb.maxcs, rb.clbrkt, rb.psi)


def test_admission_by_pool_and_removal(gpu):
    e = clmd.Ensemble(clmd.ens_config(5000, 8, ftcsi=10))
    box, arrs = replica_inputs(3000, 0.03, 0.7, 1)
    s1 = e.add(3000, box, 0.7, *arrs)
    box2, arrs2 = replica_inputs(2500, 0.03, 0.7, 2)
    assert e.add(2500, box2, 0.7, *arrs2) is None  # no room: 2000 atoms free
    assert e.free_atoms() == 2000
    e.step(1)
    e.remove(s1)
    assert e.free_atoms() == 5000
    s2 = e.add(2500, box2, 0.7, *arrs2)
    assert s2 is not None
    e.step(1)
    assert e.results()[s2].step == 10
