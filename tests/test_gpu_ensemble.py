"""Ensembles (batched / served replicas) on the GPU against the FP64 oracle.

Bars: mixed precision relative force error <= 1e-5 against the
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


@pytest.mark.parametrize("precision,tol,threads", [
    (clmd.PREC_MIXED, 1e-5, 0), (clmd.PREC_FP64, 1e-12, 0),
    (clmd.PREC_MIXED, 1e-5, 256 | clmd.ENS_LEAN), (clmd.PREC_MIXED, 1e-5, 512 | clmd.ENS_LEAN),
    (clmd.PREC_FP64, 1e-12, 128 | clmd.ENS_LEAN),
    (clmd.PREC_MIXED, 1e-5, 1024 | clmd.ens_lanes(2)),
    (clmd.PREC_MIXED, 1e-5, 256 | clmd.ENS_LEAN | clmd.ens_lanes(4))])
def test_ensemble_forces_against_oracle(gpu, precision, tol, threads):
    """Every block shape the autotuner may pick (the default per-class
    shapes and the register-lean ones) against the FP64 oracle."""
    e = clmd.Ensemble(clmd.ens_config(20000, 8, precision=precision, ftcsi=50,
                                      threads=threads))
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


def test_mixed_ensemble_nose_hoover_tracks_fp64(gpu):
    """The mixed ensemble (FP32 pair terms, the implicit Nose-Hoover velocity
    step solved in closed form) against the FP64 ensemble (the reference's
    Newton sweeps, int-verlet-nh-mav.f:105-147) on the same replicas over one
    50-step window: velocities and ekin within 1e-6 relative, PSI within 1e-6
    of its scale 3NkT dt steps / Q (the FP32 pair terms set these gaps)."""
    specs = [(1500, 0.05, 0.7), (800, 0.02, 0.8), (3000, 0.04, 0.75)]
    out = {}
    for prec in (clmd.PREC_MIXED, clmd.PREC_FP64):
        e = clmd.Ensemble(clmd.ens_config(20000, 8, precision=prec, ftcsi=50))
        slots = []
        for k, (n, rho, temp) in enumerate(specs):
            box, arrs = replica_inputs(n, rho, temp, 300 + k)
            slots.append(e.add(n, box, temp, *arrs))
        e.step(1)
        res = e.results()
        out[prec] = [(e.state(sl)[0], res[sl]) for sl in slots]
    for (n, rho, temp), (a, ra), (b, rb) in zip(specs, out[clmd.PREC_MIXED],
                                                out[clmd.PREC_FP64]):
        assert ra.status == 0 and rb.status == 0 and ra.step == rb.step == 50
        va = np.stack([a.vx, a.vy, a.vz])
        vb = np.stack([b.vx, b.vy, b.vz])
        dv = np.linalg.norm(va - vb) / np.linalg.norm(vb)
        scale = 3.0 * n * temp * 0.005 * 50 / (n * temp * 0.25)
        dpsi = abs(ra.psi - rb.psi) / scale
        dek = abs(ra.ekin - rb.ekin) / rb.ekin
        print(f"N={n}: dv {dv:.2e} dpsi {dpsi:.2e} dekin {dek:.2e}")
        assert dv <= 1e-6 and dpsi <= 1e-6 and dek <= 1e-6, (n, dv, dpsi, dek)


def test_unsupported_block_shape_rejected(gpu):
    """Only the compiled shapes are accepted (a kernel launched with another
    block size would index its per-warp buffers out of range)."""
    for bad in (300, 64, 1024 | clmd.ENS_LEAN, -1):
        with pytest.raises(clmd.ClmdError):
            clmd.Ensemble(clmd.ens_config(4000, 2, threads=bad))


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


def test_reordered_replica_against_oracle(gpu):
    """A replica whose positions do not fit in shared memory keeps its atoms
    in cell order (reordered at every rebuild).  Seen through the API it is
    in atom order: labels (the smallest atom number of each cluster) bit-exact
    and mixed forces within 1e-5 against the oracle on the positions it
    reports, after several windows of reordering."""
    e = clmd.Ensemble(clmd.ens_config(30000, 2, ftcsi=20))
    n, rho = 12000, 0.3
    box, arrs = replica_inputs(n, rho, 0.7, 8)
    slot = e.add(n, box, 0.7, *arrs)
    e.step(3)
    st, _ = e.state(slot)  # positions at the next analysis step
    e.step(1)
    _, cl = e.state(slot)  # labels of that analysis
    res = e.results()[slot]
    assert res.status == 0 and res.nrebuild >= 3
    cfg = clmd.lj_config(n, rho, 0.7)
    o = orc.Oracle(cfg, neighbor_mode=1)
    z0 = np.zeros(n)
    o.set_state(clmd.State(st.x, st.y, st.z, z0, z0, z0, z0, z0, z0),
                scalars=orc.scalars_init(cfg))
    o.neighbor(0)
    o.stoddard(0)
    assert np.array_equal(cl, o.clusters()["cl"])
    assert o.clusters()["cs"].max() > 2
    norm, per_atom = force_errors(st, oracle_forces(n, box, st).get_state())
    assert norm <= 1e-5 and per_atom <= 1e-4, (norm, per_atom)


@pytest.mark.parametrize("n", [2000, 11000])  # 11000: reordered slots
def test_replica_same_alone_and_in_mix(gpu, n):
    rho, temp = 0.04, 0.7
    box, arrs = replica_inputs(n, rho, temp, 42)
    alone = clmd.Ensemble(clmd.ens_config(n + 2000, 2, ftcsi=25, threads=256))
    sa = alone.add(n, box, temp, *arrs, csover=51, budget=400)
    alone.step(4)
    mix = clmd.Ensemble(clmd.ens_config(60000 + n, 40, ftcsi=25, threads=256))
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


def served_requests():
    """A small trace: staggered arrivals, sizes across the size classes,
    budgets that are and are not multiples of the window, low thresholds so
    that some replicas nucleate."""
    rng = np.random.default_rng(3)
    reqs = []
    for k in range(14):
        r = clmd.Request()
        r.arrival = 0.002 * k
        r.natom = int(np.exp(rng.uniform(np.log(150), np.log(7000))))
        r.rho = float(rng.uniform(0.02, 0.05))
        r.temp = float(rng.uniform(0.65, 0.75))
        r.budget = int(rng.choice([300, 450, 800]))
        r.csover = int(rng.choice([4, 6, 101]))
        r.seed = 500 + k
        reqs.append(r)
    return reqs


def test_served_trace_completes_with_pool_admission(gpu):
    reqs = served_requests()
    total = sum(r.natom for r in reqs)
    biggest = max(r.natom for r in reqs)
    # a pool smaller than the trace: later requests wait for retirements
    e = clmd.Ensemble(clmd.ens_config(max(biggest, total // 3), 64, ftcsi=50, threads=256))
    out, st = e.serve(reqs, 300.0)
    assert st.admitted == len(reqs) and st.completed == len(reqs)
    assert st.peak_atoms <= max(biggest, total // 3)
    assert e.free_atoms() == max(biggest, total // 3)  # everything retired
    for r, o in zip(reqs, out):
        assert o.done in (1, 2)
        assert o.admitted >= o.arrival and o.finished >= o.admitted
        if o.done == 2:
            assert o.steps == r.budget
        else:
            assert o.clbrkt <= o.steps <= r.budget
    assert any(o.done == 1 for o in out) and any(o.done == 2 for o in out)
    assert st.atom_steps == sum(o.natom * o.steps for o in out)


def test_served_replica_same_alone_and_in_trace(gpu):
    """Continuous batching changes nothing about a request's trajectory: the
    served trace and each request served alone agree on steps, outcome and
    the step the threshold cluster was first seen."""
    reqs = served_requests()
    e = clmd.Ensemble(clmd.ens_config(sum(r.natom for r in reqs), 64, ftcsi=50, threads=256))
    mix, _ = e.serve(reqs, 300.0)
    for k in (0, 5, 9, 13):
        a = clmd.Ensemble(clmd.ens_config(reqs[k].natom, 1, ftcsi=50, threads=256))
        r = clmd.Request()
        C_ = type(r)
        for f, _t in C_._fields_:
            setattr(r, f, getattr(reqs[k], f))
        r.arrival = 0.0
        alone, _ = a.serve([r], 300.0)
        assert (alone[0].steps, alone[0].done, alone[0].clbrkt) == \
            (mix[k].steps, mix[k].done, mix[k].clbrkt), k
        a.close()


def test_balanced_step_same_trajectories(gpu):
    """clmd_ens_step_timed only changes how many steps a launch covers (its
    boundaries fall inside windows): run to the same budget, every replica
    ends bit-identical to plain steps."""
    rng = np.random.default_rng(9)
    specs = [(int(n), float(rng.uniform(0.02, 0.05)), 0.7, 70 + k)
             for k, n in enumerate([150, 400, 900, 2200, 5000])]

    def build():
        e = clmd.Ensemble(clmd.ens_config(10000, 8, ftcsi=20, threads=256))
        slots = []
        for n, rho, temp, sd in specs:
            box, arrs = replica_inputs(n, rho, temp, sd)
            slots.append(e.add(n, box, temp, *arrs, csover=10**6, budget=600))
        return e, slots

    a, sa = build()
    while any(r.done == 0 for r in a.results().values()):
        a.step(1)
    b, sb = build()
    launches, small_done = 0, None
    while any(r.done == 0 for r in b.results().values()):
        b.step_timed(0.5)
        launches += 1
        if small_done is None and b.results()[sb[0]].done:
            small_done = launches
    # every replica ran about 0.5 ms per launch: the smallest finished its
    # 600 steps in far fewer launches than the largest
    assert small_done < launches / 2
    for p, q in zip(sa, sb):
        ra, rb = a.results()[p], b.results()[q]
        assert (ra.step, ra.done, ra.psi) == (rb.step, rb.done, rb.psi)
        xa, ca = a.state(p)
        xb, cb = b.state(q)
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(getattr(xa, k), getattr(xb, k)), k
        assert np.array_equal(ca, cb)


@pytest.mark.parametrize("precision", [clmd.PREC_MIXED, clmd.PREC_FP64])
def test_nose_hoover_solve_converges_over_long_runs(gpu, precision):
    """1.5e9 atom-steps of Nose-Hoover without CLMD_ERR_NH_NOCONVERGE.  FP64:
    the reference's per-component relative test (int-verlet-nh-mav.f:140-147)
    passes because its sweep reaches an exact fixed point; a sweep evaluated
    with fused multiply-adds does not, and failed here about once per 4e8
    atom-steps.  Mixed: the closed-form root's Newton steps must settle above
    the rounding noise of f(p) (a limit at 1e-16 of the scale stalled on 3 of
    these 128 replicas)."""
    rng = np.random.default_rng(12)
    e = clmd.Ensemble(clmd.ens_config(128 * 4000, 128, ftcsi=100, threads=256,
                                      precision=precision))
    for k in range(128):
        rho, temp = float(rng.uniform(0.03, 0.05)), float(rng.uniform(0.65, 0.85))
        box, arrs = replica_inputs(4000, rho, temp, 9000 + k)
        e.add(4000, box, temp, *arrs, csover=10**6, budget=3000)
    while any(r.done == 0 and r.status == 0 for r in e.results().values()):
        e.step(5)
    res = e.results().values()
    assert all(r.status == 0 for r in res), [r.status for r in res if r.status]
    assert all(r.step == 3000 for r in res)


def test_bulk_upload_download_in_slot_order(gpu):
    """clmd_ens_upload/download move every occupied slot's x..vz in slot
    order, whether the slots' pool ranges abut or not (a removal and a
    re-admission leave them out of order)."""
    import ctypes as C
    e = clmd.Ensemble(clmd.ens_config(40000, 8, ftcsi=10, threads=256))
    sizes = [1200, 700, 12000, 900]  # 12000: positions beyond shared memory, slots reordered
    slots = []
    for k, n in enumerate(sizes):
        box, arrs = replica_inputs(n, 0.03, 0.7, 300 + k)
        slots.append(e.add(n, box, 0.7, *arrs))
    e.remove(slots[1])
    box, arrs = replica_inputs(500, 0.03, 0.7, 399)
    slots[1] = e.add(500, box, 0.7, *arrs)  # reuses slot 1 inside the freed range
    e.step(1)
    occ = sorted(slots)
    total = sum(e.natom[s] for s in occ)
    bufs = [np.zeros(total) for _ in range(6)]
    ptrs = [b.ctypes.data_as(C.POINTER(C.c_double)) for b in bufs]
    assert e.lib.clmd_ens_download(e.h, *ptrs) == 0
    h = 0
    for s in occ:
        st, _ = e.state(s)
        n = e.natom[s]
        for k, name in enumerate(("x", "y", "z", "vx", "vy", "vz")):
            assert np.array_equal(bufs[k][h:h + n], getattr(st, name)), (s, name)
        h += n
    for b in bufs:
        b *= 1.0 + 1e-9
    assert e.lib.clmd_ens_upload(e.h, *ptrs) == 0
    h = 0
    for s in occ:
        st, _ = e.state(s)
        n = e.natom[s]
        assert np.array_equal(bufs[0][h:h + n], st.x)
        assert np.array_equal(bufs[5][h:h + n], st.vz)
        h += n


def test_mean_first_passage_matches_per_replica_tables(gpu):
    """clmd_ens_mfpt (helpers/passage-time.f + mpt.f on the device) against
    the same statistics computed here from every replica's first-passage
    table (clmd_ens_fpt)."""
    rng = np.random.default_rng(21)
    e = clmd.Ensemble(clmd.ens_config(60 * 1500, 64, ftcsi=25, threads=256))
    slots = []
    for k in range(60):
        n = int(rng.integers(300, 1500))
        box, arrs = replica_inputs(n, float(rng.uniform(0.03, 0.05)), 0.65, 700 + k)
        slots.append(e.add(n, box, 0.65, *arrs, csover=10**6, budget=400))
    e.remove(slots[7])  # a freed slot does not count
    del slots[7]
    e.step(20)
    cap = 64
    mean, sem, cnt = e.mfpt(cap)
    tab = np.array([e.fpt(s, cap) for s in sorted(slots)], dtype=np.int64)
    for j in range(cap):
        t = tab[:, j][tab[:, j] >= 0].astype(np.float64)
        assert cnt[j] == len(t)
        if len(t) == 0:
            assert mean[j] == -1.0
            continue
        m = t.sum() / len(t)
        assert mean[j] == m
        np.testing.assert_allclose(sem[j], np.sqrt(max((t * t).sum() / len(t) - m * m, 0.0)
                                                   / len(t)), rtol=1e-12, atol=1e-9)
    assert cnt[0] == len(slots) and cnt[4] > 0  # every replica has monomers; some dimers+


def test_first_passage_follows_reference_helpers(gpu):
    """Each replica's first-passage table is helpers/passage-time.f:55-75
    (the oracle's restatement) applied to that replica's record of
    (analysis step, largest cluster size), polled window by window; pooled
    over the replicas, clmd_ens_mfpt is helpers/mpt.f:73-110 with the
    reference's ts/500000 scaling (nanoseconds at a 2 fs step), the same
    counts and standard errors."""
    rng = np.random.default_rng(33)
    win = 25
    e = clmd.Ensemble(clmd.ens_config(40 * 1500, 40, ftcsi=win, threads=256))
    slots = []
    for k in range(40):
        n = int(rng.integers(300, 1500))
        box, arrs = replica_inputs(n, float(rng.uniform(0.03, 0.05)), 0.65, 900 + k)
        slots.append(e.add(n, box, 0.65, *arrs, csover=10**6, budget=0))
    rec = {s: ([], []) for s in slots}
    for w in range(1, 25):
        e.step(1)
        res = e.results()
        for s in slots:
            assert res[s].step == win * w and res[s].status == 0
            rec[s][0].append(win * (w - 1))  # the analysis opens each window
            rec[s][1].append(res[s].maxcs)
    cap = 128
    pool_ts, pool_cs = [], []
    for s in slots:
        pt, _ = orc.passage_time(rec[s][0], rec[s][1], 1, cap)
        assert np.array_equal(e.fpt(s, cap), pt[1:]), s
        for j in range(1, cap + 1):
            if pt[j] >= 0:
                pool_ts.append(pt[j])
                pool_cs.append(j)
    m, sd, cnt = orc.mpt(pool_ts, pool_cs, 1, cap)
    mean, sem, ecnt = e.mfpt(cap)
    assert np.array_equal(ecnt, cnt)
    for j in range(cap):
        if cnt[j] == 0:
            assert mean[j] == -1.0
            continue
        np.testing.assert_allclose(mean[j] / 500000, m[j], rtol=1e-12)
        if np.isnan(sd[j]):  # all passages at one step: mpt.f's sqrt of a rounding residue
            assert sem[j] <= 1e-6 * mean[j]
        else:
            assert abs(sem[j] / 500000 - sd[j]) <= 1e-12 * m[j] + 1e-9 * sd[j]
    assert cnt[0] == len(slots) and cnt[3] > 0


def test_graph_replay_same_as_direct_launches(gpu, monkeypatch):
    """The window sequence replayed from a CUDA graph (default) and issued
    launch by launch (CLMD_ENS_GRAPHS=0) give bit-identical replicas, also
    across a membership change (a replica finishing).  (Balanced steps are
    left out: how many steps they run depends on measured times.)"""
    rng = np.random.default_rng(5)
    specs = [(int(rng.integers(200, 6000)), float(rng.uniform(0.02, 0.05)), 600 + k)
             for k in range(24)]

    def run():
        e = clmd.Ensemble(clmd.ens_config(sum(n for n, _, _ in specs), 32, ftcsi=20,
                                          threads=256))
        slots = []
        for k, (n, rho, sd) in enumerate(specs):
            box, arrs = replica_inputs(n, rho, 0.7, sd)
            slots.append(e.add(n, box, 0.7, *arrs, csover=10**6, budget=60 if k == 3 else 400))
        for _ in range(4):
            e.step(1)  # replica 3 finishes after 3 windows: the launch set changes
        e.step(3)
        ms, _ = e.last_ms()
        assert max(ms) > 0
        return e, slots

    monkeypatch.setenv("CLMD_ENS_GRAPHS", "0")
    a, sa = run()
    monkeypatch.delenv("CLMD_ENS_GRAPHS")
    b, sb = run()
    for p, q in zip(sa, sb):
        ra, rb = a.results()[p], b.results()[q]
        assert (ra.step, ra.done, ra.psi, ra.ekin) == (rb.step, rb.done, rb.psi, rb.ekin)
        xa, _ = a.state(p)
        xb, _ = b.state(q)
        for k in ("x", "vx", "az"):
            assert np.array_equal(getattr(xa, k), getattr(xb, k)), k
    assert a.results()[sa[3]].done == 2


def test_failed_replica_is_isolated(gpu):
    """A replica that fails (two atoms started 0.3 sigma apart: the skin is
    exceeded in the first steps, neighbor-pbc-mav.f:48-51) stops with its own
    status; the replicas beside it run on bit-identically to a batch without
    it, and the batch keeps stepping."""
    good = [(1500, 0.03, 81), (900, 0.04, 82), (3000, 0.02, 83)]

    def build(with_bad):
        e = clmd.Ensemble(clmd.ens_config(8000, 8, ftcsi=20, threads=256))
        slots = []
        for n, rho, sd in good:
            box, arrs = replica_inputs(n, rho, 0.7, sd)
            slots.append(e.add(n, box, 0.7, *arrs, csover=10**6, budget=400))
        bad = None
        if with_bad:
            box, arrs = replica_inputs(1000, 0.03, 0.7, 84)
            x, y, z = arrs[0].copy(), arrs[1].copy(), arrs[2].copy()
            x[1], y[1], z[1] = x[0] + 0.3, y[0], z[0]
            bad = e.add(1000, box, 0.7, x, y, z, *arrs[3:], csover=10**6, budget=400)
        return e, slots, bad

    a, sa, bad = build(True)
    b, sb, _ = build(False)
    for e in (a, b):
        for _ in range(20):
            e.step(1)
    ra = a.results()
    assert ra[bad].status != 0 and ra[bad].step < 400
    for p, q in zip(sa, sb):
        x, y = ra[p], b.results()[q]
        assert x.status == 0 and (x.step, x.done, x.psi) == (y.step, y.done, y.psi)
        xa, _ = a.state(p)
        xb, _ = b.state(q)
        assert np.array_equal(xa.x, xb.x) and np.array_equal(xa.vz, xb.vz)


CLUSTER_SIZES = [(12000, 0.03), (26000, 0.02), (52000, 0.04)]  # 2, 8 and 16 CTAs


@pytest.mark.parametrize("precision,tol", [(clmd.PREC_MIXED, 1e-5), (clmd.PREC_FP64, 1e-12)])
def test_cluster_replicas_against_oracle(gpu, precision, tol):
    """Replicas too large for one SM's shared memory run on thread-block
    clusters (2-16 CTAs, positions in global memory, cluster barriers and
    distributed-shared-memory reductions).  After two windows with list
    rebuilds and analyses: forces on the engine's positions against the FP64
    oracle (1e-5 mixed, 1e-12 FP64) and the Stillinger labels bit-exact."""
    e = clmd.Ensemble(clmd.ens_config(sum(n for n, _ in CLUSTER_SIZES) + 1000, 4,
                                      precision=precision, ftcsi=25))
    slots = []
    for k, (n, rho) in enumerate(CLUSTER_SIZES):
        box, arrs = replica_inputs(n, rho, 0.7, 300 + k)
        slots.append((e.add(n, box, 0.7, *arrs, csover=10**6), n, box))
    e.step(2)
    res = e.results()
    states = {}
    for s, n, box in slots:
        r = res[s]
        assert r.status == 0 and r.step == 50 and r.nrebuild >= 3, (n, r.status, r.step)
        st, _ = e.state(s)  # positions at the next analysis step
        states[s] = st
        norm, per_atom = force_errors(st, oracle_forces(n, box, st).get_state())
        assert norm <= tol and per_atom <= 10 * tol, (n, norm, per_atom)
    e.step(1)  # opens with the analysis of those positions
    for s, n, box in slots:
        st = states[s]
        _, cl = e.state(s)
        cfg = clmd.lj_config(n, n / box ** 3, 0.7)
        o = orc.Oracle(cfg, neighbor_mode=1, label_mode=1)
        z0 = np.zeros(n)
        o.set_state(clmd.State(st.x, st.y, st.z, z0, z0, z0, z0, z0, z0),
                    scalars=orc.scalars_init(cfg))
        o.neighbor(0)
        o.stoddard(0)
        assert np.array_equal(cl, o.clusters()["cl"]), n
        assert e.results()[s].step == 75


def test_cluster_replica_matches_single_cta_and_mix(gpu, monkeypatch):
    """The same large replica on a cluster, alone and beside small replicas
    (bit-identical: its cluster size depends on its own size only), and on
    one CTA (CLMD_ENS_CLUSTERS=0: the same steps, sums in another order,
    so agreeing to rounding over one window)."""
    n, rho, temp = 20000, 0.03, 0.7
    box, arrs = replica_inputs(n, rho, temp, 77)

    def run(extra, clusters=True):
        if not clusters:
            monkeypatch.setenv("CLMD_ENS_CLUSTERS", "0")
        e = clmd.Ensemble(clmd.ens_config(n + 30000, 24, ftcsi=25))
        monkeypatch.delenv("CLMD_ENS_CLUSTERS", raising=False)
        rng = np.random.default_rng(4)
        for k in range(extra):
            m = int(rng.integers(300, 2500))
            b2, a2 = replica_inputs(m, 0.04, 0.75, 2000 + k)
            e.add(m, b2, 0.75, *a2, csover=51)
        s = e.add(n, box, temp, *arrs, csover=10**6)
        e.step(2)
        st, cl = e.state(s)
        r = e.results()[s]
        e.close()
        return st, cl, r

    a, ca, ra = run(0)
    b, cb, rb = run(12)
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert np.array_equal(ca, cb) and ra.psi == rb.psi and ra.step == rb.step == 50
    c, cc, rc = run(0, clusters=False)
    assert rc.step == 50 and rc.nrebuild == ra.nrebuild
    for k in ("x", "y", "z"):
        np.testing.assert_allclose(getattr(c, k), getattr(a, k), rtol=0, atol=1e-9 * box)
    np.testing.assert_allclose(c.vx, a.vx, rtol=0, atol=1e-8)
    assert abs(rc.psi - ra.psi) <= 1e-9 * abs(ra.psi) + 1e-14


def test_step_io_matches_upload_step_download(gpu):
    """clmd_ens_step_io (the window kernel reads each replica's x..vz from
    pinned host memory when it takes the replica and writes them back when
    it leaves it) against clmd_ens_upload + clmd_ens_step + clmd_ens_download:
    the same host arrays bit for bit, with a cluster-size replica among small
    ones, a replica finished earlier (its part is not touched) and the host
    arrays changed between calls (the kernel reads them)."""
    import ctypes as C
    import torch

    sizes = [400, 1800, 3500, 700, 12000, 2500]

    def make():
        e = clmd.Ensemble(clmd.ens_config(sum(sizes) + 5000, 16, ftcsi=25))
        slots = []
        for k, n in enumerate(sizes):
            box, arrs = replica_inputs(n, 0.03, 0.75, 300 + k)
            slots.append(e.add(n, box, 0.75, *arrs, csover=10**6,
                               budget=25 if k == 3 else 0))
        e.step(2)  # replica 3 spends its budget: finished
        return e, slots

    total = sum(sizes)
    bufs = []
    for _ in range(2):
        bufs.append([torch.empty(total, dtype=torch.float64).pin_memory() for _ in range(6)])
    ptr = [[C.cast(t.data_ptr(), C.POINTER(C.c_double)) for t in b] for b in bufs]
    e1, s1 = make()
    e2, s2 = make()
    assert e1.results()[s1[3]].done == 2
    for e, p in ((e1, ptr[0]), (e2, ptr[1])):
        assert e.lib.clmd_ens_download(e.h, *p) == 0
    for a, b in zip(*bufs):
        assert torch.equal(a, b)
    # the host copies are what the kernel starts from: change them alike
    for b in bufs:
        b[3][100:200] *= 1.01
        b[0][sizes[0] + 17] += 0.05
    for t in bufs[1]:
        t[sum(sizes[:3]):sum(sizes[:4])] = -1.0  # the finished replica's part
    for _ in range(2):
        assert e1.lib.clmd_ens_upload(e1.h, *ptr[0]) == 0
        e1.step(2)
        assert e1.lib.clmd_ens_download(e1.h, *ptr[0]) == 0
        e2.step_io(2, ptr[1])
    lo, hi = sum(sizes[:3]), sum(sizes[:4])
    for a, b in zip(*bufs):
        assert torch.equal(a[:lo], b[:lo]) and torch.equal(a[hi:], b[hi:])
        assert torch.all(b[lo:hi] == -1.0)
    r1, r2 = e1.results(), e2.results()
    for k in range(len(sizes)):
        assert r1[s1[k]].step == r2[s2[k]].step and r1[s1[k]].psi == r2[s2[k]].psi
        st1, cl1 = e1.state(s1[k])
        st2, cl2 = e2.state(s2[k])
        for name in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(getattr(st1, name), getattr(st2, name)), (k, name)
        assert np.array_equal(cl1, cl2)
    # memory the device cannot address is refused
    plain = [np.zeros(total) for _ in range(6)]
    with pytest.raises(clmd.ClmdError):
        e2.step_io(1, [a.ctypes.data_as(C.POINTER(C.c_double)) for a in plain])
    e1.close()
    e2.close()
