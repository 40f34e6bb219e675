"""Benchmark of the LJ MD step + nucleation analysis on B200.

Default workload (--workload batched): the batched nucleation ensemble the
headline metric is quoted on -- 4096 independent replicas per GPU, N
log-uniform in [200, 8000] (8.65 M atoms), rho* uniform in [0.01, 0.05],
T* uniform in [0.65, 0.85], reduced LJ (rc 2.5, initial list radius 2.8,
adaptive skin, nbtim 10), Nose-Hoover dt* = 0.005 (Q = N T* 0.25), Stillinger
clustering every 100 steps, each replica stopping when its largest cluster
exceeds 50 atoms (chk_nucleation, csover = 51) or after 2e5 steps; mixed
precision (FP32 pair terms, Kahan FP32 sums, FP64 positions, velocities,
PSI and energies).  Seeded synthetic starts (pairs >= 0.9 sigma apart,
Maxwell-Boltzmann velocities, stopdead on the device).

A bench step is one window: every running replica advances 100 steps
(analysis + chk_nucleation first).  metric = atom-steps/s.

  value   device-resident windows, whole-job atom-steps / max-over-ranks time.
  e2e     per window every running replica's x, v go host->device from pinned
          memory and back through the C ABI (clmd_ens_step_io: the window
          kernel reads a replica's state from the host arrays when it takes
          the replica and writes it back when it leaves it, so transfers
          overlap the other replicas' compute; + a 16-byte status per
          replica).  separate_copies: the same with clmd_ens_upload, step,
          clmd_ens_download one after the other.
  roofline  the window kernels (k_ens, 4 size classes concurrently), CUDA
          events inside the library; 120 algorithmic bytes per atom-step
          (x, v FP64 and a FP32, read + written) against measured HBM.
  fp64_ensemble_same_ensemble  the same replicas as an all-FP64 ensemble
          (same kernels, FP64 pair terms and sums).
  fp64_dropin_same_ensemble  the FP64 drop-in (one system at a time, the
          plain engine) timed on replicas at the size quantiles, summed over
          the whole ensemble: the "vs FP64" of the metric.
  mixed_vs_fp64_sample  64 replicas run mixed, FP64 and as an FP64 twin
          (1e-13 apart) for 1e4 steps: per-replica energy drift, mixed - FP64
          against the twin's spread, the drift of the energy the truncated
          force conserves, the cluster-size distribution.
  served  the served workload on the same GPU: a bounded Poisson window at 200
          requests/s served with continuous batching; p50/p99 request
          latency (censored requests at their lower bound), time to
          nucleation (wall and step), aggregate atom-steps/s.  Under
          "drained": a 1 s window of the same arrivals served until every
          request finished (90 s cap), so its percentiles are uncensored
          when everything finished.
  cpu_baseline  the serial C restatement of the reference (the oracle) on
          one pinned core, on 16 replicas at the midpoints of 16 size strata,
          3 timed 100-step windows: the rate of exactly that timed work.

--workload dropin: one FP64 system of N = 262,144 atoms (rho* = 0.02, T* =
0.7, velocity Verlet, Stillinger every 100 steps), a bench step = one
analysis cycle of 100 steps.

--workload nvt: one mixed-precision system of N = 2,097,152 atoms (rho* =
0.05, T* = 0.75, Nose-Hoover with Q = N T* 0.25, FP32 pair terms with Kahan
FP32 sums, FP64 positions, velocities, PSI and energies), ten Wolde-Frenkel
clustering (>= 5 neighbours within 1.5 sigma) every 50 steps; a bench step =
one analysis cycle of 50 steps.

--impl reference runs the serial C restatement of the reference (the
reference is Fortran 77 and no Fortran compiler exists on either machine),
rank 0 only, on one pinned core: for the batched workload each bench step
is one 100-step window of the 16-replica stratified sample (inputs from the
oracle's own copy of the start generator: the engine library is never
loaded), plus an all-core figure under an extra key.

Multi-GPU: independent replicas per rank (seeds offset by rank); the path has
no data exchange; value = all ranks' atom-steps / max-over-ranks time.
"""
import argparse
import ctypes as C
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "fortran-cluster-md_b200")
ORACLE = os.path.join(REPO, "oracle")
sys.path.insert(0, PKG)

import clmd  # noqa: E402

WORKLOAD = dict(name="lj-fp64-dropin", natom=262144, rho=0.02, temp=0.7, rc=2.5, rskin=2.8,
                atskin=1.5, dt=0.005, nbtim=10, ftcsi=100, seed=1234,
                integrator=clmd.INT_VERLET, ethst="-", clustering=clmd.CLU_STILLINGER,
                precision=clmd.PREC_FP64)
# mixed-precision NVT: Nose-Hoover (Q = N T* 0.25), ten Wolde-Frenkel every 50
NVT = dict(WORKLOAD, name="lj-mixed-nvt", natom=2097152, rho=0.05, temp=0.75, ftcsi=50,
           seed=4321, integrator=clmd.INT_NOSE, ethst="N", clustering=clmd.CLU_FRENKEL,
           precision=clmd.PREC_MIXED)
BYTES_PER_ATOM_STEP = 144  # FP64: x, v, a read + written


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_config(w):
    return clmd.lj_config(w["natom"], w["rho"], w["temp"], rc=w["rc"], rskin=w["rskin"],
                          atskin=w["atskin"], dt=w["dt"], nbtim=w["nbtim"], ftcsi=w["ftcsi"],
                          integrator=w["integrator"], ethst=w["ethst"],
                          clustering=w["clustering"], precision=w["precision"], atnenum=5)


def make_state(cfg, seed, temp):
    n = cfg.natom
    x, y, z, vx, vy, vz = clmd.init_random(n, (cfg.boxx, cfg.boxy, cfg.boxz), 0.9, temp, seed)
    return clmd.State(x, y, z, vx, vy, vz, np.zeros(n), np.zeros(n), np.zeros(n))


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(name="k_cycle_fp64_dropin"):
    """DRAM bytes per launch of a kernel from its committed ncu summary."""
    p = os.path.join(REPO, "profiles", name + ".md")
    if not os.path.exists(p):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, dev):
        self.dev = dev
        self.proc = None
        self.path = f"/tmp/clmd_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [t.strip() for t in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for k, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(k)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (serial C restatement of the reference)
# ---------------------------------------------------------------------------
def cpu_cycle_estimate(w, budget_s=15.0):
    """Seconds the serial reference algorithm needs for one analysis cycle
    (100 steps + 1 Stillinger analysis) at the full workload, from a bounded
    sample run on one core:
      - t_step: oracle integrator steps at full N (force + integration; the
        list kept by the oracle's cell variant so that no O(N^2) rebuild
        falls inside the sample),
      - t_rebuild: the reference's all-pairs rebuild (neighbor-pbc-mav.f
        :73-99) timed on a sample of rows at full N, scaled by the pair count,
      - t_label: the Stillinger routine (O(N^2) rescan) timed at N/8 and
        scaled by N^2.
    Returns (seconds per cycle of ftcsi steps, description)."""
    sys.path.insert(0, ORACLE)
    import orc

    n = w["natom"]
    cfg = make_config(w)
    st = make_state(cfg, w["seed"], w["temp"])
    o = orc.Oracle(cfg, neighbor_mode=1)
    o.set_state(st, scalars=orc.scalars_init(cfg))
    o.stopdead(-1)
    o.neighbor(0)
    o.zero_acc()
    o.accatom()
    # steps without a rebuild
    t_steps, nstep = 0.0, 0
    i = 1
    while nstep < 5 and i < 50:
        r0 = o.scalars().nrebuild
        t = time.perf_counter()
        o.integrator(i)
        dt = time.perf_counter() - t
        if o.scalars().nrebuild == r0:
            t_steps += dt
            nstep += 1
        i += 1
    t_step = t_steps / max(nstep, 1)
    # all-pairs rebuild on a row sample
    rows = max(200, min(4000, int(budget_s * 0.4 / (n * 4.8e-9))))
    t = time.perf_counter()
    pairs = o.neighbor_rows_sample(0, rows)
    t_pairs = time.perf_counter() - t
    t_rebuild = t_pairs / pairs * (n * (n - 1) / 2)
    o.close()
    # labelling on a sample of at most 32768 atoms, scaled by N^2
    div = max(8, n // 32768)
    ws = dict(w, natom=n // div)
    cfs = make_config(ws)
    sts = make_state(cfs, w["seed"], w["temp"])
    o = orc.Oracle(cfs, neighbor_mode=1)
    o.set_state(sts, scalars=orc.scalars_init(cfs))
    o.neighbor(0)
    t = time.perf_counter()
    o.stoddard(0)
    t_label = (time.perf_counter() - t) * float(div * div)
    o.close()
    cyc = w["ftcsi"]
    rebuilds = cyc / w["nbtim"]
    cycle = cyc * t_step + rebuilds * t_rebuild + t_label
    desc = (f"serial oracle, 1 core: {nstep} MD steps at N={n} ({t_step*1e3:.1f} ms/step), "
            f"all-pairs rebuild on {rows} rows ({pairs} pair tests) scaled to N(N-1)/2 "
            f"({t_rebuild:.1f} s/rebuild, {rebuilds:.0f} per {cyc} steps), cluster labelling "
            f"at N/{div} scaled by {div * div} ({t_label:.1f} s/analysis)")
    return cycle, desc


def reference_arm(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = w["natom"]
    units = []
    desc = ""
    # each step is a bounded sample; the whole run stays within ~2-3 minutes
    budget = min(10.0, max(1.5, 120.0 / max(1, args.warmup + args.steps)))
    for k in range(args.warmup + args.steps):
        cyc, desc = cpu_cycle_estimate(w, budget_s=budget)
        if k >= args.warmup:
            units.append(cyc)
    per_cycle = statistics.mean(units)
    value = n * w["ftcsi"] / per_cycle
    line = {
        "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_cycle * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": w_dtype(w), "data": "synthetic (seeded)",
        "config": config_json(w, args.gpus),
        "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": 1, "kind": "port",
                         "sample": desc},
        "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def w_dtype(w):
    return "f32+f64" if w["precision"] == clmd.PREC_MIXED else "f64"


def config_json(w, ngpu):
    nh = w["integrator"] == clmd.INT_NOSE
    return {"workload": f"{w['name']}-N{w['natom']}-rho{w['rho']}-T{w['temp']}",
            "natom": w["natom"], "rho": w["rho"], "T": w["temp"], "rc": w["rc"],
            "rskin0": w["rskin"], "dt": w["dt"],
            "integrator": "nose-hoover (Q = N T* 0.25)" if nh else "velocity-verlet",
            "precision": "mixed (FP32 pair terms, Kahan FP32 sums)"
                         if w["precision"] == clmd.PREC_MIXED else "fp64",
            "clustering": ("ten-wolde-frenkel (>= 5 neighbours within 1.5 sigma)"
                           if w["clustering"] == clmd.CLU_FRENKEL else "stillinger-1.5sigma")
                          + f" every {w['ftcsi']}",
            "steps_per_bench_step": w["ftcsi"],
            "l2": "flushed between timed steps (256 MB write)",
            "parallelism": f"replicas x{ngpu}"}


# ---------------------------------------------------------------------------
# engine arm
# ---------------------------------------------------------------------------
def start_system(cfg, state):
    """main.f's start with the writers off: commons from the config
    (read-3d.f:263-276), stopdead(-1), neighbor(0), a = 0, AccAtom, the
    Nose-Hoover PSI start (main.f:156-160), stoddard(-1)."""
    g = clmd.System(cfg)
    g.set_state(state, scalars=clmd.scalars_init(cfg))
    g.stopdead(-1)
    g.neighbor(0)
    g.zero_acc()
    g.accatom()
    if cfg.integrator == clmd.INT_NOSE:
        s = g.scalars()
        s.psi = (2.0 * s.ekin - 3.0 * cfg.natom * clmd.CIKB * cfg.att) / cfg.Q
        g.set_scalars(s)
    g.stoddard(-1)
    return g


def pinned(n, torch):
    return torch.empty(n, dtype=torch.float64).pin_memory()


class Ranks:
    """One process per GPU, launched by torchrun (RANK / WORLD_SIZE /
    LOCAL_RANK / MASTER_* from the environment).  The path has no exchange:
    ranks run independent replicas (seed + 1000 * rank) and meet only for the
    timing barrier and the max / sum of their numbers.  backend "nccl" on
    GPUs; "gloo" runs the same logic on CPU processes."""

    def __init__(self, backend="nccl", timeout_s=300):
        import torch
        self.torch = torch
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = self.world > 1
        self.cuda = backend == "nccl"
        if self.cuda:
            torch.cuda.set_device(self.local if self.dist else 0)
        if self.dist:
            import datetime
            torch.distributed.init_process_group(
                backend, timeout=datetime.timedelta(seconds=timeout_s))

    @property
    def device(self):
        return self.local if self.dist else 0

    def barrier(self):
        if self.dist:
            self.torch.distributed.barrier()
        if self.cuda:
            self.torch.cuda.synchronize()

    def _reduce(self, x, op):
        if not self.dist:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64,
                              device="cuda" if self.cuda else "cpu")
        self.torch.distributed.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        return self._reduce(x, self.torch.distributed.ReduceOp.MAX if self.dist else None)

    def sum(self, x):
        return self._reduce(x, self.torch.distributed.ReduceOp.SUM if self.dist else None)

    def close(self):
        if self.dist:
            self.torch.distributed.barrier()
            self.torch.distributed.destroy_process_group()


def engine_arm(args, w):
    import torch

    rk = Ranks(timeout_s=180)
    rank, world, dist, dev = rk.rank, rk.world, rk.dist, rk.device
    clmd.set_device(dev)
    barrier, max_over_ranks, sum_over_ranks = rk.barrier, rk.max, rk.sum

    n = w["natom"]
    cyc = w["ftcsi"]
    cfg = make_config(w)
    state = make_state(cfg, w["seed"] + rank, w["temp"])
    g = start_system(cfg, state)
    stream = torch.cuda.ExternalStream(g.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")

    step = 0
    for _ in range(args.warmup):
        g.run(step, cyc)
        step += cyc
    # ---- value: device-resident cycles
    clocks = Clocks(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    l0 = g.kernel_launches()
    s0 = g.scalars()
    barrier()
    clocks.start()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        evs[k][0].record(stream)
        g.run(step, cyc)
        evs[k][1].record(stream)
        step += cyc
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    launches = g.kernel_launches() - l0
    s1 = g.scalars()
    rebuilds = s1.nrebuild - s0.nrebuild
    # fixed kernels per cycle + the host-side calls of run()
    ms_max = max_over_ranks(ms)
    units = sum_over_ranks(float(n) * cyc * args.steps)
    value = units / (ms_max / 1e3)

    # ---- roofline: the step kernel alone (100 steps per launch)
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(3)]
    for a, b in kev:
        with torch.cuda.stream(stream):
            flush.zero_()
        a.record(stream)
        g.steps(step, cyc)
        b.record(stream)
        step += cyc
    torch.cuda.synchronize()
    kms = statistics.mean(x.elapsed_time(y) for x, y in kev)
    peak, peak_kind = measured_peaks()
    # mixed Nose-Hoover keeps the accelerations FP32 between its passes
    per_atom = BYTES_PER_ATOM_STEP_MIXED if w.get("precision") == clmd.PREC_MIXED \
        else BYTES_PER_ATOM_STEP
    alg = per_atom * n * cyc
    achieved = alg / (kms / 1e3) / 1e9
    # the committed captures are of the default sizes; DRAM traffic grows
    # with the atoms (both states exceed L2)
    base = WORKLOAD if w["name"] == WORKLOAD["name"] else NVT
    traffic = profiled_traffic("k_cycle_fp64_dropin" if base is WORKLOAD else "k_cycle_mixed_nvt")
    if traffic is not None:
        traffic *= n / base["natom"]

    # ---- e2e: host buffers through the C ABI
    st_h = g.get_state()
    bufs = [pinned(n, torch) for _ in range(9)]
    for b, a in zip(bufs, st_h.arrays()):
        b.numpy()[:] = a
    csi = pinned(n + 1, torch)
    lib = g.lib
    dp = [C.cast(b.data_ptr(), C.POINTER(C.c_double)) for b in bufs]
    view = clmd.ClusterView()
    view.csi = C.cast(csi.data_ptr(), C.POINTER(C.c_int32))
    sc = clmd.Scalars()
    barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        lib.clmd_set_state(g.h, *dp, None, None)
        nxt = C.c_int32(0)
        lib.clmd_run(g.h, step, cyc, C.byref(nxt))
        step += cyc
        lib.clmd_get_state(g.h, *dp, C.byref(sc))
        lib.clmd_get_clusters(g.h, C.byref(view))
    e2e_s = time.perf_counter() - t0
    barrier()
    e2e_max = max_over_ranks(e2e_s)
    e2e_value = units / e2e_max
    h2d = 9 * 8 * n
    d2h = 9 * 8 * n + 4 * (n + 1) + C.sizeof(clmd.Scalars)
    status = g.scalars().status

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cyc_s, desc = cpu_cycle_estimate(w)
            cpu = {"value": n * cyc / cyc_s, "unit": "atom-steps/s", "cores": 1, "kind": "port",
                   "sample": desc}
        line = {
            "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": w_dtype(w), "data": "synthetic (seeded)",
            "config": config_json(w, world),
            "e2e": {"value": e2e_value, "unit": "atom-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": f"k_cycle ({cyc} "
                                   + ("Nose-Hoover" if w["integrator"] == clmd.INT_NOSE
                                      else "velocity-Verlet") + " steps per launch)",
                         "algorithmic_bytes_per_launch": alg, "kernel_ms": kms,
                         "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "clocks": clk,
            "list_rebuilds_in_timed_region": int(rebuilds),
            "device_status": status,
        }
        print(json.dumps(line), flush=True)
    g.close()
    rk.close()


# ---------------------------------------------------------------------------
# batched ensemble: mixed precision vs the FP64 drop-in (the default workload)
# ---------------------------------------------------------------------------
ENSEMBLE = dict(name="batched", replicas=4096, nmin=200, nmax=8000, rho=(0.01, 0.05),
                temp=(0.65, 0.85), csover=51, budget=200000, ftcsi=100, seed=7)
BYTES_PER_ATOM_STEP_MIXED = 120  # x, v FP64 + a FP32, read + written


def ensemble_specs(nrep, seed, nmin=200, nmax=8000):
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(nmin), np.log(nmax), nrep)).astype(int)
    rho = rng.uniform(*ENSEMBLE["rho"], nrep)
    temp = rng.uniform(*ENSEMBLE["temp"], nrep)
    return [(int(n[k]), float(rho[k]), float(temp[k]), seed * 100003 + k) for k in range(nrep)]


def nh_config(n, rho, temp):
    return clmd.lj_config(n, rho, temp, integrator=clmd.INT_NOSE, ethst="N", ftcsi=100,
                          csover=ENSEMBLE["csover"], clwait=0, clnuctrl="X")


def dropin_rate(n, rho, temp, seed, steps=300):
    """atom-steps/s of the FP64 drop-in (one system at a time) on one
    replica: Nose-Hoover, Stillinger every 100 steps."""
    import torch
    cfg = nh_config(n, rho, temp)
    st = make_state(cfg, seed, temp)
    g = start_system(cfg, st)
    s = g.scalars()
    s.psi = (2.0 * s.ekin - 3.0 * n * clmd.CIKB * cfg.att) / cfg.Q  # main.f:158-160
    g.set_scalars(s)
    g.run(0, 100)
    stream = torch.cuda.ExternalStream(g.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    g.run(100, steps)
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b)
    g.close()
    return n * steps / (ms / 1e3)


# ---------------------------------------------------------------------------
# The reference's serial algorithm on the host (the oracle: a C restatement of
# the Fortran, all-pairs neighbour list, Nose-Hoover, Stillinger every 100
# steps, chk_nucleation), on a fixed sample of the ensemble's replicas.  It
# builds its inputs with the oracle's own copy of the start generator, so a
# process that runs only this never loads the engine library.
# ---------------------------------------------------------------------------
ORACLE_SAMPLE = 16  # replicas, one per 1/16 quantile of the size distribution


def oracle_sample_specs(specs, k=ORACLE_SAMPLE):
    """The replicas at the midpoints of k equal size strata (sorted by N)."""
    order = sorted(range(len(specs)), key=lambda i: (specs[i][0], i))
    return [specs[order[int((2 * q + 1) / (2 * k) * (len(order) - 1))]] for q in range(k)]


class OracleSample:
    """The sample's replicas on the oracle, advanced window by window
    (main.f's loop: stoddard + chk_nucleation every 100 steps, then the
    integrator), each from the start sequence the engine runs at admission
    (stopdead, neighbor(0), AccAtom, the NH PSI start, stoddard(-1))."""

    def __init__(self, sample):
        sys.path.insert(0, ORACLE)
        import orc
        self.reps = []
        for n, rho, temp, sd in sample:
            cfg = nh_config(n, rho, temp)
            L = cfg.boxx
            x, y, z, vx, vy, vz = orc.init_random(n, (L, L, L), 0.9, temp, sd)
            z0 = np.zeros(n)
            o = orc.Oracle(cfg, neighbor_mode=0)
            o.set_state(clmd.State(x, y, z, vx, vy, vz, z0, z0, z0),
                        scalars=orc.scalars_init(cfg))
            o.stopdead(-1)
            o.neighbor(0)
            o.zero_acc()
            o.accatom()
            sc = o.scalars()
            sc.psi = (2.0 * sc.ekin - 3.0 * n * clmd.CIKB * cfg.att) / cfg.Q  # main.f:96-101
            sc.s = 0.0
            o.set_scalars(sc)
            o.stoddard(-1)
            self.reps.append([o, n, 0, False])  # oracle, N, next step, stopped

    def window(self, steps=100):
        """One window of every running replica: (seconds, atom-steps)."""
        done = 0
        t0 = time.perf_counter()
        for r in self.reps:
            o, n, step, stopped = r
            if stopped:
                continue
            st, nxt = o.run(step, steps)
            if st or nxt < 0 or o.scalars().status:  # nucleated (chk_nucleation) or failed
                nxt = abs(nxt)
                r[3] = True
            done += n * (nxt - step)
            r[2] = nxt
        return time.perf_counter() - t0, done

    def atoms(self):
        return sum(r[1] for r in self.reps)

    def close(self):
        for r in self.reps:
            r[0].close()


def pin_one_core():
    """Pins this process to one host core (the first it may use)."""
    try:
        core = min(os.sched_getaffinity(0))
        os.sched_setaffinity(0, {core})
        return core
    except (AttributeError, OSError):
        return None


def oracle_sample_run(sample, warm, timed, pin=True):
    """warm + timed windows of the sample on one pinned core: (atom-steps/s
    over the timed windows, per-window seconds, description)."""
    core = pin_one_core() if pin else None
    os_ = OracleSample(sample)
    for _ in range(warm):
        os_.window()
    secs, work = [], 0
    for _ in range(timed):
        t, w = os_.window()
        secs.append(t)
        work += w
    os_.close()
    rate = work / max(sum(secs), 1e-12)
    desc = (f"oracle (serial C restatement of the reference: all-pairs list, Nose-Hoover, "
            f"Stillinger + chk_nucleation every 100 steps) on 1 core (cpu {core}), "
            f"{len(sample)} replicas at the midpoints of 16 size strata of the ensemble "
            f"(N = {sorted(sp[0] for sp in sample)}, {sum(sp[0] for sp in sample)} atoms), "
            f"{timed} timed 100-step windows after {warm} untimed")
    return rate, secs, desc


def _oracle_child(sample, warm, timed, q):
    q.put(oracle_sample_run(sample, warm, timed))


def oracle_sample_in_child(sample, warm, timed):
    """oracle_sample_run in a spawned process (its own pinned core; the
    caller's threads and GPU context stay as they are)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_oracle_child, args=(sample, warm, timed, q))
    p.start()
    out = q.get()
    p.join()
    return out


def _oracle_core_worker(sample, core, barrier, q):
    try:
        os.sched_setaffinity(0, {core})
    except (AttributeError, OSError):
        pass
    os_ = OracleSample(sample)
    os_.window()  # untimed
    barrier.wait()
    t, w = os_.window()
    os_.close()
    q.put((t, w))


def oracle_all_cores(sample):
    """Every host core runs its own copy of the sample for one timed window
    at the same time (the reference is serial: a host runs independent
    replicas side by side): whole-host atom-steps / the slowest core's time."""
    import multiprocessing as mp
    cores = sorted(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else [0]
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(len(cores))
    q = ctx.Queue()
    ps = [ctx.Process(target=_oracle_core_worker, args=(sample, c, barrier, q)) for c in cores]
    for p in ps:
        p.start()
    got = [q.get() for _ in ps]
    for p in ps:
        p.join()
    return sum(w for _, w in got) / max(t for t, _ in got), len(cores)


def batched_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    specs = ensemble_specs(args.replicas, ENSEMBLE["seed"])
    sample = oracle_sample_specs(specs)
    all_rate, ncores = (None, None)
    if not args.no_all_cores:
        all_rate, ncores = oracle_all_cores(sample)
    core = pin_one_core()
    os_ = OracleSample(sample)
    for _ in range(args.warmup):
        os_.window()
    secs, work = [], 0
    for _ in range(args.steps):
        t, w = os_.window()
        secs.append(t)
        work += w
    os_.close()
    value = work / sum(secs)
    desc = (f"oracle (serial C restatement of the reference: all-pairs list, Nose-Hoover, "
            f"Stillinger + chk_nucleation every 100 steps) on 1 core (cpu {core}), "
            f"{len(sample)} replicas at the midpoints of 16 size strata of the ensemble "
            f"(N = {sorted(sp[0] for sp in sample)}), one bench step = one 100-step window "
            f"of each")
    line = {
        "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sum(secs) / len(secs) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": batched_config_json(args, sum(sp[0] for sp in specs), [0, 0, 0, 0], 1),
        "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": 1, "kind": "port",
                         "sample": desc},
        "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "sample_atom_steps_per_step": work / len(secs),
        "all_cores": ({"value": all_rate, "unit": "atom-steps/s", "cores": ncores,
                       "how": "one copy of the sample per core at once, one timed window, "
                              "whole-host atom-steps / slowest core's time"}
                      if all_rate else None),
    }
    print(json.dumps(line), flush=True)


def batched_config_json(args, total, tuned, ngpu):
    return {"workload": f"batched-ensemble-{args.replicas}x(N=200..8000 log-uniform, "
                        "rho*=0.01..0.05, T*=0.65..0.85)-NoseHoover-mixed",
            "replicas_per_gpu": args.replicas, "atoms_per_gpu": total,
            "steps_per_bench_step": 100, "clustering": "stillinger-1.5sigma every 100",
            "stop": "largest cluster > 50 (csover=51) or 2e5 steps",
            "threads_per_size_class": [clmd.shape_name(t) for t in tuned],
            "l2": "window state (~1 GB) larger than L2; no flush needed",
            "parallelism": f"replicas x{ngpu}"}


U_RC = 4.0 * (2.5 ** -12 - 2.5 ** -6)  # the LJ pair energy at the cut-off (sigma = eps = 1)


def pairs_within(st, box, rc=2.5):
    """Pairs nearer than rc (minimum image) in a replica's positions."""
    from scipy.spatial import cKDTree
    p = np.mod(np.stack([st.x, st.y, st.z], 1), box)
    p[p >= box] = 0.0
    return len(cKDTree(p, boxsize=box).query_pairs(rc))


def precision_check(specs, nsample=64, windows=100):
    """Energy drift and cluster sizes of mixed precision against FP64, replica
    by replica.  The same nsample replicas run three times -- mixed, FP64 and
    an FP64 twin whose start differs by 1e-13 in one velocity -- for 100 +
    windows x 100 Nose-Hoover steps.  Per replica the drift of the conserved
    H = ekin + epot + Q PSI^2/2 + 3 N kT s (main.f:106,142) from step 100 to
    the end is taken twice: with the reference's epot, whose unshifted
    cut-off adds U(rc) to H at every pair that crosses rc (so H changes
    while the vapour condenses even with exact arithmetic), and with the
    energy the truncated force conserves, H - U(rc) x (pairs within rc).
    Reported: the mixed - FP64 difference per replica against the twin's
    (the spread chaos alone gives), and the cluster-size distribution at the
    end (every cluster of every replica) as a total variation distance."""
    sample = specs[:nsample]
    runs = {}
    for name, prec, twin in (("mixed", clmd.PREC_MIXED, False), ("fp64", clmd.PREC_FP64, False),
                             ("fp64_twin", clmd.PREC_FP64, True)):
        e = clmd.Ensemble(clmd.ens_config(sum(n for n, _, _, _ in sample) + 64, len(sample),
                                          precision=prec, integrator=clmd.INT_NOSE,
                                          ftcsi=ENSEMBLE["ftcsi"], threads=256))
        slots = []
        for n, rho, temp, sd in sample:
            box = (n / rho) ** (1.0 / 3.0)
            x, y, z, vx, vy, vz = clmd.init_random(n, (box, box, box), 0.9, temp, sd)
            if twin:
                vx = vx.copy()
                vx[1] *= 1.0 + 1e-13
            slots.append(e.add(n, box, temp, x, y, z, vx, vy, vz, csover=10**6, budget=0))

        def H(r, n, temp):
            return r.ekin + r.epot + 0.5 * (n * temp * 0.25) * r.psi ** 2 + 3.0 * n * temp * r.s

        e.step(1)  # the start sequence and a first window: energies defined
        res0 = e.results()
        h0, hs0 = [], []
        for k, (n, rho, temp, _) in zip(slots, sample):
            st, _ = e.state(k)
            h0.append(H(res0[k], n, temp))
            hs0.append(h0[-1] - U_RC * pairs_within(st, (n / rho) ** (1.0 / 3.0)))
        e.step(windows)
        res = e.results()
        d, ds, sizes = [], [], []
        for j, (k, (n, rho, temp, _)) in enumerate(zip(slots, sample)):
            st, cl = e.state(k)
            h = H(res[k], n, temp)
            hs = h - U_RC * pairs_within(st, (n / rho) ** (1.0 / 3.0))
            d.append((h - h0[j]) / abs(h0[j]))
            ds.append((hs - hs0[j]) / abs(hs0[j]))
            c = np.bincount(cl)[1:]
            sizes.extend(c[c > 0].tolist())
            assert res[k].status == 0, (name, k, res[k].status)
        runs[name] = (np.array(d), np.array(ds), np.bincount(sizes))
        e.close()
    dm, dsm, hm = runs["mixed"]
    df, dsf, hf = runs["fp64"]
    dt, dst, _ = runs["fp64_twin"]
    gap, chaos = np.abs(dm - df), np.abs(dt - df)
    m = max(len(hm), len(hf))
    pa = np.pad(hm, (0, m - len(hm))).astype(float)
    pb = np.pad(hf, (0, m - len(hf))).astype(float)
    tv = 0.5 * np.abs(pa / pa.sum() - pb / pb.sum()).sum()
    steps = windows * 100
    return {
        "replicas": nsample, "steps": steps, "from_step": 100,
        "relative_drift_of_H": {
            "mixed_median": float(np.median(np.abs(dm))),
            "fp64_median": float(np.median(np.abs(df))),
            "mixed_minus_fp64_median": float(np.median(gap)),
            "mixed_minus_fp64_max": float(gap.max()),
            "fp64_twin_minus_fp64_median": float(np.median(chaos)),
            "fp64_twin_minus_fp64_max": float(chaos.max()),
            "replicas_within_3x_twin_spread_plus_1e-6": int((gap <= 3 * chaos + 1e-6).sum())},
        "relative_drift_of_shifted_H": {
            "mixed_median": float(np.median(np.abs(dsm))),
            "mixed_max": float(np.abs(dsm).max()),
            "fp64_median": float(np.median(np.abs(dsf))),
            "fp64_max": float(np.abs(dsf).max()),
            "fp64_twin_max": float(np.abs(dst).max()),
            "replicas_mixed_within_1e-4": int((np.abs(dsm) <= 1e-4).sum())},
        "cluster_size_distribution_tv_distance": float(tv)}


def mixed_force_error(e, slots, specs_by_slot, nsample=3):
    """Relative force error of the mixed engine against the FP64 oracle on
    the engine's own positions (normwise and worst atom above 1% of max)."""
    sys.path.insert(0, ORACLE)
    import orc
    worst_n, worst_a = 0.0, 0.0
    for k in list(slots)[:nsample]:
        n = specs_by_slot[k][0]
        st, _ = e.state(k)
        rho = specs_by_slot[k][1]
        cfg = clmd.lj_config(n, rho, 0.7)
        o = orc.Oracle(cfg, neighbor_mode=1)
        z0 = np.zeros(n)
        o.set_state(clmd.State(st.x, st.y, st.z, z0, z0, z0, z0, z0, z0),
                    scalars=orc.scalars_init(cfg))
        o.neighbor(0)
        o.zero_acc()
        o.accatom()
        r = o.get_state()
        a = np.stack([st.ax, st.ay, st.az], 1)
        b = np.stack([r.ax, r.ay, r.az], 1)
        worst_n = max(worst_n, np.linalg.norm(a - b) / np.linalg.norm(b))
        mag = np.linalg.norm(b, axis=1)
        big = mag > 0.01 * mag.max()
        worst_a = max(worst_a, (np.linalg.norm(a - b, axis=1)[big] / mag[big]).max())
        o.close()
    return worst_n, worst_a


def batched_arm(args):
    import torch

    rk = Ranks(timeout_s=300)
    rank, world, dev = rk.rank, rk.world, rk.device
    clmd.set_device(dev)
    barrier = rk.barrier

    specs = ensemble_specs(args.replicas, ENSEMBLE["seed"] + 1000 * rank)
    total = sum(sp[0] for sp in specs)
    e = clmd.Ensemble(clmd.ens_config(total + 1024, len(specs), precision=clmd.PREC_MIXED,
                                      integrator=clmd.INT_NOSE, ftcsi=ENSEMBLE["ftcsi"],
                                      threads=args.threads))
    t0 = time.perf_counter()
    slots = {}
    for n, rho, temp, sd in specs:
        box = (n / rho) ** (1.0 / 3.0)
        x, y, z, vx, vy, vz = clmd.init_random(n, (box, box, box), 0.9, temp, sd)
        slots[e.add(n, box, temp, x, y, z, vx, vy, vz, csover=ENSEMBLE["csover"], clwait=0,
                    budget=ENSEMBLE["budget"])] = (n, rho, temp, sd)
    log(f"rank {rank}: admitted {len(slots)} replicas, {total} atoms in "
        f"{time.perf_counter()-t0:.1f} s")
    e.step(1)  # the start sequences + a first window
    tuned = e.autotune() if args.threads == 0 else [args.threads] * 4
    for _ in range(max(0, args.warmup - 1)):
        e.step(1)

    # ---- value: device-resident windows
    r0 = {k: v.step for k, v in e.results().items()}
    l0 = e.launches()
    clocks = Clocks(dev)
    kern_ms, kern_bytes = [], []
    pt0 = e.pair_terms()
    barrier()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    t = time.perf_counter()
    for _ in range(args.steps):
        e.step(1)
        ms, at = e.last_ms()
        kern_ms.append(max(ms))
        kern_bytes.append(sum(at) * ENSEMBLE["ftcsi"] * BYTES_PER_ATOM_STEP_MIXED)
    ev1.record()
    torch.cuda.synchronize()
    el = time.perf_counter() - t
    clk = clocks.stop()
    barrier()
    res = e.results()
    atom_steps = sum(slots[k][0] * (res[k].step - r0[k]) for k in slots)
    el_max = rk.max(el)
    units = rk.sum(float(atom_steps))
    value = units / el_max
    launches = e.launches() - l0
    pair_terms = e.pair_terms() - pt0

    # ---- roofline: the window kernels (size classes run concurrently)
    peak, peak_kind = measured_peaks()
    achieved = sum(kern_bytes) / (sum(kern_ms) / 1e3) / 1e9

    # ---- e2e: host buffers through the C ABI every window
    bufs = [torch.empty(total, dtype=torch.float64).pin_memory() for _ in range(6)]
    dp = [C.cast(b.data_ptr(), C.POINTER(C.c_double)) for b in bufs]
    lib = e.lib
    lib.clmd_ens_download(e.h, *dp)

    def e2e_run(streamed):
        r0 = e.results()
        barrier()
        t = time.perf_counter()
        for _ in range(args.steps):
            if streamed:
                # one call: the window kernel reads each running replica's
                # x, v from the pinned arrays when it takes the replica and
                # writes them back when it leaves it
                e.step_io(1, dp)
            else:
                lib.clmd_ens_upload(e.h, *dp)
                e.step(1)
                lib.clmd_ens_download(e.h, *dp)
        el = time.perf_counter() - t
        barrier()
        r1 = e.results()
        units = rk.sum(float(sum(slots[k][0] * (r1[k].step - r0[k].step) for k in slots)))
        running = sum(slots[k][0] for k in slots if r0[k].done == 0 and r0[k].status == 0)
        return units / rk.max(el), running

    e2e_copies, _ = e2e_run(False)
    e2e_value, running = e2e_run(True)
    h2d = 6 * 8 * running
    d2h = 6 * 8 * running + 16 * len(slots)

    line = None
    extra = dict(pcheck=None, rates=[], dropin_value=None)
    ferr_n = ferr_a = None
    if rank == 0 and not args.no_extras:
        ferr_n, ferr_a = mixed_force_error(e, slots, slots)
    e.close()
    rk.barrier()
    # ---- the same replicas as an all-FP64 ensemble (same kernels, FP64
    # pair terms and sums): how much of the gain is batching, how much
    # mixed precision
    fp64_value, fp64_tuned = (None, []) if args.no_extras else fp64_ensemble_rate(specs, args)
    if rank == 0 and not args.no_extras:
        pcheck = precision_check(specs)
        order = sorted(slots, key=lambda k: slots[k][0])
        picks = [order[int(q * (len(order) - 1))] for q in np.linspace(0, 1, args.dropin_sample)]
        rates = [(slots[k][0], dropin_rate(*slots[k])) for k in picks]
        ln = np.log([r[0] for r in rates])
        lr = np.log([r[1] for r in rates])
        t_drop = sum(slots[k][0] * 100 / float(np.exp(np.interp(np.log(slots[k][0]), ln, lr)))
                     for k in slots)
        dropin_value = sum(slots[k][0] * 100 for k in slots) / t_drop
        extra = dict(pcheck=pcheck, rates=rates, dropin_value=dropin_value)
    # ---- served leg: a bounded Poisson window of requests on this GPU
    served = None if (args.no_served or args.no_extras) else served_leg(args, rk)
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            v, secs, desc = oracle_sample_in_child(oracle_sample_specs(specs), 1, 3)
            cpu = {"value": v, "unit": "atom-steps/s", "cores": 1, "kind": "port",
                   "sample": desc, "seconds_per_window": secs}
        dropin_value = extra["dropin_value"]
        line = {
            "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el_max / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic (seeded)",
            "config": batched_config_json(args, total, tuned, world),
            "e2e": {"value": e2e_value, "unit": "atom-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "how": "clmd_ens_step_io per window: the window kernel reads every running "
                           "replica's x, v from pinned host memory when it takes the replica "
                           "and writes them back when it leaves it",
                    "separate_copies": e2e_copies},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profiled_traffic("k_ens_batched"),
                         "kernel": "k_ens (one window = 100 Nose-Hoover steps per replica; "
                                   "4 size classes concurrently)",
                         "algorithmic_bytes_per_atom_step": BYTES_PER_ATOM_STEP_MIXED,
                         "kernel_ms_per_window": statistics.mean(kern_ms),
                         "peak_kind": peak_kind,
                         "limiter": {
                             "what": "issue- and latency-bound, not HBM: each replica's working "
                                     "set stays in shared memory and L2 (DRAM traffic is a "
                                     "tenth of the algorithmic bytes); the work is the pair "
                                     "terms (FP64 minimum image + cut-off test, FP32 LJ "
                                     "term) and the per-step phases between barriers",
                             "pair_terms_per_s": pair_terms / (sum(kern_ms) / 1e3),
                             "pair_terms_per_atom_step": pair_terms / max(1.0, atom_steps),
                             "ncu": "profiles/k_ens_batched.md (lanes per warp instruction, "
                                    "warps active, issue active, FP64/FP32 pipes)"}},
            "cpu_baseline": cpu,
            "clocks": clk,
            "fp64_ensemble_same_ensemble": fp64_value,
            "fp64_ensemble_threads_per_size_class": [clmd.shape_name(t) for t in fp64_tuned],
            "speedup_vs_fp64_ensemble": value / fp64_value if fp64_value else None,
            "fp64_dropin_same_ensemble": dropin_value,
            "speedup_vs_fp64_dropin": value / dropin_value if dropin_value else None,
            "dropin_sample_rates": [[n, r] for n, r in extra["rates"]],
            "force_rel_err_vs_fp64": {"normwise": ferr_n, "worst_atom": ferr_a},
            "mixed_vs_fp64_sample": extra["pcheck"],
            "nucleated": sum(1 for r in res.values() if r.done == 1),
            "served": served,
        }
        print(json.dumps(line), flush=True)
    rk.close()


def fp64_ensemble_rate(specs, args, windows=3):
    """atom-steps/s of the all-FP64 ensemble on the same replicas (whole
    windows, after the start window and the tuner)."""
    import torch
    total = sum(sp[0] for sp in specs)
    e = clmd.Ensemble(clmd.ens_config(total + 1024, len(specs), precision=clmd.PREC_FP64,
                                      integrator=clmd.INT_NOSE, ftcsi=ENSEMBLE["ftcsi"],
                                      threads=args.threads))
    for n, rho, temp, sd in specs:
        box = (n / rho) ** (1.0 / 3.0)
        x, y, z, vx, vy, vz = clmd.init_random(n, (box, box, box), 0.9, temp, sd)
        e.add(n, box, temp, x, y, z, vx, vy, vz, csover=ENSEMBLE["csover"], clwait=0,
              budget=ENSEMBLE["budget"])
    e.step(1)
    tuned = e.autotune() if args.threads == 0 else [args.threads] * 4
    e.step(1)
    r0 = {k: v.step for k, v in e.results().items()}
    torch.cuda.synchronize()
    t = time.perf_counter()  # timed like the mixed value: whole windows, host clock
    for _ in range(windows):
        e.step(1)
    torch.cuda.synchronize()
    el = time.perf_counter() - t
    res = e.results()
    work = sum(e.natom[k] * (res[k].step - r0[k]) for k in res)
    e.close()
    return work / el, tuned


# served solves: Poisson arrivals, continuous batching (clmd_serve)
# ---------------------------------------------------------------------------
SERVED = dict(rate=200.0, nmin=100, nmax=50000, rho=(0.01, 0.05), temp=(0.65, 0.85),
              budget=(1e4, 1e6), csover=101, ftcsi=100, seed=11)
POOL_BYTES_PER_ATOM = 9 * 8 + 3 * 8 + 192 * 4 + 6 * 4  # x..vzn, a, ELL list, int scratch


def served_trace(arrival_s, seed):
    """Poisson arrivals at SERVED['rate'] over [0, arrival_s): N log-uniform,
    rho*/T* uniform, step budgets log-uniform, threshold largest cluster > 100."""
    rng = np.random.default_rng(seed)
    reqs, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / SERVED["rate"])
        if t >= arrival_s:
            break
        r = clmd.Request()
        r.arrival = t
        r.natom = int(np.exp(rng.uniform(np.log(SERVED["nmin"]), np.log(SERVED["nmax"]))))
        r.rho = float(rng.uniform(*SERVED["rho"]))
        r.temp = float(rng.uniform(*SERVED["temp"]))
        r.budget = int(np.exp(rng.uniform(*np.log(SERVED["budget"]))))
        r.csover = SERVED["csover"]
        r.seed = seed * 1000003 + len(reqs)
        reqs.append(r)
    return reqs


def served_config_json(args, nreq, pool, ngpu):
    return {"workload": f"served-poisson-{SERVED['rate']:.0f}req/s-for-{args.arrival_seconds}s"
                        "(N=100..50000 log-uniform, rho*=0.01..0.05, T*=0.65..0.85, "
                        "budget 1e4..1e6 log-uniform)-NoseHoover-mixed",
            "requests_per_gpu": nreq, "pool_atoms": pool,
            "admission": "free HBM: atom pool sized from cudaMemGetInfo",
            "stop": "largest cluster > 100 (csover=101) or budget",
            "window_steps": SERVED["ftcsi"], "max_seconds": args.serve_seconds,
            "l2": "no flush; resident state grows past L2 as requests arrive",
            "parallelism": f"independent traces x{ngpu}"}


def run_served(args, rk, arrival_s, serve_s, max_slots):
    """One served trace on this rank's GPU: the atom pool from free HBM, a
    short untimed trace first (block shapes, code paths), then the Poisson
    trace.  Returns (results, stats, clocks, launches, pool atoms, requests)."""
    import torch
    dev = rk.device
    free, _ = torch.cuda.mem_get_info(dev)
    pool = int(min(args.pool_fraction * free / POOL_BYTES_PER_ATOM, 2**31 - 1))
    reqs = served_trace(arrival_s, SERVED["seed"] + 1000 * rk.rank)
    e = clmd.Ensemble(clmd.ens_config(pool, max_slots, precision=clmd.PREC_MIXED,
                                      integrator=clmd.INT_NOSE, ftcsi=SERVED["ftcsi"],
                                      threads=args.threads or 0))
    warm = served_trace(0.25, SERVED["seed"] + 999 + 1000 * rk.rank)
    for r in warm:
        r.arrival = 0.0
        r.budget = 400
    e.serve(warm, 30.0)
    rk.barrier()
    clocks = Clocks(dev)
    l0 = e.launches()
    clocks.start()
    out, st = e.serve(reqs, serve_s)
    clk = clocks.stop()
    launches = e.launches() - l0
    e.close()
    return out, st, clk, launches, pool, reqs


def served_summary(out, st, nreq, serve_s):
    """Latency percentiles of a served trace.  A request still running when
    the loop stops is censored: its latency is at least (stop - arrival), so
    a percentile that reaches into the censored ones is a lower bound."""
    lat = np.array([o.finished - o.arrival for o in out if o.done in (1, 2)])
    nuc = np.array([o.finished - o.arrival for o in out if o.done == 1])
    nuc_steps = np.array([o.clbrkt for o in out if o.done == 1])
    wait = np.array([o.admitted - o.arrival for o in out if o.admitted >= 0])
    unfinished = [o for o in out if o.done == 0]
    # every request, the censored ones at their lower bound
    lat_all = np.array([o.finished - o.arrival if o.done in (1, 2) else st.wall - o.arrival
                        for o in out])

    def pct(a, q):
        return float(np.percentile(a, q)) if len(a) else None
    cens = len(unfinished) / max(1, len(out))
    return {
        "latency_s": {"p50": pct(lat_all, 50), "p99": pct(lat_all, 99),
                      "p50_is_lower_bound": cens > 0.5, "p99_is_lower_bound": cens > 0.01,
                      "completed_p50": pct(lat, 50), "completed_p99": pct(lat, 99),
                      "time_to_nucleation_p50": pct(nuc, 50),
                      "time_to_nucleation_p99": pct(nuc, 99),
                      "nucleation_step_p50": pct(nuc_steps, 50),
                      "nucleation_step_p99": pct(nuc_steps, 99),
                      "admission_wait_p50": pct(wait, 50), "admission_wait_p99": pct(wait, 99)},
        "requests": {"arrived": nreq, "admitted": st.admitted, "completed": st.completed,
                     "nucleated": int(len(nuc)), "censored": len(unfinished),
                     "peak_resident": st.peak_resident, "peak_atoms": int(st.peak_atoms)},
        "wall_s": st.wall, "serve_cap_s": serve_s,
    }


def big_replica_ms_per_step(n=50000, rho=0.03, temp=0.75, windows=3):
    """Device ms per MD step of one n-atom replica alone on the GPU (the
    served workload's largest size), on a thread-block cluster and, with
    CLMD_ENS_CLUSTERS=0, on one CTA: (cluster ms, single-CTA ms, CTAs)."""
    import torch
    out = []
    for clusters in (True, False):
        if not clusters:
            os.environ["CLMD_ENS_CLUSTERS"] = "0"
        try:
            e = clmd.Ensemble(clmd.ens_config(n + 16, 2, precision=clmd.PREC_MIXED,
                                              integrator=clmd.INT_NOSE, ftcsi=100))
        finally:
            os.environ.pop("CLMD_ENS_CLUSTERS", None)
        box = (n / rho) ** (1.0 / 3.0)
        x, y, z, vx, vy, vz = clmd.init_random(n, (box, box, box), 0.9, temp, 4242)
        slot = e.add(n, box, temp, x, y, z, vx, vy, vz, csover=10**6, budget=0)
        e.step(1)
        torch.cuda.synchronize()
        s0 = e.results()[slot].step
        t = time.perf_counter()
        e.step(windows)
        torch.cuda.synchronize()
        el = time.perf_counter() - t
        out.append(el * 1e3 / (e.results()[slot].step - s0))
        e.close()
    cs = 2
    while cs < 16 and cs * 6144 < n:
        cs *= 2
    return out[0], out[1], cs


def served_leg(args, rk):
    """The served workload inside the default bench: a bounded Poisson window at 200
    requests/s (N log-uniform in [100, 50000], rho* and T* uniform, budgets
    log-uniform in [1e4, 1e6], threshold largest cluster > 100), served with
    continuous batching on this GPU until every request finished or the cap
    passed.  Aggregate atom-steps/s and the latency percentiles."""
    out, st, clk, launches, pool, reqs = run_served(args, rk, args.served_arrival,
                                                    args.served_cap, args.served_slots)
    units = rk.sum(st.atom_steps)
    wall = rk.max(st.wall)
    d = {"workload": f"served-poisson-{SERVED['rate']:.0f}req/s-for-{args.served_arrival}s"
                     "(N=100..50000 log-uniform, rho*=0.01..0.05, T*=0.65..0.85, budget "
                     "1e4..1e6 log-uniform, stop at largest cluster > 100)-NoseHoover-mixed",
         "value": units / wall, "unit": "atom-steps/s", "gpu_launches": int(launches),
         "pool_atoms": pool, "max_resident_replicas": args.served_slots, "clocks": clk}
    d.update(served_summary(out, st, len(reqs), args.served_cap))
    if args.served_drain_arrival > 0:
        # a shorter trace served until every request finished (or the cap):
        # percentiles without censored requests, as far as the cap allows
        out2, st2, _, _, _, reqs2 = run_served(args, rk, args.served_drain_arrival,
                                               args.served_drain_cap, args.served_slots)
        dd = {"workload": f"served-poisson-{SERVED['rate']:.0f}req/s-for-"
                          f"{args.served_drain_arrival}s, served until drained "
                          f"(cap {args.served_drain_cap}s), same distributions",
              "value": rk.sum(st2.atom_steps) / rk.max(st2.wall), "unit": "atom-steps/s"}
        dd.update(served_summary(out2, st2, len(reqs2), args.served_drain_cap))
        d["drained"] = dd
    if rk.rank == 0:
        cl_ms, cta_ms, cs = big_replica_ms_per_step()
        d["one_replica_50000_atoms"] = {
            "ms_per_step_cluster": cl_ms, "ms_per_step_one_cta": cta_ms,
            "cluster_ctas": cs, "speedup": cta_ms / cl_ms,
            "note": "alone on the GPU, whole 100-step windows, host clock"}
    return d


def served_arm(args):
    rk = Ranks(timeout_s=600)
    clmd.set_device(rk.device)
    out, st, clk, launches, pool, reqs = run_served(args, rk, args.arrival_seconds,
                                                    args.serve_seconds, args.served_slots)
    wall = rk.max(st.wall)
    units = rk.sum(st.atom_steps)
    value = units / wall
    if rk.rank == 0:
        admitted_atoms = sum(o.natom for o in out if o.admitted >= 0)
        cpu = None
        if rk.world == 1 and not args.no_cpu_baseline:
            specs = [(r.natom, r.rho, r.temp, r.seed) for r in reqs]
            v, secs, desc = oracle_sample_in_child(oracle_sample_specs(specs), 1, 2)
            cpu = {"value": v, "unit": "atom-steps/s", "cores": 1, "kind": "port",
                   "sample": desc, "seconds_per_window": secs}
        line = {
            "metric": "atom-steps/s (served)", "value": value, "unit": "atom-steps/s",
            "n_gpus": rk.world, "steps": st.windows, "warmup": 1,
            "ms_per_step": wall / max(1, st.windows) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded Poisson trace)",
            "config": served_config_json(args, len(reqs), pool, rk.world),
            "e2e": {"value": value, "unit": "atom-steps/s",
                    "h2d_bytes_per_step": 48 * admitted_atoms / max(1, st.windows),
                    "d2h_bytes_per_step": 16 * st.peak_resident,
                    "note": "the served loop is end to end: host start states in, "
                            "per-window status out, wall clock"},
            "gpu_launches": int(launches),
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        line.update(served_summary(out, st, len(reqs), args.serve_seconds))
        print(json.dumps(line), flush=True)
    rk.close()


def served_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    reqs = served_trace(args.arrival_seconds, SERVED["seed"])
    specs = [(r.natom, r.rho, r.temp, r.seed) for r in reqs]
    v, secs, desc = oracle_sample_run(oracle_sample_specs(specs), args.warmup, args.steps)
    line = {
        "metric": "atom-steps/s (served)", "value": v, "unit": "atom-steps/s",
        "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sum(secs) / len(secs) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Poisson trace)",
        "config": served_config_json(args, len(reqs), 0, 1),
        "cpu_baseline": {"value": v, "unit": "atom-steps/s", "cores": 1, "kind": "port",
                         "sample": desc},
        "e2e": {"value": v, "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10, help="timed analysis cycles (100 MD steps)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--natom", type=int, default=0, help="dropin/nvt: atoms (0 = the workload's)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-all-cores", action="store_true",
                    help="reference arm: skip the all-core figure")
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "dropin", "nvt", "served"])
    ap.add_argument("--arrival-seconds", type=float, default=1.0,
                    help="served: length of the Poisson arrival window")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="served: wall-clock cap of the served loop")
    ap.add_argument("--pool-fraction", type=float, default=0.5,
                    help="served: share of free HBM given to the atom pool")
    ap.add_argument("--replicas", type=int, default=4096)
    ap.add_argument("--threads", type=int, default=0, help="0 = autotune")
    ap.add_argument("--dropin-sample", type=int, default=8)
    ap.add_argument("--no-served", action="store_true",
                    help="batched: leave out the served leg")
    ap.add_argument("--no-extras", action="store_true",
                    help="batched: only value, e2e and roofline (no FP64 comparisons, "
                         "precision check or served leg; for profiler runs)")
    ap.add_argument("--served-arrival", type=float, default=10.0,
                    help="batched: Poisson arrival window of the served leg (s)")
    ap.add_argument("--served-drain-arrival", type=float, default=1.0,
                    help="served leg: seconds of arrivals of a second trace served until "
                         "drained (0: skip)")
    ap.add_argument("--served-drain-cap", type=float, default=90.0,
                    help="served leg: wall-clock cap of the drained trace")
    ap.add_argument("--served-cap", type=float, default=30.0,
                    help="batched: wall-clock cap of the served leg (s)")
    ap.add_argument("--served-slots", type=int, default=16384,
                    help="served: resident replicas at most (the ensemble's slots)")
    args = ap.parse_args()
    if args.workload == "nvt":
        w = dict(NVT, natom=args.natom or NVT["natom"])
    else:
        w = dict(WORKLOAD, natom=args.natom or WORKLOAD["natom"])
    if args.workload == "served":
        if args.impl == "reference":
            served_reference_arm(args)
        else:
            served_arm(args)
        return
    if args.workload == "batched":
        if args.impl == "reference":
            batched_reference_arm(args)
        else:
            batched_arm(args)
        return
    if args.impl == "reference":
        reference_arm(args, w)
    else:
        engine_arm(args, w)


if __name__ == "__main__":
    main()
