"""Benchmark of the LJ MD step + cluster analysis on B200.

Workload (the configuration the headline metric is quoted on that fits one
GPU): N = 262,144 atoms, rho* = 0.02, T* = 0.7, reduced LJ units, cut-off
2.5 sigma, initial list radius 2.8 sigma (skin 0.3, adaptive, nbtim = 10),
velocity Verlet dt* = 0.005, Stillinger clustering (1.5 sigma) with the size
histogram every 100 steps -- the FP64 drop-in.  Seeded synthetic start:
positions uniform with every pair >= 0.9 sigma apart, Maxwell-Boltzmann
velocities, then stopdead(-1) and the first list/forces.

A bench step is one analysis cycle of main.f's loop: stoddard + the
histogram, then 100 integrator steps.  metric = atom-steps/s.

  value   device-resident: K cycles timed with CUDA events on the engine's
          stream; L2 (126 MB) is flushed with a 256 MB write between cycles
          (outside the timed events).
  e2e     the same cycles through the C ABI with host buffers: per cycle the
          state (x, v, a) goes host->device from pinned memory, the cycle
          runs, and the state plus the cluster histogram come back.
  roofline  the step kernel (k_cycle, one launch = 100 steps), timed alone
          with CUDA events; algorithmic bytes = 144 B per atom-step (read
          and write x, v, a in FP64) against the measured copy bandwidth.
  cpu_baseline  the serial C restatement of the reference (the oracle) on one
          host core, on a bounded sample of the same workload.

--impl reference times that serial C restatement alone (the reference is
Fortran 77 and no Fortran compiler exists on either machine), rank 0 only.

Multi-GPU: independent replicas, one per rank (seed + rank): the path has no
data exchange; value = all ranks' atom-steps / max-over-ranks time.
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
                atskin=1.5, dt=0.005, nbtim=10, ftcsi=100, seed=1234)
BYTES_PER_ATOM_STEP = 144  # FP64: x, v, a read + written


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_config(w):
    return clmd.lj_config(w["natom"], w["rho"], w["temp"], rc=w["rc"], rskin=w["rskin"],
                          atskin=w["atskin"], dt=w["dt"], nbtim=w["nbtim"], ftcsi=w["ftcsi"])


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


def profiled_traffic():
    """DRAM bytes per k_cycle launch from the committed ncu summary."""
    p = os.path.join(REPO, "profiles", "k_cycle_fp64_dropin.md")
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
    Returns (seconds per cycle, description)."""
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
    # Stillinger labelling at N/8, scaled by N^2
    ws = dict(w, natom=n // 8)
    cfs = make_config(ws)
    sts = make_state(cfs, w["seed"], w["temp"])
    o = orc.Oracle(cfs, neighbor_mode=1)
    o.set_state(sts, scalars=orc.scalars_init(cfs))
    o.neighbor(0)
    t = time.perf_counter()
    o.stoddard(0)
    t_label = (time.perf_counter() - t) * 64.0
    o.close()
    rebuilds = 100.0 / w["nbtim"]
    cycle = 100 * t_step + rebuilds * t_rebuild + t_label
    desc = (f"serial oracle, 1 core: {nstep} MD steps at N={n} ({t_step*1e3:.1f} ms/step), "
            f"all-pairs rebuild on {rows} rows ({pairs} pair tests) scaled to N(N-1)/2 "
            f"({t_rebuild:.1f} s/rebuild, {rebuilds:.0f} per 100 steps), Stillinger labelling "
            f"at N/8 scaled by 64 ({t_label:.1f} s/analysis)")
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
    value = n * 100 / per_cycle
    line = {
        "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_cycle * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": config_json(w, args.gpus),
        "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": 1, "kind": "port",
                         "sample": desc},
        "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_json(w, ngpu):
    return {"workload": f"{w['name']}-N{w['natom']}-rho{w['rho']}-T{w['temp']}",
            "natom": w["natom"], "rho": w["rho"], "T": w["temp"], "rc": w["rc"],
            "rskin0": w["rskin"], "dt": w["dt"], "integrator": "velocity-verlet",
            "clustering": "stillinger-1.5sigma", "steps_per_bench_step": 100,
            "l2": "flushed between timed steps (256 MB write)",
            "parallelism": f"replicas x{ngpu}"}


# ---------------------------------------------------------------------------
# engine arm
# ---------------------------------------------------------------------------
def start_system(cfg, state):
    """main.f's start with the writers off: commons from the config
    (read-3d.f:263-276), stopdead(-1), neighbor(0), a = 0, AccAtom, stoddard(-1)."""
    g = clmd.System(cfg)
    g.set_state(state, scalars=clmd.scalars_init(cfg))
    g.stopdead(-1)
    g.neighbor(0)
    g.zero_acc()
    g.accatom()
    g.stoddard(-1)
    return g


def pinned(n, torch):
    return torch.empty(n, dtype=torch.float64).pin_memory()


def engine_arm(args, w):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = world > 1
    if dist:
        import datetime
        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    dev = local if dist else 0
    torch.cuda.set_device(dev)
    clmd.set_device(dev)

    def barrier():
        if dist:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
        return float(t.item())

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
    alg = BYTES_PER_ATOM_STEP * n * cyc
    achieved = alg / (kms / 1e3) / 1e9
    traffic = profiled_traffic()

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
            cpu = {"value": n * 100 / cyc_s, "unit": "atom-steps/s", "cores": 1, "kind": "port",
                   "sample": desc}
        line = {
            "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": config_json(w, world),
            "e2e": {"value": e2e_value, "unit": "atom-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "k_cycle (100 velocity-Verlet steps per launch)",
                         "algorithmic_bytes_per_launch": alg, "kernel_ms": kms,
                         "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "clocks": clk,
            "list_rebuilds_in_timed_region": int(rebuilds),
            "device_status": status,
        }
        print(json.dumps(line), flush=True)
    g.close()
    if dist:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


# ---------------------------------------------------------------------------
# batched ensemble (configs "batched"): mixed precision vs the FP64 drop-in
# ---------------------------------------------------------------------------
def ensemble_specs(nrep, seed, nmin=200, nmax=8000):
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(nmin), np.log(nmax), nrep)).astype(int)
    rho = rng.uniform(0.01, 0.05, nrep)
    temp = rng.uniform(0.65, 0.85, nrep)
    return [(int(n[k]), float(rho[k]), float(temp[k]), seed * 100003 + k) for k in range(nrep)]


def dropin_rate(n, rho, temp, seed, steps=300):
    """atom-steps/s of the FP64 drop-in (one system per launch sequence) on
    one replica: Nose-Hoover, Stillinger every 100 steps."""
    import torch
    cfg = clmd.lj_config(n, rho, temp, integrator=clmd.INT_NOSE, ethst="N", ftcsi=100)
    st = make_state(cfg, seed, temp)
    g = start_system(cfg, st)
    s = g.scalars()
    sumv2 = 2.0 * s.ekin
    s.psi = (sumv2 - 3.0 * n * clmd.CIKB * cfg.att) / cfg.Q
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


def batched_arm(args):
    import torch
    torch.cuda.set_device(0)
    clmd.set_device(0)
    specs = ensemble_specs(args.replicas, 7)
    total = sum(sp[0] for sp in specs)
    e = clmd.Ensemble(clmd.ens_config(total + 1024, len(specs), precision=clmd.PREC_MIXED,
                                      integrator=clmd.INT_NOSE, ftcsi=100,
                                      threads=args.threads))
    t0 = time.perf_counter()
    slots = {}
    for n, rho, temp, sd in specs:
        box = (n / rho) ** (1.0 / 3.0)
        x, y, z, vx, vy, vz = clmd.init_random(n, (box, box, box), 0.9, temp, sd)
        slots[e.add(n, box, temp, x, y, z, vx, vy, vz, csover=51, clwait=0,
                    budget=200000)] = (n, rho, temp, sd)
    log(f"admitted {len(slots)} replicas, {total} atoms in {time.perf_counter()-t0:.1f} s")
    e.step(1)  # start sequences + first window (warm-up)
    for _ in range(args.warmup - 1):
        e.step(1)
    tuned = e.autotune() if args.threads == 0 else [args.threads] * 4
    r0 = {k: v.step for k, v in e.results().items()}
    torch.cuda.synchronize()
    l0 = e.launches()
    t = time.perf_counter()
    for _ in range(args.steps):
        e.step(1)
    torch.cuda.synchronize()
    el = time.perf_counter() - t
    res = e.results()
    atom_steps = sum(slots[k][0] * (res[k].step - r0[k]) for k in slots)
    value = atom_steps / el
    done = sum(1 for r in res.values() if r.done == 1)
    # the FP64 drop-in on the same ensemble: per-replica rates on a stratified
    # sample, total time for every replica's steps, same atom-steps
    order = sorted(slots, key=lambda k: slots[k][0])
    picks = [order[int(q * (len(order) - 1))] for q in np.linspace(0, 1, args.dropin_sample)]
    rates = []
    for k in picks:
        n, rho, temp, sd = slots[k]
        rates.append((n, dropin_rate(n, rho, temp, sd)))
    ln = np.log([r[0] for r in rates])
    lr = np.log([r[1] for r in rates])
    t_drop = 0.0
    for k in slots:
        n = slots[k][0]
        rate = float(np.exp(np.interp(np.log(n), ln, lr)))
        t_drop += n * (res[k].step - r0[k]) / rate
    dropin_value = atom_steps / t_drop
    line = {
        "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded)",
        "config": {"workload": f"batched-{len(slots)}-replicas-N200-8000-NH-mixed",
                   "replicas": len(slots), "atoms": total, "steps_per_bench_step": 100,
                   "threads_per_size_class": tuned, "parallelism": "replicas"},
        "fp64_dropin_same_ensemble": dropin_value,
        "speedup_vs_fp64_dropin": value / dropin_value,
        "dropin_sample_rates": [[n, r] for n, r in rates],
        "nucleated": done, "gpu_launches": int(e.launches() - l0),
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20, help="timed analysis cycles (100 MD steps)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--natom", type=int, default=WORKLOAD["natom"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="dropin", choices=["dropin", "batched"])
    ap.add_argument("--replicas", type=int, default=4096)
    ap.add_argument("--threads", type=int, default=0, help="0 = autotune")
    ap.add_argument("--dropin-sample", type=int, default=8)
    args = ap.parse_args()
    w = dict(WORKLOAD, natom=args.natom)
    if args.workload == "batched":
        batched_arm(args)
        return
    if args.impl == "reference":
        reference_arm(args, w)
    else:
        engine_arm(args, w)


if __name__ == "__main__":
    main()
