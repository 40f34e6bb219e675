"""TEST INFRASTRUCTURE ONLY: ctypes bindings of the C oracle (liborc.so).

The oracle is the serial FP64 restatement of the reference's hot path
(clmd_oracle.c).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
legs use it, as the checker and as the CPU baseline; the engine never calls
it.  Its methods mirror clmd.System so parity tests read the same on both.

The oracle shares the engine's ABI structs (Config, Scalars, ClusterView are
plain layouts of include/clmd.h), imported from the engine's binding module
without loading the engine library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "fortran-cluster-md_b200"))
import clmd  # noqa: E402  (structs only)

LIB_PATH = os.path.join(HERE, "liborc.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    d = C.POINTER(C.c_double)
    i = C.POINTER(C.c_int32)
    sig = {
        "orc_create": ([C.POINTER(clmd.Config)], P),
        "orc_destroy": ([P], None),
        "orc_set_neighbor_mode": ([P, C.c_int], None),
        "orc_scalars_init": ([C.POINTER(clmd.Config), C.POINTER(clmd.Scalars)], None),
        "orc_set_state": ([P, d, d, d, d, d, d, d, d, d, i, C.POINTER(clmd.Scalars)], None),
        "orc_get_state": ([P, d, d, d, d, d, d, d, d, d, C.POINTER(clmd.Scalars)], None),
        "orc_neighbor": ([P, i], C.c_int),
        "orc_accatom": ([P], C.c_int),
        "orc_zero_acc": ([P], C.c_int),
        "orc_integrator": ([P, C.c_int32], C.c_int),
        "orc_thermostat": ([P, C.c_int32], C.c_int),
        "orc_stopdead": ([P, C.c_int32], C.c_int),
        "orc_stoddard": ([P, C.c_int32], C.c_int),
        "orc_chk_nucleation": ([P, i], C.c_int),
        "orc_thermostat_clu": ([P, C.c_int32, C.c_char, C.c_int32], C.c_int),
        "orc_rates": ([P, C.c_int32, C.c_int32, C.c_char_p, C.c_char_p], C.c_int),
        "orc_run": ([P, C.c_int32, C.c_int32, i], C.c_int),
        "orc_get_halflist": ([P, i, C.c_int64, i, C.POINTER(C.c_int64)], C.c_int),
        "orc_get_clusters": ([P, C.POINTER(clmd.ClusterView)], C.c_int),
        "orc_neighbor_rows_sample": ([P, C.c_int32, C.c_int32], C.c_int64),
        "orc_readdata": ([C.c_char_p, C.POINTER(clmd.Config), i, i], C.c_int),
        "orc_set_label_mode": ([P, C.c_int], None),
        "orc_get_liquid": ([P, i], C.c_int),
        "orc_init_random": ([C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                             C.c_double, C.c_uint64, d, d, d, d, d, d], C.c_int),
        "orc_passage_time": ([i, i, C.c_int32, C.c_int32, C.c_int32, C.c_int32, i, i],
                             C.c_int),
        "orc_mpt": ([i, i, C.c_int32, C.c_int32, C.c_int32, d, d, i], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def ptr(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def scalars_init(cfg):
    s = clmd.Scalars()
    load().orc_scalars_init(C.byref(cfg), C.byref(s))
    return s


def init_random(n, box, rmin, kt_over_m, seed):
    """The engine's seeded start, computed here without the engine library
    (byte-identical to clmd.init_random)."""
    arrs = [np.zeros(n) for _ in range(6)]
    bx, by, bz = box
    st = load().orc_init_random(n, bx, by, bz, rmin, kt_over_m, seed,
                                *[ptr(a, C.c_double) for a in arrs])
    if st:
        raise RuntimeError(f"orc_init_random failed: {st}")
    return tuple(arrs)


def passage_time(ts, cs, startsize, endsize, warmup=0):
    """helpers/passage-time.f on one run: (first-passage step per size
    0..endsize, -1 where never reached; probab.largest counts)."""
    ts = np.ascontiguousarray(ts, dtype=np.int32)
    cs = np.ascontiguousarray(cs, dtype=np.int32)
    pt = np.zeros(endsize + 1, dtype=np.int32)
    pb = np.zeros(endsize + 1, dtype=np.int32)
    load().orc_passage_time(ptr(ts, C.c_int32), ptr(cs, C.c_int32), len(ts), startsize,
                            endsize, warmup, ptr(pt, C.c_int32), ptr(pb, C.c_int32))
    return pt, pb


def mpt(ts, cs, startsize, endsize):
    """helpers/mpt.f over pooled (step, size) passage lines: per size
    startsize..endsize (mean of ts/500000, standard error, count)."""
    ts = np.ascontiguousarray(ts, dtype=np.int32)
    cs = np.ascontiguousarray(cs, dtype=np.int32)
    n = endsize - startsize + 1
    m, sd = np.zeros(n), np.zeros(n)
    cnt = np.zeros(n, dtype=np.int32)
    st = load().orc_mpt(ptr(ts, C.c_int32), ptr(cs, C.c_int32), len(ts), startsize, endsize,
                        ptr(m, C.c_double), ptr(sd, C.c_double), ptr(cnt, C.c_int32))
    if st:
        raise RuntimeError(f"orc_mpt failed: {st}")
    return m, sd, cnt


def readdata(path):
    cfg = clmd.Config()
    nt = C.c_int32(0)
    sc = C.c_int32(0)
    st = load().orc_readdata(path.encode(), C.byref(cfg), C.byref(nt), C.byref(sc))
    if st:
        raise RuntimeError(f"orc_readdata({path}) failed: {st}")
    return cfg, nt.value, sc.value


class Oracle:
    def __init__(self, cfg, neighbor_mode=0, label_mode=0):
        self.lib = load()
        self.cfg = cfg
        self.n = cfg.natom
        self.h = self.lib.orc_create(C.byref(cfg))
        self.lib.orc_set_neighbor_mode(self.h, neighbor_mode)
        self.lib.orc_set_label_mode(self.h, label_mode)

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_neighbor_mode(self, mode):
        self.lib.orc_set_neighbor_mode(self.h, mode)

    def set_state(self, state=None, api=None, scalars=None):
        arrs = state.arrays() if state is not None else [None] * 9
        arrs = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
                for a in arrs]
        a = np.ascontiguousarray(api, dtype=np.int32) if api is not None else None
        self.lib.orc_set_state(self.h, *[ptr(v, C.c_double) for v in arrs],
                               ptr(a, C.c_int32),
                               C.byref(scalars) if scalars is not None else None)
        return 0

    def get_state(self):
        arrs = [np.zeros(self.n) for _ in range(9)]
        self.lib.orc_get_state(self.h, *[ptr(v, C.c_double) for v in arrs], None)
        return clmd.State(*arrs)

    def scalars(self):
        s = clmd.Scalars()
        self.lib.orc_get_state(self.h, *([None] * 9), C.byref(s))
        return s

    def set_scalars(self, s):
        self.lib.orc_set_state(self.h, *([None] * 10), C.byref(s))

    def neighbor(self, step):
        s = C.c_int32(step)
        st = self.lib.orc_neighbor(self.h, C.byref(s))
        return st, s.value

    def accatom(self):
        return self.lib.orc_accatom(self.h)

    def zero_acc(self):
        return self.lib.orc_zero_acc(self.h)

    def accwall(self):
        return 0

    def integrator(self, step):
        return self.lib.orc_integrator(self.h, step)

    def thermostat(self, step):
        return self.lib.orc_thermostat(self.h, step)

    def stopdead(self, step):
        return self.lib.orc_stopdead(self.h, step)

    def thermostat_clu(self, step, eclth, ecltim):
        return self.lib.orc_thermostat_clu(self.h, step, eclth.encode(), ecltim)

    def stoddard(self, step):
        return self.lib.orc_stoddard(self.h, step)

    def chk_nucleation(self, step):
        s = C.c_int32(step)
        st = self.lib.orc_chk_nucleation(self.h, C.byref(s))
        return st, s.value

    def rates(self, step, ctrat, out, log=None):
        """rates.f: appends to out (unit 67); the write(*,1) lines to log."""
        return self.lib.orc_rates(self.h, step, ctrat, os.fsencode(out),
                                  os.fsencode(log) if log else None)

    def run(self, first, nsteps):
        nxt = C.c_int32(0)
        st = self.lib.orc_run(self.h, first, nsteps, C.byref(nxt))
        return st, nxt.value

    def halflist(self):
        n = C.c_int64(0)
        self.lib.orc_get_halflist(self.h, None, 0, None, C.byref(n))
        lst = np.zeros(max(n.value, 1), dtype=np.int32)
        idx = np.zeros(self.n, dtype=np.int32)
        self.lib.orc_get_halflist(self.h, ptr(lst, C.c_int32), n.value, ptr(idx, C.c_int32),
                                  C.byref(n))
        return lst[: n.value], idx

    def clusters(self):
        out = {}
        v = clmd.ClusterView()
        for name, dt, kind in clmd.CLUSTER_FIELDS:
            a = np.zeros(self.n + (1 if kind == "N1" else 0), dtype=dt)
            out[name] = a
            setattr(v, name, ptr(a, C.c_int32 if dt == np.int32 else C.c_double))
        self.lib.orc_get_clusters(self.h, C.byref(v))
        return out

    def liquid(self):
        """1 for the atoms the last ten Wolde-Frenkel analysis found liquid."""
        out = np.zeros(self.n, dtype=np.int32)
        self.lib.orc_get_liquid(self.h, ptr(out, C.c_int32))
        return out

    def neighbor_rows_sample(self, i0, i1):
        return self.lib.orc_neighbor_rows_sample(self.h, i0, i1)
