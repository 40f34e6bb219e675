"""Python host mirror of the engine's C ABI (include/clmd.h), over ctypes.

The product is libclmd.so (CUDA, sm_100a) next to this file; this module only
binds it.  `System` wraps one device-resident system and exposes the
reference's subroutine surface under the reference's names (neighbor,
accatom, integrator, thermostat, stopdead, stoddard, chk_nucleation) plus
the device-resident main loop `run`.  There is no CPU fallback: creating a
System raises if the library is missing or no GPU is visible.

Reduced-unit configurations (sigma = eps = m = 1, kB*T = T*) are built by
`lj_config`; the reference's internal Boltzmann constant is kept, so
att = T* / CIKB.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libclmd.so")

MXSORTS = 10
MXA = 6000
CIKB = 1.38066e-6
CIMU = 1.66056

OK = 0
ERR_SKIN = 1
ERR_LIST_OVERFLOW = 2
ERR_NH_NOCONVERGE = 3
ERR_BAD_SPECIES = 4
ERR_ARG = 5
ERR_CUDA = 6
ERR_NOMEM = 7
ERR_NO_DEVICE = 8
ERR_TIMEOUT = 9

INT_VERLET = 0
INT_NOSE = 1
CLU_STILLINGER = 0
CLU_FRENKEL = 1
PREC_FP64 = 0
PREC_MIXED = 1


class Config(C.Structure):
    """clmd_config (include/clmd.h)."""

    _fields_ = [
        ("apmas", C.c_double * MXSORTS),
        ("apsig", C.c_double * MXSORTS),
        ("apeps", C.c_double * MXSORTS),
        ("att", C.c_double),
        ("atskin", C.c_double),
        ("atrcut", C.c_double),
        ("atrskin", C.c_double),
        ("Q", C.c_double),
        ("boxx", C.c_double),
        ("boxy", C.c_double),
        ("boxz", C.c_double),
        ("dt", C.c_double),
        ("nlist_cap", C.c_int64),
        ("natom", C.c_int32),
        ("atsorts", C.c_int32),
        ("apnum", C.c_int32 * MXSORTS),
        ("atnenum", C.c_int32),
        ("nbtim", C.c_int32),
        ("btim", C.c_int32),
        ("csover", C.c_int32),
        ("clwait", C.c_int32),
        ("ftcsi", C.c_int32),
        ("integrator", C.c_int32),
        ("clustering", C.c_int32),
        ("precision", C.c_int32),
        ("apth", C.c_char * MXSORTS),
        ("ethst", C.c_char),
        ("clnuctrl", C.c_char),
        ("forcevar", C.c_char), ("pad", C.c_char * 3),
    ]


class Scalars(C.Structure):
    """clmd_scalars (include/clmd.h)."""

    _fields_ = [
        ("ekin", C.c_double),
        ("sumv2", C.c_double),
        ("epot", C.c_double),
        ("H", C.c_double),
        ("psi", C.c_double),
        ("s", C.c_double),
        ("atrskin", C.c_double),
        ("dmms", C.c_double),
        ("dmmsu", C.c_double),
        ("dmmax", C.c_double),
        ("dmmav", C.c_double),
        ("dmmh", C.c_double * 256),
        ("virial", C.c_double),
        ("npairs_half", C.c_int64),
        ("dmmst", C.c_int32),
        ("dmmi", C.c_int32),
        ("clbrkt", C.c_int32),
        ("cnum", C.c_int32),
        ("cnumf", C.c_int32),
        ("cstep", C.c_int32),
        ("cbiggest", C.c_int32),
        ("cbiggestf", C.c_int32),
        ("clookfor", C.c_int32),
        ("clookforf", C.c_int32),
        ("status", C.c_int32),
        ("fail_step", C.c_int32),
        ("nh_iters", C.c_int32),
        ("nrebuild", C.c_int32),
        ("last_rebuild_step", C.c_int32),
        ("aborted", C.c_int32),
        ("maxcs", C.c_int32),
        ("pad", C.c_int32),
    ]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if name == "dmmh" else v
        return out


_I32P = C.POINTER(C.c_int32)
_F64P = C.POINTER(C.c_double)


class ClusterView(C.Structure):
    """clmd_cluster_view (include/clmd.h)."""

    _fields_ = [
        ("cl", _I32P), ("cs", _I32P), ("csi", _I32P),
        ("cek", _F64P), ("ceks", _F64P),
        ("clf", _I32P), ("csf", _I32P), ("csif", _I32P),
        ("cekf", _F64P), ("ceksf", _F64P),
        ("cgs", _I32P), ("cgsa", _I32P), ("cgsf", _I32P), ("cgsfa", _I32P),
        ("cfpt", _I32P), ("cfptf", _I32P),
    ]


class EnsConfig(C.Structure):
    """clmd_ens_config (include/clmd.h)."""

    _fields_ = [
        ("rc", C.c_double), ("rskin", C.c_double), ("atskin", C.c_double), ("dt", C.c_double),
        ("max_atoms", C.c_int64), ("max_replicas", C.c_int32), ("list_stride", C.c_int32),
        ("precision", C.c_int32), ("integrator", C.c_int32), ("ftcsi", C.c_int32),
        ("nbtim", C.c_int32), ("threads", C.c_int32), ("pad", C.c_int32),
    ]


class ReplicaSpec(C.Structure):
    """clmd_replica_spec (include/clmd.h)."""

    _fields_ = [
        ("box", C.c_double), ("temp", C.c_double), ("Q", C.c_double), ("natom", C.c_int32),
        ("csover", C.c_int32), ("clwait", C.c_int32), ("budget", C.c_int32),
        ("ethst", C.c_char), ("pad", C.c_char * 7),
    ]


class ReplicaResult(C.Structure):
    """clmd_replica_result (include/clmd.h)."""

    _fields_ = [
        ("ekin", C.c_double), ("epot", C.c_double), ("psi", C.c_double), ("s", C.c_double),
        ("slot", C.c_int32), ("natom", C.c_int32), ("step", C.c_int32), ("status", C.c_int32),
        ("done", C.c_int32), ("clbrkt", C.c_int32), ("maxcs", C.c_int32),
        ("nrebuild", C.c_int32),
    ]


class RatesAcc(C.Structure):
    """clmd_rates_acc (include/clmd.h): the /CVTPP/ counters of rates()."""

    _fields_ = [("mcts", C.c_double), ("omcts", C.c_double), ("ccn", C.c_int32),
                ("cen", C.c_int32)]


class Request(C.Structure):
    """clmd_request (include/clmd.h)."""

    _fields_ = [
        ("arrival", C.c_double), ("rho", C.c_double), ("temp", C.c_double),
        ("seed", C.c_uint64), ("natom", C.c_int32), ("budget", C.c_int32),
        ("csover", C.c_int32), ("pad", C.c_int32),
    ]


class RequestResult(C.Structure):
    """clmd_request_result (include/clmd.h)."""

    _fields_ = [
        ("arrival", C.c_double), ("admitted", C.c_double), ("finished", C.c_double),
        ("natom", C.c_int32), ("steps", C.c_int32), ("done", C.c_int32), ("clbrkt", C.c_int32),
        ("status", C.c_int32), ("pad", C.c_int32),
    ]


class ServeStats(C.Structure):
    """clmd_serve_stats (include/clmd.h)."""

    _fields_ = [
        ("wall", C.c_double), ("atom_steps", C.c_double), ("windows", C.c_int32),
        ("admitted", C.c_int32), ("completed", C.c_int32), ("peak_resident", C.c_int32),
        ("peak_atoms", C.c_int64),
    ]


# (name, dtype, length kind) of every cluster output: "N" or "N1" (= N+1)
CLUSTER_FIELDS = [
    ("cl", np.int32, "N"), ("cs", np.int32, "N"), ("csi", np.int32, "N1"),
    ("cek", np.float64, "N"), ("ceks", np.float64, "N1"),
    ("clf", np.int32, "N"), ("csf", np.int32, "N1"), ("csif", np.int32, "N1"),
    ("cekf", np.float64, "N1"), ("ceksf", np.float64, "N1"),
    ("cgs", np.int32, "N"), ("cgsa", np.int32, "N"), ("cgsf", np.int32, "N1"),
    ("cgsfa", np.int32, "N1"), ("cfpt", np.int32, "N"), ("cfptf", np.int32, "N"),
]


def ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


_lib = None


def load(path: str = LIB_PATH):
    """Loads libclmd.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"libclmd.so not found at {path}: build it with `make -C {HERE}` "
            "(the engine has no CPU fallback)")
    lib = C.CDLL(path)
    P = C.c_void_p
    d = C.POINTER(C.c_double)
    i = C.POINTER(C.c_int32)
    sig = {
        "clmd_create": ([C.POINTER(Config), C.POINTER(P)], C.c_int),
        "clmd_destroy": ([P], C.c_int),
        "clmd_set_state": ([P, d, d, d, d, d, d, d, d, d, i, C.POINTER(Scalars)], C.c_int),
        "clmd_get_state": ([P, d, d, d, d, d, d, d, d, d, C.POINTER(Scalars)], C.c_int),
        "clmd_get_scalars": ([P, C.POINTER(Scalars)], C.c_int),
        "clmd_set_scalars": ([P, C.POINTER(Scalars)], C.c_int),
        "clmd_clear_status": ([P], C.c_int),
        "clmd_neighbor": ([P, i], C.c_int),
        "clmd_accatom": ([P], C.c_int),
        "clmd_accwall": ([P], C.c_int),
        "clmd_zero_acc": ([P], C.c_int),
        "clmd_integrator": ([P, C.c_int32], C.c_int),
        "clmd_thermostat": ([P, C.c_int32], C.c_int),
        "clmd_stopdead": ([P, C.c_int32], C.c_int),
        "clmd_stoddard": ([P, C.c_int32], C.c_int),
        "clmd_chk_nucleation": ([P, i], C.c_int),
        "clmd_run": ([P, C.c_int32, C.c_int32, i], C.c_int),
        "clmd_steps": ([P, C.c_int32, C.c_int32], C.c_int),
        "clmd_set_device": ([C.c_int], C.c_int),
        "clmd_get_halflist": ([P, i, C.c_int64, i, C.POINTER(C.c_int64)], C.c_int),
        "clmd_get_clusters": ([P, C.POINTER(ClusterView)], C.c_int),
        "clmd_synchronize": ([P], C.c_int),
        "clmd_stream": ([P], C.c_void_p),
        "clmd_kernel_launches": ([P], C.c_int64),
        "clmd_init_random": ([C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                              C.c_double, C.c_uint64, d, d, d, d, d, d], C.c_int),
        "clmd_status_string": ([C.c_int], C.c_char_p),
        "clmd_last_status": ([], C.c_int32),
        "clmd_struct_size": ([C.c_int], C.c_int64),
        "clmd_scalars_init": ([C.POINTER(Config), C.POINTER(Scalars)], None),
        "clmd_ens_create": ([C.POINTER(EnsConfig), C.POINTER(P)], C.c_int),
        "clmd_ens_destroy": ([P], C.c_int),
        "clmd_ens_add": ([P, C.POINTER(ReplicaSpec), d, d, d, d, d, d, i], C.c_int),
        "clmd_ens_step": ([P, C.c_int32], C.c_int),
        "clmd_ens_step_timed": ([P, C.c_float], C.c_int),
        "clmd_ens_autotune": ([P, i], C.c_int),
        "clmd_ens_results": ([P, C.POINTER(ReplicaResult), C.c_int32, i], C.c_int),
        "clmd_ens_poll": ([P, C.POINTER(ReplicaResult), C.c_int32, i], C.c_int),
        "clmd_ens_remove": ([P, C.c_int32], C.c_int),
        "clmd_serve": ([P, C.POINTER(Request), C.c_int32, C.c_double,
                        C.POINTER(RequestResult), C.POINTER(ServeStats)], C.c_int),
        "clmd_ens_get_state": ([P, C.c_int32, d, d, d, d, d, d, d, d, d, i], C.c_int),
        "clmd_ens_fpt": ([P, C.c_int32, i, C.c_int32], C.c_int),
        "clmd_ens_mfpt": ([P, C.c_int32, d, d, i], C.c_int),
        "clmd_get_config": ([P, C.POINTER(Config)], C.c_int),
        "clmd_write_rst": ([P, C.c_char_p, C.c_int32], C.c_int),
        "clmd_read_rst": ([P, C.c_char_p, i], C.c_int),
        "clmd_write_csi": ([P, C.c_int32, C.c_char_p, C.c_char_p], C.c_int),
        "clmd_write_fpt": ([P, C.c_char_p], C.c_int),
        "clmd_rates": ([P, C.c_int32, C.c_int32, C.POINTER(RatesAcc), C.c_char_p, C.c_char_p],
                       C.c_int),
        "clmd_thermostat_clu": ([P, C.c_int32, C.c_char, C.c_int32], C.c_int),
        "clmd_ens_write_rst": ([P, C.c_int32, C.c_char_p, C.c_int32], C.c_int),
        "clmd_ens_write_fpt": ([P, C.c_int32, C.c_double, C.c_char_p], C.c_int),
        "clmd_ens_upload": ([P, d, d, d, d, d, d], C.c_int),
        "clmd_ens_last_ms": ([P, C.POINTER(C.c_float), C.POINTER(C.c_int64)], C.c_int),
        "clmd_ens_download": ([P, d, d, d, d, d, d], C.c_int),
        "clmd_ens_step_io": ([P, C.c_int32, d, d, d, d, d, d], C.c_int),
        "clmd_ens_free_atoms": ([P], C.c_int64),
        "clmd_ens_launches": ([P], C.c_int64),
        "clmd_ens_pair_terms": ([P, C.POINTER(C.c_int64)], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def set_device(dev: int):
    st = load().clmd_set_device(dev)
    if st:
        raise ClmdError(st, "clmd_set_device")


def status_string(code: int) -> str:
    return load().clmd_status_string(code).decode()


class ClmdError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        super().__init__(f"{what}: status {code} ({status_string(code)})")


def lj_config(n, rho, temp, *, rc=2.5, rskin=2.8, atskin=1.5, dt=0.005, nbtim=10,
              integrator=INT_VERLET, clustering=CLU_STILLINGER, ftcsi=100, csover=0,
              clwait=0, clnuctrl="-", ethst="-", q=None, atnenum=5, btim=0,
              precision=PREC_FP64, nlist_cap=0, species=None) -> Config:
    """A reduced-unit LJ configuration (sigma = eps = m = 1) at number density
    rho and temperature T* in a cubic box; `species` optionally gives a second
    species as dict(n=..., sigma=..., eps=..., mass=..., thermo='X')."""
    c = Config()
    L = (n / rho) ** (1.0 / 3.0)
    c.boxx = c.boxy = c.boxz = L
    c.natom = n
    c.apmas[0] = 1.0
    c.apsig[0] = 1.0
    c.apeps[0] = 1.0
    apth = [b"-"] * MXSORTS
    if species:
        n2 = species["n"]
        c.atsorts = 2
        c.apnum[0] = n - n2
        c.apnum[1] = n2
        c.apmas[1] = species.get("mass", 1.0)
        c.apsig[1] = species.get("sigma", 1.0)
        c.apeps[1] = species.get("eps", 1.0)
        apth[1] = species.get("thermo", "-").encode()
    else:
        c.atsorts = 1
        c.apnum[0] = n
    c.apth = b"".join(apth)
    c.att = temp / CIKB
    c.atskin = atskin
    c.atrcut = rc
    c.atrskin = rskin
    c.dt = dt
    c.nbtim = nbtim
    c.btim = btim
    c.integrator = integrator
    c.clustering = clustering
    c.ftcsi = ftcsi
    c.csover = csover
    c.clwait = clwait
    c.clnuctrl = clnuctrl.encode()
    c.ethst = ethst.encode()
    c.atnenum = atnenum
    c.precision = precision
    c.nlist_cap = nlist_cap
    # Q = N T* (0.5)^2 in reduced units (the Q_in of the deck times m sigma^2)
    c.Q = q if q is not None else n * temp * 0.25
    return c


def init_random(n, box, rmin, kt_over_m, seed):
    """Seeded start: positions uniform with all pairs >= rmin apart,
    Maxwell-Boltzmann velocities (host code in libclmd.so)."""
    lib = load()
    arrs = [np.zeros(n) for _ in range(6)]
    bx, by, bz = box
    st = lib.clmd_init_random(n, bx, by, bz, rmin, kt_over_m, seed,
                              *[ptr(a, C.c_double) for a in arrs])
    if st:
        raise ClmdError(st, "clmd_init_random")
    x, y, z, vx, vy, vz = arrs
    return x, y, z, vx, vy, vz


def scalars_init(cfg: Config) -> Scalars:
    s = Scalars()
    load().clmd_scalars_init(C.byref(cfg), C.byref(s))
    return s


@dataclass
class State:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    ax: np.ndarray
    ay: np.ndarray
    az: np.ndarray

    def copy(self):
        return State(*[getattr(self, k).copy() for k in self.__dataclass_fields__])

    def arrays(self):
        return [getattr(self, k) for k in self.__dataclass_fields__]


class System:
    """One device-resident system (clmd_system*)."""

    def __init__(self, cfg: Config):
        self.lib = load()
        self.cfg = cfg
        self.n = cfg.natom
        h = C.c_void_p()
        st = self.lib.clmd_create(C.byref(cfg), C.byref(h))
        if st:
            raise ClmdError(st, "clmd_create")
        self.h = h

    def close(self):
        if self.h:
            self.lib.clmd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st, what):
        if st not in (OK,) and st > ERR_BAD_SPECIES:
            raise ClmdError(st, what)
        return st

    # -- state -------------------------------------------------------------
    def set_state(self, state: State | None = None, api=None, scalars: Scalars | None = None):
        arrs = state.arrays() if state is not None else [None] * 9
        arrs = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
                for a in arrs]
        a = np.ascontiguousarray(api, dtype=np.int32) if api is not None else None
        st = self.lib.clmd_set_state(self.h, *[ptr(v, C.c_double) for v in arrs],
                                     ptr(a, C.c_int32),
                                     C.byref(scalars) if scalars is not None else None)
        return self._chk(st, "clmd_set_state")

    def get_state(self) -> State:
        arrs = [np.zeros(self.n) for _ in range(9)]
        st = self.lib.clmd_get_state(self.h, *[ptr(v, C.c_double) for v in arrs], None)
        self._chk(st, "clmd_get_state")
        return State(*arrs)

    def scalars(self) -> Scalars:
        s = Scalars()
        self._chk(self.lib.clmd_get_scalars(self.h, C.byref(s)), "clmd_get_scalars")
        return s

    def set_scalars(self, s: Scalars):
        return self._chk(self.lib.clmd_set_scalars(self.h, C.byref(s)), "clmd_set_scalars")

    def clear_status(self):
        return self.lib.clmd_clear_status(self.h)

    # -- the reference's subroutines ------------------------------------------
    def neighbor(self, step):
        s = C.c_int32(step)
        st = self._chk(self.lib.clmd_neighbor(self.h, C.byref(s)), "neighbor")
        return st, s.value

    def accatom(self):
        return self._chk(self.lib.clmd_accatom(self.h), "accatom")

    def accwall(self):
        return self._chk(self.lib.clmd_accwall(self.h), "accwall")

    def zero_acc(self):
        return self._chk(self.lib.clmd_zero_acc(self.h), "zero_acc")

    def integrator(self, step):
        return self._chk(self.lib.clmd_integrator(self.h, step), "integrator")

    def thermostat(self, step):
        return self._chk(self.lib.clmd_thermostat(self.h, step), "thermostat")

    def thermostat_clu(self, step, eclth, ecltim):
        """scalev-clu.f: cluster and gas scaled separately every ecltim."""
        self._chk(self.lib.clmd_thermostat_clu(self.h, step, eclth.encode(), ecltim),
                  "thermostat_clu")

    def stopdead(self, step):
        return self._chk(self.lib.clmd_stopdead(self.h, step), "stopdead")

    def stoddard(self, step):
        return self._chk(self.lib.clmd_stoddard(self.h, step), "stoddard")

    def chk_nucleation(self, step):
        s = C.c_int32(step)
        st = self._chk(self.lib.clmd_chk_nucleation(self.h, C.byref(s)), "chk_nucleation")
        return st, s.value

    def run(self, first, nsteps):
        nxt = C.c_int32(0)
        st = self._chk(self.lib.clmd_run(self.h, first, nsteps, C.byref(nxt)), "run")
        return st, nxt.value

    def steps(self, first, nsteps):
        """nsteps integrator() calls in one launch of the step kernel."""
        return self._chk(self.lib.clmd_steps(self.h, first, nsteps), "steps")

    def synchronize(self):
        return self._chk(self.lib.clmd_synchronize(self.h), "synchronize")

    def stream(self):
        return self.lib.clmd_stream(self.h)

    def kernel_launches(self):
        return self.lib.clmd_kernel_launches(self.h)

    # -- outputs -------------------------------------------------------------
    def write_rst(self, path, mxa=0):
        """wrt-rst.f: the reference's restart file (+ the engine record)."""
        self._chk(self.lib.clmd_write_rst(self.h, os.fsencode(path), mxa), "write_rst")

    def read_rst(self, path):
        """read-rst.f: state from a restart file, then neighbor(btim);
        returns btim."""
        st = C.c_int32(0)
        self._chk(self.lib.clmd_read_rst(self.h, os.fsencode(path), C.byref(st)), "read_rst")
        return st.value

    def write_csi(self, step, csi_path, fsi_path=None):
        """wrt-csi.f / wrt-csi-fre.f: append this analysis to the files."""
        self._chk(self.lib.clmd_write_csi(self.h, step, os.fsencode(csi_path),
                                          os.fsencode(fsi_path) if fsi_path else None),
                  "write_csi")

    def rates(self, step, ctrat, acc, out, log=None):
        """rates.f: evaporation/condensation of the largest cluster (appends
        to out; the size-change lines go to log, None = stdout)."""
        self._chk(self.lib.clmd_rates(self.h, step, ctrat, C.byref(acc), os.fsencode(out),
                                      os.fsencode(log) if log else None), "rates")

    def write_fpt(self, path):
        """wrt-fpt.f: append the first-passage table."""
        self._chk(self.lib.clmd_write_fpt(self.h, os.fsencode(path)), "write_fpt")

    def halflist(self):
        """(atnlist, atnidx) in the reference's layout (1-based values)."""
        n = C.c_int64(0)
        self._chk(self.lib.clmd_get_halflist(self.h, None, 0, None, C.byref(n)), "halflist")
        lst = np.zeros(max(n.value, 1), dtype=np.int32)
        idx = np.zeros(self.n, dtype=np.int32)
        self._chk(self.lib.clmd_get_halflist(self.h, ptr(lst, C.c_int32), n.value,
                                             ptr(idx, C.c_int32), C.byref(n)), "halflist")
        return lst[: n.value], idx

    def clusters(self) -> dict:
        out = {}
        v = ClusterView()
        for name, dt, kind in CLUSTER_FIELDS:
            a = np.zeros(self.n + (1 if kind == "N1" else 0), dtype=dt)
            out[name] = a
            setattr(v, name, ptr(a, C.c_int32 if dt == np.int32 else C.c_double))
        self._chk(self.lib.clmd_get_clusters(self.h, C.byref(v)), "clusters")
        return out


ENS_LEAN = 0x10000  # CLMD_ENS_LEAN: the 64-register variant of a 128/256/512-thread CTA
ENS_LANES_SHIFT = 20  # CLMD_ENS_LANES_SHIFT: 1 << field lanes per atom (mixed forces)


def ens_lanes(n):
    """The block-shape bits for n (1, 2 or 4) lanes per atom in the mixed
    force pass."""
    return {1: 0, 2: 1, 4: 2}[n] << ENS_LANES_SHIFT


def shape_name(shape):
    """A block shape as text: '256', '256 lean (64 regs)', '1024, 2 lanes/atom'."""
    t = shape & 0xFFFF
    out = f"{t} lean (64 regs)" if shape & ENS_LEAN else str(t)
    lanes = 1 << ((shape >> ENS_LANES_SHIFT) & 3)
    return out + (f", {lanes} lanes/atom" if lanes > 1 else "")


def ens_config(max_atoms, max_replicas, *, precision=PREC_MIXED, integrator=INT_NOSE, ftcsi=100,
               rc=2.5, rskin=2.8, atskin=1.5, dt=0.005, nbtim=10, list_stride=0, threads=0):
    c = EnsConfig()
    c.rc, c.rskin, c.atskin, c.dt = rc, rskin, atskin, dt
    c.max_atoms, c.max_replicas = max_atoms, max_replicas
    c.list_stride, c.precision, c.integrator = list_stride, precision, integrator
    c.ftcsi, c.nbtim, c.threads = ftcsi, nbtim, threads
    return c


class Ensemble:
    """Independent replicas advanced together (clmd_ensemble*)."""

    def __init__(self, cfg: EnsConfig):
        self.lib = load()
        self.cfg = cfg
        h = C.c_void_p()
        st = self.lib.clmd_ens_create(C.byref(cfg), C.byref(h))
        if st:
            raise ClmdError(st, "clmd_ens_create")
        self.h = h
        self.natom = {}

    def close(self):
        if self.h:
            self.lib.clmd_ens_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, natom, box, temp, x, y, z, vx, vy, vz, *, csover=0, clwait=0, budget=0,
            ethst="N", q=0.0):
        """Admits a replica; returns its slot, or None if there is no room."""
        sp = ReplicaSpec()
        sp.natom, sp.box, sp.temp, sp.Q = natom, box, temp, q
        sp.csover, sp.clwait, sp.budget = csover, clwait, budget
        sp.ethst = ethst.encode()
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, vx, vy, vz)]
        slot = C.c_int32(-1)
        st = self.lib.clmd_ens_add(self.h, C.byref(sp), *[ptr(a, C.c_double) for a in arrs],
                                   C.byref(slot))
        if st == ERR_NOMEM:
            return None
        if st:
            raise ClmdError(st, "clmd_ens_add")
        self.natom[slot.value] = natom
        return slot.value

    def step(self, nwin=1):
        st = self.lib.clmd_ens_step(self.h, nwin)
        if st:
            raise ClmdError(st, "clmd_ens_step")

    def step_io(self, nwin, ptrs):
        """clmd_ens_step_io: upload, nwin windows and download in one call,
        the copies done by the window kernel.  ptrs: six ctypes double
        pointers to pinned host arrays in the upload/download layout."""
        st = self.lib.clmd_ens_step_io(self.h, nwin, *ptrs)
        if st:
            raise ClmdError(st, "clmd_ens_step_io")

    def step_timed(self, ms):
        """Balanced step: each replica runs as many MD steps as fit in about
        ms of device time (at least one)."""
        st = self.lib.clmd_ens_step_timed(self.h, ms)
        if st:
            raise ClmdError(st, "clmd_ens_step_timed")

    def autotune(self):
        """Block shape per replica-size class, picked by timing (7 windows):
        threads per CTA, | ENS_LEAN for the 64-register variant."""
        out = (C.c_int32 * 4)()
        st = self.lib.clmd_ens_autotune(self.h, out)
        if st:
            raise ClmdError(st, "clmd_ens_autotune")
        return list(out)

    def results(self):
        cap = len(self.natom) + 1
        out = (ReplicaResult * cap)()
        n = C.c_int32(0)
        st = self.lib.clmd_ens_results(self.h, out, cap, C.byref(n))
        if st:
            raise ClmdError(st, "clmd_ens_results")
        return {out[k].slot: out[k] for k in range(n.value)}

    def poll(self):
        """Cheap per-window status (full record only for finished replicas)."""
        cap = len(self.natom) + 1
        out = (ReplicaResult * cap)()
        n = C.c_int32(0)
        st = self.lib.clmd_ens_poll(self.h, out, cap, C.byref(n))
        if st:
            raise ClmdError(st, "clmd_ens_poll")
        return {out[k].slot: out[k] for k in range(n.value)}

    def serve(self, requests, max_seconds):
        """Runs a request trace (a sequence of Request) through the served
        loop; returns (list of RequestResult, ServeStats)."""
        n = len(requests)
        reqs = (Request * max(n, 1))(*requests)
        out = (RequestResult * max(n, 1))()
        stats = ServeStats()
        st = self.lib.clmd_serve(self.h, reqs, n, max_seconds, out, C.byref(stats))
        if st:
            raise ClmdError(st, "clmd_serve")
        return [out[k] for k in range(n)], stats

    def remove(self, slot):
        st = self.lib.clmd_ens_remove(self.h, slot)
        if st:
            raise ClmdError(st, "clmd_ens_remove")
        self.natom.pop(slot, None)

    def state(self, slot):
        n = self.natom[slot]
        arrs = [np.zeros(n) for _ in range(9)]
        cl = np.zeros(n, dtype=np.int32)
        st = self.lib.clmd_ens_get_state(self.h, slot, *[ptr(a, C.c_double) for a in arrs],
                                         ptr(cl, C.c_int32))
        if st:
            raise ClmdError(st, "clmd_ens_get_state")
        return State(*arrs), cl

    def fpt(self, slot, cap=128):
        a = np.zeros(cap, dtype=np.int32)
        st = self.lib.clmd_ens_fpt(self.h, slot, ptr(a, C.c_int32), cap)
        if st:
            raise ClmdError(st, "clmd_ens_fpt")
        return a

    def mfpt(self, cap=128):
        """Per size 1..cap: (mean first-passage step, standard error, count)
        over the occupied slots (helpers/mpt.f on the device)."""
        mean, sem = np.zeros(cap), np.zeros(cap)
        cnt = np.zeros(cap, dtype=np.int32)
        st = self.lib.clmd_ens_mfpt(self.h, cap, ptr(mean, C.c_double), ptr(sem, C.c_double),
                                    ptr(cnt, C.c_int32))
        if st:
            raise ClmdError(st, "clmd_ens_mfpt")
        return mean, sem, cnt

    def write_rst(self, slot, path, mxa=0):
        st = self.lib.clmd_ens_write_rst(self.h, slot, os.fsencode(path), mxa)
        if st:
            raise ClmdError(st, "clmd_ens_write_rst")

    def write_fpt(self, slot, dt, path):
        st = self.lib.clmd_ens_write_fpt(self.h, slot, dt, os.fsencode(path))
        if st:
            raise ClmdError(st, "clmd_ens_write_fpt")

    def last_ms(self):
        """Device ms and atoms of the last window, per size class."""
        ms = (C.c_float * 4)()
        at = (C.c_int64 * 4)()
        self.lib.clmd_ens_last_ms(self.h, ms, at)
        return list(ms), list(at)

    def free_atoms(self):
        return self.lib.clmd_ens_free_atoms(self.h)

    def launches(self):
        return self.lib.clmd_ens_launches(self.h)

    def pair_terms(self):
        """Pair terms the force passes of the current replicas evaluated."""
        t = C.c_int64(0)
        st = self.lib.clmd_ens_pair_terms(self.h, C.byref(t))
        if st:
            raise ClmdError(st, "clmd_ens_pair_terms")
        return t.value
