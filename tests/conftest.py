"""Shared test setup: import paths, the gpu marker, state builders.

CPU tests (default) check the oracle against the golden fixtures and known
answers, and the C ABI's exports; `-m gpu` tests are the parity tests of the
CUDA engine against the oracle, through the C ABI.
"""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "fortran-cluster-md_b200")
for p in (PKG, os.path.join(REPO, "oracle"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libclmd.so")


def have_gpu():
    try:
        import torch  # noqa: F401  (only to ask whether a device exists)
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not have_gpu():
        pytest.skip("no CUDA device")
    import clmd
    clmd.load()
    return True


def random_state(cfg, seed, rmin=0.9, temp=None):
    """Seeded start: uniform positions with pairs >= rmin, MB velocities, a=0."""
    import clmd
    n = cfg.natom
    kt = temp if temp is not None else cfg.att * clmd.CIKB
    x, y, z, vx, vy, vz = clmd.init_random(n, (cfg.boxx, cfg.boxy, cfg.boxz), rmin, kt, seed)
    return clmd.State(x, y, z, vx, vy, vz, np.zeros(n), np.zeros(n), np.zeros(n))


def start_pair(g, o, cfg, state, api=None):
    """The start sequence (commons from the config as read-3d.f:263-276,
    stopdead(-1), neighbor(0), a = 0, AccAtom) on the engine g and the oracle
    o from one input.  stopdead's rescale factor comes from a global sum
    whose rounding depends on summation order, so the oracle's post-stopdead
    state is handed to both; from there on the FP64 velocity-Verlet path has
    no sum that feeds back into per-atom values."""
    import orc
    o.set_state(state, api=api, scalars=orc.scalars_init(cfg))
    o.stopdead(-1)
    g.set_state(o.get_state(), api=api, scalars=o.scalars())
    for s_ in (g, o):
        s_.neighbor(0)
        s_.zero_acc()
        s_.accatom()
