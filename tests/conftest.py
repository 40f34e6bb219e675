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


def droplet_state(cfg, seed, ndrop, radius, spacing=1.1, rmin=0.9, temp=None):
    """A vapour holding `ndrop` liquid-like droplets: simple-cubic blobs of
    the given spacing (every interior atom has 6 neighbours at `spacing`)
    inside spheres of `radius`, the other atoms from the seeded start
    generator (no pair nearer than rmin) with those within rmin of a
    droplet's sphere removed; Maxwell-Boltzmann velocities.  The oracle and
    the engine then get identical inputs."""
    import clmd
    import orc
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    n, L = cfg.natom, cfg.boxx
    g = np.arange(-radius, radius + 1e-9, spacing)
    gx, gy, gz = np.meshgrid(g, g, g, indexing="ij")
    blob = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], 1)
    blob = blob[np.linalg.norm(blob, axis=1) <= radius]
    centres = []
    while len(centres) < ndrop:
        c = rng.uniform(0, L, 3)
        if all(np.linalg.norm((c - q + L / 2) % L - L / 2) > 2 * radius + 3 for q in centres):
            centres.append(c)
    drops = (np.concatenate([blob + c for c in centres]) % L) if ndrop else np.zeros((0, 3))
    need = n - len(drops)
    assert need > 0
    rho = n / L ** 3
    margin = int(1.5 * rho * ndrop * 4.19 * (radius + rmin) ** 3) + 64
    for attempt in range(8):
        m = need + margin
        gx_, gy_, gz_, _, _, _ = orc.init_random(m, (L, L, L), rmin, 0.0, seed * 7919 + attempt)
        gas = np.stack([gx_, gy_, gz_], 1)
        if ndrop:
            d, _ = cKDTree(np.array(centres) % L, boxsize=L).query(gas)
            gas = gas[d > radius + rmin]
        if len(gas) >= need:
            break
        margin *= 2
    else:
        raise RuntimeError("droplet_state: could not place the vapour")
    pos = np.concatenate([drops, gas[:need]])
    pos[pos >= L] -= L
    kt = temp if temp is not None else cfg.att * clmd.CIKB
    v = rng.normal(0.0, np.sqrt(kt), (n, 3))
    z = np.zeros(n)
    return clmd.State(pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(),
                      v[:, 0].copy(), v[:, 1].copy(), v[:, 2].copy(), z, z.copy(), z.copy())
