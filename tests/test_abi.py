"""The C ABI boundary on CPU: libclmd.so loads, exports every function and
common block that include/*.h declares, and its struct layouts match the
bindings.  No compute call needs a GPU here."""
import ctypes as C
import os
import re

import pytest

import clmd
from conftest import REPO

HEADERS = [os.path.join(REPO, "include", h) for h in ("clmd.h", "clmd_f77.h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b([a-z_][a-z0-9_]*)\s*\(", text, re.M):
            name = m.group(1)
            if name in ("sizeof", "if", "return"):
                continue
            names.add(name)
    return sorted(names)


def declared_commons():
    text = open(HEADERS[1]).read()
    return re.findall(r"^extern\s+\w+\s+(\w+_);", text, re.M)


def test_library_loads():
    lib = clmd.load()
    assert lib is not None


@pytest.mark.parametrize("name", declared_functions())
def test_function_exported(name):
    lib = C.CDLL(clmd.LIB_PATH)
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


@pytest.mark.parametrize("name", declared_commons())
def test_common_block_exported(name):
    lib = C.CDLL(clmd.LIB_PATH)
    assert C.c_char.in_dll(lib, name) is not None


def test_struct_layouts_match_bindings():
    lib = clmd.load()
    assert lib.clmd_struct_size(0) == C.sizeof(clmd.Config)
    assert lib.clmd_struct_size(1) == C.sizeof(clmd.Scalars)
    assert lib.clmd_struct_size(2) == C.sizeof(clmd.ClusterView)
    assert lib.clmd_struct_size(3) == C.sizeof(clmd.EnsConfig)
    assert lib.clmd_struct_size(4) == C.sizeof(clmd.ReplicaSpec)
    assert lib.clmd_struct_size(5) == C.sizeof(clmd.ReplicaResult)
    assert lib.clmd_struct_size(6) == C.sizeof(clmd.Request)
    assert lib.clmd_struct_size(7) == C.sizeof(clmd.RequestResult)
    assert lib.clmd_struct_size(8) == C.sizeof(clmd.ServeStats)


def test_no_device_is_reported_not_faked():
    """Without a GPU the engine refuses to create a system: no CPU path."""
    from conftest import have_gpu
    if have_gpu():
        pytest.skip("a GPU is visible")
    cfg = clmd.lj_config(100, 0.05, 0.7)
    with pytest.raises(clmd.ClmdError) as e:
        clmd.System(cfg)
    assert e.value.code == clmd.ERR_NO_DEVICE


def test_status_strings_carry_reference_messages():
    assert "Skin radius exceeded" in clmd.status_string(clmd.ERR_SKIN)
    assert "Neighborlist is nearly full" in clmd.status_string(clmd.ERR_LIST_OVERFLOW)
    assert "did not converge" in clmd.status_string(clmd.ERR_NH_NOCONVERGE)


def test_init_random_respects_min_distance():
    import numpy as np
    n, L = 400, 20.0
    x, y, z, vx, vy, vz = clmd.init_random(n, (L, L, L), 0.9, 0.7, 5)
    p = np.stack([x, y, z], 1)
    d = p[:, None, :] - p[None, :, :]
    d -= L * np.round(d / L)
    r2 = (d ** 2).sum(-1) + np.eye(n) * 1e9
    assert r2.min() >= 0.81 - 1e-12
    assert 0.5 < np.var(np.concatenate([vx, vy, vz])) < 0.9
