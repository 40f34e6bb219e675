"""The .3d deck (read-3d.f:11-302): the oracle's restatement and the
library's reader (clmd_f77_readdata, filling the common blocks) agree on
decks in the reference's fixed-column format, versions 1.30 and 1.12, and
apply the reference's unit conversions (nm -> A, u -> 1e-27 kg,
K -> 1e-17 J, Q * m sigma^2)."""
import ctypes as C
import os

import numpy as np
import pytest

import clmd
import orc
from conftest import REPO

MXA, MXS = 6000, 10
MXN = MXA * MXA // 4


class ATOMP(C.Structure):
    _fields_ = [("natom", C.c_int32), ("atsorts", C.c_int32), ("apnum", C.c_int32 * MXS),
                ("apmas", C.c_double * MXS), ("apsig", C.c_double * MXS),
                ("apeps", C.c_double * MXS), ("appr", C.c_double * MXS),
                ("appa", C.c_double * MXS), ("atskin", C.c_double), ("atrskin", C.c_double),
                ("atrcut", C.c_double), ("att", C.c_double), ("psi", C.c_double),
                ("Q", C.c_double), ("s", C.c_double), ("atnlist", C.c_int32 * MXN),
                ("atnidx", C.c_int32 * MXA), ("api", C.c_int32 * MXA),
                ("apnnum", C.c_int32 * MXS), ("atnenum", C.c_int32),
                ("apsym", C.c_char * (2 * MXS)), ("apsymi", C.c_char * (2 * MXA)),
                ("apth", C.c_char * MXS), ("apNch", C.c_char * MXS), ("rndctrl", C.c_char)]


class BOXPP(C.Structure):
    _fields_ = [("boxx", C.c_double), ("boxy", C.c_double), ("boxz", C.c_double)]


class TIMEP(C.Structure):
    _fields_ = [("dt", C.c_double), ("ntim", C.c_int32), ("btim", C.c_int32),
                ("sctim", C.c_int32), ("nbtim", C.c_int32), ("chgNtim", C.c_int32)]


class DMMPP(C.Structure):
    _fields_ = [("dmmh", C.c_double * 256), ("dmmx", C.c_double), ("dmmy", C.c_double),
                ("dmmz", C.c_double), ("dmms", C.c_double), ("dmmsu", C.c_double),
                ("dmmax", C.c_double), ("dmmav", C.c_double), ("dmmst", C.c_int32),
                ("dmmi", C.c_int32)]


DECKS = ["nose_vapour.3d", "silent_v112.3d"]


@pytest.mark.parametrize("deck", DECKS)
def test_deck_readers_agree(deck):
    path = os.path.join(REPO, "tests", "golden", deck)
    cfg, ntim, sctim = orc.readdata(path)
    lib = clmd.load()
    lib.clmd_f77_readdata.argtypes = [C.c_char_p]
    P = ATOMP.in_dll(lib, "atomp_")
    # a fresh program's commons: read-3d.f:255 scales whatever Q holds, and
    # decks older than 1.2 do not read one
    P.Q = 0.0
    assert lib.clmd_f77_readdata(path.encode()) == 0
    B = BOXPP.in_dll(lib, "boxpp_")
    T = TIMEP.in_dll(lib, "timep_")
    D = DMMPP.in_dll(lib, "dmmpp_")
    assert P.natom == cfg.natom == 2000
    assert P.atsorts == cfg.atsorts == 2
    assert list(P.apnum[:2]) == list(cfg.apnum[:2]) == [1500, 500]
    for f in ("apmas", "apsig", "apeps"):
        assert list(getattr(P, f)[:2]) == list(getattr(cfg, f)[:2]), f
    for f in ("atskin", "atrcut", "atrskin", "att", "Q"):
        assert getattr(P, f) == getattr(cfg, f), f
    assert (B.boxx, B.boxy, B.boxz) == (cfg.boxx, cfg.boxy, cfg.boxz)
    assert T.dt == cfg.dt and T.nbtim == cfg.nbtim and T.ntim == ntim and T.sctim == sctim
    # unit conversions (read-3d.f:152-161, 246-261)
    assert cfg.boxx == 15.80 * 10
    assert cfg.apmas[0] == 40.0 * clmd.CIMU
    assert cfg.apsig[0] == 0.3405 * 10.0
    assert cfg.apeps[0] == 120.0 * clmd.CIKB
    assert cfg.atrcut == 2.5 * cfg.apsig[0]
    assert list(P.api[:2000]) == [1] * 1500 + [2] * 500
    # the skin history is seeded (read-3d.f:263-269)
    assert D.dmmh[0] == (cfg.atrskin - cfg.atrcut) / float(np.float32(cfg.nbtim))
    if deck.startswith("nose"):
        assert cfg.Q == 750.0 * cfg.apmas[0] * cfg.apsig[0] * cfg.apsig[0]
        assert cfg.atnenum == 5 and cfg.ethst == b"N"
        assert cfg.csover == 51 and cfg.clwait == 200 and cfg.clnuctrl == b"X"
    else:
        assert cfg.Q == 0.0 and cfg.atnenum == 0


def test_common_block_sizes_cover_layout():
    lib = clmd.load()
    # the library defines the commons at least as large as the .inc files say
    assert C.sizeof(ATOMP) <= 36060592
    assert ATOMP.in_dll(lib, "atomp_") is not None
