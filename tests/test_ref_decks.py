"""The reference's own input decks (tests/golden/ref_decks, copied byte for
byte from the reference's cluster/ folder) read by the library's .3d reader
(clmd_f77_readdata, into the common blocks) and by the oracle's, checked
against values derived by hand from read-3d.f:

  * column rules: `(41X,A)` takes column 42 (a label padded with a TAB is
    shorter, so sample.3d's first species gets a blank thermostat flag),
    `(40X,I10)` for ntim (read-3d.f:114), blanks ignored in numbers;
  * version gates (read-3d.f:100,121,133,170,175,182,186,193,198): a 1.11
    deck has no nucleation block, a 1.12 deck no Q and no atnenum;
  * unit conversions (:152-161, :246-248, :255, :259-261): nm -> 10 A,
    u -> cimu, K -> cikb, Q * m sigma^2 of species 1, radii in sigma(1);
  * the skin ring (:263-269);
  * the CRLF deck (sample-v1.12.3d) reads like its LF twin (gfortran ends a
    formatted record at CR LF);
  * two decks the reference itself cannot read stop with an error:
    sample-v1.2.3d declares version 1.12 but carries the 1.2 Q line, so
    every later read shifts by one line and an I10 field meets text;
    sample-old.3d declares 1.12 without the nucleation block, so csover's
    I10 field meets a ruler line.
"""
import ctypes as C
import os

import numpy as np
import pytest

import clmd
import orc
from conftest import REPO
from test_deck import ATOMP, BOXPP, DMMPP, TIMEP

DIR = os.path.join(REPO, "tests", "golden", "ref_decks")
CIMU, CIKB = 1.66056, 1.38066e-6


class ENERG(C.Structure):
    _fields_ = [("ekin", C.c_double), ("sumv2", C.c_double), ("epot", C.c_double),
                ("ekinA", C.c_double * 10), ("H", C.c_double), ("ewall", C.c_double),
                ("ewallsum", C.c_double), ("fwall", C.c_double), ("fwallsum", C.c_double),
                ("ecltim", C.c_int32), ("ethst", C.c_char), ("eclth", C.c_char)]


SIG1 = 0.3405 * 10.0
COMMON = dict(dt=2.0, ntim=100000, btim=0, sctim=1000, box=20.0 * 10, att=150.0,
              atskin=1.8 * SIG1, atrcut=5.0 * SIG1, atrskin=5.2 * SIG1, nbtim=100, ftcsi=1000)

EXPECT = {
    "sample.3d": dict(
        COMMON, natom=1000, atsorts=2, apnum=[125, 875], apmas=[40.0 * CIMU, 4.0 * CIMU],
        apsig=[SIG1, 0.258 * 10.0], apeps=[120.0 * CIKB, 10.22 * CIKB], apth=b" X",
        ethst=b"X", Q=2.0 * (40.0 * CIMU) * SIG1 * SIG1, atnenum=5, clnuctrl=b"-", csover=15,
        clwait=10000, ecltim=200, eclth=b"-", chgNtim=500),
    "sample-v1.12.3d": dict(
        COMMON, natom=1000, atsorts=2, apnum=[125, 875], apmas=[40.0 * CIMU, 4.0 * CIMU],
        apsig=[SIG1, 0.258 * 10.0], apeps=[120.0 * CIKB, 10.22 * CIKB], apth=b"-X",
        ethst=b"X", Q=0.0, atnenum=0, clnuctrl=b"-", csover=15, clwait=10000, ecltim=200,
        eclth=b"-", chgNtim=500),
    "test1.3d": dict(
        COMMON, natom=512, atsorts=1, apnum=[512], apmas=[40.0 * CIMU], apsig=[SIG1],
        apeps=[120.0 * CIKB], apth=b"X", ethst=b"-", Q=0.0, atnenum=0, clnuctrl=b"\x00",
        csover=0, clwait=0, ecltim=200, eclth=b"-", chgNtim=500),
}
UNREADABLE = ["sample-v1.2.3d", "sample-old.3d"]


MXA = 6000


class CVTPP(C.Structure):
    """cvtpp.inc:17-20 (the layout of include/clmd_f77.h)."""
    _fields_ = [("cek", C.c_double * MXA), ("cekf", C.c_double * (MXA + 1)),
                ("ceks", C.c_double * (MXA + 1)), ("ceksf", C.c_double * (MXA + 1)),
                ("mcts", C.c_double), ("omcts", C.c_double),
                ("cl", C.c_int32 * MXA), ("clf", C.c_int32 * MXA), ("cs", C.c_int32 * MXA),
                ("csf", C.c_int32 * (MXA + 1)), ("cc", C.c_int32 * MXA),
                ("ccf", C.c_int32 * MXA), ("csi", C.c_int32 * (MXA + 1)),
                ("csif", C.c_int32 * (MXA + 1)), ("cgs", C.c_int32 * MXA),
                ("cgsf", C.c_int32 * (MXA + 1)), ("cgsa", C.c_int32 * MXA),
                ("cgsfa", C.c_int32 * (MXA + 1)), ("cnum", C.c_int32), ("cnumf", C.c_int32),
                ("cfpt", C.c_int32 * MXA), ("cfptf", C.c_int32 * MXA), ("ccn", C.c_int32),
                ("cen", C.c_int32), ("ctrat", C.c_int32), ("cstep", C.c_int32),
                ("csover", C.c_int32), ("cbiggest", C.c_int32), ("cbiggestf", C.c_int32),
                ("clookfor", C.c_int32), ("clookforf", C.c_int32), ("clwait", C.c_int32),
                ("clbrkt", C.c_int32), ("clnuctrl", C.c_char)]


def _fresh_commons(lib):
    """The values a fresh program's commons hold in the fields that the
    older decks do not read."""
    P = ATOMP.in_dll(lib, "atomp_")
    P.Q = 0.0
    P.atnenum = 0
    cv = CVTPP.in_dll(lib, "cvtpp_")
    cv.csover = 0
    cv.clwait = 0
    cv.clnuctrl = b"\x00"


@pytest.fixture(scope="module")
def lib():
    lib = clmd.load()
    lib.clmd_f77_readdata.argtypes = [C.c_char_p]
    lib.clmd_f77_readdata.restype = C.c_int
    return lib


def cvtpp_scalars(lib):
    cv = CVTPP.in_dll(lib, "cvtpp_")
    return cv.csover, cv.clwait, cv.clnuctrl


@pytest.mark.parametrize("deck", sorted(EXPECT))
def test_oracle_reader_on_reference_deck(deck):
    e = EXPECT[deck]
    cfg, ntim, sctim = orc.readdata(os.path.join(DIR, deck))
    n = e["atsorts"]
    assert (cfg.natom, cfg.atsorts) == (e["natom"], n)
    assert list(cfg.apnum[:n]) == e["apnum"]
    assert list(cfg.apmas[:n]) == e["apmas"]
    assert list(cfg.apsig[:n]) == e["apsig"]
    assert list(cfg.apeps[:n]) == e["apeps"]
    assert bytes(cfg.apth[:n]) == e["apth"]
    assert (cfg.boxx, cfg.boxy, cfg.boxz) == (e["box"],) * 3
    assert (cfg.dt, ntim, cfg.btim, sctim, cfg.nbtim) == \
        (e["dt"], e["ntim"], e["btim"], e["sctim"], e["nbtim"])
    assert (cfg.att, cfg.atskin, cfg.atrcut, cfg.atrskin) == \
        (e["att"], e["atskin"], e["atrcut"], e["atrskin"])
    assert cfg.Q == e["Q"] and cfg.atnenum == e["atnenum"] and cfg.ftcsi == e["ftcsi"]
    assert cfg.ethst == e["ethst"]
    assert (cfg.csover, cfg.clwait) == (e["csover"], e["clwait"])
    assert cfg.clnuctrl == e["clnuctrl"]


@pytest.mark.parametrize("deck", sorted(EXPECT))
def test_library_reader_on_reference_deck(lib, deck):
    e = EXPECT[deck]
    _fresh_commons(lib)
    assert lib.clmd_f77_readdata(os.path.join(DIR, deck).encode()) == 0
    P = ATOMP.in_dll(lib, "atomp_")
    B = BOXPP.in_dll(lib, "boxpp_")
    T = TIMEP.in_dll(lib, "timep_")
    D = DMMPP.in_dll(lib, "dmmpp_")
    E = ENERG.in_dll(lib, "energ_")
    n = e["atsorts"]
    assert (P.natom, P.atsorts) == (e["natom"], n)
    assert list(P.apnum[:n]) == e["apnum"]
    assert list(P.apmas[:n]) == e["apmas"]
    assert list(P.apsig[:n]) == e["apsig"]
    assert list(P.apeps[:n]) == e["apeps"]
    assert bytes(P.apth[:n]) == e["apth"]
    assert list(P.api[:e["natom"]]) == sum(([k + 1] * e["apnum"][k] for k in range(n)), [])
    assert (B.boxx, B.boxy, B.boxz) == (e["box"],) * 3
    assert (T.dt, T.ntim, T.btim, T.sctim, T.nbtim, T.chgNtim) == \
        (e["dt"], e["ntim"], e["btim"], e["sctim"], e["nbtim"], e["chgNtim"])
    assert (P.att, P.atskin, P.atrcut, P.atrskin) == \
        (e["att"], e["atskin"], e["atrcut"], e["atrskin"])
    assert P.Q == e["Q"] and P.atnenum == e["atnenum"]
    assert E.ethst == e["ethst"] and E.eclth == e["eclth"] and E.ecltim == e["ecltim"]
    assert cvtpp_scalars(lib) == (e["csover"], e["clwait"], e["clnuctrl"])
    # read-3d.f:263-269: the skin ring, REAL(nbtim)
    ring = (e["atrskin"] - e["atrcut"]) / float(np.float32(e["nbtim"]))
    assert all(D.dmmh[k] == ring for k in range(256))
    assert D.dmmsu == 256.0 * (e["atrskin"] - e["atrcut"]) / float(np.float32(e["nbtim"]))
    assert (D.dmmst, D.dmmi, D.dmms) == (0, 0, 0.0)


def test_crlf_deck_reads_like_its_lf_twin(tmp_path):
    raw = open(os.path.join(DIR, "sample-v1.12.3d"), "rb").read()
    assert b"\r\n" in raw
    lf = tmp_path / "lf.3d"
    lf.write_bytes(raw.replace(b"\r\n", b"\n"))
    a, na, sa = orc.readdata(os.path.join(DIR, "sample-v1.12.3d"))
    b, nb, sb = orc.readdata(str(lf))
    assert bytes(a) == bytes(b) and (na, sa) == (nb, sb)


@pytest.mark.parametrize("deck", UNREADABLE)
def test_decks_the_reference_cannot_read_are_rejected(lib, deck):
    path = os.path.join(DIR, deck)
    with pytest.raises(RuntimeError):
        orc.readdata(path)
    assert lib.clmd_f77_readdata(path.encode()) != 0


@pytest.mark.parametrize("field,ok", [("2.0", 2.0), ("125", 0.00125), ("-1.5E3", -1500.0),
                                      ("1.5D-1", 0.15), ("12E3", 0.12), ("1.0+2", 100.0),
                                      ("1.2.3", None), ("--5", None), ("1X", None)])
def test_real_field_rules(tmp_path, field, ok):
    """Fw.d (read-3d.f's F14.5 box size): implied point, exponent forms,
    and the fields gfortran rejects."""
    lines = open(os.path.join(DIR, "sample.3d")).read().split("\n")
    k = next(i for i, l in enumerate(lines) if l.startswith("box size in X-direction"))
    lines[k] = lines[k][:41] + field.rjust(14)
    p = tmp_path / "d.3d"
    p.write_text("\n".join(lines))
    if ok is None:
        with pytest.raises(RuntimeError):
            orc.readdata(str(p))
    else:
        cfg, _, _ = orc.readdata(str(p))
        assert cfg.boxx == ok * 10
