"""libeu3d.so on the CPU: it loads, exports every entry point include/eu3d.h
declares, and its host-side parts (file readers, initial-state construction)
match the reference's semantics. No compute call needs a device here."""
import ctypes
import os
import re
import tempfile

import numpy as np
import pytest

import eu3d_cases as cases
from conftest import ROOT
from helpers import golden_mechanism, interior, n_unequal


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(eu_\w+)\s*\(", text))
    return names


def test_exports_every_declared_symbol(eu3d_lib):
    lib = eu3d_lib.library()
    names = declared_symbols()
    assert len(names) >= 15
    for n in sorted(names):
        assert hasattr(lib, n), n
    assert lib.eu_abi_version() == 1


def test_mechanism_parser_matches_reference_tables(eu3d_lib):
    got = eu3d_lib.parse_mechanism(cases.MECH_JA919, cases.THERMO)
    want = golden_mechanism()
    assert got["ns"] == want.ns == 9 and got["nr"] == want.nr == 19
    for k in ["mw", "coeff_lo", "coeff_hi", "af", "bf", "eaf", "stoi_f", "stoi_b", "tb"]:
        assert np.array_equal(got[k], getattr(want, k)), k


def test_parser_errors_are_statuses(eu3d_lib):
    with pytest.raises(eu3d_lib.EU3DError) as e:
        eu3d_lib.parse_mechanism("/nonexistent/mech.txt", cases.THERMO)
    assert e.value.name == "EU_ERR_IO"
    d = tempfile.mkdtemp()
    bad = os.path.join(d, "bad.txt")
    with open(bad, "w") as f:
        f.write("!\nNS\tNR\tTB\nx\ty\tz\n")
    with pytest.raises(eu3d_lib.EU3DError):
        eu3d_lib.parse_mechanism(bad, cases.THERMO)


def test_grid_reader_keeps_reference_precision(eu3d_lib):
    """FileReader stores numbers at 6 significant digits (src/FileReader.cpp:33-41)."""
    d = tempfile.mkdtemp()
    g = os.path.join(d, "grid.txt")
    with open(g, "w") as f:
        f.write("#The grid file\ntotal_ni    33\nxa  0.0\nxb  0.0123456789\ntotal_nj 17\nya 0\nyb 0.08\n"
                "total_nk 9\nza 0\nzb 0.02  # comment\nbc 2\n")
    cfg = eu3d_lib.Config()
    assert eu3d_lib.library().eu_read_grid(g.encode(), ctypes.byref(cfg)) == 0
    assert (cfg.total_ni, cfg.total_nj, cfg.total_nk, cfg.bc) == (33, 17, 9, 2)
    assert cfg.xb == 0.0123457 and cfg.yb == 0.08 and cfg.zb == 0.02
    assert eu3d_lib.library().eu_read_grid(b"/nonexistent", ctypes.byref(cfg)) == 4


def test_node_coordinates_match_reference(ref_lib):
    ext = (0.0, 0.17, 0.0, 0.08, 0.0, 0.02)
    ref = ref_lib.from_grid(281, 141, 16, ext, cases.MECH_JA919, cases.THERMO)
    x, y, z = ref.nodes()
    for got, want in zip([cases.node_coordinates(281, 0.0, 0.17), cases.node_coordinates(141, 0.0, 0.08),
                          cases.node_coordinates(16, 0.0, 0.02)], [x, y, z]):
        assert np.array_equal(got, want)


def test_host_initial_state_matches_reference(eu3d_lib, ref_lib):
    """eu_initial_state == Flowfield::FieldInitial's derived fields, value for value."""
    ext = (0.0, 0.008, 0.0, 0.004, 0.0, 0.004)
    ref = ref_lib.from_grid(17, 9, 9, ext, cases.MECH_JA919, cases.THERMO)
    x, y, z = ref.nodes()
    mech = golden_mechanism()
    prim = cases.shock_bubble(x, y, z, mech.mw, 9, radius=1.5e-3, shock_x=1e-3, standoff=2e-3, seed=11)
    ref.set_primitive(*prim)
    p, cs, T, E = eu3d_lib.initial_state(mech, 17, 9, 9, *prim)
    names = ["P", "D", "U", "V", "W", "H", "Gamma"]
    for q, n in enumerate(names):
        assert n_unequal(interior(p[q:q + 1]), interior(ref.get(n))) == 0, n
    assert n_unequal(interior(p[7:]), interior(ref.get("Yi"))) == 0
    assert n_unequal(interior(cs), interior(ref.get("CS"))) == 0
    assert n_unequal(interior(T), interior(ref.get("T"))) == 0
    assert n_unequal(interior(E), interior(ref.get("E"))) == 0
