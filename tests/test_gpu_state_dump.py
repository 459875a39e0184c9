"""EU3D_STATE_V1_LE state dumps (the reference's Euler::Output format,
src/Euler.cpp:1540-1598), written and read through the C ABI.

The dump is parsed here independently with numpy, following the reference's
writer: a header line, a line of 17 integers and two doubles (NS, total and
local node counts, rank coordinates, block counts, rank, rank count,
iteration, output number, time, dt), a line of column names, then 22 + 5 NS
little-endian doubles per interior node in (i, j, k) order, k fastest.
"""
import os
import tempfile

import numpy as np
import pytest

import eu3d_cases as cases
from helpers import golden, interior, n_unequal

pytestmark = pytest.mark.gpu

FIXED = ["X", "Y", "Z", "D", "T", "U", "V", "W", "E", "Wav", "Rgas", "Cp", "P", "H", "Gamma", "C", "Ma"]


def parse_dump(path):
    with open(path, "rb") as f:
        magic = f.readline().decode().strip()
        sizes = f.readline().decode().split()
        names = f.readline().decode().split()
        rows = np.frombuffer(f.read(), dtype="<f8")
    head = [int(v) for v in sizes[:17]] + [float(v) for v in sizes[17:]]
    return magic, head, names, rows.reshape(-1, len(names))


def bubble(gpu):
    z = golden("bubble_25x13x13_s20.npz")
    s = gpu.Solver(int(z["ni"]), int(z["nj"]), int(z["nk"]), tuple(z["extent"]), arith="strict",
                   record_sources=True)
    s.load_mechanism(cases.MECH_JA919, cases.THERMO)
    s.set_primitive(*[z[f"prim_{k}"] for k in "PTUVWY"])
    return s, z


def test_dump_layout_matches_the_reference_writer(gpu):
    s, z = bubble(gpu)
    ni, nj, nk = int(z["ni"]), int(z["nj"]), int(z["nk"])
    s.step(5, float(z["dt"]))
    path = os.path.join(tempfile.mkdtemp(), "state_check_5_rank0.bin")
    s.write_state(path, iteration=5, num=5, final_time=5 * float(z["dt"]), dt=float(z["dt"]))
    magic, head, names, rows = parse_dump(path)
    ns = 9
    assert magic == "EU3D_STATE_V1_LE"
    assert head[:17] == [ns, ni, nj, nk, ni, nj, nk, 0, 0, 0, 1, 1, 1, 0, 1, 5, 5]
    assert head[17] == 5 * float(z["dt"]) and head[18] == float(z["dt"])
    want = FIXED + [f"{f}{n}" for f in ("Di", "Yi", "Mc") for n in range(ns)] + \
        [f"CS{n}" for n in range(ns + 4)] + [f"CMS{n}" for n in range(ns)] + ["Nchem"]
    assert names == want and rows.shape == (ni * nj * nk, 22 + 5 * ns)
    col = {n: q for q, n in enumerate(names)}
    x, y, zc = s.nodes()
    X, Y, Z = np.meshgrid(x[2:-2], y[2:-2], zc[2:-2], indexing="ij")
    for name, grid in (("X", X), ("Y", Y), ("Z", Z)):
        assert np.array_equal(rows[:, col[name]], grid.ravel()), name
    for name in ["D", "T", "U", "V", "W", "E", "Wav", "Rgas", "Cp", "P", "H", "Gamma", "C", "Ma", "Nchem"]:
        assert np.array_equal(rows[:, col[name]], interior(s.get(name)).ravel()), name
    for field, planes in (("Di", ns), ("Yi", ns), ("Mc", ns), ("CS", ns + 4), ("CMS", ns)):
        got = interior(s.get(field))
        for n in range(planes):
            assert np.array_equal(rows[:, col[f"{field}{n}"]], got[n].ravel()), (field, n)


def test_restart_from_dump_continues_bitwise(gpu):
    a, z = bubble(gpu)
    dt = float(z["dt"])
    a.step(5, dt)
    path = os.path.join(tempfile.mkdtemp(), "state.bin")
    a.write_state(path, iteration=5, num=1, final_time=5 * dt, dt=dt)
    b, _ = bubble(gpu)
    assert b.read_state(path) == (5, 1, 5 * dt, dt)
    a.step(5, dt)
    b.step(5, dt)
    for f in ["CS", "T", "E", "Nchem"]:
        assert n_unequal(interior(a.get(f)), interior(b.get(f))) == 0, f


def test_dump_of_another_size_is_refused(gpu):
    a, z = bubble(gpu)
    a.step(1, float(z["dt"]))
    path = os.path.join(tempfile.mkdtemp(), "state.bin")
    a.write_state(path)
    other = gpu.Solver(int(z["ni"]) + 1, int(z["nj"]), int(z["nk"]), tuple(z["extent"]))
    other.load_mechanism(cases.MECH_JA919, cases.THERMO)
    with pytest.raises(gpu.EU3DError) as e:
        other.read_state(path)
    assert e.value.name == "EU_ERR_INVALID_ARGUMENT"


def test_async_dump_is_the_state_at_the_call(gpu):
    """eu_output_async: the dump holds the state at the call even when steps
    run before the file is waited for, and its bytes are eu_write_state's."""
    a, z = bubble(gpu)
    b, _ = bubble(gpu)
    dt = float(z["dt"])
    for s in (a, b):
        s.step(3, dt)
    d = tempfile.mkdtemp()
    a.output_async(os.path.join(d, "async.bin"), "state", iteration=3, num=2, final_time=3 * dt, dt=dt)
    a.step(4, dt)  # the time loop goes on while the snapshot is written
    a.output_wait()
    b.write_state(os.path.join(d, "sync.bin"), iteration=3, num=2, final_time=3 * dt, dt=dt)
    with open(os.path.join(d, "async.bin"), "rb") as f1, open(os.path.join(d, "sync.bin"), "rb") as f2:
        assert f1.read() == f2.read()
    # and the handle that went on stepping is where it should be
    b.step(4, dt)
    assert n_unequal(interior(a.get("CS")), interior(b.get("CS"))) == 0


def reference_tecplot(x, y, z, fields):
    """The reference's Tecplot writer (Euler::Output, src/Euler.cpp:1600-1790)
    restated: header, zone line, then each variable over every haloed node
    with k outermost and i fastest, one value per line as an ostream writes a
    double by default (%g)."""
    nx, ny, nz = len(x), len(y), len(z)
    lines = ["Variables = X,Y,Z,T,D,P,U,V,Ma,Y1,Y2,Y3,Y4,Y5,Y6,Y7", f"ZONE I={nx}\tJ={ny}\tK={nz}",
             "datapacking=block"]
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    for a in [X, Y, Z] + fields:
        lines += [format_g(v) for v in np.transpose(a, (2, 1, 0)).ravel()]
    return lines


def format_g(v):
    """One double as C's printf("%g") writes it on Linux: a NaN keeps its sign
    ("-nan" for the sign bit set), which Python's own %g drops."""
    if np.isnan(v):
        return "-nan" if np.signbit(v) else "nan"
    return "%g" % v


def test_tecplot_output_matches_the_reference_writer(gpu, port_lib):
    """The Tecplot file against the reference writer's format applied to the C
    restatement's fields after the same FP64 strict steps: identical header
    and zone lines and node order; values equal to the six significant digits
    written (one unit in the sixth digit where a last-bit difference crosses
    a rounding boundary)."""
    from helpers import golden_mechanism
    z = golden("bubble_25x13x13_s20.npz")
    dt = float(z["dt"])
    s = gpu.Solver(int(z["ni"]), int(z["nj"]), int(z["nk"]), tuple(z["extent"]), arith="strict")
    s.load_mechanism(cases.MECH_JA919, cases.THERMO)
    s.set_primitive(*[z[f"prim_{k}"] for k in "PTUVWY"])
    s.step(6, dt)
    path = os.path.join(tempfile.mkdtemp(), "Series0_0.dat")
    s.write_tecplot(path)
    p = port_lib(int(z["ni"]), int(z["nj"]), int(z["nk"]), z["x"], z["y"], z["z"], golden_mechanism())
    p.set_primitive(*[z[f"prim_{k}"] for k in "PTUVWY"])
    p.step(6, dt)
    fields = [p.get(n)[0] for n in ("T", "D", "P", "U", "V", "Ma")] + list(p.get("Yi")[:7])
    want = reference_tecplot(z["x"], z["y"], z["z"], fields)
    got = open(path).read().split("\n")
    assert got[-1] == "" and len(got) - 1 == len(want)
    assert got[:3] == want[:3]
    g = np.array([float(v) for v in got[3:-1]]).reshape(16, -1)
    w = np.array([float(v) for v in want[3:]]).reshape(16, -1)
    assert np.array_equal(g[:3], w[:3])  # node coordinates
    # corner halo nodes that no boundary pass fills hold 0/0 in both codes
    assert np.array_equal(np.isnan(g), np.isnan(w))
    ok = np.isnan(w) | (np.abs(g - w) <= 1.2e-5 * np.abs(w))
    assert ok.all()
    assert (np.array(got[3:-1]) == np.array(want[3:])).mean() > 0.999


def test_tecplot_output_in_mixed_precision(gpu):
    """In mixed precision the file holds the handle's own FP64 fields (formed
    from the conserved state for output), written as the reference writes
    them: the text equals the writer's format applied to eu_get_field."""
    z = golden("bubble_25x13x13_s20.npz")
    s = gpu.Solver(int(z["ni"]), int(z["nj"]), int(z["nk"]), tuple(z["extent"]), arith="fast", precision="mixed")
    s.load_mechanism(cases.MECH_JA919, cases.THERMO)
    s.set_primitive(*[z[f"prim_{k}"] for k in "PTUVWY"])
    s.step(6, float(z["dt"]))
    path = os.path.join(tempfile.mkdtemp(), "Series0_0.dat")
    s.output_async(path, "tecplot")
    s.output_wait()
    fields = [s.get(n)[0] for n in ("T", "D", "P", "U", "V", "Ma")] + list(s.get("Yi")[:7])
    x, y, zc = s.nodes()
    assert open(path).read().split("\n")[:-1] == reference_tecplot(x, y, zc, fields)
