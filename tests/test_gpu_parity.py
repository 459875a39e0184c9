"""Parity of the CUDA timestep (libeu3d.so) with the reference, on a B200.

The reference's outputs come from the committed golden fixtures (produced by
the reference's own CPU code, tests/golden/make_golden.py) and, at sizes the
fixtures do not cover, from the CPU restatement oracle/eu3d_oracle.c, which is
pinned value-for-value to the reference (tests/test_oracle_pin.py).

Tolerances:
  strict arithmetic (no FMA): relative L-inf per field <= 1e-11 after 3 steps
    (conserved variables <= 1e-12; primitives such as a near-zero transverse
    velocity carry the cancellation of their division),
    <= 1e-9 per conserved variable after 100 steps (the required bound), Nchem exact;
  fast arithmetic (FMA): <= 1e-9 per conserved variable after 100 steps;
  mixed precision (FP32 MUSCL/AUSM): species mass-fraction L1 error <= 1e-3 of
    the FP64 run, stated, not exact.
"""
import numpy as np
import pytest

import eu3d_cases as cases
from helpers import golden, golden_mechanism, init_state, interior, n_unequal, rel_linf

pytestmark = pytest.mark.gpu

FIELDS = ["CS", "T", "E", "P", "D", "U", "V", "W", "H", "Gamma", "Yi", "Nchem", "CMS", "Mc", "Di", "Wav", "Rgas",
          "Cp", "C", "Ma"]


def solver_from_golden(eu3d, z, arith="strict", precision="fp64", chemistry="stiff"):
    ext = tuple(float(v) for v in z["extent"])
    s = eu3d.Solver(int(z["ni"]), int(z["nj"]), int(z["nk"]), ext, arith=arith, precision=precision,
                    chemistry=chemistry, record_sources=True)
    s.load_mechanism(cases.MECH_JA919, cases.THERMO)
    if "init_CS" in z:
        s.set_state(init_state(z))
    else:
        s.set_primitive(*[z[f"prim_{k}"] for k in "PTUVWY"])
    return s


def test_nodes_match_reference(gpu):
    z = golden("rsbi_17x13x4_s3.npz")
    s = solver_from_golden(gpu, z)
    for got, want in zip(s.nodes(), (z["x"], z["y"], z["z"])):
        assert np.array_equal(got, want)


def test_strict_three_steps_every_field(gpu):
    z = golden("rsbi_17x13x4_s3.npz")
    s = solver_from_golden(gpu, z)
    st = s.step(int(z["steps"]), float(z["dt"]))
    assert st["nonfinite"] == 0
    for f in FIELDS:
        got = interior(s.get(f))
        want = z[f"out_{f}"]
        if f == "Nchem":
            assert n_unequal(got, want) == 0
        else:
            tol = 1e-12 if f in ("CS", "Di") else 1e-11
            assert rel_linf(got, want).max() <= tol, (f, rel_linf(got, want).max())


@pytest.mark.parametrize("arith", ["strict", "fast"])
def test_hundred_steps_conserved_variables(gpu, arith):
    """The required bound: relative L-inf <= 1e-9 per conserved variable after 100 steps."""
    z = golden("rsbi_36x18x3_s100.npz")
    s = solver_from_golden(gpu, z, arith=arith)
    st = s.step(int(z["steps"]), float(z["dt"]))
    assert st["max_nchem"] == int(z["out_Nchem"].max())
    err = rel_linf(interior(s.get("CS")), z["out_CS"])
    assert err.max() <= 1e-9, err
    assert n_unequal(interior(s.get("Nchem")), z["out_Nchem"]) == 0
    assert rel_linf(interior(s.get("T")), z["out_T"]).max() <= 1e-9


@pytest.mark.parametrize("arith", ["strict", "fast"])
def test_shock_bubble_twenty_steps(gpu, arith):
    z = golden("bubble_25x13x13_s20.npz")
    s = solver_from_golden(gpu, z, arith=arith)
    s.step(int(z["steps"]), float(z["dt"]))
    err = rel_linf(interior(s.get("CS")), z["out_CS"])
    assert err.max() <= (1e-11 if arith == "strict" else 1e-9), err
    assert rel_linf(interior(s.get("CMS")), z["out_CMS"]).max() <= 1e-8
    assert n_unequal(interior(s.get("Nchem")), z["out_Nchem"]) == 0


@pytest.mark.parametrize("arith", ["strict", "fast"])
def test_shock_bubble_hundred_steps(gpu, arith):
    """The required bound on the 3-D case: 100 steps of the shock-bubble (the
    shock runs through the whole perturbed sphere) against the reference's
    own CPU run, relative L-inf <= 1e-9 per conserved variable, Nchem exact."""
    z = golden("bubble_33x17x17_s100.npz")
    s = solver_from_golden(gpu, z, arith=arith)
    st = s.step(int(z["steps"]), float(z["dt"]))
    assert st["nonfinite"] == 0
    err = rel_linf(interior(s.get("CS")), z["out_CS"])
    assert err.max() <= 1e-9, err
    assert rel_linf(interior(s.get("T")), z["out_T"]).max() <= 1e-9
    assert n_unequal(interior(s.get("Nchem")), z["out_Nchem"]) == 0


def test_larger_grid_against_restatement(gpu, port_lib):
    """A grid the fixtures do not cover, against the pinned C restatement."""
    ni, nj, nk = 49, 25, 25
    ext = (0.0, 0.024, 0.0, 0.012, 0.0, 0.012)
    mech = golden_mechanism()
    x, y, zc = (cases.node_coordinates(n, a, b) for n, a, b in ((ni, 0, 0.024), (nj, 0, 0.012), (nk, 0, 0.012)))
    prim = cases.shock_bubble(x, y, zc, mech.mw, 9, radius=4e-3, shock_x=3e-3, standoff=5e-3, seed=3)
    port = port_lib(ni, nj, nk, x, y, zc, mech)
    port.set_primitive(*prim)
    s = gpu.Solver(ni, nj, nk, ext, record_sources=True)
    s.set_mechanism(mech)
    s.set_primitive(*prim)
    port.step(30, 5e-8)
    s.step(30, 5e-8)
    assert rel_linf(interior(s.get("CS")), interior(port.get("CS"))).max() <= 1e-10
    assert n_unequal(interior(s.get("Nchem")), interior(port.get("Nchem"))) == 0


def test_mixed_precision_error_is_bounded(gpu):
    """FP32 reconstruction + AUSM, FP64 update/recovery/kinetics: the species
    mass fractions stay within L1 1e-3 of the all-FP64 run (error stated)."""
    z = golden("bubble_25x13x13_s20.npz")
    a = solver_from_golden(gpu, z)
    b = solver_from_golden(gpu, z, precision="mixed")
    a.step(20, float(z["dt"]))
    b.step(20, float(z["dt"]))
    ya, yb = interior(a.get("Yi")), interior(b.get("Yi"))
    l1 = np.abs(ya - yb).sum(axis=0).mean()
    assert l1 <= 1e-3, l1
    assert rel_linf(interior(b.get("CS")), interior(a.get("CS"))).max() <= 1e-3


@pytest.mark.parametrize("dims", [(40, 20, 45), (17, 7, 32), (17, 8, 32), (33, 9, 5)])
def test_mixed_precision_tiles_match_fp64_closely(gpu, dims):
    """The plane-tiled FP32 flux kernel on grids whose (j, k) extent is not a
    multiple of its 7 x 32 tile, on one that is exactly one tile, and on one
    with a single row in its second tile, and the one-thread-per-column kernel
    of grids thin in z (nk < 16, both precisions): after
    two steps the conserved state stays within 2e-6 of the all-FP64 run, each
    error measured against the scale of its quantity (species partial
    densities against the largest density, momentum components against the
    largest momentum component, energy against its largest value). FP32 face
    fluxes perturb each update by ~1e-7 of that scale; a wrong face or stencil
    index shows up as an O(1e-2) error. (Per plane, relative errors are
    meaningless here: trace radicals sit at 1e-49 and the transverse momenta
    at 1e-6 of the streamwise one.)"""
    ni, nj, nk = dims
    ext = (0.0, 0.02, 0.0, 0.01, 0.0, 0.012)
    x = cases.node_coordinates(ni, ext[0], ext[1])
    y = cases.node_coordinates(nj, ext[2], ext[3])
    z = cases.node_coordinates(nk, ext[4], ext[5])
    mech = gpu.parse_mechanism(cases.MECH_JA919, cases.THERMO)
    prim = cases.shock_bubble(x, y, z, mech["mw"], mech["ns"], radius=3e-3, shock_x=3e-3, standoff=5e-3, seed=5)
    p, cs, T, E = gpu.initial_state(mech, ni, nj, nk, *prim)
    dt = cases.cfl_dt(x, y, p[0], p[1], p[2], p[3], p[6], 0.5)
    out = {}
    for precision in ("fp64", "mixed"):
        s = gpu.Solver(ni, nj, nk, ext, precision=precision, arith="fast")
        s.set_mechanism(mech)
        s.set_primitive(*prim)
        s.step(2, dt)
        out[precision] = interior(s.get("CS"))
        s.close()
    a, b = out["mixed"].reshape(13, -1), out["fp64"].reshape(13, -1)
    assert np.all(np.isfinite(a))
    d = np.abs(a - b).max(axis=1)
    err = np.concatenate([d[:9] / b[:9].sum(axis=0).max(), d[9:12] / np.abs(b[9:12]).max(), d[12:] / np.abs(b[12]).max()])
    assert err.max() <= 2e-6, err


def test_deterministic(gpu):
    z = golden("bubble_25x13x13_s20.npz")
    a = solver_from_golden(gpu, z, arith="fast")
    b = solver_from_golden(gpu, z, arith="fast")
    a.step(10, float(z["dt"]))
    b.step(10, float(z["dt"]))
    assert n_unequal(a.get("CS"), b.get("CS")) == 0


def test_mixed_stiff_heavy_cells_match_fp64(gpu):
    """Igniting gas in mixed precision: cells whose predicted Nchem exceeds 4
    are advanced one warp per cell (k_react_heavy). Over 8 steps of a hot
    2H2+O2/N2 block (1300-2600 K, dt 2e-8 s) the run must reach such cells and
    stay within a species L1 (mean over cells of sum_s |dY_s|) of 1e-4 and a
    relative temperature error of 1e-4 of the FP64 stiff run."""
    ni, nj, nk = 24, 8, 8
    ext = (0.0, 0.006, 0.0, 0.002, 0.0, 0.002)
    mech = gpu.parse_mechanism(cases.MECH_JA919, cases.THERMO)
    prim = cases.hot_reacting_block(ni + 4, nj + 4, nk + 4, mech["mw"], mech["ns"])
    out, peak = {}, {}
    for precision in ("fp64", "mixed"):
        s = gpu.Solver(ni, nj, nk, ext, precision=precision, arith="fast")
        s.set_mechanism(mech)
        s.set_primitive(*prim)
        peak[precision] = 0
        for _ in range(8):
            peak[precision] = max(peak[precision], s.step(1, 2e-8)["max_nchem"])
        out[precision] = (interior(s.get("Yi")), interior(s.get("T")))
        s.close()
    assert peak["mixed"] > 4, peak
    l1 = np.abs(out["mixed"][0] - out["fp64"][0]).sum(axis=0)
    terr = np.abs(out["mixed"][1] - out["fp64"][1]) / out["fp64"][1]
    assert l1.mean() <= 1e-4 and terr.max() <= 1e-4, (l1.mean(), l1.max(), terr.max(), peak)


@pytest.mark.parametrize("precision,arith,chemistry", [("mixed", "fast", "stiff"), ("fp64", "strict", "stiff"),
                                                        ("mixed", "fast", "learned")])
def test_autotuned_launch_shapes_change_no_bits(gpu, precision, arith, chemistry):
    """Every launch shape the autotuner may pick gives bitwise the same state:
    steps after tuning equal steps with the default shapes, and tuning leaves
    the state it timed on unchanged (ragged grid: 40 x 21 x 45 nodes). In
    learned mode the tuner also picks the recovery's register target."""
    ni, nj, nk = 40, 21, 45
    ext = (0.0, 0.02, 0.0, 0.01, 0.0, 0.012)
    x, y, z = (cases.node_coordinates(n, a, b) for n, a, b in ((ni, 0, 0.02), (nj, 0, 0.01), (nk, 0, 0.012)))
    mech = gpu.parse_mechanism(cases.MECH_JA919, cases.THERMO)
    prim = cases.shock_bubble(x, y, z, mech["mw"], mech["ns"], radius=3e-3, shock_x=3e-3, standoff=5e-3, seed=5)
    out = []
    for tune in (False, True):
        s = gpu.Solver(ni, nj, nk, ext, precision=precision, arith=arith, chemistry=chemistry)
        s.set_mechanism(mech)
        s.set_primitive(*prim)
        if chemistry == "learned":
            import learned
            model, gate = learned.load()
            learned.attach(s, model, gate)
        s.step(1, 2e-8)
        before = s.get("CS")
        if tune:
            rep = s.autotune(reps=2)
            assert len(rep["flux_ms"]) >= 5 and rep["flux_ci"] in rep["flux_ms"], rep
            # learned: 3 block sizes x 4 register targets; stiff: 3 x 3 (the
            # kinetics kernel's); frozen: 3 block sizes
            assert len(rep["recover_ms"]) == {"learned": 12, "stiff": 9}.get(chemistry, 3), rep
            assert n_unequal(s.get("CS"), before) == 0
        s.step(4, 2e-8)
        out.append((s.get("CS"), s.get("T")))
        s.close()
    for a, b in zip(*out):
        assert n_unequal(a, b) == 0


@pytest.mark.parametrize("width,steps,tol", [(2.0, 40, 1e-11), (6.0, 100, 1e-10)])
def test_znd_against_restatement(gpu, port_lib, width, steps, tol):
    """The 1-D ZND initiation (2H2+O2+7Ar on the Ar variant of the mechanism,
    1 MPa / 3000 K driver at a reflecting wall, 6.67 kPa / 298 K gas ahead,
    parameters from data/input-1dZND.txt, driver edge a tanh profile `width`
    cells wide) with the ZND ghost fill, on a 401 x 2 x 2 node grid at 25 um
    spacing, against the pinned C restatement with the same ghost fill
    (strict arithmetic), Nchem exact. Each step's dt comes from the
    device-side CFL reduction at 0.5 (eu_step_cfl) and the restatement takes
    the same dt.

    The two builds start 1e-14 apart (CUDA's exp/log/pow against glibc's, in
    the last bit); the rarefaction running into the wall amplifies that. With
    the 2-cell edge the difference stays below 1e-13 for 20 steps, reaches
    1e-12 at 40 and 2e-9 by step 100 (a limiter switching branch on values
    that differ in the last bit); with a 6-cell edge it is 3e-12 at step 100.
    So the bounds: 1e-11 after 40 steps at the 2-cell edge, 1e-10 after 100 at
    the 6-cell one."""
    from oracle import Mechanism
    ni, nj, nk = 401, 2, 2
    dx = 25e-6
    ext = (0.0, (ni - 1) * dx, 0.0, dx, 0.0, dx)
    x = cases.node_coordinates(ni, ext[0], ext[1])
    y = cases.node_coordinates(nj, ext[2], ext[3])
    mech = gpu.parse_mechanism(cases.MECH_JA919_AR, cases.THERMO_AR)
    prim = cases.znd(x, y, y, mech["mw"], mech["ns"], interface_cells=width)
    port = port_lib(ni, nj, nk, x, y, y, Mechanism.from_dict(mech), boundary="znd")
    port.set_primitive(*prim)
    s = gpu.Solver(ni, nj, nk, ext, record_sources=True, boundary="znd")
    s.set_mechanism(mech)
    s.set_primitive(*prim)
    # the first dt against the host rule on the initial state (interior
    # spacings: the reference's rule takes dy from its ghost nodes, which a
    # two-node direction makes negative)
    p, cs, T, E = gpu.initial_state(mech, ni, nj, nk, *prim)
    dt0 = cases.cfl_dt(x, x, p[0], p[1], p[2], p[3], p[6], 0.5)
    peak = 0
    for n in range(steps):
        st, dt = s.step_cfl(1, 0.5)
        if n == 0:
            assert abs(dt - dt0) <= 1e-12 * dt0, (dt, dt0)
        port.step(1, dt)
        peak = max(peak, st["max_nchem"])
    assert peak >= 1
    assert rel_linf(interior(s.get("CS")), interior(port.get("CS"))).max() <= tol
    assert n_unequal(interior(s.get("Nchem")), interior(port.get("Nchem"))) == 0


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-6)])
def test_set_conserved_matches_set_state(gpu, precision, tol):
    """eu_set_conserved (CS, T, E up; the primitives formed on the device by
    the recovery) steps like eu_set_state with the full state: the recovered
    temperature is within 1e-12 of the uploaded one, and after three steps each
    conserved plane agrees to its relative tolerance (the transverse momenta,
    whose planes peak at ~1e-6 of the streamwise one, carry the primitives'
    initial rounding difference at a few 1e-10 of their own maxima)."""
    ni, nj, nk = 33, 17, 17
    ext = (0.0, 0.016, 0.0, 0.008, 0.0, 0.008)
    mech = gpu.parse_mechanism(cases.MECH_JA919, cases.THERMO)
    x, y, z = (cases.node_coordinates(n, a, b) for n, a, b in ((ni, 0, 0.016), (nj, 0, 0.008), (nk, 0, 0.008)))
    prim = cases.shock_bubble(x, y, z, mech["mw"], mech["ns"], radius=3e-3, shock_x=3e-3, standoff=5e-3, seed=5)
    p, cs, T, E = gpu.initial_state(mech, ni, nj, nk, *prim)
    st = {"CS": cs, "T": T, "E": E, "P": p[0], "D": p[1], "U": p[2], "V": p[3], "W": p[4], "H": p[5],
          "Gamma": p[6], "Yi": p[7:]}
    out = []
    for full in (True, False):
        s = gpu.Solver(ni, nj, nk, ext, precision=precision, arith="fast")
        s.set_mechanism(mech)
        if full:
            s.set_state(st)
        else:
            s.set_conserved(cs, T, E)
            t0 = np.asarray(T).reshape((1,) + s.shape)
            assert rel_linf(interior(s.get("T")), interior(t0)).max() <= 1e-12
        s.step(3, 4e-8)
        out.append((s.get("CS"), s.get("T")))
        s.close()
    for a, b in zip(out[0], out[1]):
        assert rel_linf(interior(b), interior(a)).max() <= tol


@pytest.mark.parametrize("arith", ["strict", "fast"])
def test_rk3_against_restatement(gpu, port_lib, arith):
    """The three-stage TVD Runge-Kutta advection (eu_set_time_scheme) against
    the C restatement's: 10 steps of the shock-bubble fixture's initial state,
    conserved state within 1e-10 (strict) or 1e-9 (fast) per variable, Nchem
    exact; and the scheme changes the result (it is not the Euler step)."""
    z = golden("bubble_25x13x13_s20.npz")
    mech = golden_mechanism()
    port = port_lib(int(z["ni"]), int(z["nj"]), int(z["nk"]), z["x"], z["y"], z["z"], mech)
    port.set_primitive(*[z[f"prim_{k}"] for k in "PTUVWY"])
    port.set_scheme("rk3")
    port.step(10, float(z["dt"]))
    s = solver_from_golden(gpu, z, arith=arith)
    s.set_time_scheme("rk3")
    st = s.step(10, float(z["dt"]))
    assert st["nonfinite"] == 0
    want = interior(port.get("CS"))
    assert rel_linf(interior(s.get("CS")), want).max() <= (1e-10 if arith == "strict" else 1e-9)
    assert n_unequal(interior(s.get("Nchem")), interior(port.get("Nchem"))) == 0
    ee = solver_from_golden(gpu, z, arith=arith)
    ee.step(10, float(z["dt"]))
    assert rel_linf(interior(ee.get("CS")), want).max() > 1e-6


def test_rk3_learned_mixed_stays_close(gpu):
    """RK3 with the benchmark's learned + mixed step: finite, and its species
    within L1 1e-3 of the FP64 RK3 run."""
    import learned
    z = golden("bubble_25x13x13_s20.npz")
    a = solver_from_golden(gpu, z)
    a.set_time_scheme("rk3")
    b = solver_from_golden(gpu, z, precision="mixed", chemistry="learned", arith="fast")
    model, gate = learned.load(device=0)
    learned.attach(b, model, gate)
    b.set_time_scheme("rk3")
    a.step(10, float(z["dt"]))
    st = b.step(10, float(z["dt"]))
    assert st["nonfinite"] == 0
    l1 = np.abs(interior(a.get("Yi")) - interior(b.get("Yi"))).sum(axis=0).mean()
    assert l1 <= 1e-3, l1
