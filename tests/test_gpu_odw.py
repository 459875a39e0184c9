"""The ODW ghost fill on the GPU (EU_BC_ODW, the reference's
Flowfield::FieldBoundary_3dODW, src/Flowfield.cpp:412-592): the wedge-aligned
oblique-detonation case of eu3d_cases.odw against the C restatement, whose ODW
fill is pinned bitwise to the reference's own (tests/test_oracle_pin.py)."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT
from helpers import cs_rel_linf, golden_mechanism, interior, n_unequal, rel_linf

sys.path.insert(0, os.path.join(ROOT, "eu3d-gpu_b200"))
import eu3d_cases as cases  # noqa: E402

pytestmark = pytest.mark.gpu

NI, NJ, NK = 41, 21, 6
EXT = (0.0, 0.0105, 0.0, 0.005, 0.0, 0.00125)


def _case(phi=False):
    mo = golden_mechanism()
    mech = {k: getattr(mo, k) for k in ("ns", "nr", "mw", "coeff_lo", "coeff_hi", "af", "bf", "eaf", "stoi_f",
                                         "stoi_b", "tb")}
    x, y, z = (cases.node_coordinates(n, a, b) for n, a, b in ((NI, *EXT[0:2]), (NJ, *EXT[2:4]), (NK, *EXT[4:6])))
    prim, inflow = cases.odw(x, y, z, mech, phi=cases.odw_phi(z) if phi else None)
    return mo, mech, (x, y, z), prim, inflow


def test_odw_against_restatement(gpu, port_lib):
    """FP64 strict stiff steps with the ODW ghost fill (the freestream hits the
    wedge surface, the shock it raises heats the gas): conserved state within
    1e-10 of the restatement, Nchem exact."""
    mo, mech, (x, y, z), prim, inflow = _case(phi=True)
    port = port_lib(NI, NJ, NK, x, y, z, mo, boundary="odw")
    port.set_primitive(*prim)
    port.set_inflow(*inflow)
    s = gpu.Solver(NI, NJ, NK, EXT, boundary="odw", record_sources=True)
    s.set_mechanism(mech)
    s.set_primitive(*prim)
    s.set_inflow(*inflow)
    port.step(25, 2e-8)
    s.step(25, 2e-8)
    assert rel_linf(interior(s.get("CS")), interior(port.get("CS"))).max() <= 1e-10
    assert n_unequal(interior(s.get("Nchem")), interior(port.get("Nchem"))) == 0
    t = interior(s.get("T"))
    assert t.max() > 1.5 * 293.0  # the wedge's shock heats the gas
    s.close()


def test_odw_ghost_layers_match_restatement(gpu, port_lib):
    """Every face layer of the ODW ghost fill after a step, against the
    restatement (inflow tables at x low, rebuilt outflow at x high, z mirrored
    with W reflected and the thermo rebuilt)."""
    mo, mech, (x, y, z), prim, inflow = _case()
    port = port_lib(NI, NJ, NK, x, y, z, mo, boundary="odw")
    port.set_primitive(*prim)
    port.set_inflow(*inflow)
    s = gpu.Solver(NI, NJ, NK, EXT, boundary="odw")
    s.set_mechanism(mech)
    s.set_primitive(*prim)
    s.set_inflow(*inflow)
    port.step(2, 2e-8)
    s.step(2, 2e-8)
    port.boundary()
    s.step(0, 2e-8)
    b = 2
    faces = [(slice(0, b), slice(b, -b), slice(b, -b)), (slice(-b, None), slice(b, -b), slice(b, -b)),
             (slice(b, -b), slice(0, b), slice(b, -b)), (slice(b, -b), slice(-b, None), slice(b, -b)),
             (slice(b, -b), slice(b, -b), slice(0, b)), (slice(b, -b), slice(b, -b), slice(-b, None))]
    # the GPU's ghosts as its last step's fill left them; the restatement's
    # refilled from the same interior state
    for f in ["P", "U", "V", "W", "Yi"]:
        g, r = s.get(f), port.get(f)
        for sl in faces[:1]:  # the inflow layer is independent of the interior
            assert n_unequal(g[(slice(None),) + sl], r[(slice(None),) + sl]) == 0, (f, sl)
    s.close()


def test_odw_needs_its_inflow_tables(gpu):
    mo, mech, _, prim, _ = _case()
    s = gpu.Solver(NI, NJ, NK, EXT, boundary="odw")
    s.set_mechanism(mech)
    s.set_primitive(*prim)
    with pytest.raises(gpu.EU3DError) as e:
        s.step(1, 2e-8)
    assert e.value.status == 7
    s.close()


def test_odw_learned_mixed_runs(gpu):
    """The learned + mixed step on the ODW case stays finite and close to the
    FP64 stiff step over 40 steps."""
    import learned
    mo, mech, (x, y, z), prim, inflow = _case()
    model, gate = learned.load(device=0)
    out = {}
    for kw in (dict(), dict(precision="mixed", chemistry="learned", arith="fast")):
        s = gpu.Solver(NI, NJ, NK, EXT, boundary="odw", **kw)
        s.set_mechanism(mech)
        s.set_primitive(*prim)
        s.set_inflow(*inflow)
        if kw:
            learned.attach(s, model, gate)
        st, _ = s.step_cfl(40, 0.5)
        assert st["nonfinite"] == 0
        out[bool(kw)] = interior(s.get("Yi"))
        s.close()
    l1 = np.abs(out[True] - out[False]).sum(axis=0).mean()
    assert l1 <= 1e-3, l1


def test_odw_wedge_tip_inside_the_domain(gpu, port_lib):
    """The wedge surface starting at an interior x node (eu_set_odw_wall): the
    y-low ghosts ahead of it take the freestream, behind it the reference's
    symmetry fill. FP64 strict stiff steps of the Mach 7 / 101.325 kPa / 300 K
    configuration against the restatement with the same wall start: conserved
    state within 1e-10 (momentum against the momentum scale), Nchem exact,
    every y-low ghost layer equal; the shock starts at the tip (no pressure
    rise ahead of it)."""
    mo, mech, (x, y, z), _, _ = _case()
    prim, inflow = cases.odw(x, y, z, mech, input_path=cases.INPUT_ODW_M7)
    wall = 12
    port = port_lib(NI, NJ, NK, x, y, z, mo, boundary="odw")
    port.set_primitive(*prim)
    port.set_inflow(*inflow)
    port.set_wall(wall)
    s = gpu.Solver(NI, NJ, NK, EXT, boundary="odw")
    s.set_mechanism(mech)
    s.set_primitive(*prim)
    s.set_inflow(*inflow)
    s.set_odw_wall(wall)
    port.step(25, 1e-8)
    s.step(25, 1e-8)
    assert cs_rel_linf(interior(s.get("CS")), interior(port.get("CS"))).max() <= 1e-10
    assert n_unequal(interior(s.get("Nchem")), interior(port.get("Nchem"))) == 0
    # the y-low ghosts of the primitives the flux reads, as both codes' last
    # fill left them (from the state at the start of the last step)
    ylow = (slice(None), slice(2, -2), slice(0, 2), slice(2, -2))
    speed = np.abs(port.get("U")[ylow]).max()
    for f in ["P", "D", "U", "V", "W", "H", "Gamma", "Yi"]:
        g, r = s.get(f)[ylow], port.get(f)[ylow]
        # W is rounding noise in this z-uniform flow: measured against the speed
        err = np.abs(g - r).max() / speed if f == "W" else rel_linf(g, r).max()
        assert err <= 1e-10, (f, err)
    p = interior(s.get("P"))[0]
    p0 = 101325.0
    assert np.abs(p[: wall - 4, :3] / p0 - 1).max() < 1e-6  # the freestream ahead of the tip
    assert p[wall + 4:, 0].max() > 3 * p0  # the wedge's shock behind it
    s.close()


def test_odw_wall_start_needs_the_inflow_tables(gpu):
    mo, mech, _, prim, _ = _case()
    s = gpu.Solver(NI, NJ, NK, EXT, boundary="odw")
    s.set_mechanism(mech)
    s.set_primitive(*prim)
    with pytest.raises(gpu.EU3DError) as e:
        s.set_odw_wall(5)
    assert e.value.name == "EU_ERR_NOT_READY"
    s.close()
