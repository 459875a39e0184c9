"""The CPU restatement (oracle/eu3d_oracle.c) is pinned to the reference.

1. Against the reference's own CPU code compiled from its sources (oracle/_ref):
   value-for-value equality of every field after full timesteps.
2. Against the committed golden fixtures that the reference produced
   (tests/golden/make_golden.py), which needs no reference checkout.
"""
import numpy as np
import pytest

import eu3d_cases as cases
from helpers import golden, golden_mechanism, init_state, interior, n_unequal

ALL = ["CS", "T", "E", "P", "D", "U", "V", "W", "H", "Gamma", "Yi", "Nchem", "CMS", "Mc", "Di", "Wav", "Rgas",
       "Cp", "C", "Ma"]


def port_from_golden(port_lib, z):
    mech = golden_mechanism()
    p = port_lib(int(z["ni"]), int(z["nj"]), int(z["nk"]), z["x"], z["y"], z["z"], mech)
    if "init_CS" in z:
        p.set_state(init_state(z))
    else:
        p.set_primitive(*[z[f"prim_{k}"] for k in "PTUVWY"])
    return p


@pytest.mark.parametrize("name", ["rsbi_17x13x4_s3.npz", "rsbi_36x18x3_s100.npz", "bubble_25x13x13_s20.npz",
                                  "bubble_33x17x17_s100.npz"])
def test_port_matches_golden(port_lib, name):
    z = golden(name)
    p = port_from_golden(port_lib, z)
    p.step(int(z["steps"]), float(z["dt"]))
    for f in [k[4:] for k in z.files if k.startswith("out_")]:
        got = interior(p.get(f))
        assert n_unequal(got, z[f"out_{f}"]) == 0, f


def test_golden_exercises_the_kinetics():
    z = golden("rsbi_36x18x3_s100.npz")
    assert z["out_Nchem"].max() >= 3  # substep count rises near the front
    b = golden("bubble_25x13x13_s20.npz")
    # the shock has entered the perturbed sphere: transverse momentum appears
    ns = 9
    assert np.abs(b["out_CS"][ns + 1]).max() > 1.0 and np.abs(b["out_CS"][ns + 2]).max() > 1.0


def test_thermo_points(port_lib):
    z = golden("thermo_points.npz")
    mech = golden_mechanism()
    x = np.linspace(0, 1, 9)
    p = port_lib(5, 5, 5, x, x, x, mech)
    for a, T in enumerate(z["T"]):
        for s in range(mech.ns):
            assert np.array_equal(p.thermo(T, 8.31434 / mech.mw[s], s), z["cp_h_s"][a, s, 0])
            assert np.array_equal(p.thermo(T, 8.31434, s), z["cp_h_s"][a, s, 1])


def test_port_matches_reference_rsbi(ref_lib, port_lib):
    ext = (0.0, 0.17, 0.0, 0.08, 0.0, 0.02)
    ref = ref_lib.from_grid(21, 11, 5, ext, cases.MECH_JA919, cases.THERMO)
    x, y, z = ref.nodes()
    port = port_lib(21, 11, 5, x, y, z, ref.mechanism())
    port.set_state(ref.state())
    for _ in range(2):
        ref.step(2, 3e-8)
        port.step(2, 3e-8)
        for f in ALL:
            assert n_unequal(interior(port.get(f)), interior(ref.get(f))) == 0, f


def test_port_matches_reference_bubble(ref_lib, port_lib):
    ext = (0.0, 0.008, 0.0, 0.004, 0.0, 0.004)
    ref = ref_lib.from_grid(17, 9, 9, ext, cases.MECH_JA919, cases.THERMO)
    x, y, z = ref.nodes()
    prim = cases.shock_bubble(x, y, z, ref.mechanism().mw, ref.ns, radius=1.5e-3, shock_x=1e-3, standoff=2e-3,
                              seed=7)
    ref.set_primitive(*prim)
    port = port_lib(17, 9, 9, x, y, z, ref.mechanism())
    port.set_primitive(*prim)
    for f in ["CS", "T", "E", "P", "D", "H", "Gamma"]:
        assert n_unequal(interior(port.get(f)), interior(ref.get(f))) == 0, f
    ref.step(6, 1e-7)
    port.step(6, 1e-7)
    for f in ALL:
        assert n_unequal(interior(port.get(f)), interior(ref.get(f))) == 0, f


def test_rsbi_generator_matches_reference_init(ref_lib):
    """eu3d_cases.rsbi reproduces FieldInitial/ReactionInitial's fields exactly."""
    ext = (0.0, 0.17, 0.0, 0.08, 0.0, 0.02)
    ref = ref_lib.from_grid(29, 15, 4, ext, cases.MECH_JA919, cases.THERMO)
    x, y, z = ref.nodes()
    before = {k: interior(ref.get(k)) for k in ["P", "T", "U", "Yi", "CS", "D", "H", "Gamma", "E"]}
    ref.set_primitive(*cases.rsbi(x, y, z, ref.mechanism().mw, ref.ns))
    for k, v in before.items():
        assert n_unequal(interior(ref.get(k)), v) == 0, k


def test_ghost_fill_matches_reference(ref_lib, port_lib):
    """Face ghost layers after FieldBoundary_3dRSBI (the y-front rebuilds rho, H, Gamma)."""
    ext = (0.0, 0.17, 0.0, 0.08, 0.0, 0.02)
    ref = ref_lib.from_grid(13, 9, 6, ext, cases.MECH_JA919, cases.THERMO)
    x, y, z = ref.nodes()
    port = port_lib(13, 9, 6, x, y, z, ref.mechanism())
    port.set_state(ref.state())
    ref.step(3, 3e-8)
    port.step(3, 3e-8)
    ref.boundary()
    port.boundary()
    b = 2
    faces = [(slice(0, b), slice(b, -b), slice(b, -b)), (slice(-b, None), slice(b, -b), slice(b, -b)),
             (slice(b, -b), slice(0, b), slice(b, -b)), (slice(b, -b), slice(-b, None), slice(b, -b)),
             (slice(b, -b), slice(b, -b), slice(0, b)), (slice(b, -b), slice(b, -b), slice(-b, None))]
    for f in ["P", "D", "U", "V", "W", "H", "Gamma", "T", "Yi"]:
        r, p = ref.get(f), port.get(f)
        for sl in faces:
            assert n_unequal(p[(slice(None),) + sl], r[(slice(None),) + sl]) == 0, (f, sl)


def test_znd_ghost_fill_of_the_restatement(port_lib):
    """The C restatement's ZND ghost fill (the reference's commented-out
    Flowfield::FieldBoundary_1dZND, src/Flowfield.cpp:317-411): the x-low
    ghosts mirror the first nodes with U reflected, the x-high ghosts mirror
    the last nodes with density rebuilt from the mirrored p, T, Y."""
    from oracle import Mechanism
    import eu3d
    ni, nj, nk = 12, 2, 2
    dx = 25e-6
    x = cases.node_coordinates(ni, 0.0, (ni - 1) * dx)
    y = cases.node_coordinates(nj, 0.0, dx)
    md = eu3d.parse_mechanism(cases.MECH_JA919_AR, cases.THERMO_AR)
    P, T, U, V, W, Y = cases.znd(x, y, y, md["mw"], md["ns"])
    U = U + np.linspace(10.0, 20.0, ni + 4)[:, None, None]
    o = port_lib(ni, nj, nk, x, y, y, Mechanism.from_dict(md), boundary="znd")
    o.set_primitive(P, T, U, V, W, Y)
    o.boundary()
    u, d, p = o.get("U")[0], o.get("D")[0], o.get("P")[0]
    assert np.array_equal(u[0:2, 2, 2], -u[3:1:-1, 2, 2])
    assert np.array_equal(u[ni + 2:ni + 4, 2, 2], u[ni + 1:ni - 1:-1, 2, 2])
    assert np.array_equal(p[ni + 2:ni + 4, 2, 2], p[ni + 1:ni - 1:-1, 2, 2])
    assert np.allclose(d[ni + 2:ni + 4, 2, 2], d[ni + 1:ni - 1:-1, 2, 2], rtol=1e-14)


def test_odw_ghost_fill_matches_reference(ref_lib, port_lib):
    """The restatement's ODW ghost fill against the reference's own
    Flowfield::FieldBoundary_3dODW (src/Flowfield.cpp:412-592, compiled in the
    reference but never called; the harness calls it with inflow tables the
    reference allocates and leaves empty): every face layer bitwise, on a
    state with random primitives, then three steps with that ghost fill."""
    ni, nj, nk = 14, 9, 6
    ext = (0.0, 0.013, 0.0, 0.008, 0.0, 0.005)
    ref = ref_lib.from_grid(ni, nj, nk, ext, cases.MECH_JA919, cases.THERMO)
    x, y, z = ref.nodes()
    m = ref.mechanism()
    rng = np.random.default_rng(1)
    shape = ref.shape
    P = 1e5 * (1 + 0.2 * rng.random(shape))
    T = 800 + 900 * rng.random(shape)
    U, V, W = (a * rng.standard_normal(shape) for a in (300.0, 100.0, 100.0))
    Y = rng.random((m.ns,) + shape)
    Y /= Y.sum(axis=0)
    ref.set_primitive(P, T, U, V, W, Y)
    inflow = [5e4 * (1 + rng.random((nj, nk))), 300 + 50 * rng.random((nj, nk)), 2000 + rng.random((nj, nk)),
              -300 + rng.random((nj, nk)), np.zeros((nj, nk))]
    yin = rng.random((m.ns, nj, nk))
    inflow.append(yin / yin.sum(axis=0))
    ref.set_boundary("odw")
    ref.set_inflow(*inflow)
    port = port_lib(ni, nj, nk, x, y, z, m, boundary="odw")
    port.set_state(ref.state())
    port.set_inflow(*inflow)
    ref.boundary()
    port.boundary()
    b = 2
    faces = [(slice(0, b), slice(b, -b), slice(b, -b)), (slice(-b, None), slice(b, -b), slice(b, -b)),
             (slice(b, -b), slice(0, b), slice(b, -b)), (slice(b, -b), slice(-b, None), slice(b, -b)),
             (slice(b, -b), slice(b, -b), slice(0, b)), (slice(b, -b), slice(b, -b), slice(-b, None))]
    for f in ["P", "D", "U", "V", "W", "H", "Gamma", "T", "Yi"]:
        r, p = ref.get(f), port.get(f)
        for sl in faces:
            assert n_unequal(p[(slice(None),) + sl], r[(slice(None),) + sl]) == 0, (f, sl)
    ref.step(3, 2e-8)
    port.step(3, 2e-8)
    for f in ["CS", "T", "Nchem"]:
        assert n_unequal(interior(port.get(f)), interior(ref.get(f))) == 0, f


def test_ns11_mechanism_is_rejected_as_by_the_reference(ref_lib, eu3d_lib, capfd):
    """H2_JA1119.txt (11 species with Ar and He, 5 third-body rows) is not a
    file the reference can read: Reaction::ReactionRead splits each
    stoichiometry row at tabs and calls stoi on every item
    (src/Reaction.cpp:193-214), and several rows of this file end in a tab
    followed by spaces and a carriage return, an item stoi rejects. The
    library's parser rejects it too, with an error code instead of an
    exception."""
    with pytest.raises(RuntimeError):
        ref_lib.from_grid(4, 4, 4, (0.0, 1e-3, 0.0, 1e-3, 0.0, 1e-3), cases.MECH_JA1119, cases.THERMO)
    assert "stoi" in capfd.readouterr().err
    with pytest.raises(eu3d_lib.EU3DError) as e:
        eu3d_lib.parse_mechanism(cases.MECH_JA1119, cases.THERMO)
    assert e.value.name == "EU_ERR_IO"
