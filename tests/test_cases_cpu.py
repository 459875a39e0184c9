"""The case builders (eu3d-gpu_b200/eu3d_cases.py) on the CPU: the ODW
freestream from input-ODW.txt and its composition, and the equivalence-ratio
profile of the 3-D case."""
import math
import os
import sys

import numpy as np

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "eu3d-gpu_b200"))
import eu3d_cases as cases  # noqa: E402


def _mech(eu3d):
    return eu3d.parse_mechanism(cases.MECH_JA919, cases.THERMO)


def test_h2_air_stoichiometric_mass_fractions(eu3d_lib):
    m = _mech(eu3d_lib)
    y = cases.h2_air(m["mw"], m["ns"])
    assert abs(y.sum() - 1.0) < 1e-15
    assert abs(y[cases.S_H2] - 0.0285) < 5e-4
    assert abs(y[cases.S_O2] - 0.2264) < 5e-4
    assert abs(y[cases.S_N2] - 0.7451) < 5e-4


def test_odw_freestream_follows_the_input_file(eu3d_lib):
    """P, T and Mach from input-ODW.txt; the velocity turned into the wedge
    surface by the wedge angle; Mach = speed / frozen sound speed."""
    eu3d = eu3d_lib
    m = _mech(eu3d)
    P, T, U, V, W, Y = cases.odw_inflow(m, 3, 4)
    assert np.all(P == eu3d.read_value(cases.INPUT_ODW, "P")) and np.all(T == eu3d.read_value(cases.INPUT_ODW, "T"))
    angle = math.degrees(math.atan2(-V[0, 0], U[0, 0]))
    assert abs(angle - eu3d.read_value(cases.INPUT_ODW, "angle")) < 1e-12
    g, r = cases.mixture_gamma(m, T[0, 0], Y[:, 0, 0])
    mach = math.hypot(U[0, 0], V[0, 0]) / math.sqrt(g * r * T[0, 0])
    assert abs(mach - eu3d.read_value(cases.INPUT_ODW, "Mach")) < 1e-12
    assert 1.38 < g < 1.42
    assert np.all(W == 0)


def test_odw_phi_profile():
    """1 + a normalised four-mode sine sum whose largest magnitude is 0.1."""
    z = cases.node_coordinates(97, 0.0, 0.02)
    phi = cases.odw_phi(z)
    assert phi.shape == (97,)
    assert abs(np.abs(phi - 1).max() - 0.1) < 1e-12
    assert not np.allclose(phi, cases.odw_phi(z, seed=5))


def test_odw_fields_repeat_the_inflow(eu3d_lib):
    m = _mech(eu3d_lib)
    x, y, z = (cases.node_coordinates(n, 0.0, 0.01) for n in (9, 7, 6))
    (P, T, U, V, W, Y), inflow = cases.odw(x, y, z, m, phi=cases.odw_phi(z))
    assert P.shape == (13, 11, 10) and Y.shape == (m["ns"], 13, 11, 10)
    assert np.array_equal(Y[:, 5, 4, 2:-2], inflow[5][:, 2, :])
    assert np.array_equal(U[0, 0, 2:-2], inflow[2][0])
    assert np.allclose(Y.sum(axis=0), 1.0)
