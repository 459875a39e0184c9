"""The three-stage TVD Runge-Kutta advection of the C restatement (the scheme
eu_set_time_scheme(EU_TIME_RK3) runs on the GPU, which tests/test_gpu_parity.py
holds to the restatement). The reference's TimeAdv::TVD_RK3
(src/TimeAdv.cpp:210-221) is an empty stub, so there is nothing of the
reference to compare with; instead the scheme's temporal error is checked on a
smooth case against a run with 16 times smaller steps: far below the Euler
step's and shrinking as the step shrinks."""
import numpy as np

import eu3d_cases as cases
from helpers import golden_mechanism

NI, L = 81, 0.02


def _run(port_lib, scheme, dt, n):
    """An acoustic wave in N2 carried by a 100 m/s mean flow (the upwind
    direction of every face stays fixed), n steps of dt."""
    mech = golden_mechanism()
    x = cases.node_coordinates(NI, 0.0, L)
    y = cases.node_coordinates(2, 0.0, L / (NI - 1))
    X = x[:, None, None] * np.ones((1, len(y), len(y)))
    wave = np.sin(2 * np.pi * X / L)
    P, T = 1e5 * (1 + 0.02 * wave), 300.0 * (1 + 0.02 * 0.4 / 1.4 * wave)
    Z = np.zeros_like(P)
    Y = np.zeros((mech.ns,) + P.shape)
    Y[cases.S_N2] = 1.0
    p = port_lib(NI, 2, 2, x, y, y, mech, nthreads=1)
    p.set_primitive(P, T, Z + 100.0, Z, Z, Y)
    p.set_scheme(scheme)
    p.step(n, dt)
    cs = p.get("CS")[:, 2:-2, 2:-2, 2:-2]
    p.close()
    return cs


def test_rk3_temporal_error(port_lib):
    t_end = 0.6 * (L / (NI - 1)) / 350.0 * 40  # 40 steps at an acoustic CFL of 0.6
    ref = _run(port_lib, "rk3", t_end / 640, 640)
    err = {}
    for scheme in ("ee", "rk3"):
        err[scheme] = [float(np.abs(_run(port_lib, scheme, t_end / n, n) - ref).max() / np.abs(ref).max())
                       for n in (40, 80, 160)]
    assert err["rk3"][0] < err["ee"][0] / 50, err
    assert err["rk3"][1] < err["rk3"][0] / 2 and err["rk3"][2] < err["rk3"][1] / 2, err
