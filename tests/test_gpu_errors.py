"""Error behaviour of the C ABI on a device: every failure is a status and a
message, never an exit. Failures are made on the host (bad arguments, a NaN
planted in the uploaded state, a substep cap below what a cell needs); no test
faults the GPU."""
import numpy as np
import pytest

import eu3d_cases as cases
from helpers import golden, init_state

pytestmark = pytest.mark.gpu


def rsbi_solver(eu3d, **kw):
    z = golden("rsbi_17x13x4_s3.npz")
    s = eu3d.Solver(int(z["ni"]), int(z["nj"]), int(z["nk"]), tuple(z["extent"]), **kw)
    s.load_mechanism(cases.MECH_JA919, cases.THERMO)
    s.set_state(init_state(z))
    return s, z


def test_call_order_and_arguments(gpu):
    s = gpu.Solver(9, 9, 9, (0, 1, 0, 1, 0, 1))
    with pytest.raises(gpu.EU3DError) as e:
        s.step(1, 1e-8)
    assert e.value.name == "EU_ERR_NOT_READY"
    s.load_mechanism(cases.MECH_JA919, cases.THERMO)
    with pytest.raises(gpu.EU3DError) as e:
        s.get("NoSuchField")
    assert e.value.name == "EU_ERR_INVALID_ARGUMENT"
    with pytest.raises(gpu.EU3DError) as e:
        s.load_mechanism("/nonexistent", cases.THERMO)
    assert e.value.name == "EU_ERR_IO"
    with pytest.raises(gpu.EU3DError):
        gpu.Solver(1, 9, 9, (0, 1, 0, 1, 0, 1))


def test_negative_dt_rejected(gpu):
    s, z = rsbi_solver(gpu)
    with pytest.raises(gpu.EU3DError) as e:
        s.step(1, -1e-8)
    assert e.value.name == "EU_ERR_INVALID_ARGUMENT"


def test_nonfinite_state_reported(gpu):
    s, z = rsbi_solver(gpu)
    st = init_state(z)
    st["CS"] = st["CS"].copy()
    st["CS"][0, 8, 7, 3] = np.nan
    s.set_state(st)
    with pytest.raises(gpu.EU3DError) as e:
        s.step(1, 3e-8)
    assert e.value.name == "EU_ERR_NONFINITE"
    s2, _ = rsbi_solver(gpu)  # a fresh handle on the same device still works
    s2.step(1, 3e-8)


def test_substep_cap_reported(gpu):
    z = golden("rsbi_36x18x3_s100.npz")
    s = gpu.Solver(int(z["ni"]), int(z["nj"]), int(z["nk"]), tuple(z["extent"]), max_substeps=1)
    s.load_mechanism(cases.MECH_JA919, cases.THERMO)
    s.set_state(init_state(z))
    with pytest.raises(gpu.EU3DError) as e:
        s.step(100, float(z["dt"]))
    assert e.value.name == "EU_ERR_NCHEM"
