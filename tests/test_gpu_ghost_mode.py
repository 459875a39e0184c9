"""EU_GHOSTS_STORED (eu_set_ghost_mode): the z-face ghost nodes written with
each stored interior node instead of by the ghost fill at the start of each
step. The interior state must be bitwise the reference placement's; only what
the z-face ghost nodes hold between steps differs (the interior at the step's
end instead of its start)."""
import numpy as np
import pytest

import eu3d_cases as cases
from helpers import interior, n_unequal

pytestmark = pytest.mark.gpu

STATE = ("CS", "T", "E", "P", "D", "U", "V", "W", "H", "Gamma", "Yi")


def snapshot(s):
    out = {k: s.get(k) for k in STATE}
    for k in ("T", "E", "P", "D", "U", "V", "W", "H", "Gamma"):
        out[k] = out[k][0]
    return out


def hot_block_prim(ni, nj, nk, mech):
    return cases.hot_reacting_block(ni + 4, nj + 4, nk + 4, mech["mw"], mech["ns"])


@pytest.mark.parametrize("precision,arith,chemistry,case", [
    ("fp64", "strict", "stiff", "bubble"),
    ("mixed", "fast", "stiff", "bubble"),
    ("mixed", "fast", "learned", "bubble"),
    ("mixed", "fast", "stiff", "igniting"),  # cells deferred to the warp-per-cell kinetics
])
def test_stored_z_ghosts_keep_the_interior(gpu, precision, arith, chemistry, case):
    """Three steps, a re-upload of the state (after which the next ghost fill
    forms the z faces again) and three more steps: conserved, T, E and
    primitives of every interior node bitwise equal between the two ghost
    modes, on a ragged 40 x 21 x 45 shock-bubble grid and on an igniting
    24 x 8 x 8 block; and after the steps each z-face ghost node of the stored
    run mirrors its source node (W reflected), the values the next ghost fill
    would have copied."""
    mech = gpu.parse_mechanism(cases.MECH_JA919, cases.THERMO)
    if case == "bubble":
        ni, nj, nk = 40, 21, 45
        ext = (0.0, 0.02, 0.0, 0.01, 0.0, 0.012)
        x, y, z = (cases.node_coordinates(n, 0, e) for n, e in ((ni, 0.02), (nj, 0.01), (nk, 0.012)))
        prim = cases.shock_bubble(x, y, z, mech["mw"], mech["ns"], radius=3e-3, shock_x=3e-3, standoff=5e-3, seed=5)
    else:
        ni, nj, nk = 24, 8, 8
        ext = (0.0, 0.006, 0.0, 0.002, 0.0, 0.002)
        prim = hot_block_prim(ni, nj, nk, mech)
    out = {}
    for mode in ("reference", "stored"):
        s = gpu.Solver(ni, nj, nk, ext, precision=precision, arith=arith, chemistry=chemistry)
        s.set_mechanism(mech)
        s.set_primitive(*prim)
        if chemistry == "learned":
            import learned
            model, gate = learned.load()
            learned.attach(s, model, gate)
        s.set_ghost_mode(mode)
        s.step(3, 2e-8)
        s.set_state(snapshot(s))
        st = s.step(3, 2e-8)
        assert st["nonfinite"] == 0
        if case == "igniting":
            assert st["max_nchem"] > 4, st  # some cells went to the warp-per-cell kinetics
        out[mode] = snapshot(s)
        s.close()
    ref, got = out["reference"], out["stored"]
    for k in STATE:
        a, b = np.asarray(ref[k]), np.asarray(got[k])
        if a.ndim == 3:
            a, b = a[None], b[None]
        assert n_unequal(interior(a), interior(b)) == 0, k
    # z ghosts of the stored run: ghost k' mirrors node 2 bc - 1 - k' (below)
    # and 2 (nk + bc) - 1 - k' (above), over the interior (i, j)
    bc = 2
    nz = nk + 2 * bc
    for k in ("T", "P", "D", "U", "V", "W", "H", "Gamma", "Yi"):  # the mirrored fields (not CS, E)
        a = np.asarray(got[k])
        if a.ndim == 3:
            a = a[None]
        sign = -1.0 if k == "W" else 1.0
        for g in list(range(bc)) + list(range(nk + bc, nz)):
            src = 2 * bc - 1 - g if g < bc else 2 * (nk + bc) - 1 - g
            ghost = a[:, bc:-bc, bc:-bc, g]
            want = sign * a[:, bc:-bc, bc:-bc, src]
            if precision == "mixed" and k != "T":
                # mixed precision keeps FP32 primitive planes: the interior is
                # read back from the FP64 state it was rounded from, a ghost
                # node from the FP32 plane
                want = want.astype(np.float32).astype(np.float64)
            assert n_unequal(ghost, want) == 0, (k, g)


def test_stored_z_ghosts_need_a_mirror_fill(gpu):
    """The ODW fill rebuilds the z ghosts' thermo, so the stored mode is
    refused there, with an error."""
    mech = gpu.parse_mechanism(cases.MECH_JA919, cases.THERMO)
    s = gpu.Solver(16, 8, 8, (0.0, 0.016, 0.0, 0.008, 0.0, 0.008), boundary="odw")
    s.set_mechanism(mech)
    with pytest.raises(RuntimeError):
        s.set_ghost_mode("stored")
    s.set_ghost_mode("reference")
    s.close()
