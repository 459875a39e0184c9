"""Generate the golden fixtures in tests/golden/ from the reference's own CPU code.

Runs the reference's CPU hot path, compiled from its sources by
`make -C oracle ref` (oracle/_ref/libeu3d_ref.so), and stores small inputs and
outputs as .npz files. Needs the reference checkout (for the build); the
fixtures themselves travel with the repository.

    python tests/golden/make_golden.py [bubble_hundred]

(with bubble_hundred: only the 100-step shock-bubble fixture)
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "eu3d-gpu_b200"))

from oracle import RefOracle, interior  # noqa: E402
import eu3d_cases as cases  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
FIELDS = ["CS", "T", "E", "P", "D", "U", "V", "W", "H", "Gamma", "Yi", "Nchem", "CMS", "Mc", "Di", "Wav", "Rgas",
          "Cp", "C", "Ma"]
STATE = ["CS", "T", "E", "P", "D", "U", "V", "W", "H", "Gamma", "Yi"]


def ref_for(ni, nj, nk, extent, mech=cases.MECH_JA919):
    return RefOracle.from_grid(ni, nj, nk, extent, mech, cases.THERMO, workdir=tempfile.mkdtemp(prefix="eu3d_g_"))


def sanitized_state(ref):
    """The state the next step reads. Ghost D, H, Gamma, E and CS are never read
    before the step's own ghost fill rewrites them (the reference leaves them
    uninitialised at start-up), so they are stored as zeros."""
    st = ref.state()
    b = ref.bc
    for k in ("D", "H", "Gamma", "E", "CS"):
        a = np.zeros_like(st[k])
        a[:, b:-b, b:-b, b:-b] = st[k][:, b:-b, b:-b, b:-b]
        st[k] = a
    return st


def save_case(name, ref, steps, dt, extent, fields=FIELDS, primitive=None):
    """Initial state (full, or only the primitive fields it was set from) and
    interior outputs after `steps` reference timesteps."""
    if primitive is None:
        init = {f"init_{k}": v for k, v in sanitized_state(ref).items()}
    else:
        init = {f"prim_{k}": v for k, v in zip("PTUVWY", primitive)}
    ref.step(steps, dt)
    out = {f"out_{k}": interior(ref.get(k)) for k in fields}
    x, y, z = ref.nodes()
    np.savez_compressed(os.path.join(OUT, name), ni=ref.ni, nj=ref.nj, nk=ref.nk, bc=ref.bc, steps=steps, dt=dt,
                        extent=np.array(extent), x=x, y=y, z=z, **init, **out)
    print("wrote", name)


def main():
    # mechanism + thermo tables as the reference parses them
    ext = (0.0, 0.17, 0.0, 0.08, 0.0, 0.02)
    ref = ref_for(17, 13, 4, ext)
    ref.mechanism().save_npz(os.path.join(OUT, "mech_ja919.npz"))

    # NASA thermo at the reference's own check temperatures (src/Reaction.cpp:333-335)
    temps = np.array([300.0, 999.0, 1000.0, 1001.0, 2000.0])
    mech = ref.mechanism()
    tab = np.zeros((len(temps), mech.ns, 2, 3))
    for a, T in enumerate(temps):
        for s in range(mech.ns):
            tab[a, s, 0] = ref.thermo(T, 8.31434 / mech.mw[s], s)
            tab[a, s, 1] = ref.thermo(T, 8.31434, s)
    np.savez(os.path.join(OUT, "thermo_points.npz"), T=temps, cp_h_s=tab)
    print("wrote thermo_points.npz")

    # RSBI, the reference's own initial state (FieldInitial/ReactionInitial), 3 steps
    save_case("rsbi_17x13x4_s3.npz", ref, 3, 3e-8, ext)

    # RSBI, 100 steps on a coarse thin grid: Nchem grows above 1 near the front
    r2 = ref_for(36, 18, 3, ext)
    save_case("rsbi_36x18x3_s100.npz", r2, 100, 3e-8, ext, fields=["CS", "T", "E", "Nchem", "CMS"])

    # 3-D shock-bubble: the shock enters the perturbed sphere (v, w develop), 20 steps
    ext3 = (0.0, 0.012, 0.0, 0.006, 0.0, 0.006)
    ni, nj, nk = 25, 13, 13
    r3 = ref_for(ni, nj, nk, ext3)
    x, y, z = r3.nodes()
    P, T, U, V, W, Y = cases.shock_bubble(x, y, z, r3.mechanism().mw, r3.ns, radius=2e-3, shock_x=2e-3,
                                           standoff=3e-3, seed=3)
    r3.set_primitive(P, T, U, V, W, Y)
    save_case("bubble_25x13x13_s20.npz", r3, 20, 1e-7, ext3, fields=["CS", "T", "E", "Nchem", "CMS"],
              primitive=(P, T, U, V, W, Y))
    bubble_hundred()


def bubble_hundred():
    """3-D shock-bubble over 100 steps: the shock runs through the whole
    perturbed sphere (the bound the hot path is held to is relative L-inf
    <= 1e-9 per conserved variable after 100 steps). dt from the reference's
    CFL rule at 0.25 on the initial fields (at 0.5 the reference's forward
    Euler MUSCL/AUSM step goes non-finite on this case once the shock is in
    the bubble)."""
    ext = (0.0, 0.016, 0.0, 0.008, 0.0, 0.008)
    r = ref_for(33, 17, 17, ext)
    x, y, z = r.nodes()
    prim = cases.shock_bubble(x, y, z, r.mechanism().mw, r.ns, radius=3e-3, shock_x=2.5e-3, standoff=4.5e-3, seed=3)
    r.set_primitive(*prim)
    f = {k: r.get(k)[0] for k in ("P", "D", "U", "V", "Gamma")}
    dt = cases.cfl_dt(x, y, f["P"], f["D"], f["U"], f["V"], f["Gamma"], 0.25)
    save_case("bubble_33x17x17_s100.npz", r, 100, dt, ext, fields=["CS", "T", "E", "Nchem"], primitive=prim)


if __name__ == "__main__":
    if sys.argv[1:] == ["bubble_hundred"]:
        bubble_hundred()
    else:
        main()
