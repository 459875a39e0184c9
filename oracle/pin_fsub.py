"""Pin F_sub, the FP64 work of one kinetics substep of one cell (test
infrastructure; run on the CPU, the result is recorded once).

    make -C oracle flops && python oracle/pin_fsub.py [--steps 100] [--grid 281 141 2]

Runs the thin RSBI case (the reference's own wired case: 281 x 141 x 2 nodes
over 0.17 x 0.08 x 0.02 m, dt 3e-8 s, H2_JA919) through the counting build of
the C restatement (flop_count.cpp) and divides the kinetics phase's counted
operations by the substeps it ran (sum of Nchem over all cells and steps).
"""
import argparse
import ctypes
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [HERE, os.path.join(os.path.dirname(HERE), "eu3d-gpu_b200")]

import eu3d_cases as cases  # noqa: E402
import oracle  # noqa: E402

LIB = os.path.join(HERE, "_build", "libeu3d_flops.so")


class CountingOracle(oracle.PortOracle):
    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            saved = oracle.PORT_LIB
            oracle.PORT_LIB = LIB
            try:
                cls._lib = None
                lib = oracle.PortOracle.lib.__func__(cls)
            finally:
                oracle.PORT_LIB = saved
            lib.fc_step.restype = ctypes.c_int
            lib.fc_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
            cls._lib = lib
        return cls._lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--grid", type=int, nargs=3, default=[281, 141, 2])
    ap.add_argument("--dt", type=float, default=3e-8)
    args = ap.parse_args()
    ni, nj, nk = args.grid
    ext = (0.0, 0.17, 0.0, 0.08, 0.0, 0.02)
    mech = oracle.Mechanism.from_npz(os.path.join(os.path.dirname(HERE), "tests", "golden", "mech_ja919.npz"))
    x, y, z = (cases.node_coordinates(n, a, b) for n, a, b in ((ni, ext[0], ext[1]), (nj, ext[2], ext[3]),
                                                               (nk, ext[4], ext[5])))
    o = CountingOracle(ni, nj, nk, x, y, z, mech, nthreads=1)
    o.set_primitive(*cases.rsbi(x, y, z, mech.mw, mech.ns))
    counts = np.zeros(8, dtype=np.uint64)
    sub = ctypes.c_longlong(0)
    t0 = time.time()
    for n in range(args.steps):
        rc = o.lib().fc_step(o.h, args.dt, counts.ctypes.data, ctypes.byref(sub))
        if rc:
            raise RuntimeError("a cell predicted Nchem <= 0")
    names = ["add/sub", "mul", "div", "sqrt", "exp", "log", "pow (exponent 0/1/2)", "pow (other)"]
    s = sub.value
    flops = int(counts[0] + counts[1] + counts[2] + counts[3])
    print(f"{args.steps} steps of {ni}x{nj}x{nk} ({time.time() - t0:.0f} s): {s} substeps")
    for nm, c in zip(names, counts):
        print(f"  {nm:24s} {int(c) / s:10.1f} per substep")
    print(f"F_sub = {flops / s:.0f} flop per cell-substep (add+sub+mul+div+sqrt)")


if __name__ == "__main__":
    main()
