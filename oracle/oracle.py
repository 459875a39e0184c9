"""ctypes front-ends for the CPU checkers of the EU3D hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` and
by the ``cpu_baseline`` / ``--impl reference`` legs of bench.py, never by the
library itself.

* ``RefOracle`` drives the reference's own CPU code, compiled from its sources
  by ``oracle/Makefile`` into ``oracle/_ref/libeu3d_ref.so`` (see
  ``oracle/ref_harness.cpp``).  Its fields come back in the reference's native
  layout and are converted here to structure-of-arrays planes.
* ``PortOracle`` drives the plain-C restatement ``oracle/eu3d_oracle.c``
  (``oracle/_build/libeu3d_oracle.so``), which is pinned bit-for-bit against
  ``RefOracle`` and against the fixtures in ``tests/golden/``.

Both take the same inputs: a grid (node coordinates with ghosts), mechanism
tables in the reference's layouts, and initial primitive fields.
"""
from __future__ import annotations

import ctypes
import os
import tempfile
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libeu3d_ref.so")
PORT_LIB = os.path.join(HERE, "_build", "libeu3d_oracle.so")

_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int

FIELDS_1 = ["P", "D", "T", "U", "V", "W", "H", "E", "Gamma"]


@dataclass
class Mechanism:
    """Mechanism + thermo tables in the reference's layouts (src/Reaction.cpp:156-327)."""

    ns: int
    nr: int
    mw: np.ndarray        # (ns,)
    coeff_lo: np.ndarray  # (9, ns)   Coeff0: T < 1000 K
    coeff_hi: np.ndarray  # (9, ns)   Coeff1
    af: np.ndarray        # (nr,)
    bf: np.ndarray
    eaf: np.ndarray
    stoi_f: np.ndarray    # (ns, nr)
    stoi_b: np.ndarray
    tb: np.ndarray        # (ns, nr)  third-body efficiencies (0 for ordinary reactions)

    def arrays(self):
        return [np.ascontiguousarray(a, dtype=np.float64) for a in
                (self.mw, self.coeff_lo, self.coeff_hi, self.af, self.bf, self.eaf,
                 self.stoi_f, self.stoi_b, self.tb)]

    @classmethod
    def from_npz(cls, path):
        z = np.load(path)
        return cls(int(z["ns"]), int(z["nr"]), z["mw"], z["coeff_lo"], z["coeff_hi"], z["af"], z["bf"],
                   z["eaf"], z["stoi_f"], z["stoi_b"], z["tb"])

    @classmethod
    def from_dict(cls, d):
        """From the library parser's dict (eu3d.parse_mechanism): same layouts."""
        return cls(int(d["ns"]), int(d["nr"]), *[np.asarray(d[k], dtype=np.float64) for k in
                                                  ("mw", "coeff_lo", "coeff_hi", "af", "bf", "eaf", "stoi_f",
                                                   "stoi_b", "tb")])

    def save_npz(self, path):
        np.savez(path, ns=self.ns, nr=self.nr, mw=self.mw, coeff_lo=self.coeff_lo, coeff_hi=self.coeff_hi,
                 af=self.af, bf=self.bf, eaf=self.eaf, stoi_f=self.stoi_f, stoi_b=self.stoi_b, tb=self.tb)


def write_grid_file(path, ni, nj, nk, xa, xb, ya, yb, za, zb, bc=2):
    """A grid file in the reference's ``key value`` format (input/grid-3dRSBI.txt)."""
    xa, xb, ya, yb, za, zb = (float(v) for v in (xa, xb, ya, yb, za, zb))  # repr of a plain float
    with open(path, "w") as f:
        f.write(f"total_ni    {ni}\nxa    {xa!r}\nxb    {xb!r}\n"
                f"total_nj    {nj}\nya    {ya!r}\nyb    {yb!r}\n"
                f"total_nk    {nk}\nza    {za!r}\nzb    {zb!r}\nbc    {bc}\n")


def write_input_file(path, ns, nr, p_pre=101325.0, t_pre=1000.0, m_wave=3.0):
    """An initial-condition file in the reference's format (input/input-3dRSBI.txt)."""
    with open(path, "w") as f:
        f.write(f"P_pre    {p_pre!r}\nT_pre    {t_pre!r}\nM_wave    {m_wave!r}\nNS    {ns}\nNR    {nr}\n")


def node_coordinates(total_n, a, b, bc=2, blocks=1, block=0):
    """Node coordinates with ghosts of block `block` of `blocks` along one axis:
    Mesh::Initial (src/Mesh.cpp:96-119) gives the block (total_n - 1) / blocks + 1
    nodes at the global spacing, Mesh::Boundary (:131-142) mirrors the ghosts
    about the block's end nodes."""
    n = (total_n - 1) // blocks + 1
    d = (b - a) / (total_n - 1)
    x = np.zeros(n + 2 * bc)
    for i in range(bc, n + bc):
        x[i] = a + (block * (n - 1) + i - bc) * d
    for i in range(bc):
        x[i] = 2 * x[bc] - x[2 * bc - i]
        x[n + bc + i] = 2 * x[n + bc - 1] - x[n + bc - 1 - i - 1]
    return x


class RefOracle:
    """The reference's CPU hot path (oracle/_ref). Single-threaded, as the reference."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(REF_LIB):
                raise FileNotFoundError(f"{REF_LIB} missing: run `make -C oracle ref` where the reference is present")
            lib = ctypes.CDLL(REF_LIB)
            lib.ref_create.restype = _P
            lib.ref_create.argtypes = [ctypes.c_char_p] * 4
            lib.ref_destroy.argtypes = [_P]
            lib.ref_dims.argtypes = [_P, _P]
            lib.ref_get.restype = ctypes.c_long
            lib.ref_get.argtypes = [_P, ctypes.c_char_p, _P]
            lib.ref_put.restype = ctypes.c_long
            lib.ref_put.argtypes = [_P, ctypes.c_char_p, _P]
            lib.ref_set_primitive.argtypes = [_P] * 7
            lib.ref_step.argtypes = [_P, _I, _D]
            lib.ref_boundary.argtypes = [_P]
            lib.ref_set_boundary.argtypes = [_P, _I]
            lib.ref_set_inflow.argtypes = [_P] * 7
            lib.ref_thermo.argtypes = [_P, _D, _D, _I, _P]
            cls._lib = lib
        return cls._lib

    def __init__(self, grid_path, input_path, mech_path, thermo_path):
        lib = self.lib()
        self.h = lib.ref_create(grid_path.encode(), input_path.encode(), mech_path.encode(), thermo_path.encode())
        if not self.h:
            raise RuntimeError("ref_create failed")
        d = np.zeros(7, np.int32)
        lib.ref_dims(self.h, d.ctypes.data)
        self.ni, self.nj, self.nk, self.bc, self.ns, self.nr, self.tb_count = (int(v) for v in d)
        self.shape = (self.ni + 2 * self.bc, self.nj + 2 * self.bc, self.nk + 2 * self.bc)
        self.n3 = int(np.prod(self.shape))

    @classmethod
    def from_grid(cls, ni, nj, nk, extent, mech_path, thermo_path, workdir=None):
        workdir = workdir or tempfile.mkdtemp(prefix="eu3d_ref_")
        g = os.path.join(workdir, "grid.txt")
        i = os.path.join(workdir, "input.txt")
        write_grid_file(g, ni, nj, nk, *extent)
        write_input_file(i, 9, 19)
        return cls(g, i, mech_path, thermo_path)

    def close(self):
        if self.h:
            self.lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _raw(self, name, n):
        out = np.empty(n)
        got = self.lib().ref_get(self.h, name.encode(), out.ctypes.data)
        if got != n:
            raise KeyError(f"{name}: {got}")
        return out

    def get(self, name):
        """Field as SoA planes: (nplanes, nx, ny, nz); 3-D fields have nplanes == 1."""
        if name in ("Yi", "Di", "Mc", "CMS"):
            a = self._raw(name, self.n3 * self.ns).reshape(self.n3, self.ns)
            return np.ascontiguousarray(a.T).reshape(self.ns, *self.shape)
        if name == "CS":
            a = self._raw(name, self.n3 * (self.ns + 4)).reshape(self.n3, self.ns + 4)
            return np.ascontiguousarray(a.T).reshape(self.ns + 4, *self.shape)
        return self._raw(name, self.n3).reshape(1, *self.shape)

    def put(self, name, planes):
        planes = np.asarray(planes, dtype=np.float64)
        if name in ("Yi", "Di", "Mc", "CS", "CMS"):
            a = np.ascontiguousarray(planes.reshape(planes.shape[0], -1).T)
        else:
            a = np.ascontiguousarray(planes.reshape(-1))
        got = self.lib().ref_put(self.h, name.encode(), a.ctypes.data)
        if got < 0:
            raise KeyError(name)

    def vector(self, name, n):
        return self._raw(name, n)

    def nodes(self):
        nx, ny, nz = self.shape
        return self.vector("xnode", nx), self.vector("ynode", ny), self.vector("znode", nz)

    def mechanism(self) -> Mechanism:
        ns, nr = self.ns, self.nr
        v = self.vector
        return Mechanism(ns, nr, v("Mw", ns), v("Coeff0", 9 * ns).reshape(9, ns), v("Coeff1", 9 * ns).reshape(9, ns),
                         v("Af", nr), v("Bf", nr), v("Eaf", nr), v("Stoi_F", ns * nr).reshape(ns, nr),
                         v("Stoi_B", ns * nr).reshape(ns, nr), v("React_TB", ns * nr).reshape(ns, nr))

    def set_primitive(self, P, T, U, V, W, Y):
        """Y as (ns, nx, ny, nz) planes; converted to the reference's AoS layout."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (P, T, U, V, W)]
        y = np.ascontiguousarray(np.asarray(Y, dtype=np.float64).reshape(self.ns, -1).T)
        self.lib().ref_set_primitive(self.h, *[a.ctypes.data for a in arrs], y.ctypes.data)

    def step(self, nsteps, dt):
        self.lib().ref_step(self.h, int(nsteps), float(dt))

    def boundary(self):
        self.lib().ref_boundary(self.h)

    def set_boundary(self, kind):
        """The ghost fill step() and boundary() run: "rsbi" (FieldBoundary_3dRSBI) or
        "odw" (the reference's FieldBoundary_3dODW, which Euler::Computing never calls)."""
        self.lib().ref_set_boundary(self.h, {"rsbi": 0, "odw": 1}[kind])

    def set_inflow(self, P, T, U, V, W, Y):
        """The ODW inflow tables (Uint .. Yint) over the interior (j, k) nodes."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (P, T, U, V, W, Y)]
        self.lib().ref_set_inflow(self.h, *[a.ctypes.data for a in arrs])

    def thermo(self, T, R, s):
        out = np.zeros(3)
        self.lib().ref_thermo(self.h, float(T), float(R), int(s), out.ctypes.data)
        return out

    def state(self):
        """Every persistent field of the timestep, as planes (see PortOracle.set_state)."""
        st = {n: self.get(n) for n in FIELDS_1 + ["Yi", "CS"]}
        return st


class PortOracle:
    """The plain-C restatement (oracle/eu3d_oracle.c), multithreaded over x planes."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(PORT_LIB):
                raise FileNotFoundError(f"{PORT_LIB} missing: run `make -C oracle port`")
            lib = ctypes.CDLL(PORT_LIB)
            lib.eo_create.restype = _P
            lib.eo_create.argtypes = [_I, _I, _I, _I, _P, _P, _P, _P, _I]
            lib.eo_destroy.argtypes = [_P]
            lib.eo_set_primitive.argtypes = [_P] * 7
            lib.eo_set_state.argtypes = [_P] * 12
            lib.eo_step.restype = _I
            lib.eo_step.argtypes = [_P, _I, _D]
            lib.eo_boundary.argtypes = [_P]
            lib.eo_set_boundary.argtypes = [_P, _I]
            lib.eo_set_exchange.argtypes = [_P, _I, _I]
            lib.eo_set_inflow.argtypes = [_P] * 7
            lib.eo_set_wall.argtypes = [_P, _I]
            lib.eo_set_scheme.argtypes = [_P, _I]
            lib.eo_halo_count.restype = ctypes.c_long
            lib.eo_halo_count.argtypes = [_P]
            lib.eo_halo_pack.argtypes = [_P, _I, _P]
            lib.eo_halo_unpack.argtypes = [_P, _I, _P]
            lib.eo_get.restype = _I
            lib.eo_get.argtypes = [_P, ctypes.c_char_p, _P]
            lib.eo_thermo.argtypes = [_P, _D, _D, _I, _P]
            lib.eo_muscl.argtypes = [_P, _P, _P]
            lib.eo_ausm.argtypes = [_P, _P, _P, _P, _I, _P]
            lib.eo_temperature.restype = _D
            lib.eo_temperature.argtypes = [_P, _D, _D, _P]
            cls._lib = lib
        return cls._lib

    class _Mech(ctypes.Structure):
        _fields_ = [("ns", _I), ("nr", _I)] + [(n, _P) for n in
                                                ("mw", "coeff_lo", "coeff_hi", "af", "bf", "eaf",
                                                 "stoi_f", "stoi_b", "tb")]

    def __init__(self, ni, nj, nk, x, y, z, mech: Mechanism, bc=2, nthreads=None, boundary="rsbi"):
        lib = self.lib()
        self.ni, self.nj, self.nk, self.bc = ni, nj, nk, bc
        self.ns, self.nr = mech.ns, mech.nr
        self.shape = (ni + 2 * bc, nj + 2 * bc, nk + 2 * bc)
        self.n3 = int(np.prod(self.shape))
        self._keep = mech.arrays()
        m = self._Mech(mech.ns, mech.nr, *[a.ctypes.data for a in self._keep])
        xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z)]
        nthreads = nthreads or min(os.cpu_count() or 1, 32)
        self.h = lib.eo_create(ni, nj, nk, bc, xs[0].ctypes.data, xs[1].ctypes.data, xs[2].ctypes.data,
                               ctypes.byref(m), int(nthreads))
        if not self.h:
            raise RuntimeError("eo_create failed")
        lib.eo_set_boundary(self.h, {"rsbi": 0, "znd": 1, "odw": 2}[boundary])

    def close(self):
        if self.h:
            self.lib().eo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_primitive(self, P, T, U, V, W, Y):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (P, T, U, V, W, Y)]
        self.lib().eo_set_primitive(self.h, *[a.ctypes.data for a in arrs])

    def set_state(self, st):
        order = ["CS", "T", "E", "P", "D", "U", "V", "W", "H", "Gamma", "Yi"]
        arrs = [np.ascontiguousarray(st[n], dtype=np.float64) for n in order]
        self.lib().eo_set_state(self.h, *[a.ctypes.data for a in arrs])

    def step(self, nsteps, dt):
        rc = self.lib().eo_step(self.h, int(nsteps), float(dt))
        if rc != 0:
            raise RuntimeError("oracle: a cell predicted Nchem <= 0")

    def boundary(self):
        self.lib().eo_boundary(self.h)

    def set_inflow(self, P, T, U, V, W, Y):
        """ODW x-low inflow tables over the interior (j, k) nodes: planes (nj, nk), Y (ns, nj, nk)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (P, T, U, V, W, Y)]
        self.lib().eo_set_inflow(self.h, *[a.ctypes.data for a in arrs])

    def set_scheme(self, scheme):
        """Advection time scheme: "ee" (the reference's) or "rk3" (eo_set_scheme)."""
        self.lib().eo_set_scheme(self.h, {"ee": 0, "rk3": 1}[scheme])

    def set_wall(self, first_wall_node):
        """ODW: the y-low wall starts at this local x node (eo_set_wall)."""
        self.lib().eo_set_wall(self.h, int(first_wall_node))

    def set_exchange(self, x_low, x_high):
        """x faces whose ghost nodes come from a neighbouring block (eo_halo_unpack)."""
        self.lib().eo_set_exchange(self.h, int(bool(x_low)), int(bool(x_high)))

    def halo_count(self):
        return int(self.lib().eo_halo_count(self.h))

    def halo_pack(self, face, out):
        """Fill `out` (float64, contiguous, halo_count values) with the face's message."""
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == self.halo_count()
        self.lib().eo_halo_pack(self.h, int(face), out.ctypes.data)

    def halo_unpack(self, face, msg):
        m = np.ascontiguousarray(msg, dtype=np.float64)
        assert m.size == self.halo_count()
        self.lib().eo_halo_unpack(self.h, int(face), m.ctypes.data)

    def get(self, name):
        planes = {"Yi": self.ns, "Di": self.ns, "Mc": self.ns, "CMS": self.ns, "CS": self.ns + 4}.get(name, 1)
        out = np.empty(planes * self.n3)
        got = self.lib().eo_get(self.h, name.encode(), out.ctypes.data)
        if got != planes:
            raise KeyError(name)
        return out.reshape(planes, *self.shape)

    def thermo(self, T, R, s):
        out = np.zeros(3)
        self.lib().eo_thermo(self.h, float(T), float(R), int(s), out.ctypes.data)
        return out

    def temperature(self, T0, E, Y):
        y = np.ascontiguousarray(Y, dtype=np.float64)
        return self.lib().eo_temperature(self.h, float(T0), float(E), y.ctypes.data)

    @classmethod
    def muscl(cls, f4):
        f = np.ascontiguousarray(f4, dtype=np.float64)
        lo, hi = ctypes.c_double(), ctypes.c_double()
        cls.lib().eo_muscl(f.ctypes.data, ctypes.byref(lo), ctypes.byref(hi))
        return lo.value, hi.value

    def ausm(self, lr14, yl, yr, direction):
        out = np.zeros(self.ns + 4)
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (lr14, yl, yr)]
        self.lib().eo_ausm(self.h, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, int(direction),
                           out.ctypes.data)
        return out


def interior(a, bc=2):
    """Interior nodes of a (planes, nx, ny, nz) field."""
    return a[:, bc:-bc, bc:-bc, bc:-bc]
