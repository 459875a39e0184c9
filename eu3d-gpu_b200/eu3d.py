"""Python binding of libeu3d.so (the C ABI declared in include/eu3d.h).

Thin ctypes layer used by the tests and by bench.py. The compute path is the
CUDA library; this module never computes a timestep itself and raises if the
library is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libeu3d.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double

STATUS = {0: "EU_OK", 1: "EU_ERR_INVALID_ARGUMENT", 2: "EU_ERR_CUDA", 3: "EU_ERR_OUT_OF_MEMORY", 4: "EU_ERR_IO",
          5: "EU_ERR_NONFINITE", 6: "EU_ERR_NCHEM", 7: "EU_ERR_NOT_READY", 8: "EU_ERR_UNSUPPORTED",
          9: "EU_ERR_TIMEOUT"}
PRECISION = {"fp64": 0, "mixed": 1}
CHEMISTRY = {"stiff": 0, "frozen": 1, "learned": 2}
ARITH = {"strict": 0, "fast": 1}
BOUNDARY = {"rsbi": 0, "znd": 1, "odw": 2}


class EU3DError(RuntimeError):
    def __init__(self, status, message=""):
        self.status = status
        self.name = STATUS.get(status, str(status))
        super().__init__(f"{self.name}: {message}" if message else self.name)


class Config(ctypes.Structure):
    _fields_ = [("total_ni", _I), ("total_nj", _I), ("total_nk", _I),
                ("xa", _D), ("xb", _D), ("ya", _D), ("yb", _D), ("za", _D), ("zb", _D),
                ("bc", _I), ("device", _I), ("precision", _I), ("chemistry", _I), ("arith", _I),
                ("max_substeps", _I), ("record_sources", _I), ("profile", _I), ("eager", _I), ("boundary", _I),
                ("blocks_x", _I), ("block_x", _I)]


class MechanismC(ctypes.Structure):
    _fields_ = [("ns", _I), ("nr", _I)] + [(n, _P) for n in ("mw", "coeff_lo", "coeff_hi", "af", "bf", "eaf",
                                                            "stoi_f", "stoi_b", "tb")]


class LearnedConfig(ctypes.Structure):
    _fields_ = [("tau", _D), ("frozen_y", _D), ("frozen_T", _D), ("frozen_radical", _D), ("box_lo", _P),
                ("box_hi", _P), ("out_scale", _P), ("out_eps", _P), ("out_bound", _P), ("min_nchem", _I)]


class TuneReport(ctypes.Structure):
    _fields_ = [("flux_candidates", _I), ("flux_ci", _I * 16), ("flux_ms", ctypes.c_float * 16),
                ("recover_candidates", _I), ("recover_block", _I * 16), ("recover_minblocks", _I * 16),
                ("recover_ms", ctypes.c_float * 16), ("chosen_flux_ci", _I), ("chosen_recover_block", _I),
                ("chosen_recover_minblocks", _I)]

    def as_dict(self):
        nf, nr = self.flux_candidates, self.recover_candidates
        return {"flux_ms": {int(self.flux_ci[q]): round(float(self.flux_ms[q]), 4) for q in range(nf)},
                "recover_ms": {f"{self.recover_block[q]}x{self.recover_minblocks[q]}": round(float(self.recover_ms[q]), 4)
                               for q in range(nr)},
                "flux_ci": self.chosen_flux_ci, "recover_block": self.chosen_recover_block,
                "recover_minblocks": self.chosen_recover_minblocks}


class StepStats(ctypes.Structure):
    _fields_ = [("steps", _I), ("max_nchem", _I), ("sum_nchem", ctypes.c_longlong),
                ("reacting", ctypes.c_longlong), ("learned", ctypes.c_longlong), ("fallback", ctypes.c_longlong),
                ("nonfinite", ctypes.c_longlong), ("device_ms", _D), ("phase_ms", _D * 4), ("launches", _I),
                ("routed", ctypes.c_longlong)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["phase_ms"] = list(self.phase_ms)
        return d


_lib = None


def library():
    """Load libeu3d.so (built in-tree by `make -C eu3d-gpu_b200`)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is not built; run `make -C eu3d-gpu_b200` (or __graft_entry__.build())")
        lib = ctypes.CDLL(LIB_PATH)
        lib.eu_abi_version.restype = _I
        lib.eu_read_grid.argtypes = [ctypes.c_char_p, ctypes.POINTER(Config)]
        lib.eu_read_value.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(_D)]
        lib.eu_read_value.restype = _I
        lib.eu_parse_mechanism.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(_I), ctypes.POINTER(_I)] + [_P] * 9
        lib.eu_initial_state.argtypes = [ctypes.POINTER(MechanismC), _I, _I, _I, _I] + [_P] * 10
        lib.eu_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(_P)]
        lib.eu_destroy.argtypes = [_P]
        lib.eu_last_error.restype = ctypes.c_char_p
        lib.eu_last_error.argtypes = [_P]
        lib.eu_load_mechanism.argtypes = [_P, ctypes.c_char_p, ctypes.c_char_p]
        lib.eu_set_mechanism.argtypes = [_P, ctypes.POINTER(MechanismC)]
        lib.eu_get_mechanism.argtypes = [_P, ctypes.POINTER(_I), ctypes.POINTER(_I)] + [_P] * 9
        lib.eu_node_coordinates.argtypes = [_P, _P, _P, _P]
        lib.eu_set_primitive.argtypes = [_P] * 7
        lib.eu_set_state.argtypes = [_P] * 12
        lib.eu_step.argtypes = [_P, _I, _D, ctypes.POINTER(StepStats)]
        lib.eu_step_cfl.argtypes = [_P, _I, _D, ctypes.POINTER(StepStats), ctypes.POINTER(_D)]
        lib.eu_step_cfl.restype = _I
        lib.eu_get_field.argtypes = [_P, ctypes.c_char_p, _P]
        lib.eu_sync.argtypes = [_P]
        lib.eu_device_info.argtypes = [_P, ctypes.POINTER(_P), ctypes.POINTER(ctypes.c_size_t)]
        lib.eu_write_state.argtypes = [_P, ctypes.c_char_p, _I, _I, _D, _D]
        lib.eu_write_state.restype = _I
        lib.eu_read_state.argtypes = [_P, ctypes.c_char_p, ctypes.POINTER(_I), ctypes.POINTER(_I),
                                      ctypes.POINTER(_D), ctypes.POINTER(_D)]
        lib.eu_read_state.restype = _I
        lib.eu_set_time_scheme.argtypes = [_P, _I]
        lib.eu_set_time_scheme.restype = _I
        lib.eu_set_odw_wall.argtypes = [_P, _I]
        lib.eu_set_odw_wall.restype = _I
        lib.eu_set_ghost_mode.argtypes = [_P, _I]
        lib.eu_set_ghost_mode.restype = _I
        lib.eu_output_async.argtypes = [_P, _I, ctypes.c_char_p, _I, _I, _D, _D]
        lib.eu_output_async.restype = _I
        lib.eu_output_wait.argtypes = [_P]
        lib.eu_output_wait.restype = _I
        lib.eu_write_tecplot.argtypes = [_P, ctypes.c_char_p]
        lib.eu_write_tecplot.restype = _I
        lib.eu_chem_states.argtypes = [_P, ctypes.c_longlong, _P, _P, _P, _P, _P]
        lib.eu_chem_advance.argtypes = [_P, ctypes.c_longlong, _P, _P, _P, _P, _P]
        lib.eu_set_learned.argtypes = [_P, _P, ctypes.POINTER(LearnedConfig)]
        for fn in ("eu_chem_states", "eu_chem_advance", "eu_set_learned"):
            getattr(lib, fn).restype = _I
        lib.eu_mlp_create.argtypes = [_I, ctypes.POINTER(_P)]
        lib.eu_mlp_destroy.argtypes = [_P]
        lib.eu_mlp_last_error.restype = ctypes.c_char_p
        lib.eu_mlp_last_error.argtypes = [_P]
        lib.eu_mlp_gemm.argtypes = [_P, _P, _I, _P, _I, _I, _I, _I, _P, _I, _P, _P, _P, _I, _P]
        lib.eu_mlp_init.argtypes = [_P, _I, _I, _I, _I, _I, _I, ctypes.c_uint]
        lib.eu_mlp_set_scaling.argtypes = [_P, _P, _P, _P, _P]
        lib.eu_mlp_num_params.restype = ctypes.c_longlong
        lib.eu_mlp_num_params.argtypes = [_P]
        lib.eu_mlp_get_params.argtypes = [_P, _P]
        lib.eu_mlp_set_params.argtypes = [_P, _P]
        lib.eu_mlp_loss_grad.argtypes = [_P, _I, _P, _P, _I, _P, _P]
        lib.eu_mlp_train.argtypes = [_P, _P, _P, ctypes.c_longlong, _I, _I, ctypes.c_float, ctypes.c_uint, _P]
        lib.eu_mlp_predict.argtypes = [_P, _P, ctypes.c_longlong, _P]
        lib.eu_mlp_predict_noalloc.argtypes = [_P, _P, ctypes.c_longlong, _P]
        lib.eu_autotune.argtypes = [_P, _I, _P]
        lib.eu_autotune.restype = _I
        lib.eu_batch_create.argtypes = [ctypes.POINTER(_P), _I, ctypes.POINTER(_P)]
        lib.eu_batch_step.argtypes = [_P, _I, ctypes.POINTER(_D), _P, ctypes.POINTER(_D)]
        lib.eu_batch_destroy.argtypes = [_P]
        lib.eu_batch_last_error.argtypes = [_P]
        lib.eu_batch_last_error.restype = ctypes.c_char_p
        lib.eu_batch_set_shared_kinetics.argtypes = [_P, _I]
        lib.eu_batch_launches.argtypes = [_P, ctypes.POINTER(_I), ctypes.POINTER(_I)]
        for fn in ("eu_batch_create", "eu_batch_step", "eu_batch_destroy", "eu_batch_set_shared_kinetics",
                   "eu_batch_launches"):
            getattr(lib, fn).restype = _I
        lib.eu_set_conserved.argtypes = [_P] * 4
        lib.eu_set_conserved.restype = _I
        lib.eu_set_inflow.argtypes = [_P] * 7
        lib.eu_set_inflow.restype = _I
        lib.eu_halo_bytes.argtypes = [_P, ctypes.POINTER(ctypes.c_size_t)]
        lib.eu_halo_pack.argtypes = [_P, _I, _P]
        lib.eu_halo_unpack.argtypes = [_P, _I, _P]
        lib.eu_cfl_dt.argtypes = [_P, _D, _P]
        lib.eu_step_dt_device.argtypes = [_P, _I, _P, ctypes.POINTER(StepStats)]
        for fn in ("eu_halo_bytes", "eu_halo_pack", "eu_halo_unpack", "eu_cfl_dt", "eu_step_dt_device"):
            getattr(lib, fn).restype = _I
        lib.eu_mlp_predict_fused.argtypes = [_P, _P, ctypes.c_longlong, _P]
        lib.eu_mlp_predict_fused.restype = _I
        lib.eu_mlp_predict_fused_async.argtypes = [_P, _P, ctypes.c_longlong, _P]
        lib.eu_mlp_predict_fused_async.restype = _I
        lib.eu_mlp_sync.argtypes = [_P]
        lib.eu_mlp_sync.restype = _I
        lib.eu_mlp_stream.argtypes = [_P, ctypes.POINTER(_P)]
        lib.eu_mlp_stream.restype = _I
        lib.eu_mlp_predict_noalloc.restype = _I
        for fn in ("eu_mlp_create", "eu_mlp_destroy", "eu_mlp_gemm", "eu_mlp_init", "eu_mlp_set_scaling",
                   "eu_mlp_get_params", "eu_mlp_set_params", "eu_mlp_loss_grad", "eu_mlp_train", "eu_mlp_predict"):
            getattr(lib, fn).restype = _I
        for fn in ("eu_read_grid", "eu_parse_mechanism", "eu_initial_state", "eu_create", "eu_destroy",
                   "eu_load_mechanism", "eu_set_mechanism", "eu_get_mechanism", "eu_node_coordinates",
                   "eu_set_primitive", "eu_set_state", "eu_step", "eu_get_field", "eu_sync", "eu_device_info"):
            getattr(lib, fn).restype = _I
        _lib = lib
    return _lib


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def parse_mechanism(mech_path, thermo_path):
    """Mechanism tables as the library parses them (no device needed)."""
    lib = library()
    ns, nr = _I(), _I()
    st = lib.eu_parse_mechanism(mech_path.encode(), thermo_path.encode(), ctypes.byref(ns), ctypes.byref(nr),
                                *([None] * 9))
    if st:
        raise EU3DError(st, f"parse {mech_path} / {thermo_path}")
    ns, nr = ns.value, nr.value
    out = {"mw": np.zeros(ns), "coeff_lo": np.zeros((9, ns)), "coeff_hi": np.zeros((9, ns)), "af": np.zeros(nr),
           "bf": np.zeros(nr), "eaf": np.zeros(nr), "stoi_f": np.zeros((ns, nr)), "stoi_b": np.zeros((ns, nr)),
           "tb": np.zeros((ns, nr))}
    order = ["mw", "coeff_lo", "coeff_hi", "af", "bf", "eaf", "stoi_f", "stoi_b", "tb"]
    st = lib.eu_parse_mechanism(mech_path.encode(), thermo_path.encode(), None, None,
                                *[out[k].ctypes.data for k in order])
    if st:
        raise EU3DError(st)
    out["ns"], out["nr"] = ns, nr
    return out


def read_value(path, key, default=None):
    """A numeric value of a reference-format key/value file (input-*.txt)."""
    v = _D()
    st = library().eu_read_value(str(path).encode(), key.encode(), ctypes.byref(v))
    if st == 1 and default is not None:
        return default
    if st:
        raise EU3DError(st, f"{key} in {path}")
    return v.value


def mechanism_struct(m):
    """eu_mechanism from an object/dict with the table attributes; returns (struct, keepalive)."""
    get = (lambda k: m[k]) if isinstance(m, dict) else (lambda k: getattr(m, k))
    keep = [_c(get(k)) for k in ("mw", "coeff_lo", "coeff_hi", "af", "bf", "eaf", "stoi_f", "stoi_b", "tb")]
    return MechanismC(int(get("ns")), int(get("nr")), *[a.ctypes.data for a in keep]), keep


def initial_state(mech, ni, nj, nk, P, T, U, V, W, Y, bc=2):
    """Host-only FieldInitial-derived state (no device)."""
    lib = library()
    ms, keep = mechanism_struct(mech)
    ns = ms.ns
    shape = (ni + 2 * bc, nj + 2 * bc, nk + 2 * bc)
    n3 = int(np.prod(shape))
    prim = np.zeros((7 + ns) * n3)
    cs = np.zeros((ns + 4) * n3)
    To = np.zeros(n3)
    Eo = np.zeros(n3)
    ins = [_c(a) for a in (P, T, U, V, W, Y)]
    st = lib.eu_initial_state(ctypes.byref(ms), ni, nj, nk, bc, *[a.ctypes.data for a in ins], prim.ctypes.data,
                              cs.ctypes.data, To.ctypes.data, Eo.ctypes.data)
    if st:
        raise EU3DError(st, "eu_initial_state")
    return (prim.reshape(7 + ns, *shape), cs.reshape(ns + 4, *shape), To.reshape(1, *shape), Eo.reshape(1, *shape))


class Solver:
    """One eu_handle: a haloed node grid, a mechanism and the device state."""

    def __init__(self, total_ni, total_nj, total_nk, extent, precision="fp64", chemistry="stiff", arith="strict",
                 device=0, max_substeps=0, record_sources=False, profile=False, bc=2, graphs=True, boundary="rsbi",
                 blocks_x=1, block_x=0):
        """blocks_x > 1: this handle holds x block `block_x` of the global grid
        ((total_ni - 1) / blocks_x + 1 nodes, neighbours sharing one node)."""
        lib = library()
        self.cfg = Config(int(total_ni), int(total_nj), int(total_nk), *[float(v) for v in extent], int(bc),
                          int(device), PRECISION[precision], CHEMISTRY[chemistry], ARITH[arith], int(max_substeps),
                          int(bool(record_sources)), int(bool(profile)), int(not graphs), BOUNDARY[boundary],
                          int(blocks_x), int(block_x))
        h = _P()
        st = lib.eu_create(ctypes.byref(self.cfg), ctypes.byref(h))
        if st:
            raise EU3DError(st, "eu_create")
        self.h = h
        self.ni = (int(total_ni) - 1) // max(int(blocks_x), 1) + 1
        self.nj, self.nk, self.bc = int(total_nj), int(total_nk), int(bc)
        self.shape = (self.ni + 2 * bc, self.nj + 2 * bc, self.nk + 2 * bc)
        self.n3 = int(np.prod(self.shape))
        self.ns = None

    @classmethod
    def from_grid_file(cls, path, **kw):
        cfg = Config()
        st = library().eu_read_grid(path.encode(), ctypes.byref(cfg))
        if st:
            raise EU3DError(st, path)
        return cls(cfg.total_ni, cfg.total_nj, cfg.total_nk, (cfg.xa, cfg.xb, cfg.ya, cfg.yb, cfg.za, cfg.zb),
                   bc=cfg.bc, **kw)

    def _check(self, st, what=""):
        if st:
            msg = library().eu_last_error(self.h).decode() if self.h else ""
            raise EU3DError(st, f"{what}: {msg}" if what else msg)

    def close(self):
        if getattr(self, "h", None):
            library().eu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_mechanism(self, mech_path, thermo_path):
        self._check(library().eu_load_mechanism(self.h, mech_path.encode(), thermo_path.encode()), "load_mechanism")
        self.ns = self.mechanism()["ns"]

    def set_mechanism(self, m):
        ms, keep = mechanism_struct(m)
        self._check(library().eu_set_mechanism(self.h, ctypes.byref(ms)), "set_mechanism")
        self.ns = ms.ns

    def mechanism(self):
        lib = library()
        ns, nr = _I(), _I()
        self._check(lib.eu_get_mechanism(self.h, ctypes.byref(ns), ctypes.byref(nr), *([None] * 9)))
        ns, nr = ns.value, nr.value
        out = {"mw": np.zeros(ns), "coeff_lo": np.zeros((9, ns)), "coeff_hi": np.zeros((9, ns)),
               "af": np.zeros(nr), "bf": np.zeros(nr), "eaf": np.zeros(nr), "stoi_f": np.zeros((ns, nr)),
               "stoi_b": np.zeros((ns, nr)), "tb": np.zeros((ns, nr))}
        order = ["mw", "coeff_lo", "coeff_hi", "af", "bf", "eaf", "stoi_f", "stoi_b", "tb"]
        self._check(lib.eu_get_mechanism(self.h, None, None, *[out[k].ctypes.data for k in order]))
        out["ns"], out["nr"] = ns, nr
        return out

    def nodes(self):
        x, y, z = (np.zeros(n) for n in self.shape)
        self._check(library().eu_node_coordinates(self.h, x.ctypes.data, y.ctypes.data, z.ctypes.data))
        return x, y, z

    def set_primitive(self, P, T, U, V, W, Y):
        arrs = [_c(a) for a in (P, T, U, V, W, Y)]
        self._check(library().eu_set_primitive(self.h, *[a.ctypes.data for a in arrs]), "set_primitive")

    def set_state(self, st):
        order = ["CS", "T", "E", "P", "D", "U", "V", "W", "H", "Gamma", "Yi"]
        arrs = [_c(st[n]) for n in order]
        self._check(library().eu_set_state(self.h, *[a.ctypes.data for a in arrs]), "set_state")

    def set_conserved(self, cs, T, E):
        """Upload CS, T, E and form the primitives on the device (eu_set_conserved)."""
        arrs = [_c(a) for a in (cs, T, E)]
        self._check(library().eu_set_conserved(self.h, *[a.ctypes.data for a in arrs]), "set_conserved")

    def set_inflow(self, P, T, U, V, W, Y):
        """EU_BC_ODW x-low inflow tables over the interior (j, k) nodes: planes
        (nj, nk), Y (ns, nj, nk) (eu_set_inflow)."""
        arrs = [_c(a) for a in (P, T, U, V, W, Y)]
        self._check(library().eu_set_inflow(self.h, *[a.ctypes.data for a in arrs]), "set_inflow")

    def set_time_scheme(self, scheme):
        """Advection time scheme: "ee" (the reference's Euler explicit) or
        "rk3" (three-stage TVD Runge-Kutta; eu_set_time_scheme)."""
        self._check(library().eu_set_time_scheme(self.h, {"ee": 0, "rk3": 1}[scheme]), "set_time_scheme")

    def set_ghost_mode(self, mode):
        """Where the z-face ghost nodes are formed (eu_set_ghost_mode):
        "reference" (the ghost fill at each step's start, the reference's
        outputs) or "stored" (written with each stored interior node; the same
        interior state, the z ghosts mirroring the step's end)."""
        self._check(library().eu_set_ghost_mode(self.h, {"reference": 0, "stored": 1}[mode]), "set_ghost_mode")

    def set_odw_wall(self, first_wall_node):
        """EU_BC_ODW: the y-low wall starts at this global x node; the face
        ahead of it takes the freestream (eu_set_odw_wall)."""
        self._check(library().eu_set_odw_wall(self.h, int(first_wall_node)), "set_odw_wall")

    def step(self, nsteps, dt, stats=True):
        s = StepStats()
        st = library().eu_step(self.h, int(nsteps), float(dt), ctypes.byref(s) if stats else None)
        self._check(st, "step")
        return s.as_dict() if stats else None

    def step_cfl(self, nsteps, cfl):
        """eu_step_cfl: each step's dt from the CFL rule on the device.
        Returns (stats, time advanced)."""
        s = StepStats()
        t = _D()
        self._check(library().eu_step_cfl(self.h, int(nsteps), float(cfl), ctypes.byref(s), ctypes.byref(t)),
                    "step_cfl")
        return s.as_dict(), t.value

    def get(self, name, out=None):
        """A field as (planes, nx, ny, nz) float64. out: a caller's C-contiguous
        float64 array of that size (pinned host memory makes the copy faster)."""
        planes = {"Yi": self.ns, "Di": self.ns, "Mc": self.ns, "CMS": self.ns, "CS": self.ns + 4}.get(name, 1)
        if out is None:
            out = np.empty(planes * self.n3)
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != planes * self.n3:
            raise ValueError(f"out must be C-contiguous float64 with {planes * self.n3} elements")
        self._check(library().eu_get_field(self.h, name.encode(), out.ctypes.data), f"get {name}")
        return out.reshape(planes, *self.shape)

    def sync(self):
        self._check(library().eu_sync(self.h), "sync")

    def chem_states(self, T, p, Y, cs, E):
        """Torch CUDA float64 tensors: T, p (n), Y (ns x n) -> cs (ns+4 x n), E (n)."""
        n = T.shape[0]
        self._check(library().eu_chem_states(self.h, n, T.data_ptr(), p.data_ptr(), Y.data_ptr(), cs.data_ptr(),
                                             E.data_ptr()), "chem_states")

    def chem_advance(self, cs, T, E, dt, nchem=None):
        n = T.shape[0]
        self._check(library().eu_chem_advance(self.h, n, cs.data_ptr(), T.data_ptr(), E.data_ptr(), dt.data_ptr(),
                                              None if nchem is None else nchem.data_ptr()), "chem_advance")

    def set_learned(self, model, tau, box_lo, box_hi, out_scale, frozen_y=1e-9, frozen_T=0.0,
                    frozen_radical=1e-9, out_eps=None, out_bound=None, min_nchem=0):
        """min_nchem: active cells predicted to need at most this many substeps
        take the stiff kinetics directly (0: all active cells to the model)."""
        keep = [np.ascontiguousarray(v, dtype=np.float64) for v in (box_lo, box_hi, out_scale)]
        keep += [None if v is None else np.ascontiguousarray(v, dtype=np.float64) for v in (out_eps, out_bound)]
        self._learned_keep = keep
        cfg = LearnedConfig(float(tau), float(frozen_y), float(frozen_T), float(frozen_radical),
                            *[None if v is None else v.ctypes.data for v in keep], int(min_nchem))
        self._model = model
        self._check(library().eu_set_learned(self.h, model.h, ctypes.byref(cfg)), "set_learned")

    def autotune(self, reps=10):
        """eu_autotune: pick the flux march length and recovery block size by
        timing them on the current state (restored afterwards)."""
        rep = TuneReport()
        self._check(library().eu_autotune(self.h, int(reps), ctypes.cast(ctypes.byref(rep), _P)), "autotune")
        return rep.as_dict()

    def write_state(self, path, iteration=0, num=0, final_time=0.0, dt=0.0):
        """EU3D_STATE_V1_LE dump of the current state (the reference's format)."""
        self._check(library().eu_write_state(self.h, str(path).encode(), int(iteration), int(num),
                                             float(final_time), float(dt)), "write_state")

    def read_state(self, path):
        """Restart from an EU3D_STATE_V1_LE dump; returns (iteration, num, final_time, dt)."""
        it, num, t, dt = _I(), _I(), _D(), _D()
        self._check(library().eu_read_state(self.h, str(path).encode(), ctypes.byref(it), ctypes.byref(num),
                                            ctypes.byref(t), ctypes.byref(dt)), "read_state")
        return it.value, num.value, t.value, dt.value

    def output_async(self, path, kind="state", iteration=0, num=0, final_time=0.0, dt=0.0):
        """Queue an output file of the current state (eu_output_async): kind
        "state" (EU3D_STATE_V1_LE dump) or "tecplot"; stepping may continue
        at once, output_wait() waits for the file."""
        k = {"state": 0, "tecplot": 1}[kind]
        self._check(library().eu_output_async(self.h, k, str(path).encode(), int(iteration), int(num),
                                              float(final_time), float(dt)), "output_async")

    def output_wait(self):
        self._check(library().eu_output_wait(self.h), "output_wait")

    def write_tecplot(self, path):
        """The reference's Tecplot file of the current state (eu_write_tecplot)."""
        self._check(library().eu_write_tecplot(self.h, str(path).encode()), "write_tecplot")

    def halo_bytes(self):
        """Bytes of one halo message (eu_halo_bytes)."""
        n = ctypes.c_size_t()
        self._check(library().eu_halo_bytes(self.h, ctypes.byref(n)), "halo_bytes")
        return n.value

    def halo_pack(self, face, device_ptr):
        """Queue the face's outgoing message into device memory (eu_halo_pack)."""
        self._check(library().eu_halo_pack(self.h, int(face), _P(device_ptr)), "halo_pack")

    def halo_unpack(self, face, device_ptr):
        """Queue the neighbour's message into the face's ghost planes (eu_halo_unpack)."""
        self._check(library().eu_halo_unpack(self.h, int(face), _P(device_ptr)), "halo_unpack")

    def cfl_dt(self, cfl, device_ptr):
        """Queue this block's CFL dt into device memory (eu_cfl_dt)."""
        self._check(library().eu_cfl_dt(self.h, float(cfl), _P(device_ptr)), "cfl_dt")

    def step_dt_device(self, nsteps, device_ptr, stats=True):
        """eu_step with dt read from device memory."""
        s = StepStats()
        self._check(library().eu_step_dt_device(self.h, int(nsteps), _P(device_ptr), ctypes.byref(s) if stats else None),
                    "step_dt_device")
        return s.as_dict() if stats else None

    def device_info(self):
        stream = _P()
        nbytes = ctypes.c_size_t()
        self._check(library().eu_device_info(self.h, ctypes.byref(stream), ctypes.byref(nbytes)))
        return stream.value, nbytes.value


class Batch:
    """eu_batch: independent solvers on one device advanced by one graph launch
    per step (the instances' captured timesteps as parallel branches)."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        arr = (_P * len(self.solvers))(*[s.h for s in self.solvers])
        h = _P()
        st = library().eu_batch_create(arr, len(self.solvers), ctypes.byref(h))
        if st:
            raise EU3DError(st, "eu_batch_create")
        self.h = h

    def step(self, nsteps, dt):
        """dt: one value or one per instance. Returns (per-instance stats, device ms)."""
        n = len(self.solvers)
        dts = [float(dt)] * n if np.isscalar(dt) else [float(v) for v in dt]
        darr = (_D * n)(*dts)
        stats = (StepStats * n)()
        ms = _D()
        st = library().eu_batch_step(self.h, int(nsteps), darr, ctypes.cast(stats, _P), ctypes.byref(ms))
        if st:
            raise EU3DError(st, library().eu_batch_last_error(self.h).decode())
        return [s.as_dict() for s in stats], ms.value

    def set_shared_kinetics(self, on):
        """eu_batch_set_shared_kinetics: the fallback and deferred-cell kinetics
        of all instances as one shared stage (True, the default) or inside
        each instance's branch."""
        st = library().eu_batch_set_shared_kinetics(self.h, int(bool(on)))
        if st:
            raise EU3DError(st, "eu_batch_set_shared_kinetics")

    def launches(self):
        """(kernel launches per step, of which the shared kinetics stage's)."""
        per, shared = ctypes.c_int(), ctypes.c_int()
        st = library().eu_batch_launches(self.h, ctypes.byref(per), ctypes.byref(shared))
        if st:
            raise EU3DError(st, "eu_batch_launches")
        return per.value, shared.value

    def close(self):
        if getattr(self, "h", None):
            library().eu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mlp:
    """eu_mlp: the learned-chemistry model and its tensor-core kernels."""

    def __init__(self, device=0):
        h = _P()
        st = library().eu_mlp_create(int(device), ctypes.byref(h))
        if st:
            raise EU3DError(st, "eu_mlp_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            library().eu_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st:
            raise EU3DError(st, f"{what}: {library().eu_mlp_last_error(self.h).decode()}")

    def init(self, n_in, width, hidden, n_out, members, max_batch=8192, seed=1):
        self.shape = (n_in, width, hidden, n_out, members)
        self._check(library().eu_mlp_init(self.h, n_in, width, hidden, n_out, members, max_batch, seed), "init")

    def set_scaling(self, in_shift, in_scale, out_shift, out_scale):
        a = [np.ascontiguousarray(v, dtype=np.float32) for v in (in_shift, in_scale, out_shift, out_scale)]
        self._check(library().eu_mlp_set_scaling(self.h, *[v.ctypes.data for v in a]), "set_scaling")

    def num_params(self):
        return int(library().eu_mlp_num_params(self.h))

    def get_params(self):
        out = np.zeros(self.num_params(), np.float32)
        self._check(library().eu_mlp_get_params(self.h, out.ctypes.data), "get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.num_params()
        self._check(library().eu_mlp_set_params(self.h, p.ctypes.data), "set_params")

    def loss_grad(self, member, X, T):
        """X, T: torch CUDA fp32 tensors (n x n_in, n x n_out)."""
        loss = ctypes.c_float()
        g = np.zeros(self.num_params() // self.shape[4], np.float32)
        self._check(library().eu_mlp_loss_grad(self.h, member, X.data_ptr(), T.data_ptr(), X.shape[0],
                                               ctypes.byref(loss), g.ctypes.data), "loss_grad")
        return loss.value, g

    def train(self, X, T, batch, steps, lr, seed=1):
        losses = np.zeros(self.shape[4], np.float32)
        self._check(library().eu_mlp_train(self.h, X.data_ptr(), T.data_ptr(), X.shape[0], batch, steps, lr, seed,
                                           losses.ctypes.data), "train")
        return losses

    def predict(self, X, out):
        """out: torch CUDA fp32 tensor (members x n x n_out)."""
        self._check(library().eu_mlp_predict(self.h, X.data_ptr(), X.shape[0], out.data_ptr()), "predict")

    def predict_fused(self, X, out):
        """predict() from the one persistent tensor-core kernel the learned
        timestep uses (eu_mlp_predict_fused)."""
        self._check(library().eu_mlp_predict_fused(self.h, X.data_ptr(), X.shape[0], out.data_ptr()), "predict_fused")

    def predict_fused_async(self, X, out):
        """predict_fused() queued on the model's stream without waiting
        (eu_mlp_predict_fused_async); sync() waits and checks."""
        self._check(library().eu_mlp_predict_fused_async(self.h, X.data_ptr(), X.shape[0], out.data_ptr()),
                    "predict_fused_async")

    def sync(self):
        self._check(library().eu_mlp_sync(self.h), "sync")

    def stream(self):
        """The model's CUDA stream handle (eu_mlp_stream)."""
        s = _P()
        self._check(library().eu_mlp_stream(self.h, ctypes.byref(s)), "stream")
        return s.value

    def time_fused_queue(self, X, out, reps=5):
        """Milliseconds per launch of the fused inference on X: CUDA events on
        the model's stream around reps back-to-back launches, one check at the
        end."""
        import torch
        self.predict_fused(X, out)
        stream = torch.cuda.ExternalStream(self.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            self.predict_fused_async(X, out)
        e1.record(stream)
        self.sync()
        return e0.elapsed_time(e1) / reps

    def predict_noalloc(self, X, out):
        """predict() with its scratch in the library's fixed device array
        instead of allocated buffers (eu_mlp_predict_noalloc): for callers that
        cannot allocate device memory while they run. At most ~15k rows for the
        chemistry model's shape; overlapping calls on one device race."""
        self._check(library().eu_mlp_predict_noalloc(self.h, X.data_ptr(), X.shape[0], out.data_ptr()),
                    "predict_noalloc")

    def gemm(self, A, B, bias=None, act=0, Cf=None, Cb=None, Cpre=None, stream=None):
        """C = act(A @ B.T + bias) on torch CUDA tensors (A, B bf16, row-major)."""
        M, K = A.shape
        N = B.shape[0]
        ldc = N
        for c in (Cf, Cb, Cpre):
            if c is not None:
                ldc = c.stride(0)
        ptr = lambda t: None if t is None else t.data_ptr()
        st = library().eu_mlp_gemm(self.h, A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), M, N, K,
                                   ptr(bias), int(act), ptr(Cf), ptr(Cb), ptr(Cpre), ldc, stream)
        self._check(st, "gemm")
