"""Helpers shared by the tests: fixtures on disk, layout conversions and the
parity measure."""
import os

import numpy as np

from conftest import GOLDEN

STATE_FIELDS = ["CS", "T", "E", "P", "D", "U", "V", "W", "H", "Gamma", "Yi"]


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def golden_mechanism():
    import oracle
    return oracle.Mechanism.from_npz(os.path.join(GOLDEN, "mech_ja919.npz"))


def init_state(z):
    return {k: z[f"init_{k}"] for k in STATE_FIELDS}


def interior(a, bc=2):
    return a[:, bc:-bc, bc:-bc, bc:-bc]


def rel_linf(a, ref):
    """Relative L-infinity error per plane: max|a - ref| / max|ref| (planes whose
    reference is identically zero use the absolute error)."""
    a = a.reshape(a.shape[0], -1)
    ref = ref.reshape(ref.shape[0], -1)
    num = np.abs(a - ref).max(axis=1)
    den = np.abs(ref).max(axis=1)
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


def cs_rel_linf(a, ref):
    """rel_linf over the conserved planes (species densities, then rho*u,
    rho*v, rho*w, E) with the three momentum planes measured against the
    largest momentum magnitude: in a flow uniform along z, rho*w is rounding
    noise (1e-14 against 1e3) whose own relative error says nothing."""
    e = rel_linf(a, ref)
    ns = a.shape[0] - 4
    mom = slice(ns, ns + 3)
    den = np.abs(ref[mom]).max()
    if den > 0:
        e[mom] = np.abs(a[mom] - ref[mom]).reshape(3, -1).max(axis=1) / den
    return e


def n_unequal(a, b):
    """Elements that differ in value (NaN equals NaN; -0 equals +0)."""
    a, b = np.asarray(a), np.asarray(b)
    return int(np.sum((a != b) & ~(np.isnan(a) & np.isnan(b))))
