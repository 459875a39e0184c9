"""Initial conditions of the EU3D workloads, as primitive fields over the haloed grid.

* ``rsbi`` — the reference's only wired case (reacting shock / H2 cylinder in
  air): Flowfield::FieldInitial (src/Flowfield.cpp:193-225) for p, T, u and
  Reaction::ReactionInitial (src/Reaction.cpp:412-471) for the composition,
  over every node including ghosts, as the reference fills them.
* ``znd`` — the 1-D ZND detonation initiation: a hot high-pressure driver at
  a reflecting wall next to quiescent 2H2+O2+7Ar, parameters from an
  input-1dZND.txt in the reference's key/value format (P_bound, T_bound, P, T,
  and driver_nodes, this build's addition). The reference's ZND case is dead
  code (its boundary is commented out and its initialiser hard-codes RSBI).
* ``odw`` — the oblique detonation wave cases: an H2-air freestream
  (input-ODW.txt: Mach 7.5, 40 kPa, 293 K; input-ODW-M7.txt: Mach 7,
  101.325 kPa, 300 K; both a 25 degree wedge) meeting the wedge. The
  reference's FieldBoundary_3dODW has a symmetry (reflecting) y-low face and
  x-low inflow tables it never fills; here the grid is wedge-aligned: the
  y-low face is the wedge surface, the tip at x = wedge_x (0 when the file has
  none; ahead of it the face takes the freestream, eu_set_odw_wall), and the
  freestream (the inflow tables and the initial field) arrives at the wedge
  angle. Optional equivalence ratio phi(z) for the 3-D case.
* ``shock_bubble`` — the 3-D reacting shock-bubble workload: a planar shock
  in N2 hitting a sphere of stoichiometric 2H2+O2 with a tanh interface and a
  seeded spherical-harmonic surface perturbation (l = 1..8, RMS amplitude 2 % of
  the radius). The reference hard-codes only RSBI, so this initialiser is new;
  the timestep it feeds is the reference's.

Fields come back as numpy arrays over (nx, ny, nz) = haloed node counts; the
species array is (ns, nx, ny, nz) in mechanism order.
"""
from __future__ import annotations

import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "data")
MECH_JA919 = os.path.join(DATA, "H2_JA919.txt")
MECH_JA1119 = os.path.join(DATA, "H2_JA1119.txt")
THERMO = os.path.join(DATA, "thermo.dat")
# the same mechanism with Ar as the ninth (inert) species and the thermo file
# whose ninth block is AR (thermo.dat is read by position)
MECH_JA919_AR = os.path.join(DATA, "H2_JA919_Ar.txt")
THERMO_AR = os.path.join(DATA, "thermo_Ar.dat")
INPUT_ZND = os.path.join(DATA, "input-1dZND.txt")
INPUT_ODW = os.path.join(DATA, "input-ODW.txt")
# the oblique-detonation configuration of the benchmark: Mach 7, 300 K,
# 101.325 kPa stoichiometric H2-air, the wedge tip 5 mm from the inflow face
INPUT_ODW_M7 = os.path.join(DATA, "input-ODW-M7.txt")
GRID_3DODW = os.path.join(DATA, "grid-3dODW.txt")

# species slots of H2_JA919 (H O H2O OH O2 H2 H2O2 HO2 N2)
S_H2O, S_O2, S_H2, S_N2 = 2, 4, 5, 8


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


def rsbi(x, y, z, mw, ns, p_pre=101325.0, t_pre=1000.0, m_wave=3.0):
    """The reference's RSBI initial primitives, formula for formula."""
    nx, ny, nz = len(x), len(y), len(z)
    # src/Flowfield.cpp:206-225 (gamma 1.4 and R 287 as the reference writes them)
    u_post = m_wave * (1 - (2 + 0.40 * m_wave ** 2) / (2.40 * m_wave ** 2)) * math.sqrt(1.40 * 287 * t_pre)
    p_post = p_pre * (1 + 2 * 1.4 / 2.4 * (m_wave ** 2 - 1.0))
    t_post = t_pre * (2 + 0.40 * m_wave ** 2) / (2.40 * m_wave ** 2) * p_post / p_pre
    ahead = (x >= 0.01)[:, None, None] * np.ones((1, ny, nz), bool)
    P = np.where(ahead, p_pre, p_post)
    T = np.where(ahead, t_pre, t_post)
    U = np.where(ahead, 0.0, u_post)
    V = np.zeros((nx, ny, nz))
    W = np.zeros((nx, ny, nz))
    # src/Reaction.cpp:419-470, evaluated with the C library's exp/sqrt
    cx, cy, ir = 0.038, 0.0, 0.022
    orad = 1.2 * ir
    alpha = 5
    Y = np.zeros((ns, nx, ny, nz))
    col = np.zeros((ns, nx, ny))
    for i in range(nx):
        for j in range(ny):
            d2 = (x[i] - cx) ** 2 + (y[j] - cy) ** 2
            if d2 > orad ** 2:
                mr = np.zeros(ns)
                mr[S_O2] = 1.0
                mr[S_N2] = 3.76
                tot = sum(mr[s] * mw[s] for s in range(ns))
                col[:, i, j] = [mr[s] * mw[s] / tot for s in range(ns)]
            elif d2 < ir ** 2:
                col[S_H2, i, j] = 1.0 * mw[S_H2] / (1.0 * mw[S_H2])
            else:
                r = math.sqrt(d2)
                yh2 = math.exp(-alpha * ((r - ir) / (orad - ir)) ** 2)
                col[S_H2, i, j] = yh2
                col[S_O2, i, j] = (1 - yh2) * mw[S_O2] / (mw[S_O2] + 3.76 * mw[S_N2])
                col[S_N2, i, j] = (1 - yh2) * 3.76 * mw[S_N2] / (mw[S_O2] + 3.76 * mw[S_N2])
    Y[:] = col[:, :, :, None]
    return P, T, U, V, W, Y


def normal_shock(mach, p1, t1, r_gas, gamma=1.4):
    """Post-shock (p, T, u) of a shock of Mach `mach` running into gas at rest."""
    g = gamma
    u2 = mach * (1 - (2 + (g - 1) * mach ** 2) / ((g + 1) * mach ** 2)) * math.sqrt(g * r_gas * t1)
    p2 = p1 * (1 + 2 * g / (g + 1) * (mach ** 2 - 1.0))
    t2 = t1 * (2 + (g - 1) * mach ** 2) / ((g + 1) * mach ** 2) * p2 / p1
    return p2, t2, u2


def _real_sph_harm(lmax, theta, phi):
    """Orthonormal real spherical harmonics Y_lm(theta, phi), l = 0..lmax, as a
    list of (l, m, values). Associated Legendre functions by the standard
    three-term recurrence (Condon-Shortley phase omitted)."""
    x = np.cos(theta)
    sx = np.sqrt(np.maximum(0.0, 1 - x * x))
    out = []
    pmm = np.ones_like(x)
    plm = {}
    for m in range(lmax + 1):
        if m > 0:
            pmm = pmm * (2 * m - 1) * sx
        plm[(m, m)] = pmm
        if m < lmax:
            plm[(m + 1, m)] = x * (2 * m + 1) * pmm
        for l in range(m + 2, lmax + 1):
            plm[(l, m)] = ((2 * l - 1) * x * plm[(l - 1, m)] - (l + m - 1) * plm[(l - 2, m)]) / (l - m)
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            am = abs(m)
            norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
            if m == 0:
                v = norm * plm[(l, 0)]
            elif m > 0:
                v = math.sqrt(2) * norm * plm[(l, am)] * np.cos(am * phi)
            else:
                v = math.sqrt(2) * norm * plm[(l, am)] * np.sin(am * phi)
            out.append((l, m, v))
    return out


def shock_bubble(x, y, z, mw, ns, mach=2.83, p0=101325.0, t0=300.0, radius=8e-3, shock_x=4e-3,
                 standoff=16e-3, center_yz=None, lmax=8, amplitude=0.02, seed=3, interface_cells=2.0, band=None):
    """Planar shock in N2 (moving +x) hitting a perturbed 2H2+O2 sphere.

    The sphere's centre sits `standoff` downstream of the shock; its surface is
    r_s(theta, phi) = radius * (1 + sum_{l=1..lmax} a_lm Y_lm) with a_lm drawn from
    numpy.random.default_rng(seed) and scaled to an RMS of `amplitude` over the
    sphere. The composition blends across the surface with
    f = (1 - tanh((r - r_s) / w)) / 2, w = interface_cells * dx / 2 (a 2-cell
    thick profile). Pre-shock gas and bubble are at (p0, t0) and rest.

    band: when set, the perturbation is evaluated only on nodes with
    |r - radius| < band * radius (elsewhere the interface profile is saturated
    to within ~1e-5); a faster, slightly different field for large batches."""
    nx, ny, nz = len(x), len(y), len(z)
    dx = x[3] - x[2]
    if center_yz is None:
        center_yz = (0.5 * (y[2] + y[-3]), 0.5 * (z[2] + z[-3]))
    cx = shock_x + standoff
    cy, cz = center_yz
    rng = np.random.default_rng(seed)
    modes = [(l, m) for l in range(1, lmax + 1) for m in range(-l, l + 1)]
    a = rng.standard_normal(len(modes))
    a *= amplitude * math.sqrt(4 * math.pi) / math.sqrt(np.sum(a * a))
    X, Yc, Z = np.meshgrid(x - cx, y - cy, z - cz, indexing="ij")
    r = np.sqrt(X * X + Yc * Yc + Z * Z)
    theta = np.arccos(np.clip(np.divide(Z, r, out=np.zeros_like(r), where=r > 0), -1, 1))
    phi = np.arctan2(Yc, X)
    pert = np.zeros_like(r)
    sel = np.abs(r - radius) < band * radius if band is not None else np.ones(r.shape, bool)
    harm = {(l, m): v for l, m, v in _real_sph_harm(lmax, theta[sel], phi[sel])}
    acc = np.zeros(int(sel.sum()))
    for coef, (l, m) in zip(a, modes):
        acc += coef * harm[(l, m)]
    pert[sel] = acc
    rs = radius * (1 + pert)
    w = 0.5 * interface_cells * dx
    f = 0.5 * (1 - np.tanh((r - rs) / w))
    y_h2 = 2 * mw[S_H2] / (2 * mw[S_H2] + mw[S_O2])
    Y = np.zeros((ns, nx, ny, nz))
    Y[S_H2] = f * y_h2
    Y[S_O2] = f * (1 - y_h2)
    Y[S_N2] = 1 - f
    r_n2 = 8.31434 * 1000 / mw[S_N2]
    p2, t2, u2 = normal_shock(mach, p0, t0, r_n2)
    behind = (x < shock_x)[:, None, None] * np.ones((1, ny, nz), bool)
    P = np.where(behind, p2, p0)
    T = np.where(behind, t2, t0)
    U = np.where(behind, u2, 0.0)
    V = np.zeros((nx, ny, nz))
    W = np.zeros((nx, ny, nz))
    # shocked gas is pure N2 (the sphere sits fully downstream of the shock)
    Y[:, behind] = 0.0
    Y[S_N2, behind] = 1.0
    return P, T, U, V, W, Y


def cfl_dt(x, y, P, D, U, V, G, cfl, bc=2):
    """Flowfield::CFLcondition (src/Flowfield.cpp:272-304): dt from dx, dy only."""
    dx = x[1] - x[0]
    dy = y[1] - y[0]
    s = (slice(bc, -bc),) * 3
    C = np.sqrt(G[s] * P[s] / D[s])
    t = np.minimum(dx / (np.abs(U[s]) + C), dy / (np.abs(V[s]) + C))
    return cfl * float(t.min())


def hot_reacting_block(nx, ny, nz, mw, ns, t_range=(1300.0, 2600.0), p_range=(1e5, 1e6), n2_max=0.6, bc=2):
    """Quiescent reacting gas over a haloed nx x ny x nz node array (ghosts
    included): T rises linearly along x over t_range, p log-linearly along y
    over p_range, and stoichiometric 2H2+O2 is diluted with 0..n2_max N2 (mass)
    along z. Velocity is zero and the fields are smooth, so a timestep is
    almost entirely kinetics: the case isolates the chemistry phase."""
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    fx = np.clip((ii - bc) / max(nx - 2 * bc - 1, 1), 0, 1)
    fy = np.clip((jj - bc) / max(ny - 2 * bc - 1, 1), 0, 1)
    fz = np.clip((kk - bc) / max(nz - 2 * bc - 1, 1), 0, 1)
    T = t_range[0] + (t_range[1] - t_range[0]) * fx
    P = p_range[0] * (p_range[1] / p_range[0]) ** fy
    n2 = n2_max * fz
    y_h2 = 2 * mw[S_H2] / (2 * mw[S_H2] + mw[S_O2])
    Y = np.zeros((ns, nx, ny, nz))
    Y[S_H2] = (1 - n2) * y_h2
    Y[S_O2] = (1 - n2) * (1 - y_h2)
    Y[S_N2] = n2
    Z = np.zeros((nx, ny, nz))
    return P, T, Z, Z.copy(), Z.copy(), Y


def front_shift(y, y_ref, product=S_H2O, min_product=1e-2, bc=2):
    """Reaction-front position error in cells between two runs' species fields
    (ns, nx, ny, nz): per (j, k) column the front is the first node along x
    whose product mass fraction reaches half the reference run's column
    maximum; returns the largest |difference| over the columns whose reference
    maximum reaches min_product (before that there is no front, only trace
    product whose half-maximum point is noise; a front missing in one run
    counts as the column length)."""
    a = y[product, bc:-bc, bc:-bc, bc:-bc]
    b = y_ref[product, bc:-bc, bc:-bc, bc:-bc]
    thr = 0.5 * b.max(axis=0)
    ok = 2 * thr >= min_product
    fa, fb = a >= thr, b >= thr
    ia = np.where(fa.any(axis=0), fa.argmax(axis=0), a.shape[0])
    ib = np.where(fb.any(axis=0), fb.argmax(axis=0), b.shape[0])
    return int(np.abs(ia - ib)[ok].max()) if ok.any() else 0


def znd(x, y, z, mw, ns, input_path=INPUT_ZND, mole=None, bc=2, interface_cells=2.0):
    """ZND initiation: driver (P_bound, T_bound) on the first driver_nodes
    interior nodes along x and the ghosts left of them, quiescent gas (P, T)
    elsewhere, at rest, one composition everywhere (default stoichiometric
    2H2 + O2 + 7 Ar on the Ar variant of the mechanism, Ar in slot 8).

    The driver edge is a tanh profile interface_cells wide (f = (1 - tanh((i -
    i_edge) / w)) / 2, ln p and T blended by f); 0 gives the sharp jump. The
    sharp 150:1 jump does not run with the reference's scheme: in the first
    step both sides are at rest, so the AUSM+ flux at the edge carries no mass
    and no energy, only the pressure force, which accelerates the first
    quiescent node while its total energy stays put; its internal energy, and
    with it T, falls below the NASA range (60 K after 2 ns, non-finite after
    12 ns)."""
    import eu3d
    p_drv = eu3d.read_value(input_path, "P_bound")
    t_drv = eu3d.read_value(input_path, "T_bound")
    p0 = eu3d.read_value(input_path, "P")
    t0 = eu3d.read_value(input_path, "T")
    n_drv = int(eu3d.read_value(input_path, "driver_nodes", 40))
    nx, ny, nz = len(x), len(y), len(z)
    if mole is None:
        mole = {S_H2: 2.0, S_O2: 1.0, S_N2: 7.0}
    tot = sum(v * mw[s] for s, v in mole.items())
    Y = np.zeros((ns, nx, ny, nz))
    for s, v in mole.items():
        Y[s] = v * mw[s] / tot
    i = np.arange(nx, dtype=np.float64)[:, None, None] * np.ones((1, ny, nz))
    if interface_cells > 0:
        f = 0.5 * (1 - np.tanh((i - (bc + n_drv - 0.5)) / interface_cells))
    else:
        f = (i < bc + n_drv).astype(np.float64)
    P = np.exp(np.log(p0) + f * (np.log(p_drv) - np.log(p0)))
    T = t0 + f * (t_drv - t0)
    Z = np.zeros((nx, ny, nz))
    return P, T, Z, Z.copy(), Z.copy(), Y


def h2_air(mw, ns, phi=1.0):
    """Mass fractions of H2-air at equivalence ratio phi (2 phi H2 + O2 + 3.76 N2
    by moles; phi = 1 gives Y_H2 0.0285, Y_O2 0.2264, Y_N2 0.7451)."""
    phi = np.asarray(phi, dtype=np.float64)
    m = {S_H2: 2.0 * phi, S_O2: np.ones_like(phi), S_N2: 3.76 * np.ones_like(phi)}
    tot = sum(v * mw[s] for s, v in m.items())
    Y = np.zeros((ns,) + phi.shape)
    for s, v in m.items():
        Y[s] = v * mw[s] / tot
    return Y


def mixture_gamma(mech, T, Y):
    """cp / cv of a mixture from the NASA polynomials (the reference's GetCpi
    form, src/Reaction.cpp:1165-1177) at temperature T; Y (ns, ...)."""
    lo = T < 1000.0
    c = np.where(lo, 1.0, 0.0)
    a = np.asarray(mech["coeff_lo"]) * c + np.asarray(mech["coeff_hi"]) * (1 - c)  # (9, ns)
    r_s = 8.31434 / np.asarray(mech["mw"])
    cp_s = r_s * (a[0] * T ** -2 + a[1] / T + a[2] + a[3] * T + a[4] * T ** 2 + a[5] * T ** 3 + a[6] * T ** 4)
    Ys = np.moveaxis(np.asarray(Y), 0, -1)
    cp = Ys @ cp_s
    r = Ys @ r_s
    return cp / (cp - r), r * 1000


def odw_inflow(mech, nj, nk, z=None, input_path=INPUT_ODW, phi=None):
    """The freestream on the interior (j, k) nodes: P, T, U, V, W planes (nj, nk)
    and Y (ns, nj, nk). The speed is Mach x the frozen sound speed of the
    mixture; the velocity points into the wedge surface at the wedge angle
    (U = V cos a, V = -V sin a). phi: equivalence ratio per k (length nk), or
    None for 1."""
    import eu3d
    p0 = eu3d.read_value(input_path, "P")
    t0 = eu3d.read_value(input_path, "T")
    mach = eu3d.read_value(input_path, "Mach")
    angle = math.radians(eu3d.read_value(input_path, "angle"))
    ns = int(mech["ns"])
    ph = np.ones(nk) if phi is None else np.asarray(phi, dtype=np.float64)
    Yk = h2_air(mech["mw"], ns, ph)  # (ns, nk)
    g, r = mixture_gamma(mech, t0, Yk)
    speed = mach * np.sqrt(g * r * t0)  # (nk,)
    P = np.full((nj, nk), p0)
    T = np.full((nj, nk), t0)
    U = np.broadcast_to(speed * math.cos(angle), (nj, nk)).copy()
    V = np.broadcast_to(-speed * math.sin(angle), (nj, nk)).copy()
    W = np.zeros((nj, nk))
    Y = np.broadcast_to(Yk[:, None, :], (ns, nj, nk)).copy()
    return P, T, U, V, W, Y


def odw_phi(z, seed=4, modes=4, amplitude=0.1, bc=2):
    """Equivalence ratio along z: 1 + sum_{m=1..modes} a_m sin(2 pi m z / L + theta_m),
    the sum scaled so its largest magnitude over the interior nodes is
    `amplitude` (a_m ~ N(0, 1), theta_m ~ U[0, 2 pi) from default_rng(seed))."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(modes)
    th = rng.uniform(0.0, 2 * math.pi, modes)
    zi = np.asarray(z)[bc:-bc]
    L = zi[-1] - zi[0] if len(zi) > 1 else 1.0
    s = sum(a[m] * np.sin(2 * math.pi * (m + 1) * (zi - zi[0]) / L + th[m]) for m in range(modes))
    peak = np.abs(s).max()
    return 1.0 + (amplitude * s / peak if peak > 0 else 0 * s)


def odw_wall_node(x, input_path=INPUT_ODW, bc=2):
    """First x node of the wedge surface: the input file's wedge_x (distance
    from the inflow face along the wedge, 0 when absent) on the haloed
    coordinates x."""
    import eu3d
    wx = eu3d.read_value(input_path, "wedge_x", 0.0)
    xi = np.asarray(x)[bc:-bc]
    return int(np.searchsorted(xi, xi[0] + wx - 1e-12))


def odw(x, y, z, mech, input_path=INPUT_ODW, phi=None, bc=2):
    """The ODW case: the freestream of odw_inflow on every node (ghosts
    included; the z ghosts repeat the nearest interior node's composition).
    Returns (P, T, U, V, W, Y) over the haloed grid and the inflow tables."""
    nx, ny, nz = len(x), len(y), len(z)
    nj, nk = ny - 2 * bc, nz - 2 * bc
    inflow = odw_inflow(mech, nj, nk, input_path=input_path, phi=phi)
    kk = np.clip(np.arange(nz) - bc, 0, nk - 1)
    fields = []
    for a in inflow[:5]:
        fields.append(np.broadcast_to(a[0][kk][None, None, :], (nx, ny, nz)).copy())
    Y = np.broadcast_to(inflow[5][:, 0, kk][:, None, None, :], (int(mech["ns"]), nx, ny, nz)).copy()
    return (*fields, Y), inflow
