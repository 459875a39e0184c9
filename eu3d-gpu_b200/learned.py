"""Learned chemistry for the EU3D timestep: training data from the stiff
integrator, training with the library's tensor-core kernels, calibration of the
trust gate, and checkpoints.

The model maps (T, log10 p, Y_0..Y_{ns-1}, log10 dt) of a cell after advection
to the change (dY_0..dY_{ns-1}, dT) that the stiff kinetics (Nchem adaptive
trapezoid substeps at fixed density and internal energy) produces over dt.

Training states come from the library's own stiff integrator (eu_chem_advance)
run along constant-volume, constant-energy trajectories. Each trajectory
starts from a mixture of stoichiometric 2H2+O2 or H2-air (Y_H2 0.0285, Y_O2
0.2264, Y_N2 0.7451) with N2, at T ~ U[300, 3500] K and p ~ logU[0.05, 5] MPa,
and each step draws dt ~ logU[1e-9, 3e-7] s. All tensors stay on the GPU
(torch provides the buffers; every computation is a libeu3d kernel).
"""
from __future__ import annotations

import ast
import json
import math
import os
import re

import numpy as np

import eu3d
import eu3d_cases as cases

HERE = os.path.dirname(os.path.abspath(__file__))
CHECKPOINT = os.path.join(HERE, "data", "chem_mlp_ja919.npz")

N_SPECIES = 9
N_IN, N_OUT = N_SPECIES + 3, N_SPECIES + 1
# The model predicts asinh(change / eps): linear below eps, logarithmic above,
# so small and large changes get comparable relative precision. With eps 1e-6
# (species) and 1e-2 K (temperature) the trust gate accepted 81 % of the
# active validation rows at a mean species L1 error of 2e-4, against 44 % for
# linear targets, 68 % for eps 1e-8 and 87 % for eps 1e-5; eps 1e-5 left a
# per-step error of ~1e-6 on the slow 800-1200 K rows, eps 1e-6 ~2e-7.
OUT_EPS = np.array([1e-6] * N_SPECIES + [1e-2])
# Cells colder than FROZEN_T with a radical pool below FROZEN_RADICAL skip the
# kinetics: along the stiff integrator's own trajectories the largest one-step
# change of any mass fraction below 800 K was 1.5e-10 (700-800 K band).
FROZEN_T, FROZEN_RADICAL, FROZEN_Y = 800.0, 1e-9, 1e-9
# Active cells predicted to need at most this many substeps take the stiff
# kinetics: a substep costs ~6 kflop in FP64 (1.4 ns a cell on a B200), the
# ensemble 0.82 MFLOP in BF16 (3.6 ns at its measured rate), so the model pays
# from about three substeps up; below that it would only add its error (in an
# induction zone the error of many cheap cells adds up: on the oblique
# detonation case it brought the ignition forward by ~2 us).
MIN_NCHEM = 4
RADICALS = (0, 1, 3, 6, 7)  # H, O, OH, H2O2, HO2 in H2_JA919's species order
WIDTH, HIDDEN, MEMBERS = 256, 3, 3
S_O2, S_H2, S_N2 = cases.S_O2, cases.S_H2, cases.S_N2


def _initial_compositions(rng, n, mw):
    """Mixtures of a reactive gas (2H2+O2 or H2-air) with N2."""
    y_h2 = 2 * mw[S_H2] / (2 * mw[S_H2] + mw[S_O2])
    bubble = np.zeros(N_SPECIES)
    bubble[S_H2], bubble[S_O2] = y_h2, 1 - y_h2
    air = np.zeros(N_SPECIES)
    air[S_H2], air[S_O2], air[S_N2] = 0.0285, 0.2264, 0.7451
    n2 = np.zeros(N_SPECIES)
    n2[S_N2] = 1.0
    f = rng.uniform(0, 1, n)
    which = rng.uniform(0, 1, n) < 0.7
    fuel = np.where(which[:, None], bubble[None, :], air[None, :])
    Y = f[:, None] * fuel + (1 - f[:, None]) * n2[None, :]
    return Y / Y.sum(axis=1, keepdims=True)


def front_states(n_max, seed=17, steps=40, dt=2e-8, device=0):
    """(T, p, Y) of the chemically active cells of igniting blocks (the stiff
    FP64 step on eu3d_cases.hot_reacting_block variants: 1100-2600 K along x,
    0.05-2 MPa along y, 0-60 % N2 along z), every step of their ignition:
    states on the reaction front itself, where the generic trajectories of
    generate() are thin. At most n_max states, drawn at random."""
    rng = np.random.default_rng(seed)
    mech = eu3d.parse_mechanism(cases.MECH_JA919, cases.THERMO)
    grid = (48, 24, 24)
    ext = (0.0, 0.012, 0.0, 0.006, 0.0, 0.006)
    out_T, out_p, out_Y = [], [], []
    for t_range, p_range in (((1100.0, 2000.0), (5e4, 1e6)), ((1300.0, 2600.0), (1e5, 2e6)),
                             ((1200.0, 2400.0), (2e5, 5e5))):
        prim = cases.hot_reacting_block(grid[0] + 4, grid[1] + 4, grid[2] + 4, mech["mw"], mech["ns"],
                                        t_range=t_range, p_range=p_range)
        s = eu3d.Solver(*grid, ext, precision="fp64", chemistry="stiff", arith="fast", device=device)
        s.set_mechanism(mech)
        s.set_primitive(*prim)
        for _ in range(steps):
            s.step(1, dt, stats=False)
            T = s.get("T")[0, 2:-2, 2:-2, 2:-2].ravel()
            P = s.get("P")[0, 2:-2, 2:-2, 2:-2].ravel()
            Y = s.get("Yi")[:, 2:-2, 2:-2, 2:-2].reshape(mech["ns"], -1)
            radical = Y[list(RADICALS)].sum(0)
            act = (Y[:N_SPECIES - 1].sum(0) >= FROZEN_Y) & ((T >= FROZEN_T) | (radical >= FROZEN_RADICAL))
            out_T.append(T[act])
            out_p.append(P[act])
            out_Y.append(Y[:, act].T)
        s.close()
    T, P, Y = np.concatenate(out_T), np.concatenate(out_p), np.concatenate(out_Y)
    if T.size > n_max:
        pick = rng.choice(T.size, n_max, replace=False)
        T, P, Y = T[pick], P[pick], Y[pick]
    return T, P, Y


def generate(solver, n_traj, n_steps, seed=11, t_range=(300.0, 3500.0), p_range=(5e4, 5e6), dt_range=(1e-9, 3e-7),
             max_substeps=20000, with_nchem=False, init=None):
    """(inputs, targets) as torch CUDA fp32 tensors, up to n_traj * n_steps rows
    (with_nchem: and each row's Nchem, the stiff kinetics' substeps for it).

    A trajectory is dropped from the first step that leaves the physical
    range: more than max_substeps substeps (the solver handle's cap), a
    non-finite or out-of-range temperature, a mass fraction below -1e-8, or a
    single-step change of any mass fraction above 0.5. At the extreme corners
    of the sampled (T, p, dt) box the linearised trapezoid scheme can overshoot
    into such states; they are far from the workloads' flows and would only
    teach the model the scheme's instability."""
    import torch
    rng = np.random.default_rng(seed)
    mech = solver.mechanism()
    ns = mech["ns"]
    dev = "cuda"
    if init is not None:  # given start states (T, p, Y rows)
        T0, p0, Y0 = (np.asarray(a, dtype=np.float64) for a in init)
        n_traj = T0.size
    else:
        T0 = rng.uniform(*t_range, n_traj)
        p0 = np.exp(rng.uniform(math.log(p_range[0]), math.log(p_range[1]), n_traj))
        Y0 = _initial_compositions(rng, n_traj, mech["mw"])
    T = torch.tensor(T0, device=dev, dtype=torch.float64)
    p = torch.tensor(p0, device=dev, dtype=torch.float64)
    Yp = torch.tensor(np.ascontiguousarray(Y0.T), device=dev, dtype=torch.float64)
    cs = torch.zeros(ns + 4, n_traj, device=dev, dtype=torch.float64)
    E = torch.zeros(n_traj, device=dev, dtype=torch.float64)
    solver.chem_states(T, p, Yp, cs, E)
    mw = torch.tensor(mech["mw"], device=dev, dtype=torch.float64)
    X = torch.empty(n_traj * n_steps, ns + 3, device=dev, dtype=torch.float32)
    Tg = torch.empty(n_traj * n_steps, ns + 1, device=dev, dtype=torch.float32)
    keep = torch.zeros(n_traj * n_steps, device=dev, dtype=torch.bool)
    Ng = torch.zeros(n_traj * n_steps, device=dev, dtype=torch.int32)
    alive = torch.ones(n_traj, device=dev, dtype=torch.bool)
    nchem = torch.zeros(n_traj, device=dev, dtype=torch.int32)
    for k in range(n_steps):
        dt = torch.exp(torch.empty(n_traj, device=dev, dtype=torch.float64).uniform_(
            math.log(dt_range[0]), math.log(dt_range[1])))
        D = cs[:ns].sum(0)
        Y = cs[:ns] / D
        P = T * D * (8.31434 * 1000 * (Y / mw[:, None]).sum(0))
        rows = slice(k * n_traj, (k + 1) * n_traj)
        X[rows, 0] = T.float()
        X[rows, 1] = torch.log10(P).float()
        X[rows, 2:2 + ns] = Y.T.float()
        X[rows, ns + 2] = torch.log10(dt).float()
        T_before, Y_before = T.clone(), Y.clone()
        solver.chem_advance(cs, T, E, dt, nchem)
        Y_after = cs[:ns] / cs[:ns].sum(0)
        alive &= (nchem > 0) & (nchem < max_substeps) & torch.isfinite(T) & (T > 250.0) & (T < 4500.0)
        alive &= (Y_after.min(0).values > -1e-8) & ((Y_after - Y_before).abs().max(0).values < 0.5)
        keep[rows] = alive
        Ng[rows] = nchem
        Tg[rows, :ns] = (Y_after - Y_before).T.float()
        Tg[rows, ns] = (T - T_before).float()
    if with_nchem:
        return X[keep].contiguous(), Tg[keep].contiguous(), Ng[keep].contiguous()
    return X[keep].contiguous(), Tg[keep].contiguous()


def _eps(eps, like):
    import torch
    return torch.tensor(OUT_EPS if eps is None else eps, device=like.device, dtype=like.dtype)


def to_model_space(T, eps=None):
    """Targets as the model learns them: asinh(change / eps) per output
    (eps <= 0: the change itself)."""
    import torch
    e = _eps(eps, T)
    return torch.where(e > 0, torch.asinh(T / e.clamp_min(1e-300)), T)


def from_model_space(Tt, eps=None):
    import torch
    e = _eps(eps, Tt)
    return torch.where(e > 0, e * torch.sinh(Tt), Tt)


def active_rows(X):
    """Rows the step's classifier hands to the model (the others skip
    chemistry): some reactive species, and hot or radical-bearing."""
    Y = X[:, 2:2 + N_SPECIES]
    reactive = Y[:, :N_SPECIES - 1].sum(1)  # all but the inert N2 (last species)
    radical = Y[:, list(RADICALS)].sum(1)
    return (reactive >= FROZEN_Y) & ((X[:, 0] >= FROZEN_T) | (radical >= FROZEN_RADICAL))


def fit(X, T, steps=4000, batch=4096, lr=1e-3, seed=5, members=MEMBERS, log=None):
    """Train an ensemble on device tensors (T in model space); returns (model, scaling dict)."""
    m = eu3d.Mlp()
    m.init(N_IN, WIDTH, HIDDEN, N_OUT, members, max_batch=max(batch, 65536), seed=seed)
    xm, xs = X.mean(0), X.std(0).clamp_min(1e-12)
    tm, ts = T.mean(0), T.std(0).clamp_min(1e-12)
    scaling = {"in_shift": xm.cpu().numpy(), "in_scale": (1 / xs).cpu().numpy(), "out_shift": tm.cpu().numpy(),
               "out_scale": (1 / ts).cpu().numpy()}
    m.set_scaling(scaling["in_shift"], scaling["in_scale"], scaling["out_shift"], scaling["out_scale"])
    done = 0
    chunk = 500
    while done < steps:
        k = min(chunk, steps - done)
        # cosine decay of the learning rate over the run (to 2 % of lr)
        frac = (done + 0.5 * k) / max(steps, 1)
        cur = lr * (0.02 + 0.98 * 0.5 * (1 + math.cos(math.pi * frac)))
        losses = m.train(X, T, batch=batch, steps=k, lr=cur, seed=seed + done)
        done += k
        if log:
            log(f"step {done}: batch loss per member {np.round(losses, 5).tolist()}")
    return m, scaling


def predict(model, X, members=MEMBERS):
    import torch
    out = torch.empty(members, X.shape[0], N_OUT, device="cuda")
    model.predict(X, out)
    return out


def calibrate(model, scaling, X, T, target=2e-4, members=MEMBERS, eps=None, bound=None):
    """The trust gate, formed as the step kernel forms it: the input box (the
    trained range), the output bound (1.25 x the largest change in the data,
    unless given), and the spread threshold tau: the largest spread whose
    accepted rows keep the mean species L1 error (physical units; T holds the
    physical changes) below target. Only rows the classifier would hand to the
    model count."""
    import torch
    act = active_rows(X)
    X, T = X[act].contiguous(), T[act]
    eps = OUT_EPS if eps is None else np.asarray(eps, dtype=np.float64)
    bound = (1.25 * T.abs().max(0).values.double().cpu().numpy()) if bound is None else np.asarray(bound)
    out = predict(model, X, members)
    mean = from_model_space(out.mean(0), eps)
    spread = (out.std(0, unbiased=False) * torch.tensor(scaling["out_scale"], device="cuda")).max(1).values
    box_lo, box_hi = X.min(0).values, X.max(0).values
    inside = ((mean.abs() <= torch.tensor(bound, device="cuda", dtype=mean.dtype)).all(1)
              & torch.isfinite(mean).all(1))
    spread = torch.where(inside, spread, torch.full_like(spread, float("inf")))
    err = (mean[:, :N_SPECIES] - T[:, :N_SPECIES]).abs().sum(1)
    err = torch.where(inside, err, torch.zeros_like(err))
    order = torch.argsort(spread)
    cum = torch.cumsum(err[order], 0) / torch.arange(1, err.numel() + 1, device="cuda")
    ok = ((cum <= target) & torch.isfinite(spread[order])).nonzero()
    idx = int(ok[-1]) if ok.numel() else 0
    tau = float(spread[order[idx]])
    acc = spread <= tau
    accepted = float(acc.float().mean())
    return {"tau": tau, "accepted_fraction": accepted, "active_rows": int(act.sum()),
            "box_lo": box_lo.double().cpu().numpy(), "box_hi": box_hi.double().cpu().numpy(),
            "out_eps": eps, "out_bound": bound,
            "l1_accepted": float(err[acc].mean()) if accepted > 0 else float("nan"),
            "l1_accepted_max": float(err[acc].max()) if accepted > 0 else float("nan")}


def save(path, model, scaling, gate, meta=None):
    np.savez(path, params=model.get_params(), shape=np.array([N_IN, WIDTH, HIDDEN, N_OUT, MEMBERS]),
             **scaling, tau=gate["tau"], box_lo=gate["box_lo"], box_hi=gate["box_hi"], out_eps=gate["out_eps"],
             out_bound=gate["out_bound"],
             frozen=np.array([FROZEN_Y, FROZEN_T, FROZEN_RADICAL]), min_nchem=np.array(gate.get("min_nchem", 0)),
             meta=np.array(json.dumps(meta or {})))


def load_meta(z):
    """The training record of a checkpoint (JSON; older ones hold a Python
    literal)."""
    text = str(z["meta"])
    try:
        return dict(json.loads(text))
    except ValueError:  # a Python repr: inf and nan are bare names there
        return dict(ast.literal_eval(re.sub(r"\bnan\b", "None", re.sub(r"\binf\b", "1e999", text))))


def load(path=CHECKPOINT, device=0):
    z = np.load(path)
    n_in, width, hidden, n_out, members = (int(v) for v in z["shape"])
    m = eu3d.Mlp(device)
    m.init(n_in, width, hidden, n_out, members, max_batch=65536, seed=1)
    m.set_scaling(z["in_shift"], z["in_scale"], z["out_shift"], z["out_scale"])
    m.set_params(z["params"])
    gate = {"tau": float(z["tau"]), "box_lo": z["box_lo"], "box_hi": z["box_hi"], "out_scale": z["out_scale"],
            "out_eps": z["out_eps"] if "out_eps" in z.files else None,
            "out_bound": z["out_bound"] if "out_bound" in z.files else None}
    fz = z["frozen"] if "frozen" in z.files else np.array([FROZEN_Y, FROZEN_T, FROZEN_RADICAL])
    gate.update(frozen_y=float(fz[0]), frozen_T=float(fz[1]), frozen_radical=float(fz[2]))
    gate["min_nchem"] = int(z["min_nchem"]) if "min_nchem" in z.files else MIN_NCHEM
    return m, gate


def attach(solver, model, gate):
    """Install a loaded model and its gate on a solver handle."""
    solver.set_learned(model, gate["tau"], gate["box_lo"], gate["box_hi"], gate["out_scale"],
                       frozen_y=gate["frozen_y"], frozen_T=gate["frozen_T"], frozen_radical=gate["frozen_radical"],
                       out_eps=gate["out_eps"], out_bound=gate["out_bound"], min_nchem=gate.get("min_nchem", 0))


def front_check(model, gate, steps=20, dt=2e-8, grid=(40, 16, 16), device=0):
    """Largest reaction-front shift (cells, eu3d_cases.front_shift) of the
    learned + mixed step against the plain FP64 stiff step over `steps` steps
    of an igniting validation block (1300-2500 K along x, 0.1-0.8 MPa along y,
    0-50 % N2 along z: not the benchmark's block), with the given gate."""
    import eu3d_cases as cases
    mech = eu3d.parse_mechanism(cases.MECH_JA919, cases.THERMO)
    ext = (0.0, grid[0] * 2.5e-4, 0.0, grid[1] * 2.5e-4, 0.0, grid[2] * 2.5e-4)
    prim = cases.hot_reacting_block(grid[0] + 4, grid[1] + 4, grid[2] + 4, mech["mw"], mech["ns"],
                                    t_range=(1300.0, 2500.0), p_range=(1e5, 8e5), n2_max=0.5)
    ys = {}
    for name, chem, prec in (("stiff", "stiff", "fp64"), ("learned", "learned", "mixed")):
        s = eu3d.Solver(*grid, ext, precision=prec, chemistry=chem, arith="fast", device=device)
        s.set_mechanism(mech)
        s.set_primitive(*prim)
        if chem == "learned":
            attach(s, model, gate)
        ys[name] = []
        for _ in range(steps):
            s.step(1, dt)
            ys[name].append(s.get("Yi"))
        s.close()
    return max(cases.front_shift(a, b) for a, b in zip(ys["learned"], ys["stiff"]))


def tighten_for_front(model, gate, max_shift=1, tries=5, log=print):
    """Halve the gate's tau until the validation block's reaction front stays
    within max_shift cells of the stiff run at every step."""
    g = dict(gate)
    g.setdefault("frozen_y", FROZEN_Y)
    g.setdefault("frozen_T", FROZEN_T)
    g.setdefault("frozen_radical", FROZEN_RADICAL)
    for _ in range(tries):
        shift = front_check(model, g)
        log(f"tau {g['tau']:.4g}: front shift {shift} cells")
        if shift <= max_shift:
            return g, shift
        g["tau"] *= 0.5
    return g, shift
