"""The learned-chemistry step on the GPU.

* Plumbing: with the gate rejecting every cell and no cell frozen, the learned
  path (classify -> queue -> ensemble -> gate -> stiff fallback queue) must give
  exactly the stiff path's result.
* Gate: cells outside the input box fall back; the counts add up.
* Conservation: an accepted prediction changes neither the density nor the
  momentum and energy of a cell; the species change is projected onto element
  conservation, so sum Y = 1 holds.
"""
import numpy as np
import pytest

import eu3d_cases as cases
from helpers import golden, golden_mechanism, interior, n_unequal

pytestmark = pytest.mark.gpu

NS = 9


def bubble(gpu, chemistry, precision="fp64"):
    z = golden("bubble_25x13x13_s20.npz")
    s = gpu.Solver(int(z["ni"]), int(z["nj"]), int(z["nk"]), tuple(z["extent"]), chemistry=chemistry,
                   precision=precision, arith="fast")
    s.load_mechanism(cases.MECH_JA919, cases.THERMO)
    s.set_primitive(*[z[f"prim_{k}"] for k in "PTUVWY"])
    return s, z


def random_model(gpu, seed=1):
    m = gpu.Mlp()
    m.init(NS + 3, 256, 3, NS + 1, 3, max_batch=4096, seed=seed)
    m.set_scaling(np.zeros(NS + 3), np.ones(NS + 3), np.zeros(NS + 1), np.ones(NS + 1) * 1e3)
    return m


def test_reject_all_equals_stiff(gpu):
    a, z = bubble(gpu, "stiff")
    b, _ = bubble(gpu, "learned")
    m = random_model(gpu)
    big = np.full(NS + 3, 1e30)
    b.set_learned(m, tau=-1.0, box_lo=-big, box_hi=big, out_scale=np.ones(NS + 1), frozen_y=-1.0)
    sa = a.step(10, float(z["dt"]))
    sb = b.step(10, float(z["dt"]))
    assert sb["learned"] == 0 and sb["fallback"] == sb["reacting"] == z["ni"] * z["nj"] * z["nk"]
    for f in ["CS", "T", "E", "Nchem"]:
        assert n_unequal(interior(a.get(f)), interior(b.get(f))) == 0, f
    assert sa["max_nchem"] == sb["max_nchem"]


def test_frozen_cells_skip_chemistry(gpu):
    b, z = bubble(gpu, "learned")
    m = random_model(gpu)
    big = np.full(NS + 3, 1e30)
    b.set_learned(m, tau=-1.0, box_lo=-big, box_hi=big, out_scale=np.ones(NS + 1), frozen_y=1e-9)
    st = b.step(1, float(z["dt"]))
    Y = interior(b.get("Yi"))
    reactive = (Y[:8].sum(0) >= 1e-9).sum()
    assert 0 < st["reacting"] < z["ni"] * z["nj"] * z["nk"]
    assert abs(st["reacting"] - reactive) <= 0.05 * reactive + 10


def test_accepted_prediction_conserves(gpu):
    b, z = bubble(gpu, "learned")
    m = random_model(gpu, seed=3)
    big = np.full(NS + 3, 1e30)
    b.set_learned(m, tau=1e30, box_lo=-big, box_hi=big, out_scale=np.ones(NS + 1), frozen_y=1e-9)
    st = b.step(1, float(z["dt"]))
    assert st["learned"] == st["reacting"] > 0 and st["fallback"] == 0
    Y = interior(b.get("Yi"))
    assert np.abs(Y.sum(0) - 1).max() < 1e-12
    assert (Y >= 0).all()


def test_gate_box_sends_cells_to_fallback(gpu):
    b, z = bubble(gpu, "learned")
    m = random_model(gpu)
    lo = np.full(NS + 3, -1e30)
    hi = np.full(NS + 3, 1e30)
    hi[0] = 0.0  # every temperature is above the box
    b.set_learned(m, tau=1e30, box_lo=lo, box_hi=hi, out_scale=np.ones(NS + 1), frozen_y=1e-9)
    st = b.step(1, float(z["dt"]))
    assert st["learned"] == 0 and st["fallback"] == st["reacting"] > 0


def hot_mixture(gpu, chemistry, precision="fp64"):
    """A quiescent 24 x 8 x 8 block of reacting gas: T from 1300 to 2600 K along x,
    p from 0.1 to 1 MPa along y, 2H2+O2 diluted with 0-60 % N2 along z. No flux
    acts (velocity 0, smooth fields), so a step is the kinetics."""
    ni, nj, nk = 24, 8, 8
    ext = (0.0, 0.024, 0.0, 0.008, 0.0, 0.008)
    mech = gpu.parse_mechanism(cases.MECH_JA919, cases.THERMO)
    prim = cases.hot_reacting_block(ni + 4, nj + 4, nk + 4, mech["mw"], mech["ns"])
    s = gpu.Solver(ni, nj, nk, ext, chemistry=chemistry, precision=precision, arith="fast")
    s.set_mechanism(mech)
    s.set_primitive(*prim)
    return s


def test_trained_model_replaces_stiff_substeps(gpu):
    """What the trained network gains over the stiff kinetics alone, at the
    committed gate: every cell the model advances is a trapezoid substep the
    stiff kinetics does not run, and the rejected cells take the stiff
    kinetics' own substeps (the same FP64 arithmetic). The gate is tight (tau
    calibrated for a mean species L1 of 5e-6 per step, then halved until the
    reaction front of an igniting validation block does not move), so on this
    block of hot reacting gas it takes about 2 % of the cells. Here every
    active cell goes to the model (min_nchem 0): on this block each cell needs
    one substep, so the default Nchem routing (learned.MIN_NCHEM) would give
    them all to the stiff kinetics and the model none. The species error (mean
    over cells of sum_s |dY_s| against the stiff step) stays within 1e-4."""
    import learned
    dt = 5e-8
    a = hot_mixture(gpu, "stiff")
    b = hot_mixture(gpu, "learned")
    model, gate = learned.load()
    learned.attach(b, model, dict(gate, min_nchem=0))
    sa = a.step(1, dt)
    sb = b.step(1, dt)
    n = 24 * 8 * 8
    assert sa["reacting"] == n and sb["reacting"] == n
    assert sb["learned"] + sb["fallback"] == n and sb["routed"] == 0, sb
    assert sb["learned"] >= 0.005 * n, sb
    assert sb["sum_nchem"] <= sa["sum_nchem"] - sb["learned"], (sa["sum_nchem"], sb["sum_nchem"], sb["learned"])
    ya, yb = interior(a.get("Yi")), interior(b.get("Yi"))
    l1 = np.abs(ya - yb).sum(axis=0)
    assert l1.mean() <= 1e-4, l1.mean()
    assert np.allclose(yb.sum(axis=0), 1.0, atol=1e-12)
    print(f"stiff substeps {sa['sum_nchem']}, learned path {sb['sum_nchem']}; learned cells {sb['learned']} of {n}; "
          f"species L1 mean {l1.mean():.2e} max {l1.max():.2e}")


@pytest.mark.parametrize("chemistry,precision", [("stiff", "fp64"), ("stiff", "mixed"), ("learned", "mixed"),
                                                 ("learned", "fp64")])
def test_graph_replay_equals_eager_launches(gpu, chemistry, precision):
    """A timestep replayed from its captured CUDA graph is the same launches as
    the eager path: bitwise the same state, the same statistics. Covers the
    learned phase (device-side queue lengths, the fused model kernel) and a
    change of the gate's tau between calls, which recaptures the graph."""
    import learned
    out = {}
    for graphs in (False, True):
        ni, nj, nk = 24, 8, 8
        ext = (0.0, 0.024, 0.0, 0.008, 0.0, 0.008)
        mech = gpu.parse_mechanism(cases.MECH_JA919, cases.THERMO)
        prim = cases.hot_reacting_block(ni + 4, nj + 4, nk + 4, mech["mw"], mech["ns"])
        s = gpu.Solver(ni, nj, nk, ext, chemistry=chemistry, precision=precision, arith="fast", graphs=graphs)
        s.set_mechanism(mech)
        s.set_primitive(*prim)
        stats = []
        if chemistry == "learned":  # every active cell to the model, so it runs inside the graph
            model, gate = learned.load()
            learned.attach(s, model, dict(gate, min_nchem=0))
        stats.append(s.step(3, 2e-8))
        if chemistry == "learned":
            learned.attach(s, model, dict(gate, tau=gate["tau"] * 3, min_nchem=0))
        stats.append(s.step(2, 2e-8))
        keep = ("max_nchem", "sum_nchem", "reacting", "learned", "fallback", "launches")
        out[graphs] = ([{k: st[k] for k in keep} for st in stats], s.get("CS"), s.get("T"), s.get("Yi"))
        s.close()
    assert out[False][0] == out[True][0]
    for a, b in zip(out[False][1:], out[True][1:]):
        assert n_unequal(a, b) == 0


@pytest.mark.parametrize("shared", [True, False])
def test_batch_of_uneven_instances_equals_one_by_one(gpu, shared):
    """A batch of instances of different sizes and modes (stiff FP64, stiff
    mixed, learned + mixed with and without the Nchem routing, frozen)
    advanced by one graph launch per step gives each instance bitwise the
    state and statistics it reaches stepping alone, with the fallback and
    deferred-cell kinetics of all instances as one shared stage (one launch
    per kinetics stage for the instances of one flavour) or inside each
    instance's branch; the handles stay usable on their own between batch
    calls."""
    import learned
    model, gate = learned.load()
    mech = gpu.parse_mechanism(cases.MECH_JA919, cases.THERMO)
    specs = [((24, 8, 8), "stiff", "fp64", 2e-8, 0), ((16, 12, 8), "learned", "mixed", 3e-8, 0),
             ((20, 6, 10), "frozen", "mixed", 2e-8, 0), ((8, 8, 8), "learned", "fp64", 1e-8, 0),
             ((20, 10, 8), "stiff", "mixed", 3e-8, 0), ((12, 12, 12), "learned", "mixed", 3e-8, None)]

    def make():
        out = []
        for (ni, nj, nk), chem, prec, _, min_nchem in specs:
            s = gpu.Solver(ni, nj, nk, (0.0, ni * 1e-3, 0.0, nj * 1e-3, 0.0, nk * 1e-3), chemistry=chem,
                           precision=prec, arith="fast")
            s.set_mechanism(mech)
            s.set_primitive(*cases.hot_reacting_block(ni + 4, nj + 4, nk + 4, mech["mw"], mech["ns"]))
            if chem == "learned":  # min_nchem 0: every active cell to the model; None: routed
                learned.attach(s, model, gate if min_nchem is None else dict(gate, min_nchem=min_nchem))
            out.append(s)
        return out

    alone = make()
    ref_stats = [s.step(3, spec[3]) for s, spec in zip(alone, specs)]
    for s, spec in zip(alone, specs):
        s.step(1, spec[3])
    together = make()
    b = gpu.Batch(together)
    b.set_shared_kinetics(shared)
    stats, ms = b.step(3, [spec[3] for spec in specs])
    assert ms > 0
    per_step, stage = b.launches()
    # shared: the two learned mixed instances drain their fallback queues in
    # one launch and, with the stiff mixed one, their deferred cells in
    # another; the learned FP64 instance (another flavour, no deferral) has
    # its own fallback launch
    assert stage == (3 if shared else 0), stage
    assert per_step > stage
    for s, spec in zip(together, specs):  # on their own between batch calls
        s.step(1, spec[3])
    keep = ("max_nchem", "sum_nchem", "learned", "fallback")
    assert sum(st["fallback"] for st in ref_stats) > 0
    for got, want in zip(stats, ref_stats):
        assert {k: got[k] for k in keep} == {k: want[k] for k in keep}
    for a, c in zip(alone, together):
        for f in ("CS", "T", "Yi"):
            assert n_unequal(a.get(f), c.get(f)) == 0, f
    b.close()


@pytest.mark.parametrize("min_nchem", [0, None])
def test_learned_front_within_one_cell(gpu, min_nchem):
    """Over 10 steps of igniting gas (24 x 8 x 8 block, 1300-2600 K along x,
    dt 2e-8 s) the learned + mixed step keeps the reaction front (the first
    node along x where H2O reaches half the stiff run's column maximum, in the
    columns where it reaches 1e-2) within one cell of the plain FP64 stiff run
    in every column, at a species L1 (mean over cells of sum_s |dY_s|) within
    1e-3. With min_nchem 0 every active cell goes to the network first, so the
    cells it advances (at least 1 % of the cell-steps here) are in the
    comparison: the test fails if the network's accepted predictions move the
    front or the species. With the committed routing (None) the cells needing
    few substeps take the stiff kinetics."""
    import learned
    model, gate = learned.load()
    if min_nchem is not None:
        gate = dict(gate, min_nchem=min_nchem)
    ys, took = {}, 0
    n = 24 * 8 * 8
    for chem, prec in (("stiff", "fp64"), ("learned", "mixed")):
        s = hot_mixture(gpu, chem, prec)
        if chem == "learned":
            learned.attach(s, model, gate)
        ys[chem] = []
        for _ in range(10):
            st = s.step(1, 2e-8)
            took += st["learned"] if chem == "learned" else 0
            ys[chem].append(s.get("Yi"))
        s.close()
    if min_nchem == 0:
        assert took >= 0.01 * 10 * n, took
    assert max(cases.front_shift(a, b) for a, b in zip(ys["learned"], ys["stiff"])) <= 1
    l1 = np.abs(interior(ys["learned"][-1]) - interior(ys["stiff"][-1])).sum(axis=0)
    assert l1.mean() <= 1e-3, l1.mean()


def test_nchem_routing_sends_cheap_cells_to_the_stiff_kinetics(gpu):
    """With min_nchem above every cell's predicted Nchem the learned step is
    the stiff step: no cell reaches the model, and the state is bitwise that of
    the mixed-precision stiff step (the same prediction, substeps and state
    rebuild). With min_nchem 0 every active cell goes to the model."""
    import learned
    dt = 2e-8
    model, gate = learned.load()
    a = hot_mixture(gpu, "stiff")
    b = hot_mixture(gpu, "learned")
    c = hot_mixture(gpu, "learned")
    learned.attach(b, model, dict(gate, min_nchem=1 << 20))
    learned.attach(c, model, dict(gate, min_nchem=0))
    sa, sb, sc = a.step(2, dt), b.step(2, dt), c.step(2, dt)
    n = 24 * 8 * 8
    assert sb["routed"] == n and sb["learned"] == 0 and sb["fallback"] == 0, sb
    assert sb["sum_nchem"] == sa["sum_nchem"] and sb["max_nchem"] == sa["max_nchem"]
    for f in ("CS", "T", "Yi"):
        assert n_unequal(a.get(f), b.get(f)) == 0, f
    assert sc["routed"] == 0 and sc["learned"] + sc["fallback"] == n, sc
    for s in (a, b, c):
        s.close()
