"""The learned-chemistry model's training kernels on the GPU against the CPU
checker oracle/mlp_oracle.py (numpy, float64 accumulation, bf16 rounding at
the device's rounding points).

Tolerances: loss within 1e-4 relative; every gradient tensor within 2e-3 of
its largest entry (fp32 accumulation order and the rare bf16 rounding flip of
an activation); predictions within 2e-3 of the output scale.
"""
import numpy as np
import pytest

import mlp_oracle as mo

pytestmark = pytest.mark.gpu

N_IN, WIDTH, HIDDEN, N_OUT, MEMBERS = 12, 256, 3, 10, 3


def make(gpu, seed=3):
    m = gpu.Mlp()
    m.init(N_IN, WIDTH, HIDDEN, N_OUT, MEMBERS, max_batch=1024, seed=seed)
    rng = np.random.default_rng(seed)
    scal = (rng.normal(size=N_IN), rng.uniform(0.5, 2, N_IN), rng.normal(size=N_OUT), rng.uniform(0.5, 2, N_OUT))
    m.set_scaling(*scal)
    return m, [np.asarray(v, np.float32) for v in scal]


def split_sizes():
    return mo.layer_sizes(N_IN, WIDTH, HIDDEN, N_OUT)


def test_params_round_trip(gpu):
    m, _ = make(gpu)
    p = m.get_params()
    per = sum(i * o + o for i, o in split_sizes())
    assert p.size == per * MEMBERS
    q = np.random.default_rng(0).normal(scale=0.05, size=p.size).astype(np.float32)
    m.set_params(q)
    assert np.array_equal(m.get_params(), q)


def test_gradients_match_cpu_oracle(gpu):
    import torch
    m, (ish, isc, osh, osc) = make(gpu)
    rng = np.random.default_rng(5)
    n = 256
    X = rng.normal(size=(n, N_IN)).astype(np.float32) * 1.3 + 0.2
    T = rng.normal(size=(n, N_OUT)).astype(np.float32)
    params = m.get_params()
    per = params.size // MEMBERS
    for member in range(MEMBERS):
        loss, g = m.loss_grad(member, torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda())
        ref_loss, ref_g = mo.loss_and_grads(params[member * per:(member + 1) * per], X, T, N_IN, WIDTH, HIDDEN, N_OUT,
                                            ish, isc, osh, osc)
        assert abs(loss - ref_loss) <= 1e-4 * ref_loss, (loss, ref_loss)
        off = 0
        for n_in, n_out in split_sizes():
            for size in (n_in * n_out, n_out):
                a, b = g[off:off + size], ref_g[off:off + size]
                assert np.abs(a - b).max() <= 2e-3 * np.abs(b).max() + 1e-12, (off, np.abs(a - b).max(), np.abs(b).max())
                off += size


def test_predict_matches_cpu_oracle(gpu):
    import torch
    m, (ish, isc, osh, osc) = make(gpu, seed=9)
    rng = np.random.default_rng(2)
    n = 1000  # not a multiple of the tile: exercises row bounds
    X = rng.normal(size=(n, N_IN)).astype(np.float32)
    out = torch.zeros(MEMBERS, n, N_OUT, device="cuda")
    m.predict(torch.from_numpy(X).cuda(), out)
    params = m.get_params()
    per = params.size // MEMBERS
    for e in range(MEMBERS):
        ref = mo.predict(params[e * per:(e + 1) * per], X, N_IN, WIDTH, HIDDEN, N_OUT, ish, isc, osh, osc)
        got = out[e].cpu().numpy()
        assert np.abs(got - ref).max() <= 2e-3 * (1 / osc).max() * max(1.0, np.abs(ref * osc).max()), e


def test_training_fits_a_smooth_map(gpu):
    """Adam on the device reduces the loss of a smooth 12 -> 10 map by >20x."""
    import torch
    m = gpu.Mlp()
    m.init(N_IN, WIDTH, HIDDEN, N_OUT, MEMBERS, max_batch=1024, seed=4)
    m.set_scaling(np.zeros(N_IN), np.ones(N_IN), np.zeros(N_OUT), np.ones(N_OUT))
    rng = np.random.default_rng(1)
    n = 65536
    X = rng.uniform(-1, 1, size=(n, N_IN)).astype(np.float32)
    A = rng.normal(size=(N_IN, N_OUT)).astype(np.float32) / 3
    T = np.sin(X @ A).astype(np.float32) + 0.1 * (X[:, :N_OUT] ** 2)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    l0 = np.array([m.loss_grad(e, Xd[:1024], Td[:1024])[0] for e in range(MEMBERS)])
    m.train(Xd, Td, batch=512, steps=400, lr=1e-3, seed=7)
    l1 = np.array([m.loss_grad(e, Xd[:1024], Td[:1024])[0] for e in range(MEMBERS)])
    assert (l1 < l0 / 20).all(), (l0, l1)


@pytest.mark.parametrize("shape", [(N_IN, WIDTH, HIDDEN, N_OUT, MEMBERS), (5, 64, 2, 3, 2), (20, 96, 1, 40, 1)])
def test_fused_inference_matches_layerwise(gpu, shape):
    """The one-kernel inference (every member's network per 128-row tile, the
    activations in shared memory, the accumulators in tensor memory, weights
    streamed by bulk copies) gives the layer-wise GEMM path's outputs bit for
    bit: the same K=16 MMA sequence, epilogues and scalings. Row counts cover
    partial, exact and many tiles (more tiles than SMs); an empty queue is the
    learned timestep's common case and is covered there."""
    import torch
    n_in, width, hidden, n_out, members = shape
    m = gpu.Mlp()
    m.init(n_in, width, hidden, n_out, members, max_batch=1024, seed=7)
    rng = np.random.default_rng(11)
    m.set_scaling(rng.normal(size=n_in), rng.uniform(0.5, 2, n_in), rng.normal(size=n_out), rng.uniform(0.5, 2, n_out))
    m.set_params(rng.normal(scale=0.08, size=m.num_params()).astype(np.float32))
    for n in (1, 127, 128, 129, 3000, 40000):
        X = torch.from_numpy(rng.normal(size=(n, n_in)).astype(np.float32)).cuda()
        a = torch.full((members, n, n_out), float("nan"), device="cuda")
        b = torch.full((members, n, n_out), float("nan"), device="cuda")
        m.predict(X, a)
        m.predict_fused(X, b)
        torch.cuda.synchronize()
        assert torch.equal(a, b), (shape, n, (a - b).abs().max().item())


def test_models_and_handles_on_two_devices(gpu):
    """Kernels whose shared memory exceeds the 48 KB default have their limit
    raised on every device they run on, not once per process: a model and a
    step on the second GPU after the first both run and agree with the first
    GPU's results (skipped with one visible GPU)."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    import eu3d_cases as cases
    rng = np.random.default_rng(11)
    X = rng.normal(size=(300, N_IN)).astype(np.float32)
    mech = gpu.parse_mechanism(cases.MECH_JA919, cases.THERMO)
    prim = cases.hot_reacting_block(20, 12, 12, mech["mw"], mech["ns"])
    out = []
    for dev in (0, 1):
        m = gpu.Mlp(device=dev)
        m.init(N_IN, WIDTH, HIDDEN, N_OUT, MEMBERS, max_batch=1024, seed=3)
        with torch.cuda.device(dev):
            xd = torch.from_numpy(X).cuda()
            od = torch.zeros(MEMBERS, X.shape[0], N_OUT, device="cuda")
            m.predict(xd, od)
            pred = od.cpu().numpy()
        s = gpu.Solver(16, 8, 8, (0.0, 0.016, 0.0, 0.008, 0.0, 0.008), precision="mixed", arith="fast", device=dev)
        s.set_mechanism(mech)
        s.set_primitive(*prim)
        s.step(2, 2e-8)
        out.append((pred, s.get("CS")))
        s.close()
        m.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
