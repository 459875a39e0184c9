"""eu_mlp_predict_noalloc: the learned-chemistry model's inference with its
scratch in the library's fixed device array instead of allocated buffers.

It exists for callers that cannot call cudaMalloc while they run (a solver
that has handed all free device memory to its own pool, a time loop that
cannot take cudaMalloc's device-wide synchronisation). Its results must be
those of eu_mlp_predict, within the model tests' tolerance (2e-3 of the output
scale), on consecutive calls that reuse the same array. The file sorts last so
that a run stopping at the first failure has run every other test first.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_IN, WIDTH, HIDDEN, N_OUT, MEMBERS = 12, 256, 3, 10, 3
SCRATCH_BYTES = 16 << 20


def max_rows():
    in_pad, out_pad = (N_IN + 15) // 16 * 16, (N_OUT + 15) // 16 * 16
    return (SCRATCH_BYTES - 1024) // (2 * in_pad + 4 * WIDTH + 4 * out_pad)


def test_noalloc_predict_matches_predict_on_consecutive_calls(gpu):
    import torch
    m = gpu.Mlp()
    m.init(N_IN, WIDTH, HIDDEN, N_OUT, MEMBERS, max_batch=4096, seed=21)
    rng = np.random.default_rng(21)
    osc = rng.uniform(0.5, 2, N_OUT)
    m.set_scaling(rng.normal(size=N_IN), rng.uniform(0.5, 2, N_IN), rng.normal(size=N_OUT), osc)
    tol = 2e-3 * float((1 / osc).max())
    # the larger call first, so the second reads an array that still holds
    # the first call's data beyond its own rows
    for call, n in enumerate((max_rows(), 1000)):
        X = torch.from_numpy(rng.normal(size=(n, N_IN)).astype(np.float32)).cuda()
        want = torch.zeros(MEMBERS, n, N_OUT, device="cuda")
        got = torch.full((MEMBERS, n, N_OUT), float("nan"), device="cuda")
        m.predict(X, want)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        m.predict_noalloc(X, got)
        torch.cuda.synchronize()
        # eu_mlp_init has loaded the fixed array: no call, the first included,
        # may take device memory
        assert torch.cuda.mem_get_info()[0] == free_before, call
        assert torch.isfinite(got).all(), call
        err = float((got - want).abs().max())
        scale = max(1.0, float(want.abs().max()))
        assert err <= tol * scale, (call, n, err)


def test_noalloc_predict_rejects_rows_beyond_the_scratch(gpu):
    import torch
    m = gpu.Mlp()
    m.init(N_IN, WIDTH, HIDDEN, N_OUT, MEMBERS, max_batch=1024, seed=22)
    m.set_scaling(np.zeros(N_IN), np.ones(N_IN), np.zeros(N_OUT), np.ones(N_OUT))
    n = max_rows() + 1
    X = torch.zeros(n, N_IN, device="cuda")
    out = torch.zeros(MEMBERS, n, N_OUT, device="cuda")
    with pytest.raises(gpu.EU3DError) as e:
        m.predict_noalloc(X, out)
    assert e.value.name == "EU_ERR_INVALID_ARGUMENT"
    assert "scratch" in str(e.value)
