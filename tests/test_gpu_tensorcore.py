"""The BF16 tensor-core GEMM (tcgen05, TMEM accumulator) against a plain
PyTorch fp32 reference of the same operation: C = act(A @ B^T + bias).

Tolerance: products of bf16 inputs are exact in fp32 and the accumulation is
fp32, so the difference from an fp32 reference is accumulation-order rounding:
|C - C_ref| <= 1e-4 * (sum_k |a_ik b_jk| + |bias_j|) + 1e-6, and bf16 outputs
within one bf16 rounding of that.
"""
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(128, 128, 64), (300, 256, 16), (1000, 256, 256), (517, 16, 256), (64, 48, 32), (129, 130, 80),
          (4096, 256, 256)]


@pytest.mark.parametrize("M,N,K", SHAPES)
@pytest.mark.parametrize("act", [0, 1])
def test_gemm_matches_fp32_reference(gpu, M, N, K, act):
    import torch
    torch.manual_seed(M * 7 + N * 3 + K)
    dev = "cuda"
    A = torch.randn(M, K, device=dev).to(torch.bfloat16)
    B = (torch.randn(N, K, device=dev) / K ** 0.5).to(torch.bfloat16)
    bias = torch.randn(N, device=dev)
    Cf = torch.empty(M, N, device=dev)
    Cb = torch.empty(M, N, device=dev, dtype=torch.bfloat16)
    Cpre = torch.empty(M, N, device=dev)
    mlp = gpu.Mlp()
    torch.cuda.synchronize()
    mlp.gemm(A, B, bias=bias, act=act, Cf=Cf, Cb=Cb, Cpre=Cpre, stream=torch.cuda.current_stream().cuda_stream)
    ref_pre = A.float() @ B.float().T + bias
    ref = torch.nn.functional.silu(ref_pre) if act else ref_pre
    scale = A.float().abs() @ B.float().abs().T + bias.abs()
    tol = 1e-4 * scale + 1e-6
    assert ((Cpre - ref_pre).abs() <= tol).all(), (Cpre - ref_pre).abs().max().item()
    assert ((Cf - ref).abs() <= tol * 1.01 + 1e-6).all(), (Cf - ref).abs().max().item()
    assert ((Cb.float() - ref).abs() <= tol + ref.abs() * 2 ** -8).all()


def test_gemm_rejects_bad_shapes(gpu):
    import torch
    mlp = gpu.Mlp()
    A = torch.zeros(16, 24, device="cuda", dtype=torch.bfloat16)
    B = torch.zeros(16, 24, device="cuda", dtype=torch.bfloat16)
    C = torch.zeros(16, 16, device="cuda")
    with pytest.raises(gpu.EU3DError) as e:
        mlp.gemm(A, B, Cf=C)  # K = 24 is not a multiple of 16
    assert e.value.name == "EU_ERR_INVALID_ARGUMENT"
