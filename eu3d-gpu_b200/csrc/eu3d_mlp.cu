// eu3d_mlp.cu — tensor-core kernels of the learned-chemistry model and their
// C entry points (declared in include/eu3d.h).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "eu3d.h"
#include "eu3d_gemm.cuh"

using namespace eu3d;

namespace {

template <int BN>
cudaError_t gemm_launch(const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, int M, int N, int K,
                        const float *bias, int act, float *Cf, __nv_bfloat16 *Cb, float *Cpre, int ldc, int *err,
                        cudaStream_t s)
{
    const size_t smem = gemm_smem_bytes<BN>();
    static bool configured = false;
    if (!configured) {
        cudaError_t e =
            cudaFuncSetAttribute(k_gemm_bf16<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess)
            return e;
        configured = true;
    }
    const dim3 grid((M + kGemmBM - 1) / kGemmBM, (N + BN - 1) / BN);
    k_gemm_bf16<BN><<<grid, kGemmThreads, smem, s>>>(A, lda, B, ldb, M, N, K, bias, act, Cf, Cb, Cpre, ldc, err);
    return cudaGetLastError();
}

} // namespace

namespace eu3d {
// C = act(A B^T + bias): A (M x K), B (N x K), row-major bf16, K % 16 == 0.
cudaError_t gemm_bf16(const void *A, int lda, const void *B, int ldb, int M, int N, int K, const float *bias, int act,
                      float *Cf, void *Cb, float *Cpre, int ldc, int *err, cudaStream_t s)
{
    auto a = static_cast<const __nv_bfloat16 *>(A);
    auto b = static_cast<const __nv_bfloat16 *>(B);
    auto cb = static_cast<__nv_bfloat16 *>(Cb);
    if (N > 128)
        return gemm_launch<256>(a, lda, b, ldb, M, N, K, bias, act, Cf, cb, Cpre, ldc, err, s);
    if (N > 64)
        return gemm_launch<128>(a, lda, b, ldb, M, N, K, bias, act, Cf, cb, Cpre, ldc, err, s);
    return gemm_launch<64>(a, lda, b, ldb, M, N, K, bias, act, Cf, cb, Cpre, ldc, err, s);
}
} // namespace eu3d
