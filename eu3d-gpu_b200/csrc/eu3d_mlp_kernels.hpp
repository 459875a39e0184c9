// eu3d_mlp_kernels.hpp — host launch interface of the learned-chemistry kernels
// (eu3d_mlp.cu). bf16 buffers are passed as void pointers so host code needs
// no CUDA half-precision headers.
#pragma once

#include <cuda_runtime.h>

namespace eu3d {

// C = epilogue(A B^T): A (M x K), B (N x K) row-major bf16; act 0 none, 1 SiLU,
// 2 times SiLU'(Z), 3 atomically accumulate into Cf (split-K partial sums).
cudaError_t gemm_bf16(const void *A, int lda, const void *B, int ldb, int M, int N, int K, const float *bias, int act,
                      float *Cf, void *Cb, float *Cpre, int ldc, const float *Z, int k_split, int *err, cudaStream_t s);
cudaError_t transpose_bf16(const void *in, int R, int C, int ldi, void *out, int ldo, cudaStream_t s);
cudaError_t pack_features(const float *X, long long n, int n_in, const int *rows, const float *shift,
                          const float *scale, void *out, int ld, cudaStream_t s);
cudaError_t mse_grad(const float *Y, int ldy, const float *T, long long n, int n_out, const int *rows,
                     const float *shift, const float *scale, void *dY, float *loss, cudaStream_t s);
cudaError_t colsum_f32(const float *A, long long R, int C, int lda, float *out, cudaStream_t s);
cudaError_t colsum_bf16(const void *A, long long R, int C, int lda, float *out, cudaStream_t s);
cudaError_t adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2, float eps,
                 float c1, float c2, cudaStream_t s);
cudaError_t refresh_weights(const float *W, int out, int in, int out_pad, int in_pad, void *Wb, void *Wt,
                            cudaStream_t s);
cudaError_t random_rows(int *rows, int count, long long n, unsigned long long key, cudaStream_t s);
cudaError_t unscale_outputs(const float *Y, long long n, int ld, int n_out, const float *shift, const float *scale,
                            float *out, cudaStream_t s);

} // namespace eu3d
