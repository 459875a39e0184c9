// eu3d_mlp.cu — tensor-core kernels of the learned-chemistry model: the BF16
// GEMM launcher (eu3d_gemm.cuh) and the element-wise kernels of training
// (feature packing, transposes, loss gradient, bias reductions, Adam).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "eu3d.h"
#include "eu3d_attr.hpp"
#include "eu3d_gemm.cuh"
#include "eu3d_mlp_fused.cuh"
#include "eu3d_mlp_kernels.hpp"

using namespace eu3d;

namespace {

template <int BN>
cudaError_t gemm_launch(const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, int M, int N, int K,
                        const float *bias, int act, float *Cf, __nv_bfloat16 *Cb, float *Cpre, int ldc, const float *Z,
                        int k_split, int *err, cudaStream_t s)
{
    const size_t smem = gemm_smem_bytes<BN>();
    static SmemLimit limit; // per instantiation, per device
    const cudaError_t e = limit.ensure(k_gemm_bf16<BN>, smem);
    if (e != cudaSuccess)
        return e;
    const dim3 grid((M + kGemmBM - 1) / kGemmBM, (N + BN - 1) / BN, k_split);
    k_gemm_bf16<BN>
        <<<grid, kGemmThreads, smem, s>>>(A, lda, B, ldb, M, N, K, bias, act, Cf, Cb, Cpre, ldc, Z, k_split, err);
    return cudaGetLastError();
}

__global__ void k_transpose_bf16(const __nv_bfloat16 *__restrict__ in, int R, int C, int ldi,
                                 __nv_bfloat16 *__restrict__ out, int ldo)
{
    __shared__ __nv_bfloat16 tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int r = r0 + y, c = c0 + threadIdx.x;
        tile[y][threadIdx.x] = (r < R && c < C) ? in[(size_t)r * ldi + c] : __float2bfloat16_rn(0.0f);
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int c = c0 + y, r = r0 + threadIdx.x;
        if (c < C && r < R)
            out[(size_t)c * ldo + r] = tile[threadIdx.x][y];
    }
}

// rows of n_in fp32 features -> (x - shift) * scale as bf16, zero padded to ld
__global__ void k_pack_features(const float *__restrict__ X, long long n, int n_in, const int *__restrict__ rows,
                                 const float *__restrict__ shift, const float *__restrict__ scale,
                                 __nv_bfloat16 *__restrict__ out, int ld)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * ld)
        return;
    const long long r = t / ld;
    const int c = int(t % ld);
    const long long src = rows ? rows[r] : r;
    float v = 0.0f;
    if (c < n_in)
        v = (X[src * n_in + c] - shift[c]) * scale[c];
    out[t] = __float2bfloat16_rn(v);
}

// dY = 2 (Y - T') / (n n_out) on the first n_out columns (T' = normalised
// target), zero on padding; accumulates sum((Y - T')^2) into loss.
__global__ void k_mse_grad(const float *__restrict__ Y, int ldy, const float *__restrict__ T, long long n, int n_out,
                           const int *__restrict__ rows, const float *__restrict__ shift,
                           const float *__restrict__ scale, __nv_bfloat16 *__restrict__ dY, float *loss)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float sq = 0.0f;
    if (t < n * ldy) {
        const long long r = t / ldy;
        const int c = int(t % ldy);
        float g = 0.0f;
        if (c < n_out) {
            const long long src = rows ? rows[r] : r;
            const float target = (T[src * n_out + c] - shift[c]) * scale[c];
            const float d = Y[t] - target;
            sq = d * d;
            g = 2.0f * d / float(n * n_out);
        }
        dY[t] = __float2bfloat16_rn(g);
    }
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0 && sq != 0.0f)
        atomicAdd(loss, sq);
}

// out[c] = sum_r A[r][c] (fp32 or bf16 source), columns < C
template <typename T>
__global__ void k_colsum(const T *__restrict__ A, long long R, int C, int lda, float *__restrict__ out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C)
        return;
    float s = 0.0f;
    for (long long r = blockIdx.y; r < R; r += gridDim.y) s += float(A[r * lda + c]);
    atomicAdd(&out[c], s);
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

// fp32 master W [out x in] -> bf16 Wb [out_pad x in_pad] and Wt [in_pad x out_pad]
__global__ void k_refresh(const float *__restrict__ W, int out, int in, int out_pad, int in_pad,
                          __nv_bfloat16 *__restrict__ Wb, __nv_bfloat16 *__restrict__ Wt)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= out_pad * in_pad)
        return;
    const int o = t / in_pad, i = t % in_pad;
    const float w = (o < out && i < in) ? W[o * in + i] : 0.0f;
    const __nv_bfloat16 b = __float2bfloat16_rn(w);
    Wb[t] = b;
    Wt[(size_t)i * out_pad + o] = b;
}

// Y [n x ld] normalised outputs of member e -> denormalised fp32 out[e][n][n_out]
__global__ void k_unscale(const float *__restrict__ Y, long long n, int ld, int n_out, const float *__restrict__ shift,
                          const float *__restrict__ scale, float *__restrict__ out)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * n_out)
        return;
    const long long r = t / n_out;
    const int c = int(t % n_out);
    out[t] = Y[r * ld + c] / scale[c] + shift[c];
}

// rows[i] = uniform index in [0, n) from a counter-based hash (splitmix64) of
// (seed, step, i): training batches drawn on the device, no host copies.
__global__ void k_random_rows(int *rows, int count, long long n, unsigned long long key)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    unsigned long long z = key + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    rows[i] = int(z % (unsigned long long)n);
}

inline unsigned blocks(long long n, int t) { return unsigned((n + t - 1) / t); }

} // namespace

namespace eu3d {

cudaError_t gemm_bf16(const void *A, int lda, const void *B, int ldb, int M, int N, int K, const float *bias, int act,
                      float *Cf, void *Cb, float *Cpre, int ldc, const float *Z, int k_split, int *err, cudaStream_t s)
{
    auto a = static_cast<const __nv_bfloat16 *>(A);
    auto b = static_cast<const __nv_bfloat16 *>(B);
    auto cb = static_cast<__nv_bfloat16 *>(Cb);
    if (k_split < 1)
        k_split = 1;
    if (N > 128)
        return gemm_launch<256>(a, lda, b, ldb, M, N, K, bias, act, Cf, cb, Cpre, ldc, Z, k_split, err, s);
    if (N > 64)
        return gemm_launch<128>(a, lda, b, ldb, M, N, K, bias, act, Cf, cb, Cpre, ldc, Z, k_split, err, s);
    return gemm_launch<64>(a, lda, b, ldb, M, N, K, bias, act, Cf, cb, Cpre, ldc, Z, k_split, err, s);
}

cudaError_t transpose_bf16(const void *in, int R, int C, int ldi, void *out, int ldo, cudaStream_t s)
{
    const dim3 grid((C + 31) / 32, (R + 31) / 32), block(32, 8);
    k_transpose_bf16<<<grid, block, 0, s>>>(static_cast<const __nv_bfloat16 *>(in), R, C, ldi,
                                             static_cast<__nv_bfloat16 *>(out), ldo);
    return cudaGetLastError();
}

cudaError_t pack_features(const float *X, long long n, int n_in, const int *rows, const float *shift,
                          const float *scale, void *out, int ld, cudaStream_t s)
{
    k_pack_features<<<blocks(n * ld, 256), 256, 0, s>>>(X, n, n_in, rows, shift, scale,
                                                         static_cast<__nv_bfloat16 *>(out), ld);
    return cudaGetLastError();
}

cudaError_t mse_grad(const float *Y, int ldy, const float *T, long long n, int n_out, const int *rows,
                     const float *shift, const float *scale, void *dY, float *loss, cudaStream_t s)
{
    k_mse_grad<<<blocks(n * ldy, 256), 256, 0, s>>>(Y, ldy, T, n, n_out, rows, shift, scale,
                                                     static_cast<__nv_bfloat16 *>(dY), loss);
    return cudaGetLastError();
}

cudaError_t colsum_f32(const float *A, long long R, int C, int lda, float *out, cudaStream_t s)
{
    const dim3 grid((C + 127) / 128, unsigned(R < 256 ? R : 256));
    k_colsum<float><<<grid, 128, 0, s>>>(A, R, C, lda, out);
    return cudaGetLastError();
}

cudaError_t colsum_bf16(const void *A, long long R, int C, int lda, float *out, cudaStream_t s)
{
    const dim3 grid((C + 127) / 128, unsigned(R < 256 ? R : 256));
    k_colsum<__nv_bfloat16><<<grid, 128, 0, s>>>(static_cast<const __nv_bfloat16 *>(A), R, C, lda, out);
    return cudaGetLastError();
}

cudaError_t adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2, float eps,
                 float c1, float c2, cudaStream_t s)
{
    k_adam<<<blocks(n, 256), 256, 0, s>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError();
}

cudaError_t refresh_weights(const float *W, int out, int in, int out_pad, int in_pad, void *Wb, void *Wt,
                            cudaStream_t s)
{
    k_refresh<<<blocks((long long)out_pad * in_pad, 256), 256, 0, s>>>(
        W, out, in, out_pad, in_pad, static_cast<__nv_bfloat16 *>(Wb), static_cast<__nv_bfloat16 *>(Wt));
    return cudaGetLastError();
}

cudaError_t random_rows(int *rows, int count, long long n, unsigned long long key, cudaStream_t s)
{
    k_random_rows<<<blocks(count, 256), 256, 0, s>>>(rows, count, n, key);
    return cudaGetLastError();
}

cudaError_t mlp_fused(const FusedMlpParams &p, const float *feat, int ld_feat, int count_host, const int *count_dev,
                      int max_rows, float *out, long long s_row, long long s_mem, int *err, int grid, cudaStream_t s)
{
    if (!fused_supported(p.in_pad, p.width, p.out_pad, p.members, p.layers))
        return cudaErrorInvalidValue;
    const size_t smem = fused_smem_bytes(p.in_pad, p.width, p.out_pad, p.layers, p.members);
    static SmemLimit limit; // per device: the largest size set so far
    const cudaError_t e = limit.ensure(k_mlp_fused, smem);
    if (e != cudaSuccess)
        return e;
    if (grid < 1)
        return cudaSuccess;
    k_mlp_fused<<<grid, kFusedThreads, smem, s>>>(p, feat, ld_feat, count_host, count_dev, max_rows, out, s_row, s_mem,
                                                  err);
    return cudaGetLastError();
}

cudaError_t pack_slabs(const void *W, int N, int K, void *out, cudaStream_t s)
{
    k_pack_slabs<<<blocks((long long)N * K, 256), 256, 0, s>>>(static_cast<const __nv_bfloat16 *>(W), N, K,
                                                                static_cast<__nv_bfloat16 *>(out));
    return cudaGetLastError();
}

cudaError_t unscale_outputs(const float *Y, long long n, int ld, int n_out, const float *shift, const float *scale,
                            float *out, cudaStream_t s)
{
    k_unscale<<<blocks(n * n_out, 256), 256, 0, s>>>(Y, n, ld, n_out, shift, scale, out);
    return cudaGetLastError();
}

} // namespace eu3d
