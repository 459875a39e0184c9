// eu3d_mlp_kernels.hpp — host launch interface of the learned-chemistry kernels
// (eu3d_mlp.cu). bf16 buffers are passed as void pointers so host code needs
// no CUDA half-precision headers.
#pragma once

#include <cuda_runtime.h>

namespace eu3d {

// The fused inference kernel (eu3d_mlp_fused.cuh): model shape, packed weight
// slabs and per-layer biases.
constexpr int kFusedMaxMembers = 8, kFusedMaxLayers = 9, kFusedSlabK = 32;
// weight-ring slots, rows per tile, tiles per job (each weight slab feeds
// the MMAs of kFusedStreams tiles); the opt-in shared-memory limit of a
// block on sm_100 (227 KB)
constexpr int kFusedStages = 5, kFusedRows = 128, kFusedStreams = 2;
constexpr size_t kFusedMaxSmem = 232448;
struct FusedMlpParams {
    int members, layers; // layers = hidden + output
    int n_in, in_pad, width, out_pad, n_out;
    const void *slabs;                                    // bf16, K-slabs of kFusedSlabK columns, core-matrix layout
    long long off[kFusedMaxMembers][kFusedMaxLayers];     // element offset of layer (e, l)'s first slab
    const float *bias[kFusedMaxMembers][kFusedMaxLayers]; // [N] per layer
    const float *in_shift, *in_scale, *out_shift, *out_scale;
};

// Biases of one member (every layer's N); the kernel keeps every member's in
// shared memory.
inline size_t fused_bias_floats(int width, int out_pad, int layers)
{
    return size_t(layers - 1) * width + out_pad;
}

// Bytes of the feature scaling and output unscaling the fused kernel keeps in
// shared memory: in_shift, in_scale [in_pad], out_shift, out_scale [out_pad].
inline size_t fused_scaling_bytes(int in_pad, int out_pad) { return (size_t(2 * in_pad + 2 * out_pad) * 4 + 15) / 16 * 16; }

// Bytes of shared memory the fused kernel needs for a model: the weight ring,
// each stream's activations and features, the members' biases, the scaling,
// the mbarriers. At least 116 KB, so that one block (and its 512 TMEM
// columns) fits per SM.
inline size_t fused_smem_bytes(int in_pad, int width, int out_pad, int layers, int members)
{
    const size_t bias = (size_t(members) * fused_bias_floats(width, out_pad, layers) * 4 + 15) / 16 * 16;
    const size_t need = size_t(kFusedStages) * width * kFusedSlabK * 2 +
                        size_t(kFusedStreams) * size_t(kFusedRows) * (size_t(width) + in_pad) * 2 + bias +
                        fused_scaling_bytes(in_pad, out_pad) + 8 * (2 * kFusedStages + 2 * kFusedStreams) + 16;
    return need > 116 * 1024 ? need : 116 * 1024;
}

// Shapes the fused kernel takes: every layer's N fits the 256 TMEM columns and
// the ring slot (sized for width), the input tile fits its buffer, and all of
// it fits a block's shared memory.
inline bool fused_supported(int in_pad, int width, int out_pad, int members, int layers)
{
    return width % 16 == 0 && width >= 16 && width <= 256 && in_pad <= 64 && out_pad <= width &&
           members >= 1 && members <= kFusedMaxMembers && layers >= 2 && layers <= kFusedMaxLayers &&
           fused_smem_bytes(in_pad, width, out_pad, layers, members) <= kFusedMaxSmem;
}

// CTAs of a fused launch over `tiles` 128-row tiles: one per tile pair, at
// most one per SM.
inline int fused_grid(long long tiles, int sms)
{
    const long long pairs = (tiles + kFusedStreams - 1) / kFusedStreams;
    return int(pairs < sms ? pairs : sms);
}

// Predictions of every member for the first `count` rows of feat (count read
// from count_dev when it is not null, capped at max_rows): out[row * s_row +
// member * s_mem + o]. `grid` CTAs (one per SM is the intent).
cudaError_t mlp_fused(const FusedMlpParams &p, const float *feat, int ld_feat, int count_host, const int *count_dev,
                      int max_rows, float *out, long long s_row, long long s_mem, int *err, int grid, cudaStream_t s);
// One layer's bf16 [N x K] weights into K-slabs (see k_pack_slabs).
cudaError_t pack_slabs(const void *W, int N, int K, void *out, cudaStream_t s);

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
