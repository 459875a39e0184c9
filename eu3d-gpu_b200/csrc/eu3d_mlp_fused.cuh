// eu3d_mlp_fused.cuh — the learned-chemistry ensemble's whole forward pass in
// one persistent tcgen05 kernel (inference only; training uses the layer-wise
// GEMMs of eu3d_gemm.cuh).
//
// One CTA of 512 threads per SM walks the 128-row tiles of the input rows
// (tile = blockIdx.x, blockIdx.x + gridDim.x, ...). The row count may be read
// from device memory when the kernel starts, so a launch needs no host-side
// count and can sit in a captured CUDA graph. For each tile and member, every
// layer runs on the tensor cores with the activations resident in shared
// memory:
//   features (fp32, scaled and rounded to bf16)          -> fin  [128 x in_pad]
//   layer l: TMEM[128 x N] = A[128 x K] * W_l[N x K]^T    (A = fin or act)
//   hidden epilogue: + bias, SiLU, bf16                    -> act  [128 x width]
//   output epilogue: + bias, / out_scale + out_shift       -> global predictions
// Weights stream through a three-slot shared-memory ring in K-slabs of 64
// columns, pre-packed in global memory in the operands' core-matrix layout so
// that each slab is one contiguous bulk copy (cp.async.bulk, completion counted
// on a "full" mbarrier); the MMAs that read a slot commit to its "empty"
// mbarrier. Thread 0 issues the copies and the MMAs; all threads run the
// epilogues: warp w reads TMEM lanes 32 (w % 4) (its rows) and the four warp
// groups take every fourth 32-column chunk of the accumulator. Every wait is bounded: on a timeout the CTA records an error,
// waits (bounded) for its copies in flight, frees its TMEM and returns.
//
// The arithmetic is the layer-wise path's: the same K=16 MMA sequence into an
// fp32 accumulator, the same bias/SiLU/bf16 epilogue, the same feature scaling
// and output unscaling.
#pragma once

#include <cuda_bf16.h>

#include "eu3d_gemm.cuh"
#include "eu3d_mlp_kernels.hpp"
#include "eu3d_tc.cuh"

namespace eu3d {

constexpr int kFusedStages = 3, kFusedRows = 128, kFusedThreads = 512, kFusedGroups = kFusedThreads / 128;

// Bytes of shared memory the kernel needs for a model.
// At least 116 KB, so that one CTA (and its 256 TMEM columns) fits per SM.
inline size_t fused_smem_bytes(int in_pad, int width)
{
    const size_t need = size_t(kFusedStages) * width * kFusedSlabK * 2 + size_t(kFusedRows) * width * 2 +
                        size_t(kFusedRows) * in_pad * 2 + 2 * kFusedStages * 8 + 16;
    return need > 116 * 1024 ? need : 116 * 1024;
}

__device__ __forceinline__ int fused_K(const FusedMlpParams &p, int l) { return l == 0 ? p.in_pad : p.width; }
__device__ __forceinline__ int fused_N(const FusedMlpParams &p, int l)
{
    return l == p.layers - 1 ? p.out_pad : p.width;
}
__device__ __forceinline__ int fused_slabs(const FusedMlpParams &p, int l)
{
    return (fused_K(p, l) + kFusedSlabK - 1) / kFusedSlabK;
}

// Position in the per-tile slab sequence (member, layer, slab).
struct SlabCursor {
    int e = 0, l = 0, s = 0;
    __device__ void advance(const FusedMlpParams &p)
    {
        if (++s == fused_slabs(p, l)) {
            s = 0;
            if (++l == p.layers) {
                l = 0;
                if (++e == p.members)
                    e = 0;
            }
        }
    }
};

__global__ void __launch_bounds__(kFusedThreads, 1)
    k_mlp_fused(const __grid_constant__ FusedMlpParams p, const float *__restrict__ feat, int ld_feat, int count_host,
                const int *__restrict__ count_dev, int max_rows, float *pred, long long s_row, long long s_mem,
                int *err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t slot_bytes = uint32_t(p.width) * kFusedSlabK * 2;
    unsigned char *ring = smem;
    unsigned char *act = ring + kFusedStages * slot_bytes;
    unsigned char *fin = act + kFusedRows * p.width * 2;
    uint64_t *full = reinterpret_cast<uint64_t *>(fin + kFusedRows * p.in_pad * 2);
    uint64_t *empty = full + kFusedStages;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(empty + kFusedStages);

    const int tid = threadIdx.x, warp = tid / 32;
    const int lrow = tid % kFusedRows, wg = tid / kFusedRows; // tile row (TMEM lane), warp group
    int count = count_dev ? *count_dev : count_host;
    count = count < max_rows ? count : max_rows;
    const int ntiles = (count + kFusedRows - 1) / kFusedRows;
    const int mine = blockIdx.x < ntiles ? (ntiles - 1 - int(blockIdx.x)) / int(gridDim.x) + 1 : 0;
    if (mine == 0)
        return;
    int per_tile = 0;
    for (int l = 0; l < p.layers; ++l) per_tile += fused_slabs(p, l);
    per_tile *= p.members;
    const long long total = (long long)mine * per_tile;

    if (warp == 0) {
        tc::tmem_alloc(tslot, 256);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int q = 0; q < kFusedStages; ++q) {
            tc::mbar_init(&full[q], 1);
            tc::mbar_init(&empty[q], 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tslot;

    // producer state (thread 0): next slab to load and its cursor
    long long gp = 0, gc = 0; // slabs loaded, slabs consumed
    SlabCursor pc;
    bool ok = true;
    auto produce = [&](long long upto) {
        while (ok && gp < upto && gp < total) {
            const int slot = int(gp % kFusedStages);
            if (gp >= kFusedStages && !tc::mbar_wait(&empty[slot], uint32_t((gp / kFusedStages - 1) & 1))) {
                ok = false;
                break;
            }
            const int N = fused_N(p, pc.l), K = fused_K(p, pc.l);
            const int k0 = pc.s * kFusedSlabK, kw = min(kFusedSlabK, K - k0);
            const uint32_t bytes = uint32_t(N) * kw * 2;
            const __nv_bfloat16 *src =
                static_cast<const __nv_bfloat16 *>(p.slabs) + p.off[pc.e][pc.l] + (long long)pc.s * N * kFusedSlabK;
            tc::mbar_arrive_expect_tx(&full[slot], bytes);
            tc::bulk_g2s(ring + slot * slot_bytes, src, bytes, &full[slot]);
            pc.advance(p);
            ++gp;
        }
    };

    // Thread 0 keeps two slabs requested ahead of the one the MMAs consume: the
    // slot of slab g + 2 was last read by slab g - 1, whose MMAs were issued
    // before slab g's, so the tensor pipe stays fed while it waits for them.
    if (tid == 0)
        produce(kFusedStages - 1);
    long long g = 0; // slabs consumed so far (all threads track it)
    for (int it = 0; it < mine && ok; ++it) {
        const int tile = int(blockIdx.x) + it * int(gridDim.x);
        const int row = tile * kFusedRows + lrow;
        const bool valid = row < count;
        // features -> fin (core-matrix layout, 8 bf16 per 16-byte chunk)
        for (int kc = wg; kc < p.in_pad / 8; kc += kFusedGroups) {
            __align__(16) __nv_bfloat16 v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int c = kc * 8 + q;
                float x = 0.0f;
                if (valid && c < p.n_in)
                    x = (feat[(long long)row * ld_feat + c] - p.in_shift[c]) * p.in_scale[c];
                v[q] = __float2bfloat16_rn(x);
            }
            *reinterpret_cast<uint4 *>(fin + (kc * kFusedRows + lrow) * 16) = *reinterpret_cast<const uint4 *>(v);
        }
        tc::fence_proxy_async();
        tc::tc_fence_before();
        __syncthreads();
        tc::tc_fence_after();
        for (int e = 0; e < p.members && ok; ++e) {
            for (int l = 0; l < p.layers; ++l) {
                const int N = fused_N(p, l), K = fused_K(p, l), ns = fused_slabs(p, l);
                const uint32_t idesc = tc::idesc_bf16_f32(kFusedRows, N);
                const uint32_t a0 = tc::smem_u32(l == 0 ? fin : act);
                if (tid == 0) {
                    for (int s = 0; s < ns && ok; ++s) {
                        const int slot = int(g % kFusedStages);
                        if (!ok || !tc::mbar_wait(&full[slot], uint32_t((g / kFusedStages) & 1))) {
                            ok = false;
                            break;
                        }
                        ++gc;
                        tc::tc_fence_after();
                        const int kw = min(kFusedSlabK, K - s * kFusedSlabK);
                        const uint32_t b0 = tc::smem_u32(ring + slot * slot_bytes);
                        for (int kk = 0; kk < kw / 16; ++kk) {
                            const int kg = s * (kFusedSlabK / 16) + kk;
                            const uint64_t ad = tc::smem_desc(a0 + kg * 2 * kFusedRows * 16, kFusedRows * 16, 128);
                            const uint64_t bd = tc::smem_desc(b0 + kk * 2 * N * 16, N * 16, 128);
                            tc::mma_bf16(tmem, ad, bd, idesc, (s > 0 || kk > 0) ? 1u : 0u);
                        }
                        tc::mma_commit(&empty[slot]);
                        ++g;
                        produce(g + kFusedStages - 1);
                    }
                    // the last commit tracks every MMA of the layer
                    if (ok && !tc::mbar_wait(&empty[int((g - 1) % kFusedStages)], uint32_t(((g - 1) / kFusedStages) & 1)))
                        ok = false;
                } else {
                    g += ns;
                }
                ok = __syncthreads_and(ok);
                if (!ok)
                    break;
                tc::tc_fence_after();
                const float *bias = p.bias[e][l];
                const uint32_t trow = tmem + (uint32_t((warp % 4) * 32) << 16);
                if (l < p.layers - 1) {
                    for (int c0 = wg * 32; c0 < N; c0 += 32 * kFusedGroups) {
                        float v[32];
                        tc::tmem_ld32(trow + c0, v);
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int cbase = c0 + j * 8;
                            if (cbase < N) {
                                __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                                for (int q = 0; q < 8; ++q) h[q] = __float2bfloat16_rn(silu(v[j * 8 + q] + bias[cbase + q]));
                                *reinterpret_cast<uint4 *>(act + ((cbase / 8) * kFusedRows + lrow) * 16) =
                                    *reinterpret_cast<const uint4 *>(h);
                            }
                        }
                    }
                    tc::fence_proxy_async();
                } else {
                    for (int c0 = wg * 32; c0 < N; c0 += 32 * kFusedGroups) {
                        float v[32];
                        tc::tmem_ld32(trow + c0, v);
                        if (valid) {
#pragma unroll
                            for (int q = 0; q < 32; ++q) {
                                const int o = c0 + q;
                                if (o < p.n_out)
                                    pred[(long long)row * s_row + (long long)e * s_mem + o] =
                                        (v[q] + bias[o]) / p.out_scale[o] + p.out_shift[o];
                            }
                        }
                    }
                }
                tc::tc_fence_before();
                __syncthreads();
                tc::tc_fence_after();
            }
        }
    }
    if (!ok && tid == 0) {
        atomicExch(err, 1);
        // copies still in flight land before the CTA's shared memory goes away
        for (long long q = gc; q < gp; ++q)
            tc::mbar_wait(&full[int(q % kFusedStages)], uint32_t((q / kFusedStages) & 1));
        if (g > 0)
            tc::mbar_wait(&empty[int((g - 1) % kFusedStages)], uint32_t(((g - 1) / kFusedStages) & 1));
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0)
        tc::tmem_dealloc(tmem, 256);
}

// Weights of one layer, bf16 [N x K] row-major, into its K-slabs of 64 columns,
// each in the core-matrix layout: element (n, k) of slab s at
// ((k' / 8) * N + n) * 8 + k' % 8, k' = k - 64 s, slabs back to back.
__global__ void k_pack_slabs(const __nv_bfloat16 *__restrict__ W, int N, int K, __nv_bfloat16 *__restrict__ out)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)N * K)
        return;
    const int n = int(t / K), k = int(t % K);
    const int s = k / kFusedSlabK, kl = k % kFusedSlabK;
    out[(long long)s * N * kFusedSlabK + ((kl / 8) * N + n) * 8 + kl % 8] = W[t];
}

} // namespace eu3d
