// eu3d_mlp_fused.cuh — the learned-chemistry ensemble's whole forward pass in
// one persistent tcgen05 kernel (inference only; training uses the layer-wise
// GEMMs of eu3d_gemm.cuh).
//
// One CTA per SM walks the 128-row tiles of the input rows (tile =
// blockIdx.x, blockIdx.x + gridDim.x, ...). The row count may be read from
// device memory when the kernel starts, so a launch needs no host-side count
// and can sit in a captured CUDA graph. A job is one (tile, member) pair: its
// layers run on the tensor cores with the activations resident in shared
// memory:
//   features (fp32, scaled and rounded to bf16)          -> fin  [128 x in_pad]
//   layer l: TMEM[128 x N] = A[128 x K] * W_l[N x K]^T    (A = fin or act)
//   hidden epilogue: + bias, SiLU, bf16                    -> act  [128 x width]
//   output epilogue: + bias, / out_scale + out_shift       -> global predictions
//
// Two jobs are in flight at once, in two streams with their own activation
// buffers and TMEM accumulators (256 columns each): while one stream's
// epilogue runs on the CUDA cores, the tensor core runs the other stream's
// layer. Roles (warp-specialised):
//   warps 0-7   epilogue of stream 0, warps 8-15 epilogue of stream 1: warp w
//               reads TMEM lanes 32 (w % 4) (its 32 rows) and the columns of
//               half (w / 4) % 2 of the accumulator's 32-column chunks;
//   warp 16     one thread issues the MMAs,
//   warp 17     one thread issues the weight copies.
// The MMA thread issues the streams' layers alternately; before a
// stream's layer it waits on that stream's "ready" mbarrier (its 8 epilogue
// warps arrive when the layer's A operand is in shared memory and its
// accumulator has been read), after it commits the MMAs to the stream's
// "accumulator full" mbarrier, on which the epilogue warps wait.
// Weights stream through a five-slot shared-memory ring in K-slabs of 32
// columns, pre-packed in global memory in the operands' core-matrix layout so
// that each slab is one contiguous bulk copy (cp.async.bulk, completion counted
// on a "full" mbarrier); the MMAs that read a slot commit to its "empty"
// mbarrier. Every wait is bounded and watches a shared abort flag: on a
// timeout the CTA records an error, every role leaves its loop, the copy and
// MMA threads wait (bounded) for their copies and MMAs in flight, and the TMEM
// is freed before the CTA returns.
//
// The arithmetic is the layer-wise inference path's: the same K=16 MMA
// sequence into an fp32 accumulator, the same bias/SiLU/bf16 epilogue (SiLU in
// its inference form, silu_fast), the same feature scaling and output
// unscaling.
#pragma once

#include <cuda_bf16.h>

#include "eu3d_gemm.cuh"
#include "eu3d_mlp_kernels.hpp"
#include "eu3d_tc.cuh"

namespace eu3d {

constexpr int kFusedEpiWarps = 8;
constexpr int kFusedMmaWarp = kFusedStreams * kFusedEpiWarps, kFusedCopyWarp = kFusedMmaWarp + 1;
constexpr int kFusedThreads = (kFusedCopyWarp + 1) * 32;
constexpr int kFusedTmemCols = 256 * kFusedStreams;

__device__ __forceinline__ int fused_K(const FusedMlpParams &p, int l) { return l == 0 ? p.in_pad : p.width; }
__device__ __forceinline__ int fused_N(const FusedMlpParams &p, int l)
{
    return l == p.layers - 1 ? p.out_pad : p.width;
}
__device__ __forceinline__ int fused_slabs(const FusedMlpParams &p, int l)
{
    return (fused_K(p, l) + kFusedSlabK - 1) / kFusedSlabK;
}

// The order in which the control thread issues layers: step k of stream 0,
// then step k of stream 1, k = 0, 1, ...; stream x has n[x] steps (step k is
// layer k % layers of its job k / layers; its jobs are x, x + 2, x + 4, ...).
struct StepCursor {
    int k = 0, x = 0;
    __device__ bool valid(const int (&n)[kFusedStreams]) const { return k < n[x]; }
    __device__ void advance(const int (&n)[kFusedStreams])
    {
        do {
            if (++x == kFusedStreams) {
                x = 0;
                ++k;
            }
        } while (k < (n[0] > n[1] ? n[0] : n[1]) && k >= n[x]);
    }
};

// Bounded mbarrier wait that gives up early when another role has aborted.
__device__ __forceinline__ bool fused_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag)
{
    for (uint32_t n = 0; n < (1u << 24); ++n) {
        if (tc::mbar_try_wait(bar, parity))
            return true;
        if ((n & 63) == 63 && *abort_flag)
            return false;
    }
    *abort_flag = 1;
    return false;
}

__global__ void __launch_bounds__(kFusedThreads, 1)
    k_mlp_fused(const __grid_constant__ FusedMlpParams p, const float *__restrict__ feat, int ld_feat, int count_host,
                const int *__restrict__ count_dev, int max_rows, float *pred, long long s_row, long long s_mem,
                int *err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t slot_bytes = uint32_t(p.width) * kFusedSlabK * 2;
    const uint32_t act_bytes = uint32_t(kFusedRows) * p.width * 2, fin_bytes = uint32_t(kFusedRows) * p.in_pad * 2;
    const uint32_t nbias = uint32_t((p.layers - 1) * p.width + p.out_pad); // fused_bias_floats
    const uint32_t bias_bytes = (uint32_t(p.members) * nbias * 4 + 15) / 16 * 16;
    unsigned char *ring = smem;
    unsigned char *act0 = ring + kFusedStages * slot_bytes;
    unsigned char *fin0 = act0 + kFusedStreams * act_bytes;
    float *sbias = reinterpret_cast<float *>(fin0 + kFusedStreams * fin_bytes); // [member][layer][N]
    uint64_t *full = reinterpret_cast<uint64_t *>(reinterpret_cast<unsigned char *>(sbias) + bias_bytes);
    uint64_t *empty = full + kFusedStages;
    uint64_t *accf = empty + kFusedStages;  // per stream: the layer's MMAs are done
    uint64_t *ready = accf + kFusedStreams; // per stream: A operand written, accumulator read
    uint32_t *tslot = reinterpret_cast<uint32_t *>(ready + kFusedStreams);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tslot + 1);

    const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
    int count = count_dev ? *count_dev : count_host;
    count = count < max_rows ? count : max_rows;
    const int ntiles = (count + kFusedRows - 1) / kFusedRows;
    const int mine = blockIdx.x < ntiles ? (ntiles - 1 - int(blockIdx.x)) / int(gridDim.x) + 1 : 0;
    if (mine == 0)
        return;
    const int jobs = mine * p.members;
    int nsteps[kFusedStreams];
    for (int x = 0; x < kFusedStreams; ++x) nsteps[x] = (jobs - x + kFusedStreams - 1) / kFusedStreams * p.layers;

    if (warp == 0) {
        tc::tmem_alloc(tslot, kFusedTmemCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int q = 0; q < kFusedStages; ++q) {
            tc::mbar_init(&full[q], 1);
            tc::mbar_init(&empty[q], 1);
        }
        for (int x = 0; x < kFusedStreams; ++x) {
            tc::mbar_init(&accf[x], 1);
            tc::mbar_init(&ready[x], kFusedEpiWarps);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // every member's biases into shared memory (read by the epilogues)
    for (int e = 0; e < p.members; ++e)
        for (int l = 0, o = e * int(nbias); l < p.layers; o += fused_N(p, l), ++l)
            for (int c = tid; c < fused_N(p, l); c += kFusedThreads) sbias[o + c] = p.bias[e][l][c];
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == kFusedMmaWarp) {
        // ------------------------------------------------------------ MMAs
        if (lane == 0) {
            long long g = 0; // slabs consumed
            bool ok = true;
            int waits[kFusedStreams] = {0, 0};
            for (StepCursor c; ok && c.valid(nsteps); c.advance(nsteps)) {
                const int x = c.x, l = c.k % p.layers;
                if (!fused_wait(&ready[x], uint32_t(waits[x]++ & 1), abort_flag)) {
                    ok = false;
                    break;
                }
                tc::tc_fence_after();
                const int N = fused_N(p, l), K = fused_K(p, l), ns = fused_slabs(p, l);
                const uint32_t idesc = tc::idesc_bf16_f32(kFusedRows, N);
                const uint32_t a0 = tc::smem_u32(l == 0 ? fin0 + x * fin_bytes : act0 + x * act_bytes);
                const uint32_t d = tmem + uint32_t(256 * x);
                for (int s = 0; s < ns; ++s) {
                    const int slot = int(g % kFusedStages);
                    if (!fused_wait(&full[slot], uint32_t((g / kFusedStages) & 1), abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc::tc_fence_after();
                    const int kw = min(kFusedSlabK, K - s * kFusedSlabK);
                    const uint32_t b0 = tc::smem_u32(ring + slot * slot_bytes);
                    for (int kk = 0; kk < kw / 16; ++kk) {
                        const int kg = s * (kFusedSlabK / 16) + kk;
                        const uint64_t ad = tc::smem_desc(a0 + kg * 2 * kFusedRows * 16, kFusedRows * 16, 128);
                        const uint64_t bd = tc::smem_desc(b0 + kk * 2 * N * 16, N * 16, 128);
                        tc::mma_bf16(d, ad, bd, idesc, (s > 0 || kk > 0) ? 1u : 0u);
                    }
                    tc::mma_commit(&empty[slot]);
                    ++g;
                }
                if (!ok)
                    break;
                tc::mma_commit(&accf[x]); // every MMA of the layer, in issue order
            }
            if (!ok) {
                *abort_flag = 1;
                atomicExch(err, 1);
                // the MMAs issued so far finish before the CTA's memory goes
                // away (the last empty commit follows every one of them)
                if (g > 0)
                    tc::mbar_wait(&empty[int((g - 1) % kFusedStages)], uint32_t(((g - 1) / kFusedStages) & 1));
            }
        }
    } else if (warp == kFusedCopyWarp) {
        // ---------------------------------------------------- weight copies
        if (lane == 0) {
            long long gp = 0; // slabs requested
            StepCursor pc;    // the step and slab of slab gp
            int ps = 0;
            bool ok = true;
            while (pc.valid(nsteps)) {
                const int slot = int(gp % kFusedStages);
                if (gp >= kFusedStages &&
                    !fused_wait(&empty[slot], uint32_t((gp / kFusedStages - 1) & 1), abort_flag)) {
                    ok = false;
                    break;
                }
                const int job = pc.x + kFusedStreams * (pc.k / p.layers), l = pc.k % p.layers;
                const int e = job % p.members;
                const int N = fused_N(p, l), K = fused_K(p, l);
                const int k0 = ps * kFusedSlabK, kw = min(kFusedSlabK, K - k0);
                const uint32_t bytes = uint32_t(N) * kw * 2;
                const __nv_bfloat16 *src =
                    static_cast<const __nv_bfloat16 *>(p.slabs) + p.off[e][l] + (long long)ps * N * kFusedSlabK;
                tc::mbar_arrive_expect_tx(&full[slot], bytes);
                tc::bulk_g2s(ring + slot * slot_bytes, src, bytes, &full[slot]);
                if (++ps == fused_slabs(p, l)) {
                    ps = 0;
                    pc.advance(nsteps);
                }
                ++gp;
            }
            if (!ok) {
                *abort_flag = 1;
                atomicExch(err, 1);
            }
            // the last copies (one per slot at most) land before the CTA's
            // shared memory goes away; earlier slots were waited for above
            for (long long q = gp > kFusedStages ? gp - kFusedStages : 0; q < gp; ++q)
                tc::mbar_wait(&full[int(q % kFusedStages)], uint32_t((q / kFusedStages) & 1));
        }
    } else {
        // ---------------------------------------- epilogue warps of stream x
        const int x = warp / kFusedEpiWarps, w8 = warp % kFusedEpiWarps;
        const int quad = w8 % 4, half = w8 / 4;
        const int lrow = quad * 32 + lane; // tile row = TMEM lane
        unsigned char *act = act0 + x * act_bytes, *fin = fin0 + x * fin_bytes;
        const uint32_t trow = tmem + uint32_t(256 * x) + (uint32_t(quad * 32) << 16);
        int accw = 0;
        bool ok = true;
        auto arrive_ready = [&]() {
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(&ready[x])) : "memory");
        };
        for (int job = x; ok && job < jobs; job += kFusedStreams) {
            const int tile = int(blockIdx.x) + (job / p.members) * int(gridDim.x), e = job % p.members;
            const int row = tile * kFusedRows + lrow;
            const bool valid = row < count;
            // features -> fin (core-matrix layout, 8 bf16 per 16-byte chunk):
            // the two column halves of the tile's rows
            for (int kc = half; kc < p.in_pad / 8; kc += 2) {
                __align__(16) __nv_bfloat16 v[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int c = kc * 8 + q;
                    float f = 0.0f;
                    if (valid && c < p.n_in)
                        f = (feat[(long long)row * ld_feat + c] - p.in_shift[c]) * p.in_scale[c];
                    v[q] = __float2bfloat16_rn(f);
                }
                *reinterpret_cast<uint4 *>(fin + (kc * kFusedRows + lrow) * 16) = *reinterpret_cast<const uint4 *>(v);
            }
            tc::fence_proxy_async();
            arrive_ready();
            for (int l = 0; l < p.layers; ++l) {
                if (!fused_wait(&accf[x], uint32_t(accw++ & 1), abort_flag)) {
                    ok = false;
                    break;
                }
                tc::tc_fence_after();
                const int N = fused_N(p, l);
                int boff = e * int(nbias);
                for (int q = 0; q < l; ++q) boff += fused_N(p, q);
                const float *bias = sbias + boff;
                if (l < p.layers - 1) {
                    // two 32-column chunks per TMEM wait (columns c0 and c0 + 64);
                    // N is a multiple of 16, so a group of 8 columns is either
                    // inside the layer or past it
                    for (int c0 = half * 32; c0 < N; c0 += 128) {
                        uint32_t raw[2][32];
                        tc::tmem_ld32_issue(trow + c0, raw[0]);
                        if (c0 + 64 < N)
                            tc::tmem_ld32_issue(trow + c0 + 64, raw[1]);
                        tc::tmem_ld_wait();
                        tc::tmem_reg_fence(raw[0]);
                        tc::tmem_reg_fence(raw[1]);
#pragma unroll
                        for (int u = 0; u < 2; ++u)
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                const int cbase = c0 + 64 * u + j * 8;
                                if (cbase < N) {
                                    const float4 b0 = *reinterpret_cast<const float4 *>(bias + cbase);
                                    const float4 b1 = *reinterpret_cast<const float4 *>(bias + cbase + 4);
                                    const float b8[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
                                    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                                    for (int q = 0; q < 8; ++q)
                                        h[q] = __float2bfloat16_rn(silu_fast(__uint_as_float(raw[u][j * 8 + q]) + b8[q]));
                                    *reinterpret_cast<uint4 *>(act + ((cbase / 8) * kFusedRows + lrow) * 16) =
                                        *reinterpret_cast<const uint4 *>(h);
                                }
                            }
                    }
                    tc::fence_proxy_async();
                    arrive_ready();
                } else {
                    for (int c0 = half * 32; c0 < N; c0 += 64) {
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
            }
        }
        if (!ok)
            atomicExch(err, 1);
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0)
        tc::tmem_dealloc(tmem, kFusedTmemCols);
}

// Weights of one layer, bf16 [N x K] row-major, into its K-slabs of
// kFusedSlabK columns, each in the core-matrix layout: element (n, k) of slab s
// at ((k' / 8) * N + n) * 8 + k' % 8, k' = k - kFusedSlabK s, slabs back to back.
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
