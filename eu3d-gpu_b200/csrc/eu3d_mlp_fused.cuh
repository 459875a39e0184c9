// eu3d_mlp_fused.cuh — the learned-chemistry ensemble's whole forward pass in
// one persistent tcgen05 kernel (inference only; training uses the layer-wise
// GEMMs of eu3d_gemm.cuh).
//
// One CTA per SM walks the 128-row tiles of the input rows (tile =
// blockIdx.x, blockIdx.x + gridDim.x, ...) two at a time. The row count may
// be read from device memory when the kernel starts, so a launch needs no
// host-side count and can sit in a captured CUDA graph. A job is one (tile
// pair, member): its layers run on the tensor cores with the activations
// resident in shared memory, each tile with its own buffers and its own
// 256-column TMEM accumulator:
//   features (fp32, scaled and rounded to bf16)          -> fin  [128 x in_pad]
//   layer l: TMEM[128 x N] = A[128 x K] * W_l[N x K]^T    (A = fin or act)
//   hidden epilogue: + bias, SiLU, bf16                    -> act  [128 x width]
//   output epilogue: + bias, / out_scale + out_shift       -> global predictions
// The pair's features are loaded once and serve every member.
//
// What bounds this kernel is the weight stream, not the tensor core: every
// job reads all of its member's weights (272 KB for 12-256-256-256-10) from
// L2, and with one 128-row tile per weight slab the SMs together drew about
// 6 TB/s from L2 while the tensor core waited. Each slab now feeds the MMAs
// of both tiles, halving the weight bytes per row. Roles (warp-specialised):
//   warps 0-15  the epilogues: warp w reads TMEM lanes 32 (w % 4) (its 32
//               rows) of tile (w / 8) and the columns of half (w / 4) % 2 of
//               the accumulator's 32-column chunks;
//   warp 16     one thread issues the MMAs,
//   warp 17     one thread issues the weight copies.
// Before a layer the MMA thread waits on the "ready" mbarrier (the 16
// epilogue warps arrive when the layer's A operands are in shared memory and
// the accumulators have been read); after it commits the layer's MMAs to the
// "accumulator full" mbarrier, on which the epilogue warps wait. While the
// epilogue runs, the copy thread fills the ring with the next layer's slabs.
// Weights stream through a five-slot shared-memory ring in K-slabs of 32
// columns (the output layer, whose 16 x 256 weights fit one slot, as a single
// slab: 2 % faster than eight 1 KB ones), pre-packed in global memory in the
// operands' core-matrix layout so
// that each slab is one contiguous bulk copy (cp.async.bulk, completion counted
// on a "full" mbarrier); the MMAs that read a slot commit to its "empty"
// mbarrier. Every wait is bounded and watches a shared abort flag: on a
// timeout the CTA records an error, every role leaves its loop, the copy and
// MMA threads wait (bounded) for their copies and MMAs in flight, and the TMEM
// is freed before the CTA returns.
//
// The arithmetic is the layer-wise inference path's: the same K=16 MMA
// sequence into an fp32 accumulator, the same bias/SiLU/bf16 epilogue (SiLU in
// its inference form, silu_fast, with x / 2 formed in one fused multiply-add
// from the halved bias kept in shared memory: bitwise the same value), the
// same feature scaling and output unscaling (their vectors in shared memory).
#pragma once

#include <cuda_bf16.h>

#include "eu3d_gemm.cuh"
#include "eu3d_mlp_kernels.hpp"
#include "eu3d_tc.cuh"

namespace eu3d {

constexpr int kFusedEpiWarps = 16; // 8 per tile
constexpr int kFusedMmaWarp = kFusedEpiWarps, kFusedCopyWarp = kFusedMmaWarp + 1;
constexpr int kFusedThreads = (kFusedCopyWarp + 1) * 32;
constexpr int kFusedTmemCols = 256 * kFusedStreams;

__device__ __forceinline__ int fused_K(const FusedMlpParams &p, int l) { return l == 0 ? p.in_pad : p.width; }
__device__ __forceinline__ int fused_N(const FusedMlpParams &p, int l)
{
    return l == p.layers - 1 ? p.out_pad : p.width;
}
// K columns per slab of layer l: kFusedSlabK, or the whole K for an output
// layer whose weights fit one ring slot (one copy instead of K / kFusedSlabK
// small ones). The packed layout is the same for any slab width.
__device__ __forceinline__ int fused_slab_k(const FusedMlpParams &p, int l)
{
    return (l == p.layers - 1 && fused_N(p, l) * fused_K(p, l) <= p.width * kFusedSlabK) ? fused_K(p, l)
                                                                                         : kFusedSlabK;
}
__device__ __forceinline__ int fused_slabs(const FusedMlpParams &p, int l)
{
    return (fused_K(p, l) + fused_slab_k(p, l) - 1) / fused_slab_k(p, l);
}

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
    // [member][layer][N]; the hidden layers' halved (the epilogue forms x / 2)
    float *sbias = reinterpret_cast<float *>(fin0 + kFusedStreams * fin_bytes);
    float *s_in_shift = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(sbias) + bias_bytes);
    float *s_in_scale = s_in_shift + p.in_pad, *s_out_shift = s_in_scale + p.in_pad;
    float *s_out_scale = s_out_shift + p.out_pad;
    uint64_t *full = reinterpret_cast<uint64_t *>(reinterpret_cast<unsigned char *>(s_in_shift) +
                                                  ((2 * p.in_pad + 2 * p.out_pad) * 4 + 15) / 16 * 16);
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
    // jobs: (pair of this CTA's tiles, member), pairs outermost; steps: the
    // jobs' layers in order
    const int pairs = (mine + kFusedStreams - 1) / kFusedStreams;
    const int nsteps = pairs * p.members * p.layers;

    if (warp == 0) {
        tc::tmem_alloc(tslot, kFusedTmemCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int q = 0; q < kFusedStages; ++q) {
            tc::mbar_init(&full[q], 1);
            tc::mbar_init(&empty[q], 1);
        }
        tc::mbar_init(accf, 1);
        tc::mbar_init(ready, kFusedEpiWarps);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // every member's biases and the scaling into shared memory (read by the
    // epilogues); the pads beyond n_in / n_out are never read
    for (int e = 0; e < p.members; ++e)
        for (int l = 0, o = e * int(nbias); l < p.layers; o += fused_N(p, l), ++l)
            for (int c = tid; c < fused_N(p, l); c += kFusedThreads)
                sbias[o + c] = l < p.layers - 1 ? 0.5f * p.bias[e][l][c] : p.bias[e][l][c];
    for (int c = tid; c < p.n_in; c += kFusedThreads) {
        s_in_shift[c] = p.in_shift[c];
        s_in_scale[c] = p.in_scale[c];
    }
    for (int c = tid; c < p.n_out; c += kFusedThreads) {
        s_out_shift[c] = p.out_shift[c];
        s_out_scale[c] = p.out_scale[c];
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == kFusedMmaWarp) {
        // ------------------------------------------------------------ MMAs
        if (lane == 0) {
            long long g = 0; // slabs consumed
            bool ok = true;
            for (int step = 0; ok && step < nsteps; ++step) {
                const int l = step % p.layers;
                if (!fused_wait(ready, uint32_t(step & 1), abort_flag)) {
                    ok = false;
                    break;
                }
                tc::tc_fence_after();
                const int N = fused_N(p, l), K = fused_K(p, l), ns = fused_slabs(p, l), sk = fused_slab_k(p, l);
                const uint32_t idesc = tc::idesc_bf16_f32(kFusedRows, N);
                for (int s = 0; s < ns; ++s) {
                    const int slot = int(g % kFusedStages);
                    if (!fused_wait(&full[slot], uint32_t((g / kFusedStages) & 1), abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc::tc_fence_after();
                    const int kw = min(sk, K - s * sk);
                    const uint32_t b0 = tc::smem_u32(ring + slot * slot_bytes);
                    // the slab feeds both tiles' MMAs, the tiles alternating so
                    // that consecutive MMAs accumulate into different TMEM
                    // columns (each tile's own MMAs keep their K order)
                    for (int kk = 0; kk < kw / 16; ++kk) {
                        const int kg = s * (sk / 16) + kk;
                        const uint64_t bd = tc::smem_desc(b0 + kk * 2 * N * 16, N * 16, 128);
                        for (int x = 0; x < kFusedStreams; ++x) {
                            const uint32_t a0 = tc::smem_u32(l == 0 ? fin0 + x * fin_bytes : act0 + x * act_bytes);
                            const uint64_t ad = tc::smem_desc(a0 + kg * 2 * kFusedRows * 16, kFusedRows * 16, 128);
                            tc::mma_bf16(tmem + uint32_t(256 * x), ad, bd, idesc, (s > 0 || kk > 0) ? 1u : 0u);
                        }
                    }
                    tc::mma_commit(&empty[slot]);
                    ++g;
                }
                if (!ok)
                    break;
                tc::mma_commit(accf); // every MMA of the layer, in issue order
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
            bool ok = true;
            for (int step = 0; ok && step < nsteps; ++step) {
                const int l = step % p.layers, e = (step / p.layers) % p.members;
                const int N = fused_N(p, l), K = fused_K(p, l), sk = fused_slab_k(p, l);
                for (int ps = 0; ps < fused_slabs(p, l); ++ps) {
                    const int slot = int(gp % kFusedStages);
                    if (gp >= kFusedStages &&
                        !fused_wait(&empty[slot], uint32_t((gp / kFusedStages - 1) & 1), abort_flag)) {
                        ok = false;
                        break;
                    }
                    const int k0 = ps * sk, kw = min(sk, K - k0);
                    const uint32_t bytes = uint32_t(N) * kw * 2;
                    const __nv_bfloat16 *src = static_cast<const __nv_bfloat16 *>(p.slabs) + p.off[e][l] +
                                               (long long)ps * N * sk;
                    tc::mbar_arrive_expect_tx(&full[slot], bytes);
                    tc::bulk_g2s(ring + slot * slot_bytes, src, bytes, &full[slot]);
                    ++gp;
                }
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
        // ------------------------------------------------- epilogue warps
        const int x = warp / 8, quad = warp % 4, half = (warp / 4) % 2;
        const int lrow = quad * 32 + lane; // tile row = TMEM lane
        const uint32_t trow = tmem + uint32_t(256 * x) + (uint32_t(quad * 32) << 16);
        unsigned char *act = act0 + x * act_bytes, *fin = fin0 + x * fin_bytes;
        bool ok = true;
        auto arrive_ready = [&]() {
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(ready)) : "memory");
        };
        // the row of tile x of pair `pair` this thread serves (rows past the
        // count, and the missing second tile of an odd last pair, are zeros
        // in and nothing out)
        auto tile_row = [&](int pair) {
            const int k = pair * kFusedStreams + x;
            return k < mine ? (int(blockIdx.x) + k * int(gridDim.x)) * kFusedRows + lrow : count;
        };
        // features of the pair -> fin (core-matrix layout, 8 bf16 per 16-byte
        // chunk): the two column halves of the tile's rows
        auto features = [&](int pair) {
            const int row = tile_row(pair);
            const bool valid = row < count;
            for (int kc = half; kc < p.in_pad / 8; kc += 2) {
                __align__(16) __nv_bfloat16 v[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int c = kc * 8 + q;
                    float f = 0.0f;
                    if (valid && c < p.n_in)
                        f = (feat[(long long)row * ld_feat + c] - s_in_shift[c]) * s_in_scale[c];
                    v[q] = __float2bfloat16_rn(f);
                }
                *reinterpret_cast<uint4 *>(fin + (kc * kFusedRows + lrow) * 16) = *reinterpret_cast<const uint4 *>(v);
            }
            tc::fence_proxy_async();
            arrive_ready();
        };
        features(0);
        for (int step = 0; ok && step < nsteps; ++step) {
            const int l = step % p.layers, job = step / p.layers;
            const int e = job % p.members, pair = job / p.members;
            if (!fused_wait(accf, uint32_t(step & 1), abort_flag)) {
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
                                const float hb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
                                __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                                for (int q = 0; q < 8; ++q)
                                    h[q] = __float2bfloat16_rn(
                                        silu_fast_half(fmaf(0.5f, __uint_as_float(raw[u][j * 8 + q]), hb[q])));
                                *reinterpret_cast<uint4 *>(act + ((cbase / 8) * kFusedRows + lrow) * 16) =
                                    *reinterpret_cast<const uint4 *>(h);
                            }
                        }
                }
                tc::fence_proxy_async();
                arrive_ready();
            } else {
                const int row = tile_row(pair);
                for (int c0 = half * 32; c0 < N; c0 += 64) {
                    float v[32];
                    tc::tmem_ld32(trow + c0, v);
                    if (row < count) {
#pragma unroll
                        for (int q = 0; q < 32; ++q) {
                            const int o = c0 + q;
                            if (o < p.n_out)
                                pred[(long long)row * s_row + (long long)e * s_mem + o] =
                                    (v[q] + bias[o]) / s_out_scale[o] + s_out_shift[o];
                        }
                    }
                }
                // the accumulators are read: the next job may start (the next
                // member on the same features, or the next pair's features)
                if (e + 1 < p.members)
                    arrive_ready();
                else if (pair + 1 < pairs)
                    features(pair + 1);
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
