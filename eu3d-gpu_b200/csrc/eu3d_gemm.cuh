// eu3d_gemm.cuh — BF16 tensor-core GEMM for sm_100a (tcgen05, TMEM accumulator).
//
//   C[M x N] = act(A[M x K] * B[N x K]^T + bias[N])
//
// A and B are row-major with K contiguous (both operands "K-major"); C is
// written as fp32 and/or bf16, optionally with the pre-activation values kept
// for a backward pass. One CTA of 128 threads computes a 128 x BN tile:
// all threads stage K-slabs of 64 into shared memory with cp.async (two stages),
// one elected thread issues the tcgen05.mma instructions (M=128, N=BN, K=16)
// into a TMEM accumulator and commits them to the stage's mbarrier, and each
// warp reads its 32 accumulator rows back with tcgen05.ld for the epilogue.
// Every mbarrier wait is bounded; on a timeout the CTA records an error, frees
// its TMEM and returns.
#pragma once

#include <cuda_bf16.h>

#include "eu3d_tc.cuh"

namespace eu3d {

constexpr int kGemmBM = 128, kGemmBK = 64, kGemmThreads = 128;

// Epilogue modes: 0 none, 1 SiLU, 2 multiply by SiLU'(Z) (backward through an
// activation whose pre-activation Z is given), 3 accumulate into Cf with
// atomics (split-K partial sums; no bias), 4 SiLU in its inference form
// (silu_fast, the fused inference kernel's activation).
enum GemmAct { kActNone = 0, kActSilu = 1, kActSiluGrad = 2, kActAccumulate = 3, kActSiluFast = 4 };

// SiLU with the hardware's approximate division (reciprocal and multiply, about
// two units in the last place): the activations are rounded to bf16 next, eight
// bits of mantissa, so the division's last bits rarely survive. For x below
// about -87 the denominator overflows and the result is 0 (the exact value is
// below 1e-36 in magnitude). Training's forward pass uses this form.
__device__ __forceinline__ float silu(float x) { return __fdividef(x, 1.0f + __expf(-x)); }

// SiLU for inference: x sigmoid(x) = h + h tanh(h), h = x / 2, with the
// hardware's approximate tanh, one special-function instruction (relative
// error below 2^-10.9) instead of the two (exponential, reciprocal) of silu();
// those instructions bound the fused inference kernel's epilogues. The value
// is rounded to bf16 next, whose spacing is 2^-8 relative, so the two forms
// give the same activation except near bf16 rounding midpoints. For large |x|
// tanh saturates at +-1 and the result is x or 0.
__device__ __forceinline__ float tanh_approx(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// silu_fast(x) from h = x / 2. A caller that forms x = a + b can form h as
// fmaf(0.5f, a, b / 2) in one instruction: scaling by 2^-1 commutes with
// rounding, so h is bitwise 0.5f * (a + b) (outside the subnormal range).
__device__ __forceinline__ float silu_fast_half(float h) { return fmaf(h, tanh_approx(h), h); }
__device__ __forceinline__ float silu_fast(float x) { return silu_fast_half(0.5f * x); }
__device__ __forceinline__ float silu_grad(float z)
{
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

template <int BN>
constexpr size_t gemm_smem_bytes()
{
    return 2 * (size_t(kGemmBM) * kGemmBK + size_t(BN) * kGemmBK) * 2 + 64;
}

// Stage a rows x 64 bf16 slab (rows r0.., columns k0..) of a row-major matrix
// into the core-matrix layout: element (r, k) at ((k/8)*rows + r)*16 + (k%8)*2.
template <int ROWS>
__device__ __forceinline__ void stage_slab(unsigned char *dst, const __nv_bfloat16 *src, int ld, int r0, int nrows,
                                           int k0, int K)
{
    constexpr int kChunks = ROWS * (kGemmBK / 8);
#pragma unroll 4
    for (int c = threadIdx.x; c < kChunks; c += kGemmThreads) {
        const int r = c / (kGemmBK / 8), kc = c % (kGemmBK / 8);
        const int gr = r0 + r, gk = k0 + kc * 8;
        const bool ok = (gr < nrows) && (gk < K);
        const __nv_bfloat16 *p = ok ? src + (size_t)gr * ld + gk : src;
        tc::cp_async16(dst + (kc * ROWS + r) * 16, p, ok);
    }
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 1)
    k_gemm_bf16(const __nv_bfloat16 *__restrict__ A, int lda, const __nv_bfloat16 *__restrict__ B, int ldb, int M,
                int N, int K, const float *__restrict__ bias, int act, float *Cf, __nv_bfloat16 *Cb, float *Cpre,
                int ldc, const float *__restrict__ Z, int k_split, int *err)
{
    static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "BN");
    constexpr int BM = kGemmBM, BK = kGemmBK;
    constexpr uint32_t kStageA = BM * BK * 2, kStageB = BN * BK * 2;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *sa[2] = {smem, smem + kStageA + kStageB};
    unsigned char *sb[2] = {smem + kStageA, smem + 2 * kStageA + kStageB};
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * (kStageA + kStageB));
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2);

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    // split-K: CTA z handles K slabs [kt0, kt1)
    const int KT_all = (K + BK - 1) / BK;
    const int per = (KT_all + k_split - 1) / k_split;
    const int kt0 = blockIdx.z * per;
    const int KT = max(0, min(KT_all, kt0 + per) - kt0);
    const int kbase = kt0 * BK;

    if (warp == 0) {
        tc::tmem_alloc(tslot, BN);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        tc::mbar_init(&bars[0], 1);
        tc::mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tslot;
    bool ok = true;

    if (KT > 0) {
        stage_slab<BM>(sa[0], A, lda, m0, M, kbase, K);
        stage_slab<BN>(sb[0], B, ldb, n0, N, kbase, K);
    }
    tc::cp_async_commit();

    constexpr uint32_t idesc = tc::idesc_bf16_f32(BM, BN);
    for (int kt = 0; kt < KT; ++kt) {
        const int s = kt & 1;
        if (kt + 1 < KT) {
            const int s1 = s ^ 1;
            if (kt >= 1) {
                // The MMAs of slab kt-1 read stage s1: thread 0 waits for their
                // commit, the barrier orders everyone's overwrite after it.
                bool w = true;
                if (threadIdx.x == 0)
                    w = tc::mbar_wait(&bars[s1], ((kt - 1) >> 1) & 1);
                if (!__syncthreads_and(w)) {
                    ok = false;
                    break;
                }
            }
            stage_slab<BM>(sa[s1], A, lda, m0, M, kbase + (kt + 1) * BK, K);
            stage_slab<BN>(sb[s1], B, ldb, n0, N, kbase + (kt + 1) * BK, K);
            tc::cp_async_commit();
            tc::cp_async_wait<1>();
        } else {
            tc::cp_async_wait<0>();
        }
        tc::fence_proxy_async();
        __syncthreads();
        tc::tc_fence_after();
        if (threadIdx.x == 0) {
            const uint32_t a0 = tc::smem_u32(sa[s]), b0 = tc::smem_u32(sb[s]);
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
                const uint64_t ad = tc::smem_desc(a0 + kk * 2 * BM * 16, BM * 16, 128);
                const uint64_t bd = tc::smem_desc(b0 + kk * 2 * BN * 16, BN * 16, 128);
                tc::mma_bf16(tmem, ad, bd, idesc, (kt > 0 || kk > 0) ? 1u : 0u);
            }
            tc::mma_commit(&bars[s]);
        }
    }
    // the last commit tracks every earlier MMA of the issuing thread
    {
        bool w = true;
        if (threadIdx.x == 0 && ok && KT > 0)
            w = tc::mbar_wait(&bars[(KT - 1) & 1], ((KT - 1) >> 1) & 1);
        ok = __syncthreads_and(ok && w);
    }
    tc::tc_fence_after();

    if (ok && KT > 0) {
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            float v[32];
            tc::tmem_ld32(tmem + (uint32_t(warp * 32) << 16) + c0, v);
            if (row < M) {
#pragma unroll
                for (int q = 0; q < 32; ++q) {
                    const int n = n0 + c0 + q;
                    if (n < N) {
                        const size_t o = (size_t)row * ldc + n;
                        if (act == kActAccumulate) {
                            atomicAdd(&Cf[o], v[q]);
                            continue;
                        }
                        float x = v[q] + (bias ? bias[n] : 0.0f);
                        if (Cpre)
                            Cpre[o] = x;
                        if (act == kActSilu)
                            x = silu(x);
                        else if (act == kActSiluFast)
                            x = silu_fast(x);
                        else if (act == kActSiluGrad)
                            x *= silu_grad(Z[o]);
                        if (Cf)
                            Cf[o] = x;
                        if (Cb)
                            Cb[o] = __float2bfloat16_rn(x);
                    }
                }
            }
        }
    } else if (threadIdx.x == 0) {
        atomicExch(err, 1);
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0)
        tc::tmem_dealloc(tmem, BN);
}

} // namespace eu3d
