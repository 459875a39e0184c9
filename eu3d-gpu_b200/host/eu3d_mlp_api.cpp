// eu3d_mlp_api.cpp — C entry points of the learned-chemistry model
// (include/eu3d.h, eu_mlp_*): handle lifetime and the tensor-core GEMM.
#include <cstdarg>
#include <cstdio>
#include <new>
#include <string>

#include <cuda_runtime.h>

#include "eu3d.h"

namespace eu3d {
cudaError_t gemm_bf16(const void *A, int lda, const void *B, int ldb, int M, int N, int K, const float *bias, int act,
                      float *Cf, void *Cb, float *Cpre, int ldc, int *err, cudaStream_t s);
}

struct eu_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    int *d_err = nullptr;
    std::string err;
};

namespace {
eu_status mfail(eu_mlp *m, eu_status s, const char *fmt, ...)
{
    if (m) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        m->err = buf;
    }
    return s;
}
} // namespace

extern "C" {

eu_status eu_mlp_create(int device, eu_mlp **out)
{
    if (!out)
        return EU_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return EU_ERR_CUDA;
    eu_mlp *m = new (std::nothrow) eu_mlp;
    if (!m)
        return EU_ERR_OUT_OF_MEMORY;
    m->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&m->d_err, sizeof(int)) != cudaSuccess || cudaMemset(m->d_err, 0, sizeof(int)) != cudaSuccess) {
        eu_mlp_destroy(m);
        return EU_ERR_CUDA;
    }
    *out = m;
    return EU_OK;
}

eu_status eu_mlp_destroy(eu_mlp *m)
{
    if (!m)
        return EU_ERR_INVALID_ARGUMENT;
    cudaSetDevice(m->device);
    if (m->stream)
        cudaStreamSynchronize(m->stream);
    if (m->d_err)
        cudaFree(m->d_err);
    if (m->stream)
        cudaStreamDestroy(m->stream);
    delete m;
    return EU_OK;
}

const char *eu_mlp_last_error(const eu_mlp *m) { return m ? m->err.c_str() : "null handle"; }

eu_status eu_mlp_gemm(eu_mlp *m, const void *A, int lda, const void *B, int ldb, int M, int N, int K, const float *bias,
                      int act, float *Cf, void *Cb, float *Cpre, int ldc, void *stream)
{
    if (!m)
        return EU_ERR_INVALID_ARGUMENT;
    if (!A || !B || M < 0 || N <= 0 || K <= 0 || (K % 16) != 0 || (lda % 8) != 0 || (ldb % 8) != 0 || lda < K ||
        ldb < K || ldc < N || (!Cf && !Cb && !Cpre) || (act != 0 && act != 1))
        return mfail(m, EU_ERR_INVALID_ARGUMENT, "gemm: K %% 16, lda/ldb %% 8 and an output are required");
    if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15)
        return mfail(m, EU_ERR_INVALID_ARGUMENT, "gemm: operands must be 16-byte aligned");
    if (M == 0)
        return EU_OK;
    cudaSetDevice(m->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : m->stream;
    cudaError_t e = eu3d::gemm_bf16(A, lda, B, ldb, M, N, K, bias, act, Cf, Cb, Cpre, ldc, m->d_err, s);
    if (e != cudaSuccess)
        return mfail(m, EU_ERR_CUDA, "gemm launch: %s", cudaGetErrorString(e));
    int herr = 0;
    e = cudaMemcpyAsync(&herr, m->d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return mfail(m, EU_ERR_CUDA, "gemm: %s", cudaGetErrorString(e));
    if (herr) {
        cudaMemsetAsync(m->d_err, 0, sizeof(int), s);
        return mfail(m, EU_ERR_TIMEOUT, "gemm: a tensor-core pipeline wait gave up");
    }
    return EU_OK;
}

} // extern "C"
