// eu3d_noalloc.cu — eu_mlp_predict_noalloc: ensemble inference of the
// learned-chemistry model whose scratch (packed inputs, hidden activations,
// normalised outputs, the tensor-core error flag) lives in one fixed array of
// this library's device memory instead of buffers the library allocates.
//
// Why: some callers cannot call cudaMalloc while they run — a flow solver that
// hands all free device memory to its own pool after start-up, where an
// allocation from a library fails or fragments the pool, or a time loop that
// cannot afford the device-wide synchronisation cudaMalloc and cudaFree may
// cause. After eu_mlp_init and eu_mlp_set_params they can still evaluate the
// model on arrays they own, through this entry point.
#include <cstdio>
#include <mutex>

#include <cuda_runtime.h>

#include "eu3d.h"
#include "eu3d_mlp_kernels.hpp"
#include "mlp_internal.hpp"

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20; // EU_MLP_NOALLOC_SCRATCH_BYTES
constexpr size_t kAlign = 256;
static_assert(kScratchBytes == EU_MLP_NOALLOC_SCRATCH_BYTES, "header and library disagree on the scratch size");

// The array is device memory of this file's own CUDA module. CUDA loads
// modules lazily, so the array takes its 16 MiB on a device when its address
// is first looked up there: eu_mlp_init does that on the model's device
// (eu3d::noalloc_setup), before the caller can give its free memory away.
// From then on the device holds the array until the process exits.
// In host code the name is only a stand-in for the symbol: the device address
// comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_lock;
unsigned char *g_scratch_addr[kMaxDevices] = {};

size_t round_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

cudaError_t lookup_locked(int device)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
        return e;
    g_scratch_addr[device] = static_cast<unsigned char *>(p);
    return cudaSuccess;
}

// Device address of the scratch array on `device` (the current device), as
// the set-up recorded it.
cudaError_t scratch_on(int device, unsigned char **out)
{
    std::lock_guard<std::mutex> guard(g_lock);
    if (!g_scratch_addr[device]) {
        const cudaError_t e = lookup_locked(device);
        if (e != cudaSuccess)
            return e;
    }
    *out = g_scratch_addr[device];
    return cudaSuccess;
}

// Rows whose scratch fits the array: the error flag and three 256-byte
// round-ups take at most 4 * kAlign; the rest is per row.
long long max_rows(const eu3d::MlpView &v)
{
    const size_t per_row = size_t(v.in_pad) * 2 + 2 * size_t(v.width) * 2 + size_t(v.out_pad) * 4;
    return (long long)((kScratchBytes - 4 * kAlign) / per_row);
}

eu_status fail_cuda(eu_mlp *m, cudaError_t e, const char *what)
{
    char msg[256];
    std::snprintf(msg, sizeof msg, "%s: %s", what, cudaGetErrorString(e));
    return eu3d::mlp_fail(m, EU_ERR_CUDA, msg);
}

} // namespace

// Set-up, with `device` current: load the array there and record its address.
// It runs at every eu_mlp_init, so a model created again after a
// cudaDeviceReset (which unloads the module and drops every allocation,
// the model's own included) records the new address.
cudaError_t eu3d::noalloc_setup(int device)
{
    if (device < 0 || device >= kMaxDevices)
        return cudaSuccess; // eu_mlp_predict_noalloc rejects such a device
    std::lock_guard<std::mutex> guard(g_lock);
    return lookup_locked(device);
}

extern "C" eu_status eu_mlp_predict_noalloc(eu_mlp *m, const float *X, long long n, float *out)
{
    if (!m || !X || !out || n < 0)
        return EU_ERR_INVALID_ARGUMENT;
    eu3d::MlpView v;
    if (!eu3d::mlp_view(m, &v))
        return eu3d::mlp_fail(m, EU_ERR_NOT_READY, "eu_mlp_init first");
    const long long limit = max_rows(v);
    if (n > limit) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "%lld rows exceed the %lld rows that the fixed %zu-byte scratch holds for this model shape",
                      n, limit, kScratchBytes);
        return eu3d::mlp_fail(m, EU_ERR_INVALID_ARGUMENT, msg);
    }
    if (v.device < 0 || v.device >= kMaxDevices)
        return eu3d::mlp_fail(m, EU_ERR_UNSUPPORTED, "device ordinal beyond the scratch table");
    cudaError_t e = cudaSetDevice(v.device);
    if (e != cudaSuccess)
        return fail_cuda(m, e, "cudaSetDevice");
    unsigned char *base = nullptr;
    if ((e = scratch_on(v.device, &base)) != cudaSuccess)
        return fail_cuda(m, e, "cudaGetSymbolAddress of the scratch array");
    if (n == 0)
        return EU_OK;

    // scratch layout: [error flag | packed inputs | hidden ping | hidden pong | outputs]
    int *err = reinterpret_cast<int *>(base);
    unsigned char *p = base + kAlign;
    void *xs = p;
    p += round_up(size_t(n) * v.in_pad * 2);
    void *h[2] = {p, nullptr};
    p += round_up(size_t(n) * v.width * 2);
    h[1] = p;
    p += round_up(size_t(n) * v.width * 2);
    float *ys = reinterpret_cast<float *>(p);

    const cudaStream_t s = v.stream;
    // The array keeps the previous call's contents; only the flag must start
    // at zero (every other byte read below is written first in this call).
#define NCK(call)                                                                                  \
    do {                                                                                           \
        const cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                                     \
            return fail_cuda(m, e_, #call);                                                        \
    } while (0)
    NCK(cudaMemsetAsync(err, 0, sizeof(int), s));
    NCK(eu3d::pack_features(X, n, v.n_in, nullptr, v.in_shift, v.in_scale, xs, v.in_pad, s));
    const int rows = int(n);
    for (int member = 0; member < v.members; ++member) {
        eu3d::MlpLayerView L;
        for (int l = 0; l < v.hidden; ++l) {
            eu3d::mlp_layer_view(m, member, l, &L);
            const void *A = l == 0 ? xs : h[(l - 1) & 1];
            const int lda = l == 0 ? v.in_pad : v.width;
            NCK(eu3d::gemm_bf16(A, lda, L.Wb, L.in_pad, rows, L.out_pad, L.in_pad, L.b, 4, nullptr, h[l & 1],
                                nullptr, v.width, nullptr, 1, err, s));
        }
        eu3d::mlp_layer_view(m, member, v.hidden, &L);
        NCK(eu3d::gemm_bf16(h[(v.hidden - 1) & 1], v.width, L.Wb, L.in_pad, rows, L.out_pad, L.in_pad, L.b, 0, ys,
                            nullptr, nullptr, v.out_pad, nullptr, 1, err, s));
        NCK(eu3d::unscale_outputs(ys, n, v.out_pad, v.n_out, v.out_shift, v.out_scale,
                                  out + (long long)member * n * v.n_out, s));
    }
    int herr = 0;
    NCK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    NCK(cudaStreamSynchronize(s));
#undef NCK
    if (herr)
        return eu3d::mlp_fail(m, EU_ERR_TIMEOUT, "a tensor-core pipeline wait gave up");
    return EU_OK;
}
