// eu3d_mlp_api.cpp — the learned-chemistry model (include/eu3d.h, eu_mlp_*):
// an ensemble of MLPs (n_in -> width x hidden SiLU layers -> n_out) trained and
// evaluated with the BF16 tensor-core GEMM (fp32 accumulation, fp32 master
// weights, Adam). All tensors stay on the device; training batches are drawn
// on the device from caller-provided fp32 arrays.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "eu3d.h"
#include "eu3d_mlp_kernels.hpp"
#include "mlp_internal.hpp"

namespace {

struct Layer {
    int in = 0, out = 0, in_pad = 0, out_pad = 0;
    float *W = nullptr, *b = nullptr;   // fp32 master, padded [out_pad x in_pad], [out_pad]
    float *gW = nullptr, *gb = nullptr; // gradients
    float *mW = nullptr, *vW = nullptr, *mb = nullptr, *vb = nullptr;
    void *Wb = nullptr, *Wt = nullptr; // bf16 [out_pad x in_pad] and [in_pad x out_pad]
};

int pad16(int n) { return (n + 15) / 16 * 16; }

} // namespace

struct eu_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    int *d_err = nullptr;
    std::string err;
    bool ready = false;
    int n_in = 0, width = 0, hidden = 0, n_out = 0, members = 0, max_batch = 0;
    int in_pad = 0, out_pad = 0;
    std::vector<std::vector<Layer>> net;
    float *in_shift = nullptr, *in_scale = nullptr, *out_shift = nullptr, *out_scale = nullptr;
    void *X = nullptr;                  // bf16 [B x in_pad]
    std::vector<float *> Z;             // fp32 [B x width] per hidden layer
    std::vector<void *> H;              // bf16 [B x width]
    float *Y = nullptr;                 // fp32 [B x out_pad]
    void *dY = nullptr;                 // bf16 [B x out_pad]
    float *dZf[2] = {nullptr, nullptr}; // fp32 [B x width]
    void *dZb[2] = {nullptr, nullptr};  // bf16 [B x width]
    void *T1 = nullptr, *T2 = nullptr;  // bf16 transposes [width x B]
    float *loss = nullptr;
    int *rows = nullptr;
    long long adam_t = 0;
    std::vector<void *> allocs;
    // inference in one persistent kernel (eu3d_mlp_fused.cuh): the bf16 weights
    // repacked into K-slabs whenever they change
    bool fused = false;
    void *slabs = nullptr;
    long long slab_off[eu3d::kFusedMaxMembers][eu3d::kFusedMaxLayers] = {};
    int sms = 0;
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

#define MCK(m, call)                                                                               \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return mfail((m), e_ == cudaErrorMemoryAllocation ? EU_ERR_OUT_OF_MEMORY : EU_ERR_CUDA, "%s: %s", #call, \
                         cudaGetErrorString(e_));                                                  \
    } while (0)

template <typename T>
cudaError_t malloc_zero(eu_mlp *m, T **p, size_t bytes)
{
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess)
        return e;
    m->allocs.push_back(q);
    *p = static_cast<T *>(q);
    return cudaMemsetAsync(q, 0, bytes, m->stream);
}

void free_all(eu_mlp *m)
{
    for (void *p : m->allocs) cudaFree(p);
    m->allocs.clear();
    m->net.clear();
    m->Z.clear();
    m->H.clear();
    m->ready = false;
}

long long params_per_member(const eu_mlp *m)
{
    long long n = 0;
    for (const Layer &L : m->net[0]) n += (long long)L.out * L.in + L.out;
    return n;
}

// forward of member e over n packed rows in m->X (on stream s). Training keeps
// the pre-activations and uses the exact-form SiLU (epilogue mode 1);
// inference uses the fused kernel's form (mode 4), so the layer-wise and fused
// predictions agree bitwise.
eu_status forward(eu_mlp *m, int e, int n, cudaStream_t s = nullptr, bool keep_pre = true)
{
    if (!s)
        s = m->stream;
    auto &net = m->net[e];
    for (int l = 0; l < m->hidden; ++l) {
        const void *A = l == 0 ? m->X : m->H[l - 1];
        const int lda = l == 0 ? m->in_pad : m->width;
        const Layer &L = net[l];
        MCK(m, eu3d::gemm_bf16(A, lda, L.Wb, L.in_pad, n, L.out_pad, L.in_pad, L.b, keep_pre ? 1 : 4, nullptr,
                               m->H[l], keep_pre ? m->Z[l] : nullptr, m->width, nullptr, 1, m->d_err, s));
    }
    const Layer &L = net[m->hidden];
    MCK(m, eu3d::gemm_bf16(m->H[m->hidden - 1], m->width, L.Wb, L.in_pad, n, L.out_pad, L.in_pad, L.b, 0, m->Y, nullptr,
                           nullptr, m->out_pad, nullptr, 1, m->d_err, s));
    return EU_OK;
}

// gradients of member e for the n rows whose forward is in the scratch buffers
// and whose output gradient is in m->dY (n % 16 == 0)
eu_status backward(eu_mlp *m, int e, int n)
{
    auto &net = m->net[e];
    const int ksplit = n >= 2048 ? 16 : (n >= 512 ? 4 : 1);
    for (Layer &L : net) {
        MCK(m, cudaMemsetAsync(L.gW, 0, sizeof(float) * L.out_pad * L.in_pad, m->stream));
        MCK(m, cudaMemsetAsync(L.gb, 0, sizeof(float) * L.out_pad, m->stream));
    }
    // output layer
    {
        Layer &L = net[m->hidden];
        void *Hl = m->H[m->hidden - 1];
        MCK(m, eu3d::transpose_bf16(m->dY, n, L.out_pad, L.out_pad, m->T1, n, m->stream));
        MCK(m, eu3d::transpose_bf16(Hl, n, m->width, m->width, m->T2, n, m->stream));
        MCK(m, eu3d::gemm_bf16(m->T1, n, m->T2, n, L.out_pad, L.in_pad, n, nullptr, 3, L.gW, nullptr, nullptr, L.in_pad,
                               nullptr, ksplit, m->d_err, m->stream));
        MCK(m, eu3d::colsum_bf16(m->dY, n, L.out_pad, L.out_pad, L.gb, m->stream));
        MCK(m, eu3d::gemm_bf16(m->dY, L.out_pad, L.Wt, L.out_pad, n, m->width, L.out_pad, nullptr, 2, m->dZf[0],
                               m->dZb[0], nullptr, m->width, m->Z[m->hidden - 1], 1, m->d_err, m->stream));
    }
    int cur = 0;
    for (int l = m->hidden - 1; l >= 0; --l) {
        Layer &L = net[l];
        const void *A = l == 0 ? m->X : m->H[l - 1];
        const int in_pad = L.in_pad;
        MCK(m, eu3d::transpose_bf16(m->dZb[cur], n, m->width, m->width, m->T1, n, m->stream));
        MCK(m, eu3d::transpose_bf16(A, n, in_pad, in_pad, m->T2, n, m->stream));
        MCK(m, eu3d::gemm_bf16(m->T1, n, m->T2, n, m->width, in_pad, n, nullptr, 3, L.gW, nullptr, nullptr, in_pad,
                               nullptr, ksplit, m->d_err, m->stream));
        MCK(m, eu3d::colsum_f32(m->dZf[cur], n, m->width, m->width, L.gb, m->stream));
        if (l > 0) {
            MCK(m, eu3d::gemm_bf16(m->dZb[cur], m->width, L.Wt, L.out_pad, n, m->width, m->width, nullptr, 2,
                                   m->dZf[cur ^ 1], m->dZb[cur ^ 1], nullptr, m->width, m->Z[l - 1], 1, m->d_err,
                                   m->stream));
            cur ^= 1;
        }
    }
    return EU_OK;
}

eu_status refresh(eu_mlp *m, int e)
{
    for (size_t l = 0; l < m->net[e].size(); ++l) {
        Layer &L = m->net[e][l];
        MCK(m, eu3d::refresh_weights(L.W, L.out_pad, L.in_pad, L.out_pad, L.in_pad, L.Wb, L.Wt, m->stream));
        if (m->fused)
            MCK(m, eu3d::pack_slabs(L.Wb, L.out_pad, L.in_pad,
                                    static_cast<uint16_t *>(m->slabs) + m->slab_off[e][l], m->stream));
    }
    return EU_OK;
}

eu_status check_err(eu_mlp *m)
{
    int herr = 0;
    MCK(m, cudaMemcpyAsync(&herr, m->d_err, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    MCK(m, cudaStreamSynchronize(m->stream));
    if (herr) {
        cudaMemsetAsync(m->d_err, 0, sizeof(int), m->stream);
        return mfail(m, EU_ERR_TIMEOUT, "a tensor-core pipeline wait gave up");
    }
    return EU_OK;
}

} // namespace

namespace eu3d {
bool mlp_shape(const eu_mlp *m, int *n_in, int *n_out, int *members)
{
    if (!m || !m->ready)
        return false;
    *n_in = m->n_in;
    *n_out = m->n_out;
    *members = m->members;
    return true;
}

int mlp_layers(const eu_mlp *m) { return m && m->ready ? m->hidden + 1 : 0; }

int mlp_batches(const eu_mlp *m, long long n)
{
    return m && m->ready && m->max_batch > 0 ? int((n + m->max_batch - 1) / m->max_batch) : 0;
}

bool mlp_view(const eu_mlp *m, MlpView *v)
{
    if (!m || !m->ready || !v)
        return false;
    *v = MlpView{m->device, m->n_in,  m->width,    m->hidden,   m->n_out,    m->members,  m->in_pad,
                 m->out_pad, m->stream, m->in_shift, m->in_scale, m->out_shift, m->out_scale};
    return true;
}

bool mlp_layer_view(const eu_mlp *m, int member, int layer, MlpLayerView *v)
{
    if (!m || !m->ready || !v || member < 0 || member >= m->members || layer < 0 || layer > m->hidden)
        return false;
    const Layer &L = m->net[member][layer];
    *v = MlpLayerView{L.in_pad, L.out_pad, L.Wb, L.b};
    return true;
}

eu_status mlp_fail(eu_mlp *m, eu_status s, const char *msg) { return mfail(m, s, "%s", msg); }

bool mlp_fused_params(const eu_mlp *m, FusedMlpParams *p)
{
    if (!m || !m->ready || !m->fused || !p)
        return false;
    *p = FusedMlpParams{};
    p->members = m->members;
    p->layers = m->hidden + 1;
    p->n_in = m->n_in;
    p->in_pad = m->in_pad;
    p->width = m->width;
    p->out_pad = m->out_pad;
    p->n_out = m->n_out;
    p->slabs = m->slabs;
    for (int e = 0; e < m->members; ++e)
        for (int l = 0; l <= m->hidden; ++l) {
            p->off[e][l] = m->slab_off[e][l];
            p->bias[e][l] = m->net[e][l].b;
        }
    p->in_shift = m->in_shift;
    p->in_scale = m->in_scale;
    p->out_shift = m->out_shift;
    p->out_scale = m->out_scale;
    return true;
}

eu_status mlp_predict_queue(eu_mlp *m, const float *feat, const int *count_dev, int max_rows, float *out,
                            long long s_row, long long s_mem, cudaStream_t s)
{
    FusedMlpParams p;
    if (!mlp_fused_params(m, &p))
        return mfail(m, EU_ERR_UNSUPPORTED, "the model's shape has no fused inference kernel");
    const int tiles = (max_rows + 127) / 128;
    const int grid = eu3d::fused_grid(tiles, m->sms);
    MCK(m, eu3d::mlp_fused(p, feat, m->n_in, 0, count_dev, max_rows, out, s_row, s_mem, m->d_err, grid, s));
    return EU_OK;
}

bool mlp_has_fused(const eu_mlp *m) { return m && m->ready && m->fused; }

int *mlp_error_flag(eu_mlp *m) { return m ? m->d_err : nullptr; }

cudaStream_t mlp_stream(const eu_mlp *m) { return m ? m->stream : nullptr; }

eu_status mlp_predict_stream(eu_mlp *m, const float *X, long long n, float *out, cudaStream_t s)
{
    for (long long r0 = 0; r0 < n; r0 += m->max_batch) {
        const int nb = int(n - r0 < m->max_batch ? n - r0 : m->max_batch);
        MCK(m, eu3d::pack_features(X + r0 * m->n_in, nb, m->n_in, nullptr, m->in_shift, m->in_scale, m->X, m->in_pad,
                                   s));
        for (int e = 0; e < m->members; ++e) {
            eu_status st = forward(m, e, nb, s, false);
            if (st != EU_OK)
                return st;
            MCK(m, eu3d::unscale_outputs(m->Y, nb, m->out_pad, m->n_out, m->out_shift, m->out_scale,
                                         out + ((long long)e * n + r0) * m->n_out, s));
        }
    }
    return EU_OK;
}
} // namespace eu3d

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
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaDeviceGetAttribute(&m->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
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
    free_all(m);
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
    cudaError_t e = eu3d::gemm_bf16(A, lda, B, ldb, M, N, K, bias, act, Cf, Cb, Cpre, ldc, nullptr, 1, m->d_err, s);
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

eu_status eu_mlp_init(eu_mlp *m, int n_in, int width, int hidden_layers, int n_out, int members, int max_batch,
                      unsigned seed)
{
    if (!m)
        return EU_ERR_INVALID_ARGUMENT;
    if (n_in < 1 || n_in > 256 || width < 16 || width > 256 || (width % 16) || hidden_layers < 1 || hidden_layers > 8 ||
        n_out < 1 || n_out > 256 || members < 1 || members > 8 || max_batch < 16 || (max_batch % 16))
        return mfail(m, EU_ERR_INVALID_ARGUMENT, "mlp sizes out of range");
    cudaSetDevice(m->device);
    free_all(m);
    m->n_in = n_in;
    m->width = width;
    m->hidden = hidden_layers;
    m->n_out = n_out;
    m->members = members;
    m->max_batch = max_batch;
    m->in_pad = pad16(n_in);
    m->out_pad = pad16(n_out);
    m->adam_t = 0;
    std::mt19937_64 rng(seed);
    m->net.assign(members, std::vector<Layer>(hidden_layers + 1));
    for (int e = 0; e < members; ++e)
        for (int l = 0; l <= hidden_layers; ++l) {
            Layer &L = m->net[e][l];
            L.in = l == 0 ? n_in : width;
            L.out = l == hidden_layers ? n_out : width;
            L.in_pad = pad16(L.in);
            L.out_pad = pad16(L.out);
            const size_t nw = size_t(L.out_pad) * L.in_pad, nb = L.out_pad;
            MCK(m, malloc_zero(m, &L.W, nw * 4));
            MCK(m, malloc_zero(m, &L.b, nb * 4));
            MCK(m, malloc_zero(m, &L.gW, nw * 4));
            MCK(m, malloc_zero(m, &L.gb, nb * 4));
            MCK(m, malloc_zero(m, &L.mW, nw * 4));
            MCK(m, malloc_zero(m, &L.vW, nw * 4));
            MCK(m, malloc_zero(m, &L.mb, nb * 4));
            MCK(m, malloc_zero(m, &L.vb, nb * 4));
            MCK(m, malloc_zero(m, &L.Wb, nw * 2));
            MCK(m, malloc_zero(m, &L.Wt, nw * 2));
            // He-uniform initialisation (SiLU layers), zero biases
            std::vector<float> w(nw, 0.0f);
            const double bound = std::sqrt(6.0 / L.in) * (l == hidden_layers ? 0.5 : 1.0);
            std::uniform_real_distribution<double> u(-bound, bound);
            for (int o = 0; o < L.out; ++o)
                for (int i = 0; i < L.in; ++i) w[size_t(o) * L.in_pad + i] = float(u(rng));
            MCK(m, cudaMemcpyAsync(L.W, w.data(), nw * 4, cudaMemcpyHostToDevice, m->stream));
            MCK(m, cudaStreamSynchronize(m->stream));
        }
    const int B = max_batch;
    MCK(m, malloc_zero(m, &m->in_shift, size_t(m->in_pad) * 4));
    MCK(m, malloc_zero(m, &m->in_scale, size_t(m->in_pad) * 4));
    MCK(m, malloc_zero(m, &m->out_shift, size_t(m->out_pad) * 4));
    MCK(m, malloc_zero(m, &m->out_scale, size_t(m->out_pad) * 4));
    {
        std::vector<float> one(256, 1.0f);
        MCK(m, cudaMemcpyAsync(m->in_scale, one.data(), size_t(m->in_pad) * 4, cudaMemcpyHostToDevice, m->stream));
        MCK(m, cudaMemcpyAsync(m->out_scale, one.data(), size_t(m->out_pad) * 4, cudaMemcpyHostToDevice, m->stream));
    }
    MCK(m, malloc_zero(m, &m->X, size_t(B) * m->in_pad * 2));
    m->Z.assign(hidden_layers, nullptr);
    m->H.assign(hidden_layers, nullptr);
    for (int l = 0; l < hidden_layers; ++l) {
        MCK(m, malloc_zero(m, &m->Z[l], size_t(B) * width * 4));
        MCK(m, malloc_zero(m, &m->H[l], size_t(B) * width * 2));
    }
    MCK(m, malloc_zero(m, &m->Y, size_t(B) * m->out_pad * 4));
    MCK(m, malloc_zero(m, &m->dY, size_t(B) * m->out_pad * 2));
    for (int q = 0; q < 2; ++q) {
        MCK(m, malloc_zero(m, &m->dZf[q], size_t(B) * width * 4));
        MCK(m, malloc_zero(m, &m->dZb[q], size_t(B) * width * 2));
    }
    int tw = width > m->in_pad ? width : m->in_pad;
    tw = tw > m->out_pad ? tw : m->out_pad;
    MCK(m, malloc_zero(m, &m->T1, size_t(B) * tw * 2));
    MCK(m, malloc_zero(m, &m->T2, size_t(B) * tw * 2));
    MCK(m, malloc_zero(m, &m->loss, 4 * sizeof(float)));
    MCK(m, malloc_zero(m, &m->rows, size_t(B) * sizeof(int)));
    m->fused = eu3d::fused_supported(m->in_pad, width, m->out_pad, members, hidden_layers + 1);
    if (m->fused) {
        long long n = 0;
        for (int e = 0; e < members; ++e)
            for (int l = 0; l <= hidden_layers; ++l) {
                m->slab_off[e][l] = n;
                n += (long long)m->net[e][l].out_pad * m->net[e][l].in_pad;
            }
        MCK(m, malloc_zero(m, &m->slabs, size_t(n) * 2));
    }
    for (int e = 0; e < members; ++e) {
        eu_status s = refresh(m, e);
        if (s != EU_OK)
            return s;
    }
    MCK(m, cudaStreamSynchronize(m->stream));
    // the no-allocation entry point's fixed array is loaded on this device now,
    // before the caller can hand its free memory to a pool of its own
    MCK(m, eu3d::noalloc_setup(m->device));
    m->ready = true;
    return EU_OK;
}

eu_status eu_mlp_set_scaling(eu_mlp *m, const float *in_shift, const float *in_scale, const float *out_shift,
                             const float *out_scale)
{
    if (!m || !in_shift || !in_scale || !out_shift || !out_scale)
        return EU_ERR_INVALID_ARGUMENT;
    if (!m->ready)
        return mfail(m, EU_ERR_NOT_READY, "eu_mlp_init first");
    cudaSetDevice(m->device);
    MCK(m, cudaMemcpyAsync(m->in_shift, in_shift, size_t(m->n_in) * 4, cudaMemcpyHostToDevice, m->stream));
    MCK(m, cudaMemcpyAsync(m->in_scale, in_scale, size_t(m->n_in) * 4, cudaMemcpyHostToDevice, m->stream));
    MCK(m, cudaMemcpyAsync(m->out_shift, out_shift, size_t(m->n_out) * 4, cudaMemcpyHostToDevice, m->stream));
    MCK(m, cudaMemcpyAsync(m->out_scale, out_scale, size_t(m->n_out) * 4, cudaMemcpyHostToDevice, m->stream));
    MCK(m, cudaStreamSynchronize(m->stream));
    return EU_OK;
}

long long eu_mlp_num_params(const eu_mlp *m)
{
    if (!m || !m->ready)
        return 0;
    return params_per_member(m) * m->members;
}

eu_status eu_mlp_get_params(eu_mlp *m, float *out)
{
    if (!m || !out)
        return EU_ERR_INVALID_ARGUMENT;
    if (!m->ready)
        return mfail(m, EU_ERR_NOT_READY, "eu_mlp_init first");
    cudaSetDevice(m->device);
    long long off = 0;
    for (auto &net : m->net)
        for (Layer &L : net) {
            std::vector<float> w(size_t(L.out_pad) * L.in_pad), b(L.out_pad);
            MCK(m, cudaMemcpyAsync(w.data(), L.W, w.size() * 4, cudaMemcpyDeviceToHost, m->stream));
            MCK(m, cudaMemcpyAsync(b.data(), L.b, b.size() * 4, cudaMemcpyDeviceToHost, m->stream));
            MCK(m, cudaStreamSynchronize(m->stream));
            for (int o = 0; o < L.out; ++o)
                for (int i = 0; i < L.in; ++i) out[off++] = w[size_t(o) * L.in_pad + i];
            for (int o = 0; o < L.out; ++o) out[off++] = b[o];
        }
    return EU_OK;
}

eu_status eu_mlp_set_params(eu_mlp *m, const float *in)
{
    if (!m || !in)
        return EU_ERR_INVALID_ARGUMENT;
    if (!m->ready)
        return mfail(m, EU_ERR_NOT_READY, "eu_mlp_init first");
    cudaSetDevice(m->device);
    long long off = 0;
    for (int e = 0; e < m->members; ++e) {
        for (Layer &L : m->net[e]) {
            std::vector<float> w(size_t(L.out_pad) * L.in_pad, 0.0f), b(L.out_pad, 0.0f);
            for (int o = 0; o < L.out; ++o)
                for (int i = 0; i < L.in; ++i) w[size_t(o) * L.in_pad + i] = in[off++];
            for (int o = 0; o < L.out; ++o) b[o] = in[off++];
            MCK(m, cudaMemcpyAsync(L.W, w.data(), w.size() * 4, cudaMemcpyHostToDevice, m->stream));
            MCK(m, cudaMemcpyAsync(L.b, b.data(), b.size() * 4, cudaMemcpyHostToDevice, m->stream));
            MCK(m, cudaStreamSynchronize(m->stream));
        }
        eu_status s = refresh(m, e);
        if (s != EU_OK)
            return s;
    }
    MCK(m, cudaStreamSynchronize(m->stream));
    return EU_OK;
}

eu_status eu_mlp_loss_grad(eu_mlp *m, int member, const float *X, const float *T, int n, float *loss_out,
                           float *grads_out)
{
    if (!m || !X || !T || !loss_out)
        return EU_ERR_INVALID_ARGUMENT;
    if (!m->ready)
        return mfail(m, EU_ERR_NOT_READY, "eu_mlp_init first");
    if (member < 0 || member >= m->members || n < 16 || n > m->max_batch || (n % 16))
        return mfail(m, EU_ERR_INVALID_ARGUMENT, "member or batch size (multiple of 16 up to max_batch)");
    cudaSetDevice(m->device);
    MCK(m, eu3d::pack_features(X, n, m->n_in, nullptr, m->in_shift, m->in_scale, m->X, m->in_pad, m->stream));
    eu_status s = forward(m, member, n);
    if (s != EU_OK)
        return s;
    MCK(m, cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream));
    MCK(m, eu3d::mse_grad(m->Y, m->out_pad, T, n, m->n_out, nullptr, m->out_shift, m->out_scale, m->dY, m->loss,
                          m->stream));
    if ((s = backward(m, member, n)) != EU_OK)
        return s;
    if ((s = check_err(m)) != EU_OK)
        return s;
    float sq = 0;
    MCK(m, cudaMemcpy(&sq, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
    *loss_out = sq / float(n * m->n_out);
    if (grads_out) {
        long long off = 0;
        for (Layer &L : m->net[member]) {
            std::vector<float> w(size_t(L.out_pad) * L.in_pad), b(L.out_pad);
            MCK(m, cudaMemcpy(w.data(), L.gW, w.size() * 4, cudaMemcpyDeviceToHost));
            MCK(m, cudaMemcpy(b.data(), L.gb, b.size() * 4, cudaMemcpyDeviceToHost));
            for (int o = 0; o < L.out; ++o)
                for (int i = 0; i < L.in; ++i) grads_out[off++] = w[size_t(o) * L.in_pad + i];
            for (int o = 0; o < L.out; ++o) grads_out[off++] = b[o];
        }
    }
    return EU_OK;
}

eu_status eu_mlp_train(eu_mlp *m, const float *X, const float *T, long long n, int batch, int steps, float lr,
                       unsigned seed, float *mean_loss)
{
    if (!m || !X || !T)
        return EU_ERR_INVALID_ARGUMENT;
    if (!m->ready)
        return mfail(m, EU_ERR_NOT_READY, "eu_mlp_init first");
    if (batch < 16 || batch > m->max_batch || (batch % 16) || n < batch || steps < 0 || !(lr > 0))
        return mfail(m, EU_ERR_INVALID_ARGUMENT, "batch must be a multiple of 16, <= max_batch and <= n");
    cudaSetDevice(m->device);
    std::vector<double> total(m->members, 0.0);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int it = 0; it < steps; ++it) {
        ++m->adam_t;
        const float c1 = 1.0f / (1.0f - std::pow(b1, float(m->adam_t)));
        const float c2 = 1.0f / (1.0f - std::pow(b2, float(m->adam_t)));
        for (int e = 0; e < m->members; ++e) {
            const unsigned long long key =
                (unsigned long long)seed * 0x100000001B3ull + (unsigned long long)m->adam_t * 131ull + e;
            MCK(m, eu3d::random_rows(m->rows, batch, n, key, m->stream));
            MCK(m, eu3d::pack_features(X, batch, m->n_in, m->rows, m->in_shift, m->in_scale, m->X, m->in_pad,
                                       m->stream));
            eu_status s = forward(m, e, batch);
            if (s != EU_OK)
                return s;
            MCK(m, cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream));
            MCK(m, eu3d::mse_grad(m->Y, m->out_pad, T, batch, m->n_out, m->rows, m->out_shift, m->out_scale, m->dY,
                                  m->loss, m->stream));
            if ((s = backward(m, e, batch)) != EU_OK)
                return s;
            for (Layer &L : m->net[e]) {
                MCK(m, eu3d::adam(L.W, L.gW, L.mW, L.vW, (long long)L.out_pad * L.in_pad, lr, b1, b2, eps, c1, c2,
                                  m->stream));
                MCK(m, eu3d::adam(L.b, L.gb, L.mb, L.vb, L.out_pad, lr, b1, b2, eps, c1, c2, m->stream));
            }
            if ((s = refresh(m, e)) != EU_OK)
                return s;
            if (it + 1 == steps) {
                float sq = 0;
                MCK(m, cudaMemcpyAsync(&sq, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
                MCK(m, cudaStreamSynchronize(m->stream));
                total[e] = sq / double(batch * m->n_out);
            }
        }
    }
    eu_status s = check_err(m);
    if (s != EU_OK)
        return s;
    if (mean_loss)
        for (int e = 0; e < m->members; ++e) mean_loss[e] = float(total[e]);
    return EU_OK;
}

eu_status eu_mlp_predict_fused(eu_mlp *m, const float *X, long long n, float *out)
{
    if (!m || !X || !out || n < 0 || n > 0x7fffffffLL)
        return EU_ERR_INVALID_ARGUMENT;
    if (!m->ready)
        return mfail(m, EU_ERR_NOT_READY, "eu_mlp_init first");
    if (!m->fused)
        return mfail(m, EU_ERR_UNSUPPORTED, "the model's shape has no fused inference kernel");
    cudaSetDevice(m->device);
    eu3d::FusedMlpParams p;
    eu3d::mlp_fused_params(m, &p);
    const long long tiles = (n + 127) / 128;
    const int grid = eu3d::fused_grid(tiles, m->sms);
    MCK(m, eu3d::mlp_fused(p, X, m->n_in, int(n), nullptr, int(n), out, m->n_out, n * m->n_out, m->d_err, grid,
                           m->stream));
    return check_err(m);
}

eu_status eu_mlp_predict_fused_async(eu_mlp *m, const float *X, long long n, float *out)
{
    if (!m || !X || !out || n < 0 || n > 0x7fffffffLL)
        return EU_ERR_INVALID_ARGUMENT;
    if (!m->ready)
        return mfail(m, EU_ERR_NOT_READY, "eu_mlp_init first");
    if (!m->fused)
        return mfail(m, EU_ERR_UNSUPPORTED, "the model's shape has no fused inference kernel");
    cudaSetDevice(m->device);
    eu3d::FusedMlpParams p;
    eu3d::mlp_fused_params(m, &p);
    const long long tiles = (n + 127) / 128;
    const int grid = eu3d::fused_grid(tiles, m->sms);
    MCK(m, eu3d::mlp_fused(p, X, m->n_in, int(n), nullptr, int(n), out, m->n_out, n * m->n_out, m->d_err, grid,
                           m->stream));
    return EU_OK;
}

eu_status eu_mlp_sync(eu_mlp *m)
{
    if (!m)
        return EU_ERR_INVALID_ARGUMENT;
    if (!m->ready)
        return mfail(m, EU_ERR_NOT_READY, "eu_mlp_init first");
    cudaSetDevice(m->device);
    return check_err(m);
}

eu_status eu_mlp_stream(eu_mlp *m, void **stream)
{
    if (!m || !stream)
        return EU_ERR_INVALID_ARGUMENT;
    *stream = m->stream;
    return EU_OK;
}

eu_status eu_mlp_predict(eu_mlp *m, const float *X, long long n, float *out)
{
    if (!m || !X || !out || n < 0)
        return EU_ERR_INVALID_ARGUMENT;
    if (!m->ready)
        return mfail(m, EU_ERR_NOT_READY, "eu_mlp_init first");
    cudaSetDevice(m->device);
    for (long long r0 = 0; r0 < n; r0 += m->max_batch) {
        const int nb = int(n - r0 < m->max_batch ? n - r0 : m->max_batch);
        MCK(m, eu3d::pack_features(X + r0 * m->n_in, nb, m->n_in, nullptr, m->in_shift, m->in_scale, m->X, m->in_pad,
                                   m->stream));
        for (int e = 0; e < m->members; ++e) {
            eu_status s = forward(m, e, nb, nullptr, false);
            if (s != EU_OK)
                return s;
            MCK(m, eu3d::unscale_outputs(m->Y, nb, m->out_pad, m->n_out, m->out_shift, m->out_scale,
                                         out + ((long long)e * n + r0) * m->n_out, m->stream));
        }
    }
    return check_err(m);
}

} // extern "C"
