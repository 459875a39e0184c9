// mlp_internal.hpp — what the solver needs from an eu_mlp (eu3d_mlp_api.cpp).
#pragma once

#include <cuda_runtime.h>

#include "eu3d.h"
#include "eu3d_mlp_kernels.hpp"

namespace eu3d {
// Model shape; false when the model is not initialised.
bool mlp_shape(const eu_mlp *m, int *n_in, int *n_out, int *members);
// Layers per member (hidden + output) and the row batches mlp_predict_stream
// splits n rows into: what it launches is, per batch, one packing kernel and
// per member one GEMM per layer and one unscaling kernel.
int mlp_layers(const eu_mlp *m);
int mlp_batches(const eu_mlp *m, long long n);
// Physical outputs of every member for n fp32 input rows, on `stream`:
// out[member][row][n_out]. Uses the model's scratch buffers.
eu_status mlp_predict_stream(eu_mlp *m, const float *X, long long n, float *out, cudaStream_t stream);

// Read-only views of an initialised model, for inference with scratch that
// the caller of these views provides (eu3d_noalloc.cu).
struct MlpView {
    int device, n_in, width, hidden, n_out, members, in_pad, out_pad;
    cudaStream_t stream;
    const float *in_shift, *in_scale, *out_shift, *out_scale;
};
struct MlpLayerView {
    int in_pad, out_pad;
    const void *Wb; // bf16 [out_pad x in_pad]
    const float *b; // [out_pad]
};
bool mlp_view(const eu_mlp *m, MlpView *v);
bool mlp_layer_view(const eu_mlp *m, int member, int layer, MlpLayerView *v);
// Loads the no-allocation entry point's fixed scratch array on `device` (the
// current device) and records its device address (eu3d_noalloc.cu); called by
// eu_mlp_init, so the array exists from the model's set-up on.
cudaError_t noalloc_setup(int device);
// Records msg as the model's last error and returns s.
eu_status mlp_fail(eu_mlp *m, eu_status s, const char *msg);
// The fused inference kernel: whether the model's shape has one, its launch
// parameters, and predictions for the rows of a device-side queue whose length
// the kernel reads from count_dev (at most max_rows): out[row * s_row + member *
// s_mem + o]. One launch of one CTA per SM, so it can be captured in a graph.
bool mlp_has_fused(const eu_mlp *m);
bool mlp_fused_params(const eu_mlp *m, FusedMlpParams *p);
eu_status mlp_predict_queue(eu_mlp *m, const float *feat, const int *count_dev, int max_rows, float *out,
                            long long s_row, long long s_mem, cudaStream_t s);
// Device flag the tensor-core kernels set when a bounded wait gives up.
int *mlp_error_flag(eu_mlp *m);
// The model's own stream (weight updates and repacking run there).
cudaStream_t mlp_stream(const eu_mlp *m);
} // namespace eu3d
