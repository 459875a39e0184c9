// mlp_internal.hpp — what the solver needs from an eu_mlp (eu3d_mlp_api.cpp).
#pragma once

#include <cuda_runtime.h>

#include "eu3d.h"

namespace eu3d {
// Model shape; false when the model is not initialised.
bool mlp_shape(const eu_mlp *m, int *n_in, int *n_out, int *members);
// Physical outputs of every member for n fp32 input rows, on `stream`:
// out[member][row][n_out]. Uses the model's scratch buffers.
eu_status mlp_predict_stream(eu_mlp *m, const float *X, long long n, float *out, cudaStream_t stream);
} // namespace eu3d
