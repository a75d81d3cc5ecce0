// rpl_mlp.h -- internal interface of the learned-source MLP: the tensor-core GEMM (rpl_gemm.cu) and the
// network's layout (rpl_mlp.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/rpl.h"

namespace rpl {

enum GemmEpilogue {
    EPI_F32 = 0,        // out_f32 = A B^T
    EPI_BIAS_GELU = 1,  // z = A B^T + bias (+ extra . wextra); out_f32 = z (optional); out_bf16 (and/or its
                        // transpose out_bf16_t) = GELU(z)
    EPI_BIAS = 2,       // out_f32 = A B^T + bias
    EPI_GELU_BWD = 3    // out_bf16 (and/or out_bf16_t) = (A B^T) * GELU'(pre)
};

struct GemmArgs {
    const __nv_bfloat16* A;  // M x K, row stride lda (elements)
    const __nv_bfloat16* B;  // N x K, row stride ldb
    int64_t lda, ldb;
    int M, N, K, epi;
    const float* bias;       // N
    const float* extra;      // M x 4 per-row extra inputs (EPI_BIAS_GELU, optional)
    const float* wextra;     // N x 4 weights of the extra inputs
    float* out_f32;          // M x N, row stride ldo
    int64_t ldo;
    __nv_bfloat16* out_bf16;    // M x N, row stride ldh
    int64_t ldh;
    __nv_bfloat16* out_bf16_t;  // N x M (transposed), row stride ldt
    int64_t ldt;
    const float* pre;        // M x N pre-activations (EPI_GELU_BWD), row stride ldp
    int64_t ldp;
    const float* clamp_lo;   // EPI_BIAS: per-column bounds the output is clamped to (both or neither)
    const float* clamp_hi;
    unsigned int* err;       // bit 4: a bounded wait gave up
    uint32_t wait_limit;     // polls before a barrier wait gives up; 0: the kernel's default
};

bool gemm_shape_ok(const GemmArgs& g, int bn);
cudaError_t launch_gemm(const GemmArgs& g, int bn, cudaStream_t s);

// Network forward over n rows (n % 128 == 0): X (row stride ldx) and E -> Y (row stride ldy), on stream s;
// GEMM wait timeouts set bit 4 of *err (the network's own error word when err is NULL).
// ylo, yhi (nbins each, optional): bounds the outputs are clamped to.
cudaError_t mlp_forward(rpl_mlp* m, const __nv_bfloat16* X, int64_t ldx, const float* E, int64_t n, float* Y,
                        int64_t ldy, bool train, cudaStream_t s, unsigned int* err, const float* ylo = nullptr,
                        const float* yhi = nullptr);

}  // namespace rpl
