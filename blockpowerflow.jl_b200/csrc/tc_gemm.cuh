// BF16 tensor-core GEMM (tcgen05, TMEM accumulator) used by the learned warm-start network.
#pragma once

#include "bpf_internal.cuh"

namespace bpf {

// D (M x N, FP32, row stride ldd) = [D +] A (M x K) B (N x K)^T; A and B K-major BF16 (row
// strides lda, ldb, multiples of 8; 16-byte aligned bases); K a multiple of 64.  splits = K
// slices over the grid (0: chosen to fill the SMs); with splits > 1 the slices add into D
// atomically (D is cleared first unless accumulate).  *err_dev is raised if a bounded wait
// gave up.
bpf_status tc_gemm_bf16_tn(bpf_ctx *ctx, int M, int N, int K, const void *A, int lda, const void *B,
                           int ldb, float *D, int ldd, bool accumulate, int *err_dev, int splits = 0);

}  // namespace bpf
