// The learned part of the solve path: a 3-layer MLP that maps a right-hand side to a warm
// start for block-GMRES and supplies a low-rank deflation basis; plain ILU(0) block-GMRES stays
// the fallback and the judge of its error (the solver always runs to the requested residual
// from whatever start it is given).
//
//   u = b / ||b||,   h1 = lrelu(W1 u + b1),   h2 = lrelu(W2 h1 + b2),   y = W3 h2 + b3,
//   x0 = s ||b|| y          (s: the data set's median ||x|| / ||b||, set at training time)
//
// Widths n -> H -> H -> n (H = 512 by default), weights in BF16 for the products with FP32
// masters, FP32 accumulation in TMEM (tc_gemm.cu), Adam on the masters.  Activations are
// stored sample-major ([p x H], feature contiguous) so that every product of the forward and
// backward passes is D = A B^T with both operands K-major; the weight gradients take the
// transposed BF16 copies that the elementwise kernels write beside the activations.
//
// Loss of a batch of p samples (x = the solver's solution of A x = b):
//   L = (1/p) sum_j ||y_j - t_j||^2 / ||t_j||^2,   t_j = x_j / (s ||b_j||).
// Dimensions: n is padded to np (multiple of 128, zero rows / columns), batches to P = 128.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "bpf_internal.cuh"
#include "dense.cuh"
#include "tc_gemm.cuh"

namespace bpf {

constexpr int kMlpBatch = 128;
constexpr float kLeak = 0.25f;

struct MlpParam {
    float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
    size_t len = 0;
};

}  // namespace bpf

struct bpf_mlp {
    bpf_ctx *ctx = nullptr;
    int n = 0, np = 0, H = 0;
    double scale = 1.0;
    long long step = 0;
    bpf::MlpParam W1, b1, W2, b2, W3, b3;
    __nv_bfloat16 *W1b = nullptr, *W2b = nullptr, *W2tb = nullptr, *W3b = nullptr, *W3tb = nullptr;
    // activations and gradients of one batch (P = 128 samples)
    __nv_bfloat16 *Ub = nullptr, *Utb = nullptr, *A1b = nullptr, *A1tb = nullptr, *A2b = nullptr,
                  *A2tb = nullptr, *dYb = nullptr, *dYtb = nullptr, *dZb = nullptr, *dZtb = nullptr;
    float *Z1 = nullptr, *Z2 = nullptr, *Y = nullptr, *dA = nullptr;
    float *bn = nullptr;      // per-sample ||b||
    float *tn = nullptr;      // per-sample ||t||^2
    double *loss = nullptr;   // device scalar
    int *err = nullptr;       // tensor-core pipeline error word
};

namespace bpf {

// ---------------------------------------------------------------------------------------
// elementwise kernels
// ---------------------------------------------------------------------------------------
__global__ void col_norms_kernel(int n, int p, const double *__restrict__ B, int ldb, float *__restrict__ out) {
    const int j = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = B[(size_t)j * ldb + i];
        s += v * v;
    }
    __shared__ double red[32];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) out[j] = (float)sqrt(t);
    }
}

// U[j][i] = b_ij / ||b_j|| (sample-major, BF16) and its transpose Ut[i][j]; zero padding for
// i >= n and j >= p.
__global__ void prep_input_kernel(int n, int np, int p, const double *__restrict__ B, int ldb,
                                  const float *__restrict__ bn, __nv_bfloat16 *__restrict__ U,
                                  __nv_bfloat16 *__restrict__ Ut) {
    const size_t total = (size_t)np * kMlpBatch;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / np), i = (int)(e % np);
        float v = 0.f;
        if (j < p && i < n) {
            const float nb = bn[j];
            v = nb > 0.f ? (float)(B[(size_t)j * ldb + i] / (double)nb) : 0.f;
        }
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        U[(size_t)j * np + i] = h;
        Ut[(size_t)i * kMlpBatch + j] = h;
    }
}

// Z (P x H) += bias; A = lrelu(Z) as BF16, sample-major and transposed; rows j >= p zero.
__global__ void bias_act_kernel(int H, int p, float *__restrict__ Z, const float *__restrict__ bias,
                                __nv_bfloat16 *__restrict__ A, __nv_bfloat16 *__restrict__ At) {
    const int total = kMlpBatch * H;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int j = e / H, c = e % H;
        float z = 0.f, a = 0.f;
        if (j < p) {
            z = Z[e] + bias[c];
            a = z > 0.f ? z : kLeak * z;
        }
        Z[e] = z;
        const __nv_bfloat16 h = __float2bfloat16_rn(a);
        A[e] = h;
        At[(size_t)c * kMlpBatch + j] = h;
    }
}

// y = Y + b3 (normalized output); forward only: X[i, j] = s ||b_j|| y_ji.
__global__ void output_kernel(int n, int np, int p, const float *__restrict__ Y, const float *__restrict__ b3,
                              const float *__restrict__ bn, double scale, double *__restrict__ X, int ldx) {
    const size_t total = (size_t)p * n;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / n), i = (int)(e % n);
        X[(size_t)j * ldx + i] = scale * (double)bn[j] * (double)(Y[(size_t)j * np + i] + b3[i]);
    }
}

// tn[j] = ||t_j||^2 with t_j = x_j / (s ||b_j||)
__global__ void target_norms_kernel(int n, const double *__restrict__ X, int ldx, const float *__restrict__ bn,
                                    double scale, float *__restrict__ tn) {
    const int j = blockIdx.x;
    const double f = bn[j] > 0.f ? 1.0 / (scale * (double)bn[j]) : 0.0;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double t = X[(size_t)j * ldx + i] * f;
        s += t * t;
    }
    __shared__ double red[32];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) tn[j] = (float)t;
    }
}

// dY = 2 w_j (y - t), w_j = 1 / (p ||t_j||^2); BF16 sample-major and transposed; the loss
// sum_j w_j ||y_j - t_j||^2 into *loss (atomic; cleared by the caller); rows j >= p zero.
// Y and dYf may be the same buffer (each element is read before it is overwritten).
__global__ void loss_grad_kernel(int n, int np, int p, const float *Y, const float *__restrict__ b3,
                                 const double *__restrict__ X, int ldx, const float *__restrict__ bn,
                                 const float *__restrict__ tn, double scale, __nv_bfloat16 *__restrict__ dY,
                                 __nv_bfloat16 *__restrict__ dYt, float *dYf, double *loss) {
    const size_t total = (size_t)np * kMlpBatch;
    double ls = 0.0;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / np), i = (int)(e % np);
        float g = 0.f;
        if (j < p && i < n) {
            const double w = tn[j] > 0.f ? 1.0 / ((double)p * (double)tn[j]) : 0.0;
            const double t = bn[j] > 0.f ? X[(size_t)j * ldx + i] / (scale * (double)bn[j]) : 0.0;
            const double d = (double)(Y[e] + b3[i]) - t;
            ls += w * d * d;
            g = (float)(2.0 * w * d);
        }
        dYf[e] = g;
        const __nv_bfloat16 h = __float2bfloat16_rn(g);
        dY[e] = h;
        dYt[(size_t)i * kMlpBatch + j] = h;
    }
    ls = warp_sum(ls);
    if ((threadIdx.x & 31) == 0 && ls != 0.0) atomicAdd(loss, ls);
}

// db[c] = sum_j G[j][c] over the batch (G: P x width, FP32)
__global__ void col_sum_kernel(int width, const float *__restrict__ G, float *__restrict__ db) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < width; c += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int j = 0; j < kMlpBatch; j++) s += G[(size_t)j * width + c];
        db[c] = s;
    }
}

// dZ = dA * lrelu'(Z) (FP32 in dA, in place) and BF16 sample-major / transposed copies
__global__ void act_back_kernel(int H, const float *__restrict__ Z, float *__restrict__ dA,
                                __nv_bfloat16 *__restrict__ dZ, __nv_bfloat16 *__restrict__ dZt) {
    const int total = kMlpBatch * H;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int j = e / H, c = e % H;
        const float g = dA[e] * (Z[e] > 0.f ? 1.f : kLeak);
        dA[e] = g;
        const __nv_bfloat16 h = __float2bfloat16_rn(g);
        dZ[e] = h;
        dZt[(size_t)c * kMlpBatch + j] = h;
    }
}

// Adam on an FP32 master with bias correction.
__global__ void adam_kernel(size_t len, float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                            const float *__restrict__ g, float lr, float b1, float b2, float c1, float c2,
                            float eps) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
        const float gg = g[e];
        const float mm = b1 * m[e] + (1.f - b1) * gg;
        const float vv = b2 * v[e] + (1.f - b2) * gg * gg;
        m[e] = mm;
        v[e] = vv;
        w[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    }
}

// BF16 copy of a rows x cols FP32 matrix, and optionally its transpose (cols x rows).
__global__ void to_bf16_kernel(int rows, int cols, const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb,
                               __nv_bfloat16 *__restrict__ wtb) {
    const size_t total = (size_t)rows * cols;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(e / cols), c = (int)(e % cols);
        const __nv_bfloat16 h = __float2bfloat16_rn(w[e]);
        wb[e] = h;
        if (wtb) wtb[(size_t)c * rows + r] = h;
    }
}

static int grid_for(bpf_ctx *ctx, size_t work) {
    return (int)std::max<size_t>(1, std::min<size_t>((work + 255) / 256, (size_t)ctx->num_sms * 16));
}

static bpf_status mlp_refresh_bf16(bpf_mlp *m) {
    bpf_ctx *ctx = m->ctx;
    to_bf16_kernel<<<grid_for(ctx, (size_t)m->H * m->np), 256, 0, ctx->stream>>>(m->H, m->np, m->W1.w, m->W1b, nullptr);
    BPF_LAUNCHED(ctx);
    to_bf16_kernel<<<grid_for(ctx, (size_t)m->H * m->H), 256, 0, ctx->stream>>>(m->H, m->H, m->W2.w, m->W2b, m->W2tb);
    BPF_LAUNCHED(ctx);
    to_bf16_kernel<<<grid_for(ctx, (size_t)m->np * m->H), 256, 0, ctx->stream>>>(m->np, m->H, m->W3.w, m->W3b, m->W3tb);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

// Forward pass of a batch of p <= 128 samples into m->Y (normalized outputs, without b3).
static bpf_status mlp_forward_core(bpf_mlp *m, int p, const double *B, int ldb) {
    bpf_ctx *ctx = m->ctx;
    const int H = m->H, np = m->np, P = kMlpBatch;
    col_norms_kernel<<<p, 256, 0, ctx->stream>>>(m->n, p, B, ldb, m->bn);
    BPF_LAUNCHED(ctx);
    prep_input_kernel<<<grid_for(ctx, (size_t)np * P), 256, 0, ctx->stream>>>(m->n, np, p, B, ldb, m->bn, m->Ub, m->Utb);
    BPF_LAUNCHED(ctx);
    BPF_TRY(tc_gemm_bf16_tn(ctx, P, H, np, m->Ub, np, m->W1b, np, m->Z1, H, false, m->err));
    bias_act_kernel<<<grid_for(ctx, (size_t)P * H), 256, 0, ctx->stream>>>(H, p, m->Z1, m->b1.w, m->A1b, m->A1tb);
    BPF_LAUNCHED(ctx);
    BPF_TRY(tc_gemm_bf16_tn(ctx, P, H, H, m->A1b, H, m->W2b, H, m->Z2, H, false, m->err));
    bias_act_kernel<<<grid_for(ctx, (size_t)P * H), 256, 0, ctx->stream>>>(H, p, m->Z2, m->b2.w, m->A2b, m->A2tb);
    BPF_LAUNCHED(ctx);
    BPF_TRY(tc_gemm_bf16_tn(ctx, P, np, H, m->A2b, H, m->W3b, H, m->Y, np, false, m->err));
    return BPF_SUCCESS;
}

// Loss and gradients of a batch (into the params' g buffers); *loss_dev = L.
static bpf_status mlp_backward_core(bpf_mlp *m, int p, const double *X, int ldx) {
    bpf_ctx *ctx = m->ctx;
    const int H = m->H, np = m->np, P = kMlpBatch;
    target_norms_kernel<<<p, 256, 0, ctx->stream>>>(m->n, X, ldx, m->bn, m->scale, m->tn);
    BPF_LAUNCHED(ctx);
    BPF_CUDA(ctx, cudaMemsetAsync(m->loss, 0, sizeof(double), ctx->stream));
    // dY (FP32 kept in Y's storage after use: the loss kernel reads Y[e] before writing dYf[e])
    loss_grad_kernel<<<grid_for(ctx, (size_t)np * P), 256, 0, ctx->stream>>>(
        m->n, np, p, m->Y, m->b3.w, X, ldx, m->bn, m->tn, m->scale, m->dYb, m->dYtb, m->Y, m->loss);
    BPF_LAUNCHED(ctx);
    col_sum_kernel<<<grid_for(ctx, np), 256, 0, ctx->stream>>>(np, m->Y, m->b3.g);
    BPF_LAUNCHED(ctx);
    // dW3 [np x H] = dY^T A2
    BPF_TRY(tc_gemm_bf16_tn(ctx, np, H, P, m->dYtb, P, m->A2tb, P, m->W3.g, H, false, m->err));
    // dA2 [P x H] = dY W3
    BPF_TRY(tc_gemm_bf16_tn(ctx, P, H, np, m->dYb, np, m->W3tb, np, m->dA, H, false, m->err));
    act_back_kernel<<<grid_for(ctx, (size_t)P * H), 256, 0, ctx->stream>>>(H, m->Z2, m->dA, m->dZb, m->dZtb);
    BPF_LAUNCHED(ctx);
    col_sum_kernel<<<grid_for(ctx, H), 256, 0, ctx->stream>>>(H, m->dA, m->b2.g);
    BPF_LAUNCHED(ctx);
    // dW2 [H x H] = dZ2^T A1
    BPF_TRY(tc_gemm_bf16_tn(ctx, H, H, P, m->dZtb, P, m->A1tb, P, m->W2.g, H, false, m->err));
    // dA1 [P x H] = dZ2 W2
    BPF_TRY(tc_gemm_bf16_tn(ctx, P, H, H, m->dZb, H, m->W2tb, H, m->dA, H, false, m->err));
    act_back_kernel<<<grid_for(ctx, (size_t)P * H), 256, 0, ctx->stream>>>(H, m->Z1, m->dA, m->dZb, m->dZtb);
    BPF_LAUNCHED(ctx);
    col_sum_kernel<<<grid_for(ctx, H), 256, 0, ctx->stream>>>(H, m->dA, m->b1.g);
    BPF_LAUNCHED(ctx);
    // dW1 [H x np] = dZ1^T U
    BPF_TRY(tc_gemm_bf16_tn(ctx, H, np, P, m->dZtb, P, m->Utb, P, m->W1.g, np, false, m->err));
    return BPF_SUCCESS;
}

static bpf_status mlp_check_err(bpf_mlp *m) {
    int h = 0;
    BPF_CUDA(m->ctx, cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->ctx->stream));
    BPF_CUDA(m->ctx, cudaStreamSynchronize(m->ctx->stream));
    if (h) return set_error(m->ctx, BPF_ERR_TIMEOUT, "mlp: a tensor-core pipeline wait timed out");
    return BPF_SUCCESS;
}

}  // namespace bpf

using namespace bpf;

extern "C" {

bpf_status bpf_mlp_destroy(bpf_mlp *m) {
    if (!m) return BPF_SUCCESS;
    if (m->ctx) cudaStreamSynchronize(m->ctx->stream);
    for (MlpParam *q : {&m->W1, &m->b1, &m->W2, &m->b2, &m->W3, &m->b3}) {
        cudaFree(q->w);
        cudaFree(q->m);
        cudaFree(q->v);
        cudaFree(q->g);
    }
    for (void *q : {(void *)m->W1b, (void *)m->W2b, (void *)m->W2tb, (void *)m->W3b, (void *)m->W3tb,
                    (void *)m->Ub, (void *)m->Utb, (void *)m->A1b, (void *)m->A1tb, (void *)m->A2b,
                    (void *)m->A2tb, (void *)m->dYb, (void *)m->dYtb, (void *)m->dZb, (void *)m->dZtb,
                    (void *)m->Z1, (void *)m->Z2, (void *)m->Y, (void *)m->dA, (void *)m->bn,
                    (void *)m->tn, (void *)m->loss, (void *)m->err})
        cudaFree(q);
    delete m;
    return BPF_SUCCESS;
}

bpf_status bpf_mlp_create(bpf_ctx *ctx, int n, int hidden, unsigned long long seed, bpf_mlp **out) {
    if (!ctx || !out) return BPF_ERR_INVALID_VALUE;
    *out = nullptr;
    if (n < 1 || hidden < 64 || hidden % 128)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "mlp: n >= 1 and hidden a multiple of 128 (got %d, %d)", n,
                         hidden);
    bpf_mlp *m = new bpf_mlp();
    m->ctx = ctx;
    m->n = n;
    m->np = ceil_div(n, 128) * 128;
    m->H = hidden;
    const int np = m->np, H = hidden, P = kMlpBatch;
    cudaError_t e = cudaSuccess;
    auto fa = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) e = cudaMemsetAsync(*p, 0, bytes, ctx->stream);
    };
    auto param = [&](MlpParam &q, size_t len) {
        q.len = len;
        fa((void **)&q.w, 4 * len);
        fa((void **)&q.m, 4 * len);
        fa((void **)&q.v, 4 * len);
        fa((void **)&q.g, 4 * len);
    };
    param(m->W1, (size_t)H * np);
    param(m->b1, H);
    param(m->W2, (size_t)H * H);
    param(m->b2, H);
    param(m->W3, (size_t)np * H);
    param(m->b3, np);
    fa((void **)&m->W1b, 2 * (size_t)H * np);
    fa((void **)&m->W2b, 2 * (size_t)H * H);
    fa((void **)&m->W2tb, 2 * (size_t)H * H);
    fa((void **)&m->W3b, 2 * (size_t)np * H);
    fa((void **)&m->W3tb, 2 * (size_t)np * H);
    fa((void **)&m->Ub, 2 * (size_t)P * np);
    fa((void **)&m->Utb, 2 * (size_t)P * np);
    fa((void **)&m->A1b, 2 * (size_t)P * H);
    fa((void **)&m->A1tb, 2 * (size_t)P * H);
    fa((void **)&m->A2b, 2 * (size_t)P * H);
    fa((void **)&m->A2tb, 2 * (size_t)P * H);
    fa((void **)&m->dYb, 2 * (size_t)P * np);
    fa((void **)&m->dYtb, 2 * (size_t)P * np);
    fa((void **)&m->dZb, 2 * (size_t)P * H);
    fa((void **)&m->dZtb, 2 * (size_t)P * H);
    fa((void **)&m->Z1, 4 * (size_t)P * H);
    fa((void **)&m->Z2, 4 * (size_t)P * H);
    fa((void **)&m->Y, 4 * (size_t)P * np);
    fa((void **)&m->dA, 4 * (size_t)P * H);
    fa((void **)&m->bn, 4 * P);
    fa((void **)&m->tn, 4 * P);
    fa((void **)&m->loss, sizeof(double));
    fa((void **)&m->err, sizeof(int) * 4);
    if (e != cudaSuccess) {
        cudaGetLastError();
        bpf_mlp_destroy(m);
        return e == cudaErrorMemoryAllocation ? set_error(ctx, BPF_ERR_ALLOC, "mlp: allocation failed")
                                              : cuda_error(ctx, e, "mlp create", __FILE__, __LINE__);
    }
    // LeCun-normal initialization (std 1/sqrt(fan_in)) on the host, seeded; biases zero
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    auto init = [&](MlpParam &q, int rows, int cols, int valid_rows, int valid_cols, float sd) {
        std::vector<float> h((size_t)rows * cols, 0.f);
        for (int r = 0; r < valid_rows; r++)
            for (int c = 0; c < valid_cols; c++) h[(size_t)r * cols + c] = sd * nd(rng);
        if (e == cudaSuccess) e = cudaMemcpy(q.w, h.data(), 4 * h.size(), cudaMemcpyHostToDevice);
    };
    init(m->W1, H, np, H, n, 1.f / std::sqrt((float)n));
    init(m->W2, H, H, H, H, 1.f / std::sqrt((float)H));
    init(m->W3, np, H, n, H, 1.f / std::sqrt((float)H));
    if (e != cudaSuccess) {
        bpf_mlp_destroy(m);
        return cuda_error(ctx, e, "mlp init", __FILE__, __LINE__);
    }
    bpf_status s = mlp_refresh_bf16(m);
    if (s != BPF_SUCCESS) {
        bpf_mlp_destroy(m);
        return s;
    }
    *out = m;
    return BPF_SUCCESS;
}

bpf_status bpf_mlp_set_scale(bpf_mlp *m, double scale) {
    if (!m || !(scale > 0.0)) return BPF_ERR_INVALID_VALUE;
    m->scale = scale;
    return BPF_SUCCESS;
}

bpf_status bpf_mlp_forward(bpf_mlp *m, int p, const double *B, int ldb, double *X, int ldx) {
    if (!m) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = m->ctx;
    if (p < 0 || (p > 0 && (!B || !X))) return set_error(ctx, BPF_ERR_INVALID_VALUE, "mlp_forward: invalid argument");
    if (ldb < m->n || ldx < m->n) return set_error(ctx, BPF_ERR_DIMENSION, "mlp_forward: leading dimension < n");
    BPF_CUDA(ctx, cudaMemsetAsync(m->err, 0, sizeof(int), ctx->stream));
    for (int j0 = 0; j0 < p; j0 += kMlpBatch) {
        const int pb = std::min(kMlpBatch, p - j0);
        BPF_TRY(mlp_forward_core(m, pb, B + (size_t)j0 * ldb, ldb));
        output_kernel<<<grid_for(ctx, (size_t)pb * m->n), 256, 0, ctx->stream>>>(
            m->n, m->np, pb, m->Y, m->b3.w, m->bn, m->scale, X + (size_t)j0 * ldx, ldx);
        BPF_LAUNCHED(ctx);
    }
    return mlp_check_err(m);
}

bpf_status bpf_mlp_gradients(bpf_mlp *m, int p, const double *B, int ldb, const double *X, int ldx,
                             double *loss) {
    if (!m) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = m->ctx;
    if (p < 1 || p > kMlpBatch || !B || !X)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "mlp_gradients: 1 <= p <= %d", kMlpBatch);
    if (ldb < m->n || ldx < m->n) return set_error(ctx, BPF_ERR_DIMENSION, "mlp_gradients: leading dimension < n");
    BPF_CUDA(ctx, cudaMemsetAsync(m->err, 0, sizeof(int), ctx->stream));
    BPF_TRY(mlp_forward_core(m, p, B, ldb));
    BPF_TRY(mlp_backward_core(m, p, X, ldx));
    if (loss) BPF_CUDA(ctx, cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    return mlp_check_err(m);
}

bpf_status bpf_mlp_train_step(bpf_mlp *m, int p, const double *B, int ldb, const double *X, int ldx,
                              double lr, double *loss) {
    BPF_TRY(bpf_mlp_gradients(m, p, B, ldb, X, ldx, loss));
    bpf_ctx *ctx = m->ctx;
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    for (MlpParam *q : {&m->W1, &m->b1, &m->W2, &m->b2, &m->W3, &m->b3}) {
        adam_kernel<<<grid_for(ctx, q->len), 256, 0, ctx->stream>>>(q->len, q->w, q->m, q->v, q->g, (float)lr,
                                                                     b1, b2, c1, c2, 1e-8f);
        BPF_LAUNCHED(ctx);
    }
    return mlp_refresh_bf16(m);
}

bpf_status bpf_mlp_params(bpf_mlp *m, int which, float **w, float **g, long long *rows, long long *cols) {
    if (!m || which < 0 || which > 5) return BPF_ERR_INVALID_VALUE;
    MlpParam *q[6] = {&m->W1, &m->b1, &m->W2, &m->b2, &m->W3, &m->b3};
    const long long r[6] = {m->H, 1, m->H, 1, m->np, 1};
    const long long c[6] = {m->np, m->H, m->H, m->H, m->H, m->np};
    if (w) *w = q[which]->w;
    if (g) *g = q[which]->g;
    if (rows) *rows = r[which];
    if (cols) *cols = c[which];
    return BPF_SUCCESS;
}

bpf_status bpf_mlp_param_copy(bpf_mlp *m, int which, int grad, float *buf, int to_network) {
    if (!m || which < 0 || which > 5 || !buf) return BPF_ERR_INVALID_VALUE;
    MlpParam *q[6] = {&m->W1, &m->b1, &m->W2, &m->b2, &m->W3, &m->b3};
    float *dev = grad ? q[which]->g : q[which]->w;
    const size_t bytes = sizeof(float) * q[which]->len;
    BPF_CUDA(m->ctx, cudaMemcpyAsync(to_network ? dev : buf, to_network ? buf : dev, bytes,
                                     cudaMemcpyDeviceToDevice, m->ctx->stream));
    if (to_network && !grad) return mlp_refresh_bf16(m);
    return BPF_SUCCESS;
}

bpf_status bpf_mlp_refresh(bpf_mlp *m) {
    if (!m) return BPF_ERR_INVALID_VALUE;
    return mlp_refresh_bf16(m);
}

bpf_status bpf_mlp_basis(bpf_mlp *m, int r, unsigned long long seed, double *Z, int ldz) {
    if (!m) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = m->ctx;
    if (r < 1 || r > 32 || 4 * r > m->n || !Z)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "mlp_basis: 1 <= rank <= 32 and 4 rank <= n");
    if (ldz < m->n) return set_error(ctx, BPF_ERR_DIMENSION, "mlp_basis: leading dimension < n");
    // The dominant output directions of the learned map: Y = f(G) on q = 4r seeded Gaussian
    // probes, Y = Q R (Cholesky-QR), R = U S V^T (host, q x q), Z = Q U(:, :r).
    const int q = 4 * r, n = m->n;
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<double> G((size_t)n * q);
    for (auto &v : G) v = nd(rng);
    bpf_status s;
    double *buf = (double *)ws_get(ctx, WS_B, sizeof(double) * (3 * (size_t)n * q + 2 * (size_t)q * q), &s);
    if (!buf) return s;
    double *Gd = buf, *Yd = buf + (size_t)n * q, *Qr = buf + 2 * (size_t)n * q;
    double *Rd = Qr + (size_t)n * q, *Ud = Rd + (size_t)q * q;
    BPF_CUDA(ctx, cudaMemcpyAsync(Gd, G.data(), sizeof(double) * G.size(), cudaMemcpyHostToDevice, ctx->stream));
    BPF_TRY(bpf_mlp_forward(m, q, Gd, n, Yd, n));
    BPF_TRY(bpf_householder(ctx, n, q, Yd, n, Rd, q));          // Yd <- Q (column-major)
    std::vector<double> R((size_t)q * q);
    BPF_CUDA(ctx, cudaMemcpyAsync(R.data(), Rd, sizeof(double) * R.size(), cudaMemcpyDeviceToHost, ctx->stream));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    // left singular vectors of R (column-major q x q): eigenvectors of R R^T by cyclic Jacobi
    std::vector<double> S((size_t)q * q, 0.0), U((size_t)q * q, 0.0);
    for (int i = 0; i < q; i++)
        for (int j = 0; j < q; j++) {
            double v = 0.0;
            for (int k = 0; k < q; k++) v += R[(size_t)k * q + i] * R[(size_t)k * q + j];
            S[(size_t)j * q + i] = v;
        }
    for (int i = 0; i < q; i++) U[(size_t)i * q + i] = 1.0;
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0.0;
        for (int a = 0; a < q; a++)
            for (int b = a + 1; b < q; b++) off += S[(size_t)b * q + a] * S[(size_t)b * q + a];
        if (off < 1e-26) break;
        for (int a = 0; a < q; a++)
            for (int b = a + 1; b < q; b++) {
                const double apq = S[(size_t)b * q + a];
                if (std::fabs(apq) < 1e-300) continue;
                const double theta = 0.5 * (S[(size_t)b * q + b] - S[(size_t)a * q + a]) / apq;
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < q; k++) {   // columns a, b of S
                    const double ska = S[(size_t)a * q + k], skb = S[(size_t)b * q + k];
                    S[(size_t)a * q + k] = c * ska - sn * skb;
                    S[(size_t)b * q + k] = sn * ska + c * skb;
                }
                for (int k = 0; k < q; k++) {   // rows a, b
                    const double sak = S[(size_t)k * q + a], sbk = S[(size_t)k * q + b];
                    S[(size_t)k * q + a] = c * sak - sn * sbk;
                    S[(size_t)k * q + b] = sn * sak + c * sbk;
                }
                for (int k = 0; k < q; k++) {
                    const double uka = U[(size_t)a * q + k], ukb = U[(size_t)b * q + k];
                    U[(size_t)a * q + k] = c * uka - sn * ukb;
                    U[(size_t)b * q + k] = sn * uka + c * ukb;
                }
            }
    }
    std::vector<int> idx(q);
    for (int i = 0; i < q; i++) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return S[(size_t)a * q + a] > S[(size_t)b * q + b]; });
    // W (row-major q x q): column c = the c-th dominant eigenvector (first r columns used)
    std::vector<double> W((size_t)q * q, 0.0);
    for (int c = 0; c < r; c++)
        for (int k = 0; k < q; k++) W[(size_t)k * q + c] = U[(size_t)idx[c] * q + k];
    BPF_CUDA(ctx, cudaMemcpyAsync(Ud, W.data(), sizeof(double) * W.size(), cudaMemcpyHostToDevice, ctx->stream));
    BPF_TRY(colmajor_to_rowmajor(ctx, n, q, Yd, n, Qr));
    BPF_TRY(tsmm(ctx, n, q, 1, Qr, 0, Ud, 0, 1.0, nullptr, 0.0, Gd, nullptr));   // Gd = Q W (row-major)
    BPF_TRY(rowmajor_to_colmajor(ctx, n, q, Gd, Yd, n));
    for (int c = 0; c < r; c++)
        BPF_CUDA(ctx, cudaMemcpyAsync(Z + (size_t)c * ldz, Yd + (size_t)c * n, sizeof(double) * n,
                                      cudaMemcpyDeviceToDevice, ctx->stream));
    return check_dev_status(ctx, "mlp_basis");
}

}  // extern "C"
