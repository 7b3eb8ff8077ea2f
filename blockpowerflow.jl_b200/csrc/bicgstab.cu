// block-BiCGSTAB: src/block_bicgstab.jl:182-299 (GPU variant; CPU twin :65-178).
//
// El Guennouni-Jbilou-Sadok block BiCGSTAB, iteration for iteration as the reference:
//   Y = N \ P; V = A Y; K = C^T V; D = C^T R; alpha = K \ D      (:364-371)
//   U = R - V alpha; R = Y alpha; X += R                          (:372-375)
//   Y = N \ U; Q = A Y; omega = |<Q,U>| / |<Q,Q>|                 (:376-378)
//   X += omega Y; R = U - omega Q                                 (:379-380)
//   D = C^T Q; beta = K \ D; U = P - omega V; P = R - U beta     (:381-387)
//   ||R||_F -> stopping test                                      (:389-398)
// The p x p solves use one Householder QR of K per iteration (the reference: geqrf + ormqr +
// trsm), kept for the second solve.  omega and ||R|| stay on the device; the host syncs once
// per chunk of iterations.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "bpf_internal.cuh"
#include "dense.cuh"
#include "prec.cuh"

namespace bpf {

static double now_s_bicg() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

__device__ __forceinline__ unsigned long long gtimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ double block_sum_b(double v, double *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double t = lane < nw ? red[lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) red[0] = t;
    }
    __syncthreads();
    double r = red[0];
    __syncthreads();
    return r;
}

// Householder QR of K (p x p, row-major) into Kf/tau (mode 0), then Out = R^{-1} Q^T D.
// mode 1 reuses Kf/tau.  One CTA; operands in global memory ordered by __syncthreads.
__global__ void __launch_bounds__(1024)
small_qr_solve_kernel(int p, const double *__restrict__ K, double *__restrict__ Kf,
                      double *__restrict__ tau, const double *__restrict__ D,
                      double *__restrict__ Out, int mode, const SolveState *st) {
    if (!st->active) return;
    __shared__ double red[32];
    __shared__ double s_scale;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    const size_t pp = (size_t)p * p;
    if (mode == 0) {
        for (size_t e = tid; e < pp; e += nt) Kf[e] = K[e];
        __syncthreads();
        for (int c = 0; c < p; c++) {
            double s = 0.0;
            for (int r = c + 1 + tid; r < p; r += nt) s += Kf[(size_t)r * p + c] * Kf[(size_t)r * p + c];
            s = block_sum_b(s, red);
            if (tid == 0) {
                const double alpha = Kf[(size_t)c * p + c];
                const double xn = sqrt(s);
                if (xn == 0.0) {
                    tau[c] = 0.0;
                    s_scale = 0.0;
                } else {
                    const double beta = -copysign(hypot(alpha, xn), alpha);
                    tau[c] = (beta - alpha) / beta;
                    s_scale = 1.0 / (alpha - beta);
                    Kf[(size_t)c * p + c] = beta;
                }
            }
            __syncthreads();
            const double t = tau[c];
            if (t != 0.0) {
                const double sc = s_scale;
                for (int r = c + 1 + tid; r < p; r += nt) Kf[(size_t)r * p + c] *= sc;
                __syncthreads();
                for (int c2 = c + 1 + warp; c2 < p; c2 += nw) {
                    double wv = 0.0;
                    for (int r = c + 1 + lane; r < p; r += 32) wv += Kf[(size_t)r * p + c] * Kf[(size_t)r * p + c2];
                    wv = (warp_sum(wv) + Kf[(size_t)c * p + c2]) * t;
                    if (lane == 0) Kf[(size_t)c * p + c2] -= wv;
                    for (int r = c + 1 + lane; r < p; r += 32) Kf[(size_t)r * p + c2] -= wv * Kf[(size_t)r * p + c];
                }
            }
            __syncthreads();
        }
    }
    // Out = Q^T D: apply H_0 .. H_{p-1} to every column of D (one warp per column)
    for (int b = warp; b < p; b += nw) {
        for (int r = lane; r < p; r += 32) Out[(size_t)r * p + b] = D[(size_t)r * p + b];
        __syncwarp();
        for (int c = 0; c < p; c++) {
            const double t = tau[c];
            if (t == 0.0) continue;
            double wv = 0.0;
            for (int r = c + 1 + lane; r < p; r += 32) wv += Kf[(size_t)r * p + c] * Out[(size_t)r * p + b];
            wv = (warp_sum(wv) + Out[(size_t)c * p + b]) * t;
            __syncwarp();
            if (lane == 0) Out[(size_t)c * p + b] -= wv;
            for (int r = c + 1 + lane; r < p; r += 32) Out[(size_t)r * p + b] -= wv * Kf[(size_t)r * p + c];
            __syncwarp();
        }
        // back substitution with R (upper triangle of Kf), column-oriented
        for (int c = p - 1; c >= 0; c--) {
            double xc = 0.0;
            if (lane == 0) {
                xc = Out[(size_t)c * p + b] / Kf[(size_t)c * p + c];
                Out[(size_t)c * p + b] = xc;
            }
            xc = __shfl_sync(0xffffffffu, xc, 0);
            __syncwarp();
            for (int r = lane; r < c; r += 32) Out[(size_t)r * p + b] -= Kf[(size_t)r * p + c] * xc;
            __syncwarp();
        }
    }
}

// Two dot products <Q,U>, <Q,Q> (deterministic two-stage); stage 2 writes omega.
__global__ void dot2_partial_kernel(size_t len, const double *__restrict__ Q,
                                    const double *__restrict__ U, double *__restrict__ part,
                                    const SolveState *st) {
    if (!st->active) return;
    __shared__ double red[32];
    double a = 0.0, b = 0.0;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
        const double q = Q[e];
        a += q * U[e];
        b += q * q;
    }
    a = block_sum_b(a, red);
    b = block_sum_b(b, red);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
    }
}

__global__ void omega_kernel(int nparts, const double *__restrict__ part, SolveState *st) {
    if (!st->active) return;
    __shared__ double red[32];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        a += part[2 * i];
        b += part[2 * i + 1];
    }
    a = block_sum_b(a, red);
    b = block_sum_b(b, red);
    if (threadIdx.x == 0) st->omega = fabs(a) / fabs(b);
}

// X += omega Y; R = U - omega Q; partial ||R||^2.
__global__ void bicg_update1_kernel(size_t len, double *__restrict__ X, const double *__restrict__ Y,
                                    double *__restrict__ R, const double *__restrict__ U,
                                    const double *__restrict__ Q, double *__restrict__ part,
                                    const SolveState *st) {
    if (!st->active) return;
    __shared__ double red[32];
    const double om = st->omega;
    double s = 0.0;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
        X[e] += om * Y[e];
        const double r = U[e] - om * Q[e];
        R[e] = r;
        s += r * r;
    }
    s = block_sum_b(s, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// U = P - omega V
__global__ void bicg_update2_kernel(size_t len, double *__restrict__ U, const double *__restrict__ P,
                                    const double *__restrict__ V, const SolveState *st) {
    if (!st->active) return;
    const double om = st->omega;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x)
        U[e] = P[e] - om * V[e];
}

// ||R|| from the partials of update1; iteration bookkeeping and the stopping test.
__global__ void bicg_step_end_kernel(int nparts, const double *__restrict__ part, SolveState *st,
                                     double *__restrict__ hist) {
    if (!st->active) return;
    __shared__ double red[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[i];
    s = block_sum_b(s, red);
    if (threadIdx.x == 0) {
        const double rn = sqrt(s);
        st->rnorm = rn;
        st->iter += 1;
        if (st->nres < st->hist_cap) hist[st->nres] = rn;
        st->nres++;
        st->solved = rn <= st->eps;
        const int tired = st->iter >= st->itmax;
        st->overtimed = (st->deadline_ns != 0ull && gtimer_ns() > st->deadline_ns);
        st->inner_tired = tired;
        st->active = !(st->solved || tired || st->overtimed);
    }
}

__global__ void bicg_init_kernel(SolveState *st, double atol, double rtol, double *hist,
                                 double timemax, int itmax) {
    const double r = st->rnorm;
    st->eps = atol + rtol * r;
    st->solved = r <= st->eps;
    st->iter = 0;
    st->itmax = itmax;
    if (st->hist_cap > 0) hist[0] = r;
    st->nres = 1;
    st->overtimed = 0;
    st->inner_tired = itmax <= 0;
    st->deadline_ns = (timemax > 0.0 && timemax < 1e15) ? gtimer_ns() + (unsigned long long)(timemax * 1e9) : 0ull;
    st->active = !(st->solved || st->inner_tired);
}

}  // namespace bpf

using namespace bpf;

extern "C" bpf_status bpf_block_bicgstab(bpf_ctx *ctx, const bpf_csr_desc *A, int p,
                                         const double *B, int ldb, double *X, int ldx,
                                         const double *Cs, int ldc, const bpf_prec *N,
                                         const bpf_bicgstab_opts *opts, bpf_stats *stats) {
    if (!ctx) return BPF_ERR_INVALID_VALUE;
    const double t0 = now_s_bicg();
    if (!A || !opts || !stats) return set_error(ctx, BPF_ERR_INVALID_VALUE, "block_bicgstab: null argument");
    const int n = A->n;
    if (A->dtype != BPF_F64) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "block_bicgstab: FP64 only");
    if (n < 1 || p < 1 || !B || !X) return set_error(ctx, BPF_ERR_INVALID_VALUE, "block_bicgstab: empty system");
    if (ldb < n || ldx < n || (Cs && ldc < n)) return set_error(ctx, BPF_ERR_DIMENSION, "Inconsistent problem size");
    if (N && N->n != n) return set_error(ctx, BPF_ERR_DIMENSION, "preconditioner size differs from the system");
    if (N) BPF_TRY(prec_reserve_z(ctx, const_cast<bpf_prec *>(N), p));
    if (p > 128) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "block_bicgstab: p=%d > 128", p);
    int itmax = opts->itmax == 0 ? 2 * n : opts->itmax;                     // :347
    const double timemax = opts->timemax > 0.0 ? opts->timemax : 1e300;
    const size_t np = (size_t)n * p, pp = (size_t)p * p;
    bpf_status s;
    double *vec = (double *)ws_get(ctx, WS_VEC, sizeof(double) * np * 10, &s);
    if (!vec) return s;
    double *Bi = vec, *Xi = vec + np, *P = vec + 2 * np, *R = vec + 3 * np, *V = vec + 4 * np,
           *Q = vec + 5 * np, *U = vec + 6 * np, *Yb = vec + 7 * np, *Ci = vec + 8 * np;
    double *small = (double *)ws_get(ctx, WS_HSCR, sizeof(double) * (6 * pp + p), &s);
    if (!small) return s;
    double *K = small, *Kf = small + pp, *D = small + 2 * pp, *alpha = small + 3 * pp,
           *beta = small + 4 * pp, *tau = small + 6 * pp;
    SolveState *st = (SolveState *)ws_get(ctx, WS_STATE, sizeof(SolveState), &s);
    if (!st) return s;
    const int hist_cap = itmax + 2;
    double *hist = (double *)ws_get(ctx, WS_HIST, sizeof(double) * hist_cap, &s);
    if (!hist) return s;
    const int nparts = ctx->num_sms * 2;
    double *part = (double *)ws_get(ctx, WS_NORM, sizeof(double) * 2 * nparts, &s);
    if (!part) return s;
    if (!ws_get(ctx, WS_PARTIAL, sizeof(double) * pp * ((size_t)ctx->num_sms * 4 + 2), &s)) return s;

    SolveState hs;
    std::memset(&hs, 0, sizeof(hs));
    hs.hist_cap = hist_cap;
    BPF_CUDA(ctx, cudaMemcpyAsync(st, &hs, sizeof(SolveState), cudaMemcpyHostToDevice, ctx->stream));
    const int base = A->index_base;
    const int *rp = A->rowptr, *ci = A->colind;
    const double *av = (const double *)A->vals;
    BPF_TRY(colmajor_to_rowmajor(ctx, n, p, B, ldb, Bi));
    const double *Cm = Bi;                                                  // C = B (:301)
    if (Cs) {
        BPF_TRY(colmajor_to_rowmajor(ctx, n, p, Cs, ldc, Ci));
        Cm = Ci;
    }
    BPF_CUDA(ctx, cudaMemsetAsync(Xi, 0, sizeof(double) * np, ctx->stream));  // :326-335
    BPF_CUDA(ctx, cudaMemcpyAsync(P, Bi, sizeof(double) * np, cudaMemcpyDeviceToDevice, ctx->stream));
    BPF_CUDA(ctx, cudaMemcpyAsync(R, Bi, sizeof(double) * np, cudaMemcpyDeviceToDevice, ctx->stream));
    BPF_TRY(frob_norm(ctx, np, R, &st->rnorm));                              // :344
    bicg_init_kernel<<<1, 1, 0, ctx->stream>>>(st, opts->atol, opts->rtol, hist,
                                               timemax - (now_s_bicg() - t0), itmax);
    BPF_LAUNCHED(ctx);
    BPF_CUDA(ctx, cudaMemcpyAsync(&hs, st, sizeof(SolveState), cudaMemcpyDeviceToHost, ctx->stream));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (opts->verbose > 0) {
        printf("BLOCK-BICGSTAB: system of size %d with %d right-hand sides\n", n, p);
        printf("%5s  %7s  %5s\n", "k", "‖Rₖ‖", "timer");
        printf("%5d  %7.1e  %.2fs\n", 0, hs.rnorm, now_s_bicg() - t0);
    }
    const int *act = &st->active;
    const int blocks = std::max(1, std::min(ceil_div((long long)np, 256), nparts));
    int launched = 0, printed = 1;
    std::vector<double> hbuf;
    bool active = hs.active != 0;
    while (active) {
        const int chunk = std::min(16, itmax - launched);
        if (chunk <= 0) break;
        for (int it = 0; it < chunk; it++) {
            const double *Yp = P;                                           // :364
            if (N) {
                BPF_TRY(prec_apply_rowmajor(ctx, N, p, P, Yb, act));
                Yp = Yb;
            }
            BPF_TRY(spmm_rowmajor(ctx, n, A->nnz, rp, ci, av, base, p, 1.0, Yp, 0.0, V, nullptr, act));  // :365
            BPF_TRY(gram(ctx, n, p, 1, Cm, 0, V, K, 1.0, false, st));      // :366
            BPF_TRY(gram(ctx, n, p, 1, Cm, 0, R, D, 1.0, false, st));      // :367
            {
                KScope ks(ctx, BPF_KC_SMALL);
                small_qr_solve_kernel<<<1, 1024, 0, ctx->stream>>>(p, K, Kf, tau, D, alpha, 0, st);  // :368-371
            }
            BPF_LAUNCHED(ctx);
            BPF_TRY(tsmm(ctx, n, p, 1, V, 0, alpha, 0, -1.0, R, 1.0, U, st));   // :372-373
            BPF_TRY(tsmm(ctx, n, p, 1, Yp, 0, alpha, 0, 1.0, nullptr, 0.0, R, st));  // :374
            BPF_TRY(axpby(ctx, np, 1.0, R, 1.0, Xi, st));                   // :375
            const double *Yu = U;                                           // :376
            if (N) {
                BPF_TRY(prec_apply_rowmajor(ctx, N, p, U, Yb, act));
                Yu = Yb;
            }
            BPF_TRY(spmm_rowmajor(ctx, n, A->nnz, rp, ci, av, base, p, 1.0, Yu, 0.0, Q, nullptr, act));  // :377
            dot2_partial_kernel<<<nparts, 256, 0, ctx->stream>>>(np, Q, U, part, st);        // :378
            BPF_LAUNCHED(ctx);
            omega_kernel<<<1, 256, 0, ctx->stream>>>(nparts, part, st);
            BPF_LAUNCHED(ctx);
            bicg_update1_kernel<<<blocks, 256, 0, ctx->stream>>>(np, Xi, Yu, R, U, Q, part, st);  // :379-380
            BPF_LAUNCHED(ctx);
            // part now holds ||R||^2 partials for step_end; D = C^T Q uses the gram workspace.
            BPF_TRY(gram(ctx, n, p, 1, Cm, 0, Q, D, 1.0, false, st));      // :381
            small_qr_solve_kernel<<<1, 1024, 0, ctx->stream>>>(p, K, Kf, tau, D, beta, 1, st);  // :382-384
            BPF_LAUNCHED(ctx);
            bicg_update2_kernel<<<blocks, 256, 0, ctx->stream>>>(np, U, P, V, st);           // :385
            BPF_LAUNCHED(ctx);
            BPF_TRY(tsmm(ctx, n, p, 1, U, 0, beta, 0, -1.0, R, 1.0, P, st));   // :386-387
            bicg_step_end_kernel<<<1, 256, 0, ctx->stream>>>(blocks, part, st, hist);        // :389-398
            BPF_LAUNCHED(ctx);
        }
        launched += chunk;
        BPF_CUDA(ctx, cudaMemcpyAsync(&hs, st, sizeof(SolveState), cudaMemcpyDeviceToHost, ctx->stream));
        BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        active = hs.active != 0;
        if (opts->verbose > 0 && hs.nres > printed) {
            int upto = std::min(hs.nres, hist_cap);
            hbuf.resize(upto);
            BPF_CUDA(ctx, cudaMemcpy(hbuf.data(), hist, sizeof(double) * upto, cudaMemcpyDeviceToHost));
            for (int q = printed; q < upto; q++)
                if (q % opts->verbose == 0) printf("%5d  %7.1e  %.2fs\n", q, hbuf[q], now_s_bicg() - t0);
            printed = upto;
        }
        if (now_s_bicg() - t0 > timemax) {
            hs.overtimed = 1;
            break;
        }
    }
    BPF_TRY(rowmajor_to_colmajor(ctx, n, p, Xi, X, ldx));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    BPF_TRY(check_dev_status(ctx, "block_bicgstab"));
    const bool solved = hs.solved != 0;
    const bool tired = hs.iter >= itmax;
    const bool overtimed = hs.overtimed != 0;
    int status = BPF_SOLVE_UNKNOWN;                                          // :402-405
    if (tired) status = BPF_SOLVE_ITMAX;
    if (solved) status = BPF_SOLVE_SOLVED;
    if (overtimed) status = BPF_SOLVE_TIMEMAX;
    stats->niter = hs.iter;
    stats->solved = solved;
    stats->status = status;
    stats->npass = 1;
    stats->n_residuals = opts->history ? std::min(hs.nres, hist_cap) : 0;
    if (opts->history && stats->residuals && stats->residuals_capacity > 0) {
        int cnt = std::min(stats->n_residuals, stats->residuals_capacity);
        BPF_CUDA(ctx, cudaMemcpy(stats->residuals, hist, sizeof(double) * cnt, cudaMemcpyDeviceToHost));
    }
    if (opts->verbose > 0) printf("\n");
    stats->timer = now_s_bicg() - t0;
    return BPF_SUCCESS;
}
