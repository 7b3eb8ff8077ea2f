// One-CTA / one-CTA-per-column kernels on p x p blocks: Cholesky of the Gram matrix (for
// Cholesky-QR), the block Householder QR update of the block Hessenberg matrix, and the
// block back substitution of block-GMRES.
//
// These replace the chains of small cuSOLVER / cuBLAS calls of the reference
// (householder! -> geqrf/orgqr, ormqr on 2p x p blocks, trsm; src/block_gmres.jl:316-375,
// src/block_utils.jl:46-53).  They are latency kernels, so: every operand a loop walks is
// staged in shared memory first (bulk coalesced or cp.async loads, never a dependent chain of
// L2 round trips), consecutive threads touch consecutive addresses, partial sums go through
// shared memory, and each phase costs one __syncthreads.  Blocks wider than the shared-memory
// budget (p > 64) keep the same code on global (L1/L2) memory.
#include <algorithm>
#include <cmath>

#include "bpf_internal.cuh"
#include "dense.cuh"
#include "small.cuh"

namespace bpf {

__device__ __forceinline__ unsigned long long small_globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Inverse of an upper-triangular p x p matrix U (row stride ldu) into X (row stride ldx), both
// in shared memory.  Column c of X = U^{-1} is computed by back substitution (x_k = 0 for
// k > c, so every column runs the same loop) by a group of L consecutive lanes that split the
// inner products and combine them with shuffles; L = 4, 2 or 1 so that the p columns fill
// the block.
__device__ void upper_inverse(int p, const double *U, int ldu, double *X, int ldx) {
    const int nt = blockDim.x;
    const int L = (nt >= 4 * p) ? 4 : ((nt >= 2 * p) ? 2 : 1);
    const int tid = threadIdx.x;
    const int q = tid % L;
    for (int c0 = 0; c0 < p; c0 += nt / L) {
        const int c = c0 + tid / L;
        const bool act = (tid / L < nt / L) && c < p;
        for (int i = p - 1; i >= 0; i--) {
            double s = 0.0;
            if (act)
                for (int k = i + 1 + q; k < p; k += L) s += U[i * ldu + k] * X[k * ldx + c];
            if (L >= 4) s += __shfl_xor_sync(0xffffffffu, s, 2);
            if (L >= 2) s += __shfl_xor_sync(0xffffffffu, s, 1);
            if (act && q == 0) X[i * ldx + c] = (i > c) ? 0.0 : (((i == c) ? 1.0 : 0.0) - s) / U[i * ldu + i];
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------------------
// Cholesky of G = R^T R (R upper), Rinv = R^{-1}, Racc <- R Racc (pass > 0) or R (pass 0).
// pass 0 may add the shift s = 11 (n p + p (p+1)) u trace(G) (shifted Cholesky-QR, Fukaya et
// al. 2020) when a pivot falls below 1e-13 of its column's norm^2; it then raises *shift_flag
// (the caller's third pass runs) and *reorth_flag reports a pivot below 1e-8.
// One phase (one __syncthreads) per column: every thread reads the unscaled pivot row.
// Shared memory: g (working matrix) and R, both p x (p+1); R falls back to the global Rtmp
// when two of them do not fit.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
chol2_kernel(int n, int p, const double *__restrict__ G, double *__restrict__ Rinv,
             double *__restrict__ Racc, double *__restrict__ Rglob, int pass, SolveState *st,
             const int *gate, const int *gate2, int *shift_flag, int *reorth_flag,
             DevStatus *ds, int r_in_smem) {
    if (st && !st->active) return;
    if (gate && *gate == 0) return;
    if (gate2 && *gate2 == 0) return;
    extern __shared__ double sm[];
    const int ld = p + 1;
    double *g = sm;
    double *R = r_in_smem ? sm + p * ld : Rglob;
    const int ldr = r_in_smem ? ld : p;
    __shared__ double s_trace;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) {
        double tr = 0.0;
        for (int i = 0; i < p; i++) tr += G[i * p + i];
        s_trace = tr;
        if (pass == 0 && shift_flag) *shift_flag = 0;
    }
    __syncthreads();
    double minratio = 1.0;
    int fail = 0;
    for (int attempt = 0; attempt < 2; attempt++) {
        const double shift = attempt == 0 ? 0.0
                                          : 11.0 * ((double)n * p + (double)p * (p + 1)) *
                                                1.1102230246251565e-16 * s_trace;
        for (int e = tid; e < p * p; e += nt) {
            const int a = e / p, b = e % p;
            g[a * ld + b] = G[e] + (a == b ? shift : 0.0);
            R[a * ldr + b] = 0.0;
        }
        __syncthreads();
        fail = 0;
        for (int j = 0; j < p; j++) {
            const double d = g[j * ld + j];
            const double ref = G[j * p + j] + shift;
            if (attempt == 0) minratio = fmin(minratio, ref > 0.0 ? d / ref : 0.0);
            if (!(d > 1e-13 * ref) || !(d > 0.0)) {
                fail = 1;
                break;
            }
            const double r = sqrt(d), dinv = 1.0 / d;
            for (int c = j + tid; c < p; c += nt) R[j * ldr + c] = (c == j) ? r : g[j * ld + c] / r;
            // trailing update of the upper triangle: 16 x 16 thread grid, rows a, columns b >= a
            const int ty = tid >> 4, tx = tid & 15;
            for (int a = j + 1 + ty; a < p; a += nt >> 4) {
                const double ga = g[j * ld + a] * dinv;
                for (int b = j + 1 + tx; b < p; b += 16)
                    if (b >= a) g[a * ld + b] -= ga * g[j * ld + b];
            }
            __syncthreads();
        }
        if (attempt == 0 && tid == 0 && pass == 0 && reorth_flag)
            *reorth_flag = (fail || minratio < 1e-8) ? 1 : 0;
        if (!fail) break;
        if (tid == 0 && shift_flag) *shift_flag = 1;
        __syncthreads();
    }
    if (fail) {
        if (tid == 0) {
            if (st) st->qr_fail = 1;
            if (ds && atomicCAS(&ds->err, 0, (int)DEV_CHOL_FAIL) == 0) ds->aux = pass;
        }
        return;
    }
    __syncthreads();
    upper_inverse(p, R, ldr, g, ld);
    __syncthreads();
    for (int e = tid; e < p * p; e += nt) Rinv[e] = g[(e / p) * ld + e % p];
    if (pass == 0) {
        for (int e = tid; e < p * p; e += nt) Racc[e] = R[(e / p) * ldr + e % p];
        return;
    }
    __syncthreads();
    for (int e = tid; e < p * p; e += nt) g[(e / p) * ld + e % p] = Racc[e];   // Racc staged
    __syncthreads();
    for (int e = tid; e < p * p; e += nt) {
        const int a = e / p, b = e % p;
        double s = 0.0;
        for (int c = a; c <= b; c++) s += R[a * ldr + c] * g[c * ld + b];
        Racc[e] = (b >= a) ? s : 0.0;
    }
}

bpf_status launch_chol(bpf_ctx *ctx, int n, int p, const double *G, double *Rinv, double *Racc,
                       double *Rtmp, int pass, SolveState *st, const int *gate, const int *gate2,
                       int *shift_flag, int *reorth_flag) {
    const size_t one = sizeof(double) * p * (p + 1);
    const int r_in_smem = (2 * one <= 200 * 1024) ? 1 : 0;
    const size_t smem = r_in_smem ? 2 * one : one;
    if (smem > 48 * 1024)
        BPF_CUDA(ctx, cudaFuncSetAttribute(chol2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
    KScope ks(ctx, BPF_KC_SMALL);
    chol2_kernel<<<1, 256, smem, ctx->stream>>>(n, p, G, Rinv, Racc, Rtmp, pass, st, gate, gate2,
                                                shift_flag, reorth_flag, ctx->dstat, r_in_smem);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

// ---------------------------------------------------------------------------------------
// Block Hessenberg QR: apply Omega_0..Omega_{j-1} to block column j (one CTA per column b).
// HY per block column i: Y_i (2p x p, explicit unit lower trapezoid) then T_i (p x p upper),
// contiguous, Omega_i^T = I - Y_i T_i^T Y_i^T.  Per step: w = Y^T seg, w2 = T^T w,
// seg -= Y w2, each a (column, row-range) split over the 256 threads with partial sums in
// shared memory.  STAGED: Y_i and T_i are copied to shared memory with cp.async, the copy of
// step i+1 in flight while step i computes (double buffer, 2 x 3 p^2 doubles).
// ---------------------------------------------------------------------------------------
__host__ __device__ inline size_t rblk_pos(int i, int j) { return (size_t)j * (j + 1) / 2 + i; }

template <bool STAGED>
__global__ void __launch_bounds__(256)
hess_apply2_kernel(int p, int k, double *__restrict__ Rblk, const double *__restrict__ HY,
                   const SolveState *st) {
    if (!st->active) return;
    const int j = k - 1;
    if (j <= 0) return;
    const int b = blockIdx.x;
    extern __shared__ __align__(16) double sm[];
    const size_t pp = (size_t)p * p;
    const int nparts = max(1, (int)blockDim.x / p);
    double *stage = sm;                                   // STAGED: 2 x 3 p^2
    double *seg = sm + (STAGED ? 6 * pp : 0);             // 2p
    double *part = seg + 2 * p;                           // nparts * p
    double *w = part + nparts * p;                        // p
    const int tid = threadIdx.x;
    const int c_of = tid % p, q_of = tid / p;
    // 16-lane groups for row-wise sums.  Both half-warps of a warp always run the same number
    // of row iterations (2p rows, stride 16, even group pairs), so the shuffles use the full
    // mask with width 16.
    const int g16 = tid >> 4, l16 = tid & 15;
    const int nvec = (int)(3 * pp / 2);  // 16-byte chunks of Y_i + T_i
    auto prefetch = [&](int i) {
        const double *src = HY + (size_t)i * 3 * pp;
        double *dst = stage + (size_t)(i & 1) * 3 * pp;
        for (int e = tid; e < nvec; e += blockDim.x) cp_async16(dst + 2 * e, src + 2 * e);
        cp_async_commit();
    };
    if (STAGED) prefetch(0);
    for (int a = tid; a < p; a += blockDim.x) seg[a] = Rblk[rblk_pos(0, j) * pp + (size_t)a * p + b];
    for (int i = 0; i < j; i++) {
        for (int a = tid; a < p; a += blockDim.x) seg[p + a] = Rblk[rblk_pos(i + 1, j) * pp + (size_t)a * p + b];
        if (STAGED) {
            if (i + 1 < j) {
                prefetch(i + 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
        }
        __syncthreads();
        const double *Y = STAGED ? stage + (size_t)(i & 1) * 3 * pp : HY + (size_t)i * 3 * pp;
        const double *T = Y + 2 * pp;
        // w partials: w[c] = sum_{r >= c} Y[r][c] seg[r], rows split in nparts ranges
        if (q_of < nparts) {
            const int c = c_of;
            const int len = (2 * p + nparts - 1) / nparts;
            const int r0 = max(c, q_of * len), r1 = min(2 * p, (q_of + 1) * len);
            double s = 0.0;
            for (int r = r0; r < r1; r++) s += Y[(size_t)r * p + c] * seg[r];
            part[q_of * p + c] = s;
        }
        __syncthreads();
        if (tid < p) {
            double s = 0.0;
            for (int q = 0; q < nparts; q++) s += part[q * p + tid];
            w[tid] = s;
        }
        __syncthreads();
        // w2 partials: w2[c] = sum_{c' <= c} T[c'][c] w[c']
        if (q_of < nparts) {
            const int c = c_of;
            const int len = (p + nparts - 1) / nparts;
            const int a0 = q_of * len, a1 = min(c + 1, (q_of + 1) * len);
            double s = 0.0;
            for (int a = a0; a < a1; a++) s += T[(size_t)a * p + c] * w[a];
            part[q_of * p + c] = s;
        }
        __syncthreads();
        if (tid < p) {
            double s = 0.0;
            for (int q = 0; q < nparts; q++) s += part[q * p + tid];
            w[tid] = s;   // now w2
        }
        __syncthreads();
        // seg[r] -= sum_c Y[r][c] w2[c]; 16 lanes per row
        for (int r = g16; r < 2 * p; r += blockDim.x >> 4) {
            double s = 0.0;
            const int cmax = min(r, p - 1);
            for (int c = l16; c <= cmax; c += 16) s += Y[(size_t)r * p + c] * w[c];
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, 16);
            if (l16 == 0) seg[r] -= s;
        }
        __syncthreads();
        for (int a = tid; a < p; a += blockDim.x) {
            Rblk[rblk_pos(i, j) * pp + (size_t)a * p + b] = seg[a];
            seg[a] = seg[p + a];
        }
        __syncthreads();
    }
    for (int a = tid; a < p; a += blockDim.x) Rblk[rblk_pos(j, j) * pp + (size_t)a * p + b] = seg[a];
}

// ---------------------------------------------------------------------------------------
// Factor F = [R_jj; C] (2p x p) by Householder QR (dlarfg conventions), store Y_j and its
// T_j (T^{-1} = diag(1/tau) + strict_upper(Y^T Y), the UT transform of Joffrain et al.),
// apply Omega_j^T to [Z_j; 0] and run the stopping test.  One CTA of 256 threads; three
// phases per Householder column.  F_SMEM: F lives in shared memory (row stride p+1) and is
// written to HY at the end; otherwise it is worked on in place in global memory.
// ---------------------------------------------------------------------------------------
template <bool F_SMEM>
__global__ void __launch_bounds__(256)
hess_factor2_kernel(int p, int k, double *__restrict__ Rblk, double *__restrict__ HY,
                    double *__restrict__ tau, double *__restrict__ Z,
                    const double *__restrict__ Cm, SolveState *st, double *__restrict__ hist,
                    double *__restrict__ scr) {
    if (!st->active) return;
    extern __shared__ double sm[];
    const int ld = p + 1;
    const int nparts = max(1, (int)blockDim.x / p);
    double *Tm = sm;                    // p x ld: T
    double *part = sm + p * ld;         // nparts * p: partial sums
    double *rowc = part + nparts * p;   // p: row c of F before the reflector update
    double *Fs = rowc + p;              // F_SMEM: 2p x ld
    __shared__ double red[32];
    __shared__ double s_scale, s_beta;
    __shared__ int s_anyzero;
    const int j = k - 1;
    const size_t pp = (size_t)p * p;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    const int m = 2 * p;
    double *Fg = HY + (size_t)j * 3 * pp;
    double *T = Fg + 2 * pp;
    double *F = F_SMEM ? Fs : Fg;
    const int ldf = F_SMEM ? ld : p;
    double *Rjj = Rblk + rblk_pos(j, j) * pp;
    double *Zj = Z + (size_t)j * pp;
    double *Zn = Z + (size_t)(j + 1) * pp;
    // W1, W2 and a copy of Z_j live in shared memory after F when F does (F_SMEM)
    double *W1 = F_SMEM ? Fs + 2 * p * ld : scr;
    double *W2 = F_SMEM ? W1 + pp : scr + pp;
    double *Zs = F_SMEM ? W2 + pp : Zj;
    double *Tinv = scr + 2 * pp;        // p x p (global scratch)
    const int c_of = tid % p, q_of = tid / p;
    for (size_t e = tid; e < pp; e += nt) {
        const int a = (int)(e / p), b = (int)(e % p);
        F[a * ldf + b] = Rjj[e];
        F[(a + p) * ldf + b] = Cm[e];
    }
    if (tid == 0) s_anyzero = 0;
    __syncthreads();
    double prev_sc = 0.0;
    for (int c = 0; c < p; c++) {
        // phase 1: norm of the sub-column, reflector scalars; scale the previous column's
        // reflector (deferred: phase 3 of that column still read it unscaled)
        if (c > 0 && prev_sc != 0.0)
            for (int r = c + tid; r < m; r += nt) F[r * ldf + c - 1] *= prev_sc;
        double s = 0.0;
        for (int r = c + 1 + tid; r < m; r += nt) {
            const double v = F[r * ldf + c];
            s += v * v;
        }
        s = warp_sum(s);
        if (lane == 0) red[warp] = s;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int q = 0; q < nw; q++) t += red[q];
            const double alpha = F[c * ldf + c];
            const double xn = sqrt(t);
            if (xn == 0.0) {
                tau[c] = 0.0;
                s_scale = 0.0;
                s_beta = alpha;
                s_anyzero = 1;
            } else {
                const double beta = -copysign(hypot(alpha, xn), alpha);
                tau[c] = (beta - alpha) / beta;
                s_scale = 1.0 / (alpha - beta);
                s_beta = beta;
            }
        }
        __syncthreads();
        const double tc = tau[c], sc = s_scale;
        // phase 2: w[c2] = F[c][c2] + sc * sum_{r>c} F[r][c] F[r][c2]  (partials); the
        // unscaled column c is read, and row c is kept aside before phase 3 rewrites it
        if (tc != 0.0 && q_of < nparts) {
            const int c2 = c_of;
            if (c2 > c) {
                const int len = (m - c - 1 + nparts - 1) / nparts;
                const int r0 = c + 1 + q_of * len, r1 = min(m, r0 + len);
                double s2 = 0.0;
                for (int r = r0; r < r1; r++) s2 += F[r * ldf + c] * F[r * ldf + c2];
                part[q_of * p + c2] = s2;
                if (q_of == 0) rowc[c2] = F[c * ldf + c2];
            }
        }
        __syncthreads();
        // phase 3: apply the reflector to columns c2 > c; the diagonal becomes beta
        if (tc != 0.0) {
            const int width = p - c - 1;
            for (int e = tid; e < (m - c) * (width + 1); e += nt) {
                const int r = c + e / (width + 1), c2 = c + e % (width + 1);
                if (c2 == c) {
                    if (r == c) F[c * ldf + c] = s_beta;
                } else {
                    double wv = 0.0;
                    for (int q = 0; q < nparts; q++) wv += part[q * p + c2];
                    wv = tc * (rowc[c2] + sc * wv);
                    const double vr = (r == c) ? 1.0 : sc * F[r * ldf + c];
                    F[r * ldf + c2] -= wv * vr;
                }
            }
        }
        prev_sc = sc;
        __syncthreads();
    }
    if (prev_sc != 0.0)
        for (int r = p + tid; r < m; r += nt) F[r * ldf + p - 1] *= prev_sc;
    __syncthreads();
    // R_jj <- upper triangle of F; F <- explicit Y (0 above, 1 on the diagonal)
    for (size_t e = tid; e < pp; e += nt) {
        const int a = (int)(e / p), b = (int)(e % p);
        Rjj[e] = (b >= a) ? F[a * ldf + b] : 0.0;
    }
    __syncthreads();
    for (size_t e = tid; e < 2 * pp; e += nt) {
        const int r = (int)(e / p), c = (int)(e % p);
        if (r < c) F[r * ldf + c] = 0.0;
        else if (r == c) F[r * ldf + c] = 1.0;
    }
    __syncthreads();
    if (F_SMEM)
        for (size_t e = tid; e < 2 * pp; e += nt) Fg[e] = F[(e / p) * ldf + e % p];
    // T^{-1} = diag(1/tau) + strict_upper(Y^T Y);  (a, c) with a < c, rows r >= c
    for (int e = tid; e < p * p; e += nt) {
        const int a = e / p, c = e % p;
        double v = 0.0;
        if (a < c) {
            for (int r = c; r < m; r++) v += F[r * ldf + a] * F[r * ldf + c];
        } else if (a == c) {
            v = (tau[c] != 0.0) ? 1.0 / tau[c] : 1.0;
        }
        Tm[a * ld + c] = v;    // T^{-1} staged in Tm, inverted into Tinv's place below
    }
    __syncthreads();
    if (!s_anyzero) {
        // Tinv (global scratch) only serves as the row-stride-p copy the inverse reads
        for (int e = tid; e < p * p; e += nt) Tinv[e] = Tm[(e / p) * ld + e % p];
        __syncthreads();
        upper_inverse(p, Tinv, p, Tm, ld);
    } else {
        // some reflector is the identity: the dlarft recurrence handles tau = 0 exactly
        for (int e = tid; e < p * p; e += nt) Tinv[e] = Tm[(e / p) * ld + e % p];
        __syncthreads();
        if (tid == 0) {
            for (int c = 0; c < p; c++) {
                for (int a = 0; a < p; a++) Tm[a * ld + c] = 0.0;
                const double t = tau[c];
                for (int a = 0; a < c; a++) {
                    double s = 0.0;
                    for (int a2 = a; a2 < c; a2++) s += Tm[a * ld + a2] * Tinv[a2 * p + c];
                    Tm[a * ld + c] = -t * s;
                }
                Tm[c * ld + c] = t;
            }
        }
    }
    __syncthreads();
    for (int e = tid; e < p * p; e += nt) T[e] = Tm[(e / p) * ld + e % p];
    if (F_SMEM) {
        for (int e = tid; e < p * p; e += nt) Zs[e] = Zj[e];
        __syncthreads();
    }
    // W1 = Y_top^T Z_j
    for (int e = tid; e < p * p; e += nt) {
        const int c = e / p, b = e % p;
        double s = 0.0;
        for (int r = c; r < p; r++) s += F[r * ldf + c] * Zs[(size_t)r * p + b];
        W1[e] = s;
    }
    __syncthreads();
    // W2 = T^T W1
    for (int e = tid; e < p * p; e += nt) {
        const int c = e / p, b = e % p;
        double s = 0.0;
        for (int c2 = 0; c2 <= c; c2++) s += Tm[c2 * ld + c] * W1[(size_t)c2 * p + b];
        W2[e] = s;
    }
    __syncthreads();
    // [Z_j; Lambda] = [Z_j; 0] - Y W2
    double ss = 0.0;
    for (size_t e = tid; e < 2 * pp; e += nt) {
        const int r = (int)(e / p), b = (int)(e % p);
        const int cmax = min(r, p - 1);
        double s = 0.0;
        for (int c = 0; c <= cmax; c++) s += F[r * ldf + c] * W2[(size_t)c * p + b];
        if (r < p) {
            Zj[e] = Zs[e] - s;
        } else {
            Zn[e - pp] = -s;
            ss += s * s;
        }
    }
    ss = warp_sum(ss);
    __syncthreads();
    if (lane == 0) red[warp] = ss;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int q = 0; q < nw; q++) t += red[q];
        const double rn = sqrt(t);
        st->rnorm = rn;
        if (st->nres < st->hist_cap) hist[st->nres] = rn;
        st->nres++;
        st->inner_iter = k;
        st->solved = rn <= st->eps;
        st->inner_tired = st->restart ? (k >= min(st->mem, st->inner_itmax)) : (k >= st->inner_itmax);
        st->overtimed = (st->deadline_ns != 0ull && small_globaltimer_ns() > st->deadline_ns);
        st->active = !(st->solved || st->inner_tired || st->overtimed);
    }
}

bpf_status launch_hess(bpf_ctx *ctx, int p, int k, double *Rblk, double *HY, double *tau,
                       double *Z, const double *Cm, SolveState *st, double *hist, double *scr) {
    KScope ks(ctx, BPF_KC_SMALL);
    const int nparts = std::max(1, 256 / p);
    const size_t pp = (size_t)p * p;
    const size_t small_a = sizeof(double) * (2 * p + nparts * p + p);
    const size_t staged_a = small_a + sizeof(double) * 6 * pp;
    // cp.async moves 16-byte chunks: the per-block stride 3 p^2 doubles is 16-byte aligned
    // only for even p.
    if (staged_a <= 220 * 1024 && p % 2 == 0) {
        if (staged_a > 48 * 1024)
            BPF_CUDA(ctx, cudaFuncSetAttribute(hess_apply2_kernel<true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)staged_a));
        hess_apply2_kernel<true><<<p, 256, staged_a, ctx->stream>>>(p, k, Rblk, HY, st);
    } else {
        hess_apply2_kernel<false><<<p, 256, small_a, ctx->stream>>>(p, k, Rblk, HY, st);
    }
    BPF_LAUNCHED(ctx);
    const size_t base_f = sizeof(double) * (p * (p + 1) + nparts * p + p);
    const size_t smem_f = base_f + sizeof(double) * (2 * p * (p + 1) + 3 * pp);
    if (smem_f <= 220 * 1024) {
        if (smem_f > 48 * 1024)
            BPF_CUDA(ctx, cudaFuncSetAttribute(hess_factor2_kernel<true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_f));
        hess_factor2_kernel<true><<<1, 256, smem_f, ctx->stream>>>(p, k, Rblk, HY, tau, Z, Cm, st, hist, scr);
    } else {
        if (base_f > 48 * 1024)
            BPF_CUDA(ctx, cudaFuncSetAttribute(hess_factor2_kernel<false>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)base_f));
        hess_factor2_kernel<false><<<1, 256, base_f, ctx->stream>>>(p, k, Rblk, HY, tau, Z, Cm, st, hist, scr);
    }
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

}  // namespace bpf
