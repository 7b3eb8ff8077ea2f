// One-CTA / one-CTA-per-column kernels on p x p blocks: Cholesky of the Gram matrix (for
// Cholesky-QR), the block Householder QR update of the block Hessenberg matrix, and the
// block back substitution of block-GMRES.
//
// These replace the chains of small cuSOLVER / cuBLAS calls of the reference
// (householder! -> geqrf/orgqr, ormqr on 2p x p blocks, trsm; src/block_gmres.jl:316-375,
// src/block_utils.jl:46-53).  They are latency kernels; the design rules are:
//  * every operand a loop walks is in shared memory (bulk async copies or coalesced loads),
//    with row strides of p+1 doubles so that both row- and column-direction sweeps by a warp
//    are free of bank conflicts;
//  * a fixed thread -> (column, row group) map, so each phase is a handful of FMAs per
//    thread with one barrier, and no thread ever runs a serial section;
//  * no global load inside a dependent loop.
// Blocks wider than the shared-memory budget (p > 64) run the same code with the large
// operands in global memory (L1/L2).
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

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

// --- mbarrier + bulk async copy (global -> shared) ---------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Bounded wait on a phase of an mbarrier (~2^21 polls); false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity) {
    for (long long it = 0; it < kSpinLimit; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 64) __nanosleep(32);
    }
    return false;
}

// Inverse of an upper-triangular p x p matrix U (row stride ldu) into X (row stride ldx), both
// in shared memory (or X in global memory).  Column c of X = U^{-1} is computed by back
// substitution (x_k = 0 for k > c, so every column runs the same loop) by a group of L
// consecutive lanes that split the inner products and combine them with shuffles; L = 4, 2
// or 1 so that the p columns fill the block.  dinv[i] = 1 / U[i][i] (shared).
__device__ void upper_inverse(int p, const double *U, int ldu, double *X, int ldx,
                              const double *dinv) {
    const int nt = blockDim.x;
    const int L = (nt >= 8 * p) ? 8 : ((nt >= 4 * p) ? 4 : ((nt >= 2 * p) ? 2 : 1));
    const int tid = threadIdx.x;
    const int q = tid % L;
    for (int c0 = 0; c0 < p; c0 += nt / L) {
        const int c = c0 + tid / L;
        const bool act = c < p;
        for (int i = p - 1; i >= 0; i--) {
            double s = 0.0;
            if (act && i < c)
                for (int k = i + 1 + q; k <= c; k += L) s += U[i * ldu + k] * X[k * ldx + c];
            if (L >= 8) s += __shfl_xor_sync(0xffffffffu, s, 4);
            if (L >= 4) s += __shfl_xor_sync(0xffffffffu, s, 2);
            if (L >= 2) s += __shfl_xor_sync(0xffffffffu, s, 1);
            if (act && q == 0) X[i * ldx + c] = (i > c) ? 0.0 : (((i == c) ? 1.0 : 0.0) - s) * dinv[i];
            __syncwarp();
        }
    }
}

// FP64 tensor-core MMA, mma.sync.aligned.m8n8k4 (row.col): lane = 4 g + t holds A[g][t],
// B[t][g] and D[g][2t], D[g][2t+1].
__device__ __forceinline__ void dmma_f64(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Small dense product on the FP64 tensor pipe: C (M x N) = op(A) (M x K) B (K x N), one 8 x 8
// output tile per warp at a time (tiles warp, warp + nwarps, ...), two accumulator chains over
// alternating k-steps of 4.  A(a, m) = TA ? A[m * lda + a] : A[a * lda + m]; B(m, c) =
// B[m * ldb + c]; out-of-range rows / columns / k read as zero.  epi(row, col, value) is
// called once per output inside M x N.  Every lane of a warp must call it (mma.sync).
template <bool TA, class Epi>
__device__ __forceinline__ void dmma_gemm(int M, int N, int K, const double *A, int lda,
                                          const double *B, int ldb, int warp, int nwarps, Epi epi) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int tn = (N + 7) >> 3, tiles = ((M + 7) >> 3) * tn;
    for (int tile = warp; tile < tiles; tile += nwarps) {
        const int a0 = (tile / tn) * 8, c0 = (tile % tn) * 8;
        const int ar = a0 + g, bc = c0 + g;
        const bool aok = ar < M, bok = bc < N;
        double d0 = 0.0, d1 = 0.0, e0 = 0.0, e1 = 0.0;
        int k0 = 0;
        for (; k0 + 8 <= K; k0 += 8) {
            const int ka = k0 + t, kb = ka + 4;
            const double a1 = aok ? (TA ? A[(size_t)ka * lda + ar] : A[(size_t)ar * lda + ka]) : 0.0;
            const double b1 = bok ? B[(size_t)ka * ldb + bc] : 0.0;
            const double a2 = aok ? (TA ? A[(size_t)kb * lda + ar] : A[(size_t)ar * lda + kb]) : 0.0;
            const double b2 = bok ? B[(size_t)kb * ldb + bc] : 0.0;
            dmma_f64(d0, d1, a1, b1);
            dmma_f64(e0, e1, a2, b2);
        }
        for (; k0 < K; k0 += 4) {
            const int ka = k0 + t;
            const bool kok = ka < K;
            const double a1 = (aok && kok) ? (TA ? A[(size_t)ka * lda + ar] : A[(size_t)ar * lda + ka]) : 0.0;
            const double b1 = (bok && kok) ? B[(size_t)ka * ldb + bc] : 0.0;
            dmma_f64(d0, d1, a1, b1);
        }
        d0 += e0;
        d1 += e1;
        const int r = a0 + g, c = c0 + 2 * t;
        if (r < M) {
            if (c < N) epi(r, c, d0);
            if (c + 1 < N) epi(r, c + 1, d1);
        }
    }
}

// ---------------------------------------------------------------------------------------
// Cholesky of G = R^T R (R upper), Rinv = R^{-1}, Racc <- R Racc (pass > 0) or R (pass 0).
// pass 0 may add the shift s = 11 (n p + p (p+1)) u trace(G) (shifted Cholesky-QR, Fukaya et
// al. 2020) when a pivot falls below 1e-13 of its column's norm^2; it then raises *shift_flag
// (the caller's third pass runs) and *reorth_flag reports a pivot below 1e-8.
//
// Right-looking elimination on [G | I] with unscaled pivot rows: step j subtracts
// (g_ja / d_j) x row j from every row a > j, in G's upper triangle (g_ab -= g_ja g_jb / d_j,
// j < a <= b) and in X (X_ac -= (g_ja / d_j) X_jc, c <= j).  At the end G = Lt D Lt^T with
// X = Lt^{-1}, so R = D^{1/2} Lt^T (R_ab = g_ab / sqrt(d_a)) and R^{-1} = Lt^{-T} D^{-1/2}
// (Rinv_ab = X_ba / sqrt(d_b)): the triangular inverse costs no serial substitution.
// Thread t owns column b = t % p and the rows a = t / p + k (nt / p); at step j it works on
// G if b > j and on X if b <= j, so both halves keep every thread busy.  One barrier per
// column; each thread's row loads are issued in batches of 8 before its stores.
// SM: X and R in shared memory (row stride p+1); otherwise in the global scratch gscr
// (2 p^2 doubles, row stride p).  g (p x (p+1)) is always in shared memory.
// ---------------------------------------------------------------------------------------
template <bool SM>
__global__ void __launch_bounds__(512)
chol3_kernel(int n, int p, const double *__restrict__ G, double *__restrict__ Rinv,
             double *__restrict__ Racc, double *__restrict__ gscr, int pass, SolveState *st,
             const int *gate, const int *gate2, int *shift_flag, int *reorth_flag,
             DevStatus *ds, int iter_tag) {
    {   // one decision per CTA: st->active may be cleared by the other stream mid-launch
        __shared__ int s_off;
        if (threadIdx.x == 0)
            s_off = ((st && !st->active) || (gate && *gate == 0) || (gate2 && *gate2 == 0)) ? 1 : 0;
        __syncthreads();
        if (s_off) return;
    }
    extern __shared__ __align__(128) double sm[];
    const int ld = p + 1;
    double *g = sm;                                   // p x ld
    double *dref = g + (size_t)p * ld;                // p: diagonal of G
    double *rs = dref + p;                            // p: 1 / sqrt(pivot)
    const int ldx = SM ? ld : p;
    double *X = SM ? rs + p : gscr;                   // p x ldx
    double *Rs = SM ? X + (size_t)p * ld : gscr + (size_t)p * p;
    __shared__ double s_trace;
    __shared__ double s_dinv[2];               // 1 / pivot of columns j (parity j & 1)
    const int tid = threadIdx.x, nt = blockDim.x;
    const int ngrp = nt / p;                  // row groups (>= 1 for p <= nt)
    const int bcol = tid % p, grp = tid / p;
    const bool owner = grp < ngrp;
    for (int e = tid; e < p * p; e += nt) {
        const int a = e / p, b = e - a * p;
        const double v = G[e];
        g[a * ld + b] = v;
        X[a * ldx + b] = (a == b) ? 1.0 : 0.0;
        if (a == b) dref[a] = v;
    }
    __syncthreads();
    if (tid < 32) {
        double t = 0.0;
        for (int i = tid; i < p; i += 32) t += dref[i];
        t = warp_sum(t);
        if (tid == 0) {
            s_trace = t;
            if (pass == 0 && shift_flag) *shift_flag = 0;
        }
    }
    __syncthreads();
    bool illcond = false;   // some pivot below 1e-8 of its column's norm^2 (attempt 0)
    int fail = 0;
    for (int attempt = 0; attempt < 2; attempt++) {
        const double shift = attempt == 0 ? 0.0
                                          : 11.0 * ((double)n * p + (double)p * (p + 1)) *
                                                1.1102230246251565e-16 * s_trace;
        if (attempt == 1) {
            for (int e = tid; e < p * p; e += nt) {
                const int a = e / p, b = e - a * p;
                g[a * ld + b] = G[e] + (a == b ? shift : 0.0);
                X[a * ldx + b] = (a == b) ? 1.0 : 0.0;
            }
        }
        if (tid == 0) s_dinv[0] = 1.0 / g[0];
        __syncthreads();
        fail = 0;
        // first row a > j of this thread's residue class (advanced incrementally)
        int a0 = grp;
        if (a0 < 1) a0 += ngrp;
        for (int j = 0; j < p; j++) {
            const double d = g[j * ld + j];
            const double ref = dref[j] + shift;
            if (attempt == 0 && !(d >= 1e-8 * ref)) illcond = true;
            if (!(d > 1e-13 * ref) || !(d > 0.0)) {
                fail = 1;
                break;
            }
            const double dinv = s_dinv[j & 1];
            if (owner) {
                const double *gj = g + (size_t)j * ld;
                if (bcol > j) {
                    const double f = gj[bcol] * dinv;
                    for (int a = a0; a <= bcol; a += 8 * ngrp) {
                        double rj[8], cur[8];
#pragma unroll
                        for (int i = 0; i < 8; i++) {
                            const int aa = a + i * ngrp;
                            if (aa <= bcol) {
                                rj[i] = gj[aa];
                                cur[i] = g[aa * ld + bcol];
                            }
                        }
#pragma unroll
                        for (int i = 0; i < 8; i++) {
                            const int aa = a + i * ngrp;
                            if (aa <= bcol) {
                                const double nv = cur[i] - rj[i] * f;
                                g[aa * ld + bcol] = nv;
                                // the next pivot: its thread publishes 1 / d_{j+1}
                                if (aa == j + 1 && bcol == j + 1) s_dinv[(j + 1) & 1] = 1.0 / nv;
                            }
                        }
                    }
                } else {
                    const double f = X[j * ldx + bcol] * dinv;
                    if (f != 0.0) {
                        for (int a = a0; a < p; a += 8 * ngrp) {
                            double rj[8], cur[8];
#pragma unroll
                            for (int i = 0; i < 8; i++) {
                                const int aa = a + i * ngrp;
                                if (aa < p) {
                                    rj[i] = gj[aa];
                                    cur[i] = X[aa * ldx + bcol];
                                }
                            }
#pragma unroll
                            for (int i = 0; i < 8; i++) {
                                const int aa = a + i * ngrp;
                                if (aa < p) X[aa * ldx + bcol] = cur[i] - rj[i] * f;
                            }
                        }
                    }
                }
            }
            if (a0 == j + 1) a0 += ngrp;
            __syncthreads();
        }
        if (attempt == 0 && tid == 0 && pass == 0 && reorth_flag)
            *reorth_flag = (fail || illcond) ? 1 : 0;
        if (!fail) break;
        if (tid == 0 && shift_flag) *shift_flag = 1;
        __syncthreads();
    }
    if (fail) {
        if (tid == 0) {
            if (st) st->qr_fail = 1;
            if (iter_tag >= 0 && st)
                atomicMin(&st->qr_fail_iter, iter_tag);
            else if (ds && atomicCAS(&ds->err, 0, (int)DEV_CHOL_FAIL) == 0)
                ds->aux = pass;
        }
        return;
    }
    for (int i = tid; i < p; i += nt) rs[i] = 1.0 / sqrt(g[i * ld + i]);
    __syncthreads();
    for (int e = tid; e < p * p; e += nt) {
        const int a = e / p, b = e - a * p;
        const double r = (b >= a) ? g[a * ld + b] * rs[a] : 0.0;
        Rs[a * ldx + b] = r;
        if (pass == 0) Racc[e] = r;
        Rinv[e] = (a <= b) ? X[b * ldx + a] * rs[b] : 0.0;
    }
    if (pass == 0) return;
    __syncthreads();
    for (int e = tid; e < p * p; e += nt) g[(e / p) * ld + e % p] = Racc[e];   // Racc staged
    __syncthreads();
    // Racc <- R Racc: (a, b) = sum_{c=a}^{b} R[a][c] Racc[c][b], four partial sums
    if (owner) {
        const int b = bcol;
        for (int a = grp; a < p; a += ngrp) {
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            int c = a;
            for (; c + 3 <= b; c += 4) {
                s0 += Rs[a * ldx + c] * g[c * ld + b];
                s1 += Rs[a * ldx + c + 1] * g[(c + 1) * ld + b];
                s2 += Rs[a * ldx + c + 2] * g[(c + 2) * ld + b];
                s3 += Rs[a * ldx + c + 3] * g[(c + 3) * ld + b];
            }
            for (; c <= b; c++) s0 += Rs[a * ldx + c] * g[c * ld + b];
            Racc[(size_t)a * p + b] = (b >= a) ? (s0 + s1) + (s2 + s3) : 0.0;
        }
    }
}

bpf_status launch_chol(bpf_ctx *ctx, int n, int p, const double *G, double *Rinv, double *Racc,
                       double *gscr, int pass, SolveState *st, const int *gate, const int *gate2,
                       int *shift_flag, int *reorth_flag, int iter_tag) {
    const int nt = p > 32 ? 512 : 256;
    const size_t one = sizeof(double) * p * (p + 1);
    const size_t extra = sizeof(double) * 2 * p;
    const bool sm = 3 * one + extra <= 200 * 1024;
    const size_t smem = (sm ? 3 * one : one) + extra;
    KScope ks(ctx, BPF_KC_CHOL, 0.0, 0.0, gate != nullptr || gate2 != nullptr);
    if (sm) {
        if (smem > 48 * 1024)
            BPF_CUDA(ctx, cudaFuncSetAttribute(chol3_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem));
        chol3_kernel<true><<<1, nt, smem, ctx->stream>>>(n, p, G, Rinv, Racc, gscr, pass, st, gate, gate2,
                                                         shift_flag, reorth_flag, ctx->dstat, iter_tag);
    } else {
        if (smem > 48 * 1024)
            BPF_CUDA(ctx, cudaFuncSetAttribute(chol3_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem));
        chol3_kernel<false><<<1, nt, smem, ctx->stream>>>(n, p, G, Rinv, Racc, gscr, pass, st, gate, gate2,
                                                          shift_flag, reorth_flag, ctx->dstat, iter_tag);
    }
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

// ---------------------------------------------------------------------------------------
// Block Hessenberg QR: apply Omega_0..Omega_{j-1} to block column j.
//
// Layout of the reflector storage HY, per block column i (hy_stride(p) doubles): Y_i
// (2p x (p+1), explicit: unit lower-triangular top, upper-triangular bottom), T_i
// (p x (p+1), upper) and R_ii^{-1} (p x p).  Omega_i^T = I - Y_i T_i^T Y_i^T acts on block
// rows i, i+1.
//
// One CTA per 8 columns of the block column; the 2p x 8 window S holds block rows i and i+1.
// Per step: W = Y_i^T S, W2 = T_i^T W, S -= Y_i W2 -- three small products on the FP64
// tensor pipe (mma.sync m8n8k4), one barrier each -- then block row i is final (written to R),
// the window slides down one block row and block row i+2 (loaded one step ahead) enters it.
// STAGED: Y_i and T_i reach shared memory by one bulk async copy per step, double buffered on
// two mbarriers (the copy of step i+1 is in flight during step i).
// ---------------------------------------------------------------------------------------
template <bool STAGED>
__global__ void __launch_bounds__(256)
hess_apply4_kernel(int p, int k, double *__restrict__ Rblk, const double *__restrict__ HY,
                   const SolveState *st, DevStatus *ds) {
    if (!st->active) return;
    const int j = k - 1;
    if (j <= 0) return;
    const int cb = blockIdx.x * 8;                 // first column of this CTA's 8
    const int ld = p + 1;
    const size_t hs = hy_stride(p);
    const size_t pp = (size_t)p * p;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int warp = tid >> 5, nw = nt >> 5;
    const int two_p = 2 * p;
    const unsigned blk = 3u * (unsigned)p * (unsigned)ld;   // doubles of [Y_i, T_i]
    extern __shared__ __align__(128) double sm[];
    double *stage = sm;                                      // STAGED: 2 x blk
    double *S = sm + (STAGED ? 2 * (size_t)blk : 0);         // window: 2p x 8
    double *W = S + (size_t)two_p * 8;                       // p x 8
    double *W2 = W + (size_t)p * 8;                          // p x 8
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int s_timeout;
    if (STAGED) {
        if (tid == 0) {
            s_timeout = 0;
            mbar_init(&bar[0], 1);
            mbar_init(&bar[1], 1);
            mbar_init_fence();
        }
        __syncthreads();
        if (tid == 0) {
            mbar_expect_tx(&bar[0], blk * 8u);
            bulk_g2s(stage, HY, blk * 8u, &bar[0]);
        }
    }
    // window: block rows 0 (rows 0..p-1) and 1 (rows p..2p-1), columns cb..cb+7
    for (int e = tid; e < two_p * 8; e += nt) {
        const int r = e >> 3, c = cb + (e & 7);
        const int br = r < p ? 0 : 1, rr = r < p ? r : r - p;
        S[e] = (c < p) ? Rblk[rblk_pos(br, j) * pp + (size_t)rr * p + c] : 0.0;
    }
    __syncthreads();
    for (int i = 0; i < j; i++) {
        // block row i+2 for the bottom half after this step (loaded ahead)
        double nxt[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int e = tid + q * nt;
            nxt[q] = 0.0;
            if (i + 2 <= j && e < p * 8) {
                const int c = cb + (e & 7);
                if (c < p) nxt[q] = Rblk[rblk_pos(i + 2, j) * pp + (size_t)(e >> 3) * p + c];
            }
        }
        const double *Y;
        if (STAGED) {
            if (!mbar_wait_bounded(&bar[i & 1], (unsigned)((i >> 1) & 1))) {
                if ((tid & 31) == 0) {
                    s_timeout = 1;
                    atomicCAS(&ds->err, 0, (int)DEV_BARRIER_TIMEOUT);
                }
            }
            Y = stage + (size_t)(i & 1) * blk;
        } else {
            Y = HY + (size_t)i * hs;
        }
        const double *T = Y + (size_t)two_p * ld;
        // W = Y^T S  (p x 8)
        dmma_gemm<true>(p, 8, two_p, Y, ld, S, 8, warp, nw, [&](int a, int c, double v) { W[a * 8 + c] = v; });
        __syncthreads();
        if (STAGED && tid == 0 && i + 1 < j && !s_timeout) {
            const int nb = (i + 1) & 1;
            mbar_expect_tx(&bar[nb], blk * 8u);
            bulk_g2s(stage + (size_t)nb * blk, HY + (size_t)(i + 1) * hs, blk * 8u, &bar[nb]);
        }
        if (STAGED && s_timeout) break;
        // W2 = T^T W
        dmma_gemm<true>(p, 8, p, T, ld, W, 8, warp, nw, [&](int a, int c, double v) { W2[a * 8 + c] = v; });
        __syncthreads();
        // S -= Y W2
        dmma_gemm<false>(two_p, 8, p, Y, ld, W2, 8, warp, nw, [&](int r, int c, double v) { S[r * 8 + c] -= v; });
        __syncthreads();
        // block row i is final; slide the window down one block row
        double *Ri = Rblk + rblk_pos(i, j) * pp;
        for (int e = tid; e < p * 8; e += nt) {
            const int c = cb + (e & 7);
            if (c < p) Ri[(size_t)(e >> 3) * p + c] = S[e];
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int e = tid + q * nt;
            if (e < p * 8) {
                S[e] = S[p * 8 + e];
                S[p * 8 + e] = nxt[q];
            }
        }
        __syncthreads();
    }
    // the top half is now block row j (R_jj before its factorization)
    if (!(STAGED && s_timeout)) {
        double *Rj = Rblk + rblk_pos(j, j) * pp;
        for (int e = tid; e < p * 8; e += nt) {
            const int c = cb + (e & 7);
            if (c < p) Rj[(size_t)(e >> 3) * p + c] = S[e];
        }
    }
}

// Row stride of the factor kernel's shared-memory matrices: p + 4 for p a multiple of 16 (the
// column sweep's 8-lane groups and the MMA fragment loads then hit distinct bank pairs), else
// p + 1; the global fallback works in place in HY (p + 1).
__host__ __device__ inline int factor_ld(int p, bool smem) {
    return (smem && p % 16 == 0) ? p + 4 : p + 1;
}

// ---------------------------------------------------------------------------------------
// Factor F = [R_jj; C] (2p x p) by Householder QR (dlarfg conventions), store Y_j, T_j (the
// compact-WY factor: T^{-1} = diag(1/tau) + strict_upper(Y^T Y), the UT transform of
// Joffrain et al.) and R_jj^{-1}, apply Omega_j^T to [Z_j; 0] and run the stopping test.
//
// C is upper triangular (it is the R factor of the Cholesky-QR of the new basis block), and
// the reflectors keep that structure: the reflector of column c has exactly p sub-diagonal
// rows, c+1..p-1 (top) and p..p+c (bottom).  Column loop: a group of G consecutive lanes
// (G a power of two) owns column c2 and splits the p reflector rows; per column c: partial
// dot products of column c against the group's column (||x||^2 for c2 = c, the update
// weights otherwise), a shuffle reduction inside the group, one barrier to publish ||x||^2,
// the reflector scalars (every thread, redundantly), the rank-1 update, a barrier.  The
// scaling of reflector c by 1/(alpha - beta) and its diagonal beta are written during
// column c+1 (nobody reads column c then).  The p x p products after the loop run as
// register-tiled dense products on the explicit Y.
// F_SMEM: F and the p x p work matrices live in shared memory; otherwise in HY / scr.
// ---------------------------------------------------------------------------------------
template <bool F_SMEM>
__global__ void __launch_bounds__(512)
hess_factor3_kernel(int p, int k, double *__restrict__ Rblk, double *__restrict__ HY,
                    double *__restrict__ tau_out, double *__restrict__ Z,
                    const double *__restrict__ Cm, SolveState *st, double *__restrict__ hist,
                    double *__restrict__ scr) {
    if (!st->active) return;
    extern __shared__ __align__(128) double sm[];
    const int gld = p + 1;            // row stride of Y_j, T_j in HY
    const int ld = factor_ld(p, F_SMEM);   // row stride of F and the work matrices
    const int j = k - 1;
    const size_t pp = (size_t)p * p;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    int G = 1;
    while (2 * G <= 32 && 2 * G * p <= nt) G *= 2;
    const int grp = tid & (G - 1), c2 = tid / G;
    const bool owner = c2 < p;
    double *Yg = HY + (size_t)j * hy_stride(p);     // Y_j: 2p x gld
    double *Tg = Yg + (size_t)2 * p * gld;          // T_j: p x gld
    double *Rig = Tg + (size_t)p * gld;             // R_jj^{-1}: p x p
    double *Rjj = Rblk + rblk_pos(j, j) * pp;
    double *Zj = Z + (size_t)j * pp;
    double *Zn = Z + (size_t)(j + 1) * pp;
    // shared: tau (p), dinv (p), then the F_SMEM matrices
    double *tau = sm;
    double *dinv = tau + p;
    double *F, *Tm, *W1, *Zs, *X;
    if (F_SMEM) {
        F = dinv + p;                    // 2p x ld
        Tm = F + (size_t)2 * p * ld;     // p x ld
        W1 = Tm + (size_t)p * ld;        // p x ld
        Zs = W1 + (size_t)p * ld;        // p x ld
        X = Zs + (size_t)p * ld;         // p x ld
    } else {
        F = Yg;
        Tm = Tg;
        W1 = scr;
        Zs = scr + (size_t)p * ld;
        X = scr + (size_t)2 * p * ld;
    }
    __shared__ double red[32];
    __shared__ double s_refl[3];   // tau, 1 / (alpha - beta), beta of the current column
    __shared__ int s_anyzero;
    for (int e = tid; e < p * p; e += nt) {
        const int a = e / p, b = e - a * p;
        F[a * ld + b] = Rjj[e];
        F[(a + p) * ld + b] = Cm[e];
        Zs[a * ld + b] = Zj[e];
    }
    if (tid == 0) s_anyzero = 0;
    __syncthreads();
    // the lanes of a group take interleaved rows r = c + 1 + grp + G i (conflict-free with
    // ld = p + 4 for p a multiple of 16)
    double prev_sc = 0.0, prev_beta = 0.0;
    for (int c = 0; c < p; c++) {
        const int r0 = c + 1 + grp;
        const int r1 = c + 1 + p;
        // deferred: finish reflector c-1 (scale, diagonal beta); its owners are idle now
        if (c > 0 && owner && c2 == c - 1) {
            for (int r = r0 - 1; r < r1 - 1; r += G) F[r * ld + c - 1] *= prev_sc;
            if (grp == 0) F[(c - 1) * ld + c - 1] = prev_beta;
        }
        // row c of column c2 before this column's update (group 0 rewrites it below)
        const double fcc2 = (owner && c2 > c) ? F[c * ld + c2] : 0.0;
        double d = 0.0;
        if (owner && c2 >= c) {
            double s0 = 0.0, s1 = 0.0;
            int r = r0;
            for (; r + G < r1; r += 2 * G) {
                s0 += F[r * ld + c] * F[r * ld + c2];
                s1 += F[(r + G) * ld + c] * F[(r + G) * ld + c2];
            }
            if (r < r1) s0 += F[r * ld + c] * F[r * ld + c2];
            d = s0 + s1;
        }
        for (int o = 1; o < G; o <<= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        // the reflector scalars, once, by the lane that owns (c, row group 0)
        if (owner && c2 == c && grp == 0) {
            const double alpha = F[c * ld + c];
            const double xn = sqrt(d);
            double tc0 = 0.0, sc0 = 0.0, beta0 = alpha;
            if (xn != 0.0) {
                beta0 = -copysign(hypot(alpha, xn), alpha);
                tc0 = (beta0 - alpha) / beta0;
                sc0 = 1.0 / (alpha - beta0);
            } else {
                s_anyzero = 1;
            }
            s_refl[0] = tc0;
            s_refl[1] = sc0;
            s_refl[2] = beta0;
            tau[c] = tc0;
        }
        __syncthreads();
        const double tc = s_refl[0], sc = s_refl[1], beta = s_refl[2];
        if (tc != 0.0 && owner && c2 > c) {
            const double w = tc * (fcc2 + sc * d);
            const double wsc = w * sc;
            for (int r = r0; r < r1; r += 8 * G) {
                double fc[8], cur[8];
#pragma unroll
                for (int i = 0; i < 8; i++)
                    if (r + i * G < r1) {
                        fc[i] = F[(r + i * G) * ld + c];
                        cur[i] = F[(r + i * G) * ld + c2];
                    }
#pragma unroll
                for (int i = 0; i < 8; i++)
                    if (r + i * G < r1) F[(r + i * G) * ld + c2] = cur[i] - wsc * fc[i];
            }
            if (grp == 0) F[c * ld + c2] = fcc2 - w;
        }
        prev_sc = sc;
        prev_beta = beta;
        __syncthreads();
    }
    if (owner && c2 == p - 1) {
        for (int r = p + grp; r < 2 * p; r += G) F[r * ld + p - 1] *= prev_sc;
        if (grp == 0) F[(p - 1) * ld + p - 1] = prev_beta;
    }
    __syncthreads();
    // R_jj <- upper triangle of the top block (kept in W1 for its inverse); 1 / diagonal
    for (int e = tid; e < p * p; e += nt) {
        const int a = e / p, b = e - a * p;
        const double v = (b >= a) ? F[a * ld + b] : 0.0;
        Rjj[e] = v;
        W1[a * ld + b] = v;
    }
    for (int i = tid; i < p; i += nt) dinv[i] = 1.0 / F[i * ld + i];
    if (tid < p) tau_out[tid] = tau[tid];
    __syncthreads();
    // F -> explicit Y (unit lower top, upper bottom)
    for (int e = tid; e < 2 * p * p; e += nt) {
        const int r = e / p, c = e - r * p;
        double *y = F + (size_t)r * ld + c;
        if (r < p) {
            if (r < c) *y = 0.0;
            else if (r == c) *y = 1.0;
        } else if (r - p > c) {
            *y = 0.0;
        }
    }
    // R_jj^{-1} (for the back substitution) into X
    upper_inverse(p, W1, ld, X, ld, dinv);
    __syncthreads();
    for (int e = tid; e < p * p; e += nt) Rig[e] = X[(e / p) * ld + e % p];
    // T^{-1} = diag(1/tau) + strict_upper(Y^T Y) into W1
    dmma_gemm<true>(p, p, 2 * p, F, ld, F, ld, warp, nw, [&](int a, int c, double v) {
        W1[a * ld + c] = (a < c) ? v : ((a == c) ? ((tau[c] != 0.0) ? 1.0 / tau[c] : 1.0) : 0.0);
    });
    __syncthreads();
    if (!s_anyzero) {
        for (int i = tid; i < p; i += nt) dinv[i] = tau[i];   // 1 / (1 / tau)
        __syncthreads();
        upper_inverse(p, W1, ld, Tm, ld, dinv);
    } else {
        // some reflector is the identity: the dlarft recurrence handles tau = 0 exactly
        if (tid == 0) {
            for (int c = 0; c < p; c++) {
                for (int a = 0; a < p; a++) Tm[a * ld + c] = 0.0;
                const double t = tau[c];
                for (int a = 0; a < c; a++) {
                    double s = 0.0;
                    for (int a2 = a; a2 < c; a2++) s += Tm[a * ld + a2] * W1[a2 * ld + c];
                    Tm[a * ld + c] = -t * s;
                }
                Tm[c * ld + c] = t;
            }
        }
    }
    __syncthreads();
    if (F_SMEM) {
        for (int e = tid; e < 2 * p * p; e += nt) {
            const int r = e / p, c = e - r * p;
            Yg[(size_t)r * gld + c] = F[r * ld + c];
        }
        for (int e = tid; e < p * p; e += nt) {
            const int a = e / p, c = e - a * p;
            Tg[(size_t)a * gld + c] = Tm[a * ld + c];
        }
    }
    // W1 = Y_top^T Z_j  (Y_top unit lower: rows m >= a)
    dmma_gemm<true>(p, p, p, F, ld, Zs, ld, warp, nw, [&](int a, int c, double v) { X[a * ld + c] = v; });
    __syncthreads();
    // W2 = T^T W1  (T upper: T^T rows m <= a; full range, zeros below)
    dmma_gemm<true>(p, p, p, Tm, ld, X, ld, warp, nw, [&](int a, int c, double v) { W1[a * ld + c] = v; });
    __syncthreads();
    // [Z_j; Lambda] = [Z_j; 0] - Y W2
    double ss = 0.0;
    dmma_gemm<false>(2 * p, p, p, F, ld, W1, ld, warp, nw, [&](int r, int c, double v) {
        if (r < p) {
            Zj[(size_t)r * p + c] = Zs[r * ld + c] - v;
        } else {
            Zn[(size_t)(r - p) * p + c] = -v;
            ss += v * v;
        }
    });
    ss = warp_sum(ss);
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
    KScope ks(ctx, BPF_KC_HESS);
    const int ld = p + 1;
    // apply: one CTA per 8 columns, 8 warps
    const size_t blk = sizeof(double) * 3 * (size_t)p * ld;
    const size_t small_a = sizeof(double) * (4 * (size_t)p * 8);
    const size_t staged_a = small_a + 2 * blk;
    const int ncb = (p + 7) / 8;
    if (staged_a <= 220 * 1024) {
        if (staged_a > 48 * 1024)
            BPF_CUDA(ctx, cudaFuncSetAttribute(hess_apply4_kernel<true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)staged_a));
        hess_apply4_kernel<true><<<ncb, 256, staged_a, ctx->stream>>>(p, k, Rblk, HY, st, ctx->dstat);
    } else {
        hess_apply4_kernel<false><<<ncb, 256, small_a, ctx->stream>>>(p, k, Rblk, HY, st, ctx->dstat);
    }
    BPF_LAUNCHED(ctx);
    const int nt = p > 64 ? 512 : 256;
    const size_t base_f = sizeof(double) * (2 * (size_t)p);
    const size_t smem_f = base_f + sizeof(double) * 6 * (size_t)p * factor_ld(p, true);
    if (smem_f <= 220 * 1024) {
        if (smem_f > 48 * 1024)
            BPF_CUDA(ctx, cudaFuncSetAttribute(hess_factor3_kernel<true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_f));
        hess_factor3_kernel<true><<<1, nt, smem_f, ctx->stream>>>(p, k, Rblk, HY, tau, Z, Cm, st, hist, scr);
    } else {
        if (base_f > 48 * 1024)
            BPF_CUDA(ctx, cudaFuncSetAttribute(hess_factor3_kernel<false>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)base_f));
        hess_factor3_kernel<false><<<1, nt, base_f, ctx->stream>>>(p, k, Rblk, HY, tau, Z, Cm, st, hist, scr);
    }
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

// ---------------------------------------------------------------------------------------
// Block back substitution R Y = Z (src/block_gmres.jl:366-375), right-looking, one launch per
// block row i (from the last): every CTA forms Y_i = R_ii^{-1} Z_i (the inverse was stored by
// the factor kernel; the product is redundant per CTA, p^3 FMAs), CTA 0 stores Y_i, and CTA
// b < i updates Z_b -= R_{b,i} Y_i.  Z_i is never written in step i.  Shared memory: R_ii^{-1},
// Z_i, Y_i and R_{b,i}, row stride p+1 (4 p (p+1) doubles; p <= 64).
// ---------------------------------------------------------------------------------------
// acc (4 x 4) = A[a0..a0+3][k0..p) B[k0..p)[c0..c0+3], A and B in shared memory.
__device__ __forceinline__ void mm_tile4(int p, const double *A, int lda, const double *B, int ldb,
                                         int a0, int c0, int k0, double acc[4][4]) {
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[i][q] = 0.0;
    if (a0 >= p || c0 >= p) return;
#pragma unroll 2
    for (int m = k0; m < p; m++) {
        double av[4], bv[4];
#pragma unroll
        for (int i = 0; i < 4; i++) av[i] = (a0 + i < p) ? A[(a0 + i) * lda + m] : 0.0;
#pragma unroll
        for (int q = 0; q < 4; q++) bv[q] = (c0 + q < p) ? B[m * ldb + c0 + q] : 0.0;
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][q] = fma(av[i], bv[q], acc[i][q]);
    }
}

__global__ void __launch_bounds__(256)
backsub3_kernel(int p, int i, const double *__restrict__ Rblk, const double *__restrict__ HY,
                double *__restrict__ Z, double *__restrict__ Y) {
    extern __shared__ __align__(128) double sm[];
    const size_t pp = (size_t)p * p;
    const int ld = p + 1;
    const int tid = threadIdx.x, nt = blockDim.x;
    double *Ri = sm, *Zi = sm + p * ld, *Yi = sm + 2 * p * ld, *Rb = sm + 3 * p * ld;
    const double *Rig = HY + (size_t)i * hy_stride(p) + (size_t)3 * p * ld;
    const int bb = blockIdx.x;
    const bool upd = bb < i;
    const double *Rbi = Rblk + rblk_pos(upd ? bb : 0, i) * pp;
    for (int e = tid; e < p * p; e += nt) {
        const int a = e / p, c = e - a * p;
        Ri[a * ld + c] = Rig[e];
        Zi[a * ld + c] = Z[(size_t)i * pp + e];
        if (upd) Rb[a * ld + c] = Rbi[e];
    }
    __syncthreads();
    // 16 x 16 threads, 4 x 4 outputs each (p <= 64)
    const int a0 = 4 * (tid >> 4), c0 = 4 * (tid & 15);
    double acc[4][4];
    mm_tile4(p, Ri, ld, Zi, ld, a0, c0, a0 < p ? a0 : 0, acc);   // R_ii^{-1} is upper
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int a = a0 + r, c = c0 + q;
            if (a < p && c < p) {
                Yi[a * ld + c] = acc[r][q];
                if (bb == 0) Y[(size_t)i * pp + (size_t)a * p + c] = acc[r][q];
            }
        }
    if (!upd) return;
    __syncthreads();
    mm_tile4(p, Rb, ld, Yi, ld, a0, c0, 0, acc);
    double *Zb = Z + (size_t)bb * pp;
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int a = a0 + r, c = c0 + q;
            if (a < p && c < p) Zb[(size_t)a * p + c] -= acc[r][q];
        }
}

// Fallback for p > 64, two launches per block row: one CTA solves Y_i = R_ii^{-1} Z_i by
// substitution on global (L1/L2) operands, then CTA b < i updates Z_b -= R_{b,i} Y_i.
__global__ void __launch_bounds__(256)
backsub_solve_global_kernel(int p, int i, const double *__restrict__ Rblk,
                            const double *__restrict__ Z, double *__restrict__ Y) {
    const size_t pp = (size_t)p * p;
    const int tid = threadIdx.x, nt = blockDim.x;
    const double *Rii = Rblk + rblk_pos(i, i) * pp;
    double *Ys = Y + (size_t)i * pp;
    for (int e = tid; e < p * p; e += nt) Ys[e] = Z[(size_t)i * pp + e];
    __syncthreads();
    const int L = (nt >= 4 * p) ? 4 : ((nt >= 2 * p) ? 2 : 1);
    const int q = tid % L;
    for (int c0 = 0; c0 < p; c0 += nt / L) {
        const int c = c0 + tid / L;
        const bool act = c < p;
        for (int r = p - 1; r >= 0; r--) {
            double s = 0.0;
            if (act)
                for (int m = r + 1 + q; m < p; m += L) s += Rii[r * p + m] * Ys[m * p + c];
            if (L >= 4) s += __shfl_xor_sync(0xffffffffu, s, 2);
            if (L >= 2) s += __shfl_xor_sync(0xffffffffu, s, 1);
            if (act && q == 0) Ys[r * p + c] = (Ys[r * p + c] - s) / Rii[r * p + r];
            __syncwarp();
        }
    }
}

__global__ void __launch_bounds__(256)
backsub_update_global_kernel(int p, int i, const double *__restrict__ Rblk,
                             const double *__restrict__ Y, double *__restrict__ Z) {
    const size_t pp = (size_t)p * p;
    const int bb = blockIdx.x;
    const double *Rbi = Rblk + rblk_pos(bb, i) * pp;
    const double *Ys = Y + (size_t)i * pp;
    double *Zb = Z + (size_t)bb * pp;
    for (int e = threadIdx.x; e < p * p; e += blockDim.x) {
        const int a = e / p, col = e % p;
        double s = 0.0;
        for (int c = 0; c < p; c++) s += Rbi[a * p + c] * Ys[c * p + col];
        Zb[e] -= s;
    }
}

bpf_status launch_backsub(bpf_ctx *ctx, int p, int k, const double *Rblk, const double *HY,
                          double *Z, double *Y) {
    KScope ks(ctx, BPF_KC_BACKSUB);
    const size_t smem = sizeof(double) * 4 * (size_t)p * (p + 1);
    const bool use_smem = p <= 64 && smem <= 220 * 1024;
    if (use_smem && smem > 48 * 1024)
        BPF_CUDA(ctx, cudaFuncSetAttribute(backsub3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
    // Every CTA of a launch only reads block row i of Z and writes rows b < i.
    for (int i = k - 1; i >= 0; i--) {
        if (use_smem) {
            backsub3_kernel<<<std::max(i, 1), 256, smem, ctx->stream>>>(p, i, Rblk, HY, Z, Y);
            BPF_LAUNCHED(ctx);
        } else {
            backsub_solve_global_kernel<<<1, 256, 0, ctx->stream>>>(p, i, Rblk, Z, Y);
            BPF_LAUNCHED(ctx);
            if (i > 0) {
                backsub_update_global_kernel<<<i, 256, 0, ctx->stream>>>(p, i, Rblk, Y, Z);
                BPF_LAUNCHED(ctx);
            }
        }
    }
    return BPF_SUCCESS;
}

}  // namespace bpf
