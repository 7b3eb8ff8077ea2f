// Batched block-GMRES: many independent systems (each its own Jacobian and right-hand-side
// block) solved by ILU(0)-preconditioned block-GMRES in ONE persistent launch, captured with the
// factorization in a CUDA graph.
//
// No counterpart in the reference, whose solvers take one system per call
// (src/block_gmres.jl:127-168); every step of a solve follows the single-system path of this
// library (which restates block_gmres!, src/block_gmres.jl:170-411): right preconditioning with
// ILU(0) (csrilu02 semantics, src/preconditioners_nvidia.jl:42-71), block Arnoldi, the block
// Hessenberg QR with the least-squares residual as the stopping test (eps = atol + rtol ||R0||,
// :223-231), back substitution and X update at the end of a cycle, restart when the basis is
// full.
//
// Design (B200):
//  * A work unit is one system and a slice of q <= 32 of its right-hand-side columns (block-GMRES
//    on the slice; a system with p columns gives ceil(p / q_max) units of nearly equal width).
//    One CTA runs a whole unit: every level of the triangular solves, the SpMM, the Gram
//    products, the Cholesky-QR and the Hessenberg update of an iteration.  Dependencies inside a
//    unit are __syncthreads (~ns) instead of grid barriers or kernel boundaries (~us), and units
//    never wait on one another: a CTA takes the next unit from an atomic counter, units sorted by
//    estimated cost (longest first), so the batch load-balances over the SMs.
//  * Each system is solved in a fill-reducing symmetric order (A_hat = A(perm, perm), minimum
//    degree by default): B is gathered through perm at the start of a unit and X scattered back
//    at its end, so no kernel of the iteration sees the permutation.
//  * Precision: the ILU(0) factors and triangular solves in FP32 (BPF_F32, the default) or FP64;
//    the SpMM, the orthogonalization, the Hessenberg least squares and X in FP64.  With FP32
//    factors the preconditioned blocks Z_j = M^{-1} V_j are kept (flexible GMRES), so X = X0 +
//    Z y satisfies the FP64 Arnoldi relation and the estimated residual is the true one.
//  * Block Gram-Schmidt twice (CGS2) and Cholesky-QR2 of the new block (diagonally scaled, with a
//    shifted first pass and a third pass when the block is ill-conditioned), all products on the
//    FP64 tensor pipe (DMMA m8n8k4).  The Hessenberg QR is per-column Householder (LAPACK
//    dlarfg convention), one group of lanes per column.
//  * No cross-CTA waits anywhere: nothing in the batched path can spin.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <type_traits>
#include <thread>
#include <vector>

#include "bpf_internal.cuh"
#include "ordering.cuh"
#include "prec.cuh"

namespace bpf {
namespace batch {

constexpr int kT = 256;        // threads per CTA
constexpr int kW = kT / 32;    // warps per CTA
constexpr int kQ = 32;         // widest column slice
constexpr int kLd = 32;        // leading dimension of the q x q scratch matrices in shared memory

// One system (device view).  Pattern, orderings and factor storage are read-only in the solve
// kernel; av / fv and the factor values are written by the factor kernel.
struct Sys {
    int n, nnz, p, pad;
    const int *rp, *ci, *diag;   // A_hat pattern (0-based)
    const int *amap;             // caller's entry k -> A_hat position
    const int *pp, *pdst, *psrc; // ILU(0) update pairs on A_hat's pattern
    const int *perm;             // perm[i] = caller's row of A_hat row i
    const double *vals;          // caller's values (device; re-read by every solve)
    double *av;                  // A_hat values
    double *fv;                  // ILU(0) factor values on A_hat's pattern
    TriKernelArgs L, U;          // level-sorted factors (L unit lower, U upper with 1/diag)
};

// One work unit: system `sys`, columns [col0, col0 + q), basis of m blocks.
struct Unit {
    int sys, col0, q, m;
    double *V;    // (m + 1) blocks n x q, row-major
    double *Z;    // m blocks: preconditioned basis
    double *Bh;   // the slice of B in A_hat's order
    double *Xh;   // the solution slice in A_hat's order
    double *R;    // Hessenberg column blocks: column j holds blocks 0..j+1 at (j(j+3)/2) q^2
    double *C2;   // (m + 1) q x q: second Gram-Schmidt pass coefficients
    double *HV;   // reflectors: column j at j (2 q + 2) q: v_c[t] at t q + c, tau_c at (q + 1) q + c,
                  // the compact-WY factor T (q x q, upper) at (q + 2) q + r q + c
    double *g;    // (m + 1) q x q: least-squares right-hand side (then y)
    double est;   // estimated cost (host ordering)
};

// Phases of a unit's solve whose SM cycles are counted (clock64 of thread 0).
enum Phase { PH_PREC = 0, PH_SPMM, PH_GRAM, PH_UPDATE, PH_CHOLQR, PH_HESS, PH_BACKSUB, PH_COUNT };

struct UnitOut {
    int niter;
    int status;    // bpf_solve_status, or -1 numeric failure, -2 zero pivot in the factorization
    int cycles;
    int pad;
    double rnorm0, rnorm;
    long long phase_cycles[PH_COUNT];
    long long total_cycles;
};

struct IO {
    const double *B;
    double *X;
    int ldb, ldx;
};

struct Cfg {
    double atol, rtol;
    int itmax;      // per unit (0: max(2 floor(n / q), 50))
    int f32;        // FP32 factors
};

struct Smem {
    double red[kW * kLd * kLd];   // Gram warp partials; aliased by the Hessenberg windows
    double gm[kLd * kLd];         // Gram / Cholesky work
    double r0[kLd * kLd];         // R of a Cholesky-QR pass
    double racc[kLd * kLd];       // accumulated R
    double rinv[kLd * kLd];       // R^{-1} of a pass
    double dsc[kLd];              // diagonal scaling
    double scal[kW];              // block reductions
    double zscale;                // scale of the stand-in columns of a zero right-hand side column
    unsigned zmask;               // zero columns of the unit's right-hand side
    int ival[3];
};

// Cycles since the last mark added to phase `ph` (thread 0 keeps the counts).
struct PhaseClock {
    long long t, acc[PH_COUNT];
    __device__ void start() {
        t = clock64();
        for (int i = 0; i < PH_COUNT; i++) acc[i] = 0;
    }
    __device__ __forceinline__ void mark(int ph) {
        if (threadIdx.x == 0) {
            const long long now = clock64();
            acc[ph] += now - t;
            t = now;
        }
    }
};

// Deterministic stand-in entry for row r of a zero right-hand-side column c: uniform in
// [-sqrt(3), sqrt(3)) (unit variance) from an integer hash of (r, c).
__device__ __forceinline__ double standin(int r, int c) {
    unsigned h = (unsigned)r * 0x9E3779B1u ^ ((unsigned)c + 1u) * 0x85EBCA77u;
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return ((double)h * (1.0 / 4294967296.0) - 0.5) * 3.4641016151377544;
}

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Sum of v over the CTA (every thread gets the total).
__device__ double cta_sum(double v, double *scratch) {
    v = warp_sum(v);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kW; w++) s += scratch[w];
    return s;
}

// ---------------------------------------------------------------------------------------
// q x q Gram product G = A^T B of two row-major n x q blocks: warps take runs of UF k-steps
// (4 rows each, all UF k-steps' fragments loaded before their DMMAs), every warp accumulates
// the whole (8 NT)^2 output, partials summed through shared memory.  dst (ld ldd) may be shared
// or global memory.
// ---------------------------------------------------------------------------------------
template <int NT>
__device__ void gram_t(const double *A, const double *B, int n, int q, double *red, double *dst, int ldd) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    constexpr int UF = NT == 1 ? 16 : (NT == 2 ? 8 : 4);
    constexpr int NC = NT <= 3 ? 2 : 1;   // independent accumulator chains (alternate k-steps)
    double acc[NC][NT][NT][2];
#pragma unroll
    for (int h = 0; h < NC; h++)
#pragma unroll
        for (int a = 0; a < NT; a++)
#pragma unroll
            for (int b = 0; b < NT; b++) acc[h][a][b][0] = acc[h][a][b][1] = 0.0;
    const int nks = (n + 3) >> 2;
    for (int ks0 = warp * UF; ks0 < nks; ks0 += kW * UF) {
        double af[UF][NT], bf[UF][NT];
#pragma unroll
        for (int u = 0; u < UF; u++) {
            const int r = (ks0 + u) * 4 + t;
#pragma unroll
            for (int i = 0; i < NT; i++) {
                const int c = i * 8 + g;
                const bool ok = r < n && c < q;
                af[u][i] = ok ? A[(size_t)r * q + c] : 0.0;
                bf[u][i] = ok ? B[(size_t)r * q + c] : 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < UF; u++)
#pragma unroll
            for (int a = 0; a < NT; a++)
#pragma unroll
                for (int b = 0; b < NT; b++)
                    dmma(acc[u % NC][a][b][0], acc[u % NC][a][b][1], af[u][a], bf[u][b]);
    }
    double *my = red + warp * kLd * kLd;
#pragma unroll
    for (int a = 0; a < NT; a++)
#pragma unroll
        for (int b = 0; b < NT; b++) {
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int h = 0; h < NC; h++) {
                s0 += acc[h][a][b][0];
                s1 += acc[h][a][b][1];
            }
            my[(a * 8 + g) * kLd + b * 8 + 2 * t] = s0;
            my[(a * 8 + g) * kLd + b * 8 + 2 * t + 1] = s1;
        }
    __syncthreads();
    for (int idx = threadIdx.x; idx < q * q; idx += kT) {
        const int a = idx / q, b = idx - a * q;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kW; w++) s += red[w * kLd * kLd + a * kLd + b];
        dst[a * ldd + b] = s;
    }
    __syncthreads();
}

// NB Gram products at once for narrow blocks (q <= 16): G_b = A_b^T B, A_b = A + b astr, in one
// sweep over the rows (B's fragments loaded once for all NB blocks), so a narrow unit pays one
// memory latency per NB basis blocks instead of one per block.  Partials of warp w, block b at
// red + (w NB + b) 256 (ld 16).
template <int NT, int NB>
__device__ void gram_nb_t(const double *A, size_t astr, const double *B, int n, int q, double *red, double *dst,
                          size_t dstr, int ldd) {
    static_assert(NT <= 2 && NB * kW * 256 <= kW * kLd * kLd, "partials must fit the reduction area");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    constexpr int UF = NT == 1 ? 16 : 8;
    constexpr int NC = 2;
    double acc[NB][NC][NT][NT][2];
#pragma unroll
    for (int k = 0; k < NB; k++)
#pragma unroll
        for (int h = 0; h < NC; h++)
#pragma unroll
            for (int a = 0; a < NT; a++)
#pragma unroll
                for (int b = 0; b < NT; b++) acc[k][h][a][b][0] = acc[k][h][a][b][1] = 0.0;
    const int nks = (n + 3) >> 2;
    for (int ks0 = warp * UF; ks0 < nks; ks0 += kW * UF) {
        double af[NB][UF][NT], bf[UF][NT];
#pragma unroll
        for (int u = 0; u < UF; u++) {
            const int r = (ks0 + u) * 4 + t;
#pragma unroll
            for (int i = 0; i < NT; i++) {
                const int c = i * 8 + g;
                const bool ok = r < n && c < q;
                bf[u][i] = ok ? B[(size_t)r * q + c] : 0.0;
#pragma unroll
                for (int k = 0; k < NB; k++) af[k][u][i] = ok ? A[k * astr + (size_t)r * q + c] : 0.0;
            }
        }
#pragma unroll
        for (int k = 0; k < NB; k++)
#pragma unroll
            for (int u = 0; u < UF; u++)
#pragma unroll
                for (int a = 0; a < NT; a++)
#pragma unroll
                    for (int b = 0; b < NT; b++)
                        dmma(acc[k][u % NC][a][b][0], acc[k][u % NC][a][b][1], af[k][u][a], bf[u][b]);
    }
#pragma unroll
    for (int k = 0; k < NB; k++) {
        double *my = red + (warp * NB + k) * 256;
#pragma unroll
        for (int a = 0; a < NT; a++)
#pragma unroll
            for (int b = 0; b < NT; b++) {
                my[(a * 8 + g) * 16 + b * 8 + 2 * t] = acc[k][0][a][b][0] + acc[k][1][a][b][0];
                my[(a * 8 + g) * 16 + b * 8 + 2 * t + 1] = acc[k][0][a][b][1] + acc[k][1][a][b][1];
            }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < NB * q * q; idx += kT) {
        const int k = idx / (q * q), r = idx - k * q * q;
        const int a = r / q, b = r - a * q;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kW; w++) s += red[(w * NB + k) * 256 + a * 16 + b];
        dst[k * dstr + a * ldd + b] = s;
    }
    __syncthreads();
}

// Gram products of blocks whose width q = 8 F + R has a thin rim (R columns past F full 8-wide
// tiles): the F x F full tiles on the DMMA pipe, the rim (G[0:8F, 8F:q], G[8F:q, 0:8F] and the
// R x R corner) with FP64 FMAs, instead of padding q to 8 (F + 1) columns, whose DMMA work is
// (F + 1)^2 / F^2 of the full tiles' (4x at q = 9).  Used for R = 1 (q = 9, 17, 25): measured
// on the 512-grid batch, the longest units with q = 9 and 17 ran 5 % faster; with R = 2 and 3
// the rim's loads and FMAs cost more than the padding they save (units with q = 26, 27 slower).  Lane (g, t) holds rows r_t of
// column 8 i + g of every full tile, as for the DMMA fragments, and loads the rim values of its
// row itself (the same cache lines); its rim partials are summed over t by shuffles, and over
// the warps through shared memory as the tiles are.  NB blocks A_b = A + b astr per sweep (the
// new block's fragments loaded once for all of them); partials of warp w, block b at
// red + (w NB + b) ld^2, ld = kLd for NB = 1 and 16 otherwise (q <= 16 then).
template <int F, int R, int NB>
__device__ void gram_rim_t(const double *A, size_t astr, const double *B, int n, int q, double *red,
                           double *dst, size_t dstr, int ldd) {
    constexpr int LD = NB == 1 ? kLd : 16;
    static_assert(8 * F + R <= LD && NB * kW * LD * LD <= kW * kLd * kLd, "partials must fit the reduction area");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    constexpr int UF = (F == 1 && NB == 1) ? 8 : (F * NB <= 2 ? 4 : 2);
    constexpr int NC = F <= 2 ? 2 : 1;
    double acc[NB][NC][F][F][2];
    double ra[NB][F][R], rb[NB][F][R], rc[NB][R][R];
#pragma unroll
    for (int k = 0; k < NB; k++) {
#pragma unroll
        for (int h = 0; h < NC; h++)
#pragma unroll
            for (int a = 0; a < F; a++)
#pragma unroll
                for (int b = 0; b < F; b++) acc[k][h][a][b][0] = acc[k][h][a][b][1] = 0.0;
#pragma unroll
        for (int i = 0; i < F; i++)
#pragma unroll
            for (int r = 0; r < R; r++) ra[k][i][r] = rb[k][i][r] = 0.0;
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
            for (int c = 0; c < R; c++) rc[k][r][c] = 0.0;
    }
    const int nks = (n + 3) >> 2;
    for (int ks0 = warp * UF; ks0 < nks; ks0 += kW * UF) {
        double af[NB][UF][F], bf[UF][F], ar[NB][UF][R], br[UF][R];
#pragma unroll
        for (int u = 0; u < UF; u++) {
            const int r = (ks0 + u) * 4 + t;
            const bool ok = r < n;
            const size_t ro = (size_t)r * q;
#pragma unroll
            for (int i = 0; i < F; i++) {
                bf[u][i] = ok ? B[ro + i * 8 + g] : 0.0;
#pragma unroll
                for (int k = 0; k < NB; k++) af[k][u][i] = ok ? A[k * astr + ro + i * 8 + g] : 0.0;
            }
#pragma unroll
            for (int c = 0; c < R; c++) {
                br[u][c] = ok ? B[ro + 8 * F + c] : 0.0;
#pragma unroll
                for (int k = 0; k < NB; k++) ar[k][u][c] = ok ? A[k * astr + ro + 8 * F + c] : 0.0;
            }
        }
#pragma unroll
        for (int k = 0; k < NB; k++)
#pragma unroll
            for (int u = 0; u < UF; u++) {
#pragma unroll
                for (int a = 0; a < F; a++)
#pragma unroll
                    for (int b = 0; b < F; b++)
                        dmma(acc[k][u % NC][a][b][0], acc[k][u % NC][a][b][1], af[k][u][a], bf[u][b]);
#pragma unroll
                for (int i = 0; i < F; i++)
#pragma unroll
                    for (int c = 0; c < R; c++) {
                        ra[k][i][c] = fma(af[k][u][i], br[u][c], ra[k][i][c]);
                        rb[k][i][c] = fma(ar[k][u][c], bf[u][i], rb[k][i][c]);
                    }
#pragma unroll
                for (int r = 0; r < R; r++)
#pragma unroll
                    for (int c = 0; c < R; c++) rc[k][r][c] = fma(ar[k][u][r], br[u][c], rc[k][r][c]);
            }
    }
    // rim partials: sum over the four row lanes t of each g
#pragma unroll
    for (int k = 0; k < NB; k++) {
#pragma unroll
        for (int i = 0; i < F; i++)
#pragma unroll
            for (int c = 0; c < R; c++) {
                ra[k][i][c] += __shfl_xor_sync(0xffffffffu, ra[k][i][c], 1);
                ra[k][i][c] += __shfl_xor_sync(0xffffffffu, ra[k][i][c], 2);
                rb[k][i][c] += __shfl_xor_sync(0xffffffffu, rb[k][i][c], 1);
                rb[k][i][c] += __shfl_xor_sync(0xffffffffu, rb[k][i][c], 2);
            }
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
            for (int c = 0; c < R; c++) {
                rc[k][r][c] += __shfl_xor_sync(0xffffffffu, rc[k][r][c], 1);
                rc[k][r][c] += __shfl_xor_sync(0xffffffffu, rc[k][r][c], 2);
            }
        double *my = red + (warp * NB + k) * LD * LD;
#pragma unroll
        for (int a = 0; a < F; a++)
#pragma unroll
            for (int b = 0; b < F; b++) {
                double s0 = 0.0, s1 = 0.0;
#pragma unroll
                for (int h = 0; h < NC; h++) {
                    s0 += acc[k][h][a][b][0];
                    s1 += acc[k][h][a][b][1];
                }
                my[(a * 8 + g) * LD + b * 8 + 2 * t] = s0;
                my[(a * 8 + g) * LD + b * 8 + 2 * t + 1] = s1;
            }
        if (t == 0) {
#pragma unroll
            for (int i = 0; i < F; i++)
#pragma unroll
                for (int c = 0; c < R; c++) {
                    my[(i * 8 + g) * LD + 8 * F + c] = ra[k][i][c];
                    my[(8 * F + c) * LD + i * 8 + g] = rb[k][i][c];
                }
            if (g == 0) {
#pragma unroll
                for (int r = 0; r < R; r++)
#pragma unroll
                    for (int c = 0; c < R; c++) my[(8 * F + r) * LD + 8 * F + c] = rc[k][r][c];
            }
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < NB * q * q; idx += kT) {
        const int k = idx / (q * q), rr = idx - k * q * q;
        const int a = rr / q, b = rr - a * q;
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < kW; w++) sum += red[(w * NB + k) * LD * LD + a * LD + b];
        dst[k * dstr + a * ldd + b] = sum;
    }
    __syncthreads();
}

template <int R>
__device__ __forceinline__ void gram_rim(const double *V, size_t vstr, int nblk, const double *W, int n, int q,
                                         double *red, double *dst, size_t dstr, int ldd) {
    const int F = q >> 3;
    int i = 0;
    if (F == 1) {
        for (; i + 2 <= nblk; i += 2) gram_rim_t<1, R, 2>(V + i * vstr, vstr, W, n, q, red, dst + i * dstr, dstr, ldd);
    }
    for (; i < nblk; i++) {
        switch (F) {
            case 1: gram_rim_t<1, R, 1>(V + i * vstr, vstr, W, n, q, red, dst + i * dstr, dstr, ldd); break;
            case 2: gram_rim_t<2, R, 1>(V + i * vstr, vstr, W, n, q, red, dst + i * dstr, dstr, ldd); break;
            default: gram_rim_t<3, R, 1>(V + i * vstr, vstr, W, n, q, red, dst + i * dstr, dstr, ldd); break;
        }
    }
}

// G_i = V_i^T W for i < nblk (V_i = V + i vstr) into dst + i dstr (ld ldd).
__device__ __noinline__ void gram(const double *V, size_t vstr, int nblk, const double *W, int n, int q,
                                  double *red, double *dst, size_t dstr, int ldd) {
    if (q > 8 && q < 32 && (q & 7) == 1) {
        gram_rim<1>(V, vstr, nblk, W, n, q, red, dst, dstr, ldd);
        return;
    }
    int i = 0;
    if (q <= 8) {
        for (; i + 4 <= nblk; i += 4) gram_nb_t<1, 4>(V + i * vstr, vstr, W, n, q, red, dst + i * dstr, dstr, ldd);
    } else if (q <= 16) {
        for (; i + 2 <= nblk; i += 2) gram_nb_t<2, 2>(V + i * vstr, vstr, W, n, q, red, dst + i * dstr, dstr, ldd);
    }
    for (; i < nblk; i++) {
        switch ((q + 7) >> 3) {
            case 1: gram_t<1>(V + i * vstr, W, n, q, red, dst + i * dstr, ldd); break;
            case 2: gram_t<2>(V + i * vstr, W, n, q, red, dst + i * dstr, ldd); break;
            case 3: gram_t<3>(V + i * vstr, W, n, q, red, dst + i * dstr, ldd); break;
            default: gram_t<4>(V + i * vstr, W, n, q, red, dst + i * dstr, ldd); break;
        }
    }
}

// ---------------------------------------------------------------------------------------
// W (n x q) = [W] + sign * sum_{i < nb} A_i C_i, A_i = A + i astr (row-major n x q), C_i = C + i
// cstr (q x q, row stride ldc).  A warp owns 8 MT consecutive rows at a time; for each block i it
// loads the fragments of all of the block's k-steps (MT + NT per k-step) before their DMMAs, so
// a block costs one memory latency.  W may be A itself (nb = 1, init = false: the warp reads its
// rows before it writes them).  No barrier inside.
// ---------------------------------------------------------------------------------------
template <int NT>
__device__ void update_t(double *W, const double *A, size_t astr, const double *C, size_t cstr, int ldc,
                         int nb, int n, int q, double sign, bool init) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    constexpr int MT = NT == 1 ? 8 : (NT == 2 ? 4 : (NT == 3 ? 4 : 2));
    constexpr int KK = 2 * NT;   // k-steps of 4 columns in a block of q <= 8 NT columns
    constexpr int RT = 8 * MT;
    for (int r0 = warp * RT; r0 < n; r0 += kW * RT) {
        double acc[MT][NT][2];
#pragma unroll
        for (int m = 0; m < MT; m++)
#pragma unroll
            for (int b = 0; b < NT; b++) {
                const int r = r0 + m * 8 + g, c = b * 8 + 2 * t;
                acc[m][b][0] = (init && r < n && c < q) ? W[(size_t)r * q + c] : 0.0;
                acc[m][b][1] = (init && r < n && c + 1 < q) ? W[(size_t)r * q + c + 1] : 0.0;
            }
        int i0 = 0;
        if constexpr (NT <= 2) {
            // narrow blocks: two blocks' fragments loaded before their DMMAs (one memory
            // latency per two blocks)
            for (; i0 + 2 <= nb; i0 += 2) {
                double bf[2][KK][NT], af[2][KK][MT];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const double *Ai = A + (i0 + h) * astr;
                    const double *Ci = C + (i0 + h) * cstr;
#pragma unroll
                    for (int k = 0; k < KK; k++) {
                        const int kc = k * 4 + t;
#pragma unroll
                        for (int b = 0; b < NT; b++) {
                            const int c = b * 8 + g;
                            bf[h][k][b] = (kc < q && c < q) ? Ci[kc * ldc + c] : 0.0;
                        }
#pragma unroll
                        for (int m = 0; m < MT; m++) {
                            const int r = r0 + m * 8 + g;
                            af[h][k][m] = (kc < q && r < n) ? Ai[(size_t)r * q + kc] : 0.0;
                        }
                    }
                }
#pragma unroll
                for (int h = 0; h < 2; h++)
#pragma unroll
                    for (int k = 0; k < KK; k++)
#pragma unroll
                        for (int m = 0; m < MT; m++)
#pragma unroll
                            for (int b = 0; b < NT; b++)
                                dmma(acc[m][b][0], acc[m][b][1], sign * af[h][k][m], bf[h][k][b]);
            }
        }
        for (int i = i0; i < nb; i++) {
            const double *Ai = A + i * astr;
            const double *Ci = C + i * cstr;
            double bf[KK][NT], af[KK][MT];
#pragma unroll
            for (int k = 0; k < KK; k++) {
                const int kc = k * 4 + t;
#pragma unroll
                for (int b = 0; b < NT; b++) {
                    const int c = b * 8 + g;
                    bf[k][b] = (kc < q && c < q) ? Ci[kc * ldc + c] : 0.0;
                }
#pragma unroll
                for (int m = 0; m < MT; m++) {
                    const int r = r0 + m * 8 + g;
                    af[k][m] = (kc < q && r < n) ? Ai[(size_t)r * q + kc] : 0.0;
                }
            }
#pragma unroll
            for (int k = 0; k < KK; k++)
#pragma unroll
                for (int m = 0; m < MT; m++)
#pragma unroll
                    for (int b = 0; b < NT; b++) dmma(acc[m][b][0], acc[m][b][1], sign * af[k][m], bf[k][b]);
        }
#pragma unroll
        for (int m = 0; m < MT; m++)
#pragma unroll
            for (int b = 0; b < NT; b++) {
                const int r = r0 + m * 8 + g, c = b * 8 + 2 * t;
                if (r < n && c < q) W[(size_t)r * q + c] = acc[m][b][0];
                if (r < n && c + 1 < q) W[(size_t)r * q + c + 1] = acc[m][b][1];
            }
    }
}

// The block update for widths q = 8 F + R with a thin rim (used for R = 1): the F x F full tiles of
// every block product on the DMMA pipe (2 F k-steps), the rim with FP64 FMAs instead of padding q
// to 8 (F + 1): the K rim (columns 8F .. q of A_i times rows 8F .. q of C_i) into the full output
// tiles, and the output rim (columns 8F .. q of W) as per-lane partial dot products over the
// lane's k-steps (k = t mod 4, the DMMA A-fragment layout) plus the corner terms of k = 8F + t,
// summed over the four lanes t of a row by shuffles after the last block.  Every lane has loaded
// its rows of A before any lane stores (the shuffles order them), so W may be A itself (nb = 1,
// init = false), as in update_t.
template <int F, int R>
__device__ void update_rim_t(double *W, const double *A, size_t astr, const double *C, size_t cstr, int ldc,
                             int nb, int n, int q, double sign, bool init) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    constexpr int MT = F == 1 ? 4 : 2;
    constexpr int KK = 2 * F;
    constexpr int RT = 8 * MT;
    for (int r0 = warp * RT; r0 < n; r0 += kW * RT) {
        double acc[MT][F][2], pr[MT][R];
#pragma unroll
        for (int m = 0; m < MT; m++) {
            const int r = r0 + m * 8 + g;
#pragma unroll
            for (int b = 0; b < F; b++) {
                const int c = b * 8 + 2 * t;
                acc[m][b][0] = (init && r < n) ? W[(size_t)r * q + c] : 0.0;
                acc[m][b][1] = (init && r < n) ? W[(size_t)r * q + c + 1] : 0.0;
            }
#pragma unroll
            for (int c = 0; c < R; c++) pr[m][c] = 0.0;
        }
        for (int i = 0; i < nb; i++) {
            const double *Ai = A + i * astr;
            const double *Ci = C + i * cstr;
            double bf[KK][F], af[KK][MT], ar[MT][R];
#pragma unroll
            for (int k = 0; k < KK; k++) {
                const int kc = k * 4 + t;
#pragma unroll
                for (int b = 0; b < F; b++) bf[k][b] = Ci[kc * ldc + b * 8 + g];
#pragma unroll
                for (int m = 0; m < MT; m++) {
                    const int r = r0 + m * 8 + g;
                    af[k][m] = r < n ? Ai[(size_t)r * q + kc] : 0.0;
                }
            }
#pragma unroll
            for (int m = 0; m < MT; m++) {
                const int r = r0 + m * 8 + g;
#pragma unroll
                for (int c = 0; c < R; c++) ar[m][c] = r < n ? sign * Ai[(size_t)r * q + 8 * F + c] : 0.0;
            }
#pragma unroll
            for (int k = 0; k < KK; k++)
#pragma unroll
                for (int m = 0; m < MT; m++)
#pragma unroll
                    for (int b = 0; b < F; b++) dmma(acc[m][b][0], acc[m][b][1], sign * af[k][m], bf[k][b]);
            // K rim into the full tiles: rows 8F + c of C_i
#pragma unroll
            for (int c = 0; c < R; c++) {
                const double *crow = Ci + (8 * F + c) * ldc + 2 * t;
#pragma unroll
                for (int b = 0; b < F; b++) {
                    const double c0 = crow[b * 8], c1 = crow[b * 8 + 1];
#pragma unroll
                    for (int m = 0; m < MT; m++) {
                        acc[m][b][0] = fma(ar[m][c], c0, acc[m][b][0]);
                        acc[m][b][1] = fma(ar[m][c], c1, acc[m][b][1]);
                    }
                }
            }
            // output rim: this lane's k-steps (columns 4 k + t of A_i) and corner row 8F + t
#pragma unroll
            for (int c = 0; c < R; c++) {
#pragma unroll
                for (int k = 0; k < KK; k++) {
                    const double cv = Ci[(k * 4 + t) * ldc + 8 * F + c];
#pragma unroll
                    for (int m = 0; m < MT; m++) pr[m][c] = fma(sign * af[k][m], cv, pr[m][c]);
                }
                if (t < R) {
                    const double cv = Ci[(8 * F + t) * ldc + 8 * F + c];
#pragma unroll
                    for (int m = 0; m < MT; m++) {
                        double a = 0.0;
#pragma unroll
                        for (int e = 0; e < R; e++)
                            if (e == t) a = ar[m][e];
                        pr[m][c] = fma(a, cv, pr[m][c]);
                    }
                }
            }
        }
#pragma unroll
        for (int m = 0; m < MT; m++)
#pragma unroll
            for (int c = 0; c < R; c++) {
                pr[m][c] += __shfl_xor_sync(0xffffffffu, pr[m][c], 1);
                pr[m][c] += __shfl_xor_sync(0xffffffffu, pr[m][c], 2);
            }
#pragma unroll
        for (int m = 0; m < MT; m++) {
            const int r = r0 + m * 8 + g;
            if (r >= n) continue;
#pragma unroll
            for (int b = 0; b < F; b++) {
                const int c = b * 8 + 2 * t;
                W[(size_t)r * q + c] = acc[m][b][0];
                W[(size_t)r * q + c + 1] = acc[m][b][1];
            }
            if (t == 0) {
#pragma unroll
                for (int c = 0; c < R; c++) {
                    double *w = W + (size_t)r * q + 8 * F + c;
                    *w = (init ? *w : 0.0) + pr[m][c];
                }
            }
        }
    }
}

template <int R>
__device__ __forceinline__ void update_rim(double *W, const double *A, size_t astr, const double *C, size_t cstr,
                                           int ldc, int nb, int n, int q, double sign, bool init) {
    switch (q >> 3) {
        case 1: update_rim_t<1, R>(W, A, astr, C, cstr, ldc, nb, n, q, sign, init); break;
        case 2: update_rim_t<2, R>(W, A, astr, C, cstr, ldc, nb, n, q, sign, init); break;
        default: update_rim_t<3, R>(W, A, astr, C, cstr, ldc, nb, n, q, sign, init); break;
    }
}

__device__ __noinline__ void update(double *W, const double *A, size_t astr, const double *C, size_t cstr,
                                    int ldc, int nb, int n, int q, double sign, bool init) {
    if (q > 8 && q < 32 && (q & 7) == 1) {
        update_rim<1>(W, A, astr, C, cstr, ldc, nb, n, q, sign, init);
        return;
    }
    switch ((q + 7) >> 3) {
        case 1: update_t<1>(W, A, astr, C, cstr, ldc, nb, n, q, sign, init); break;
        case 2: update_t<2>(W, A, astr, C, cstr, ldc, nb, n, q, sign, init); break;
        case 3: update_t<3>(W, A, astr, C, cstr, ldc, nb, n, q, sign, init); break;
        default: update_t<4>(W, A, astr, C, cstr, ldc, nb, n, q, sign, init); break;
    }
}

// The same update with global coefficients C staged through shared memory `stage` (capacity
// `cap` doubles) in chunks of blocks: every row tile of every warp reads each coefficient block,
// so they come from shared memory (row stride q + 1, no bank conflicts) instead of L1 / L2.  W is
// read and written once per chunk.  Collective: every thread of the CTA calls it.
__device__ __noinline__ void update_staged(double *W, const double *A, size_t astr, const double *C, size_t cstr,
                                           int nb, int n, int q, double sign, bool init, double *stage, int cap) {
    const int lds = q + 1, per = q * lds;
    const int chunk = max(1, cap / per);
    for (int i0 = 0; i0 < nb; i0 += chunk) {
        const int nc = min(chunk, nb - i0);
        __syncthreads();
        for (int idx = threadIdx.x; idx < nc * q * q; idx += kT) {
            const int b = idx / (q * q), r = idx - b * q * q;
            const int a = r / q, c = r - a * q;
            stage[b * per + a * lds + c] = C[(size_t)(i0 + b) * cstr + (size_t)a * q + c];
        }
        __syncthreads();
        update(W, A + (size_t)i0 * astr, astr, stage, per, lds, nc, n, q, sign, init || i0 > 0);
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------------------
// Sparse kernels: a group of 8 lanes per row (32 rows in flight per CTA), lane l holding
// columns l, l + 8, ... (CPL of them) of the row-major block, the row's (column, value) pairs
// broadcast by shuffles; the next row's metadata is loaded before the current row is worked.
// ---------------------------------------------------------------------------------------
constexpr int kG = 8;
constexpr int kNG = kT / kG;

template <int CPL>
__device__ void spmm_t(const int *__restrict__ rp, const int *__restrict__ ci, const double *__restrict__ av,
                       int n, int q, const double *X, double *Y, const double *Bsub) {
    const int lane = threadIdx.x & 31, gl = lane & (kG - 1);
    const unsigned gmask = 0xffu << (lane & ~(kG - 1));
    int i = threadIdx.x / kG;
    int rs = i < n ? __ldg(rp + i) : 0, re = i < n ? __ldg(rp + i + 1) : 0;
    for (; i < n; i += kNG) {
        const int in = i + kNG;
        const int rsn = in < n ? __ldg(rp + in) : 0, ren = in < n ? __ldg(rp + in + 1) : 0;
        double acc[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) acc[c] = 0.0;
        for (int kb = rs; kb < re; kb += kG) {
            const int k = kb + gl;
            int col = 0;
            double a = 0.0;
            if (k < re) {
                col = __ldg(ci + k);
                a = __ldg(av + k);
            }
            const int cnt = min(kG, re - kb);
            #pragma unroll 4   // several entries' loads in flight; same summation order
            for (int e = 0; e < cnt; e++) {
                const int cs = __shfl_sync(gmask, col, e, kG);
                const double as = __shfl_sync(gmask, a, e, kG);
                const double *xr = X + (size_t)cs * q + gl;
#pragma unroll
                for (int c = 0; c < CPL; c++)
                    if (gl + c * kG < q) acc[c] += as * xr[c * kG];
            }
        }
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            const int col = gl + c * kG;
            if (col < q) Y[(size_t)i * q + col] = Bsub ? Bsub[(size_t)i * q + col] - acc[c] : acc[c];
        }
        rs = rsn;
        re = ren;
    }
}

__device__ __forceinline__ void cpa4(void *smem, const void *gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem) : "memory");
}
__device__ __forceinline__ void cpa8(void *smem, const void *gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Per-group staging of the sweeps' coming positions in shared memory (three levels in flight):
// the row metadata (row, entry range) and the first kG (column, value) pairs and inverted
// diagonal of each group's first position of a level.
template <typename TF>
struct SweepStage {
    int meta[3][kNG][3];
    int col[3][kNG][kG];
    TF val[3][kNG][kG];
    TF dinv[3][kNG];
};

// One triangular factor, every level, a __syncthreads between levels.  Y rows of earlier levels
// are read with plain loads (written by this CTA before the barrier).  A group of kG lanes takes
// positions grp, grp + kNG, ... of each level.  Measured on the batched configuration, a level
// used to wait for two L2 round trips besides its gathers: the row metadata, then the row's
// entries (whose addresses need the metadata).  Here they come two and one levels ahead, by
// asynchronous copies into the shared staging St (a barrier does not wait for them, and they
// hold no registers): at the start of level l each group issues the entries of its first
// position of level l + 1 (whose metadata arrived during level l - 1) and the metadata of its
// first position of level l + 2; every thread waits for its own copies at the end of the level,
// before the barrier that makes them visible to its group.  A level then waits for the gathers
// of solved rows (and, in parallel, its rows' right-hand sides) alone.  Positions past the first
// of a level wider than kNG groups are loaded directly, one ahead.  The summation order is the
// same as one row at a time.
template <int CPL, typename TF>
__device__ void trsv_t(const TriKernelArgs &T, int q, const double *X, double *Y, SweepStage<TF> &St) {
    const int lane = threadIdx.x & 31, gl = lane & (kG - 1), grp = threadIdx.x / kG;
    const unsigned gmask = 0xffu << (lane & ~(kG - 1));
    const TF *val = std::is_same<TF, float>::value ? (const TF *)T.valf : (const TF *)T.val;
    const TF *dinv = std::is_same<TF, float>::value ? (const TF *)T.dinvf : (const TF *)T.dinv;
    const int nl = T.nlev;
    auto cp_val = [&](TF *dst, const TF *src) {
        if constexpr (sizeof(TF) == 4) cpa4(dst, src);
        else cpa8(dst, src);
    };
    // metadata of position p into stage s (lane 0 of the group)
    auto stage_meta = [&](int s, int p) {
        if (gl == 0) {
            cpa4(&St.meta[s][grp][0], T.rows + p);
            cpa4(&St.meta[s][grp][1], T.rp + p);
            cpa4(&St.meta[s][grp][2], T.rp + p + 1);
        }
    };
    // entries and diagonal of position p into stage s (its metadata already in stage s)
    auto stage_entries = [&](int s, int p) {
        const int rs = St.meta[s][grp][1], re = St.meta[s][grp][2];
        if (rs + gl < re) {
            cpa4(&St.col[s][grp][gl], T.ci + rs + gl);
            cp_val(&St.val[s][grp][gl], val + rs + gl);
        }
        if (gl == 0 && dinv) cp_val(&St.dinv[s][grp], dinv + p);
    };
    // the row at position p with row i, entries [rs, re), first pair (colk, ak), diagonal dv
    auto solve_row = [&](int i, int rs, int re, int colk, TF ak, TF dv) {
        TF acc[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            const int col = gl + c * kG;
            acc[c] = col < q ? (TF)X[(size_t)i * q + col] : (TF)0;
        }
        for (int kb = rs; kb < re; kb += kG) {
            if (kb != rs) {
                const int k = kb + gl;
                colk = 0;
                ak = (TF)0;
                if (k < re) {
                    colk = __ldg(T.ci + k);
                    ak = val[k];
                }
            }
            const int cnt = min(kG, re - kb);
            #pragma unroll 4   // several entries' loads in flight; same summation order
            for (int e = 0; e < cnt; e++) {
                const int cs = __shfl_sync(gmask, colk, e, kG);
                const TF as = __shfl_sync(gmask, ak, e, kG);
                const double *yr = Y + (size_t)cs * q + gl;
#pragma unroll
                for (int c = 0; c < CPL; c++)
                    if (gl + c * kG < q) acc[c] -= as * (TF)yr[c * kG];
            }
        }
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            const int col = gl + c * kG;
            if (col < q) Y[(size_t)i * q + col] = (double)(acc[c] * dv);
        }
    };
    // b0 .. b3: starts of levels l .. l + 3 (a level past the last one is empty)
    int b0 = __ldg(T.lev_ptr), b1 = __ldg(T.lev_ptr + min(1, nl)), b2 = __ldg(T.lev_ptr + min(2, nl)),
        b3 = __ldg(T.lev_ptr + min(3, nl));
    // prologue: metadata of levels 0 and 1, then the entries of level 0
    if (b0 + grp < b1) stage_meta(0, b0 + grp);
    if (b1 + grp < b2) stage_meta(1, b1 + grp);
    cpa_commit();
    cpa_wait_all();
    __syncthreads();
    if (b0 + grp < b1) stage_entries(0, b0 + grp);
    cpa_commit();
    cpa_wait_all();
    __syncthreads();
    for (int l = 0; l < nl; l++) {
        const int s0 = l % 3, s1 = (l + 1) % 3, s2 = (l + 2) % 3;
        const int b4 = __ldg(T.lev_ptr + min(l + 4, nl));
        // asynchronous copies for the coming levels (rows of levels l + 1 and l + 2 are written
        // only in their own levels)
        if (b1 + grp < b2) stage_entries(s1, b1 + grp);
        if (b2 + grp < b3) stage_meta(s2, b2 + grp);
        cpa_commit();
        const int p0 = b0 + grp;
        if (p0 < b1) {
            const int i = St.meta[s0][grp][0], rs = St.meta[s0][grp][1], re = St.meta[s0][grp][2];
            const int colk = rs + gl < re ? St.col[s0][grp][gl] : 0;
            const TF ak = rs + gl < re ? St.val[s0][grp][gl] : (TF)0;
            const TF dv = dinv ? St.dinv[s0][grp] : (TF)1;
            solve_row(i, rs, re, colk, ak, dv);
            // a wide level's further positions, loaded directly one ahead
            int p = p0 + kNG;
            int wi = 0, wrs = 0, wre = 0;
            if (p < b1) {
                wi = __ldg(T.rows + p);
                wrs = __ldg(T.rp + p);
                wre = __ldg(T.rp + p + 1);
            }
            for (; p < b1; p += kNG) {
                const int pw = p + kNG;
                int ni = 0, nrs = 0, nre = 0;
                if (pw < b1) {
                    ni = __ldg(T.rows + pw);
                    nrs = __ldg(T.rp + pw);
                    nre = __ldg(T.rp + pw + 1);
                }
                int c0 = 0;
                TF a0 = (TF)0;
                if (wrs + gl < wre) {
                    c0 = __ldg(T.ci + wrs + gl);
                    a0 = val[wrs + gl];
                }
                solve_row(wi, wrs, wre, c0, a0, dinv ? dinv[p] : (TF)1);
                wi = ni;
                wrs = nrs;
                wre = nre;
            }
        }
        b0 = b1;
        b1 = b2;
        b2 = b3;
        b3 = b4;
        cpa_wait_all();   // this thread's copies for levels l + 1 and l + 2 ...
        __syncthreads();  // ... visible to its group after the barrier
    }
}

__device__ __noinline__ void spmm(const Sys &S, int q, const double *X, double *Y, const double *Bsub) {
    switch ((q + kG - 1) / kG) {
        case 1: spmm_t<1>(S.rp, S.ci, S.av, S.n, q, X, Y, Bsub); break;
        case 2: spmm_t<2>(S.rp, S.ci, S.av, S.n, q, X, Y, Bsub); break;
        case 3: spmm_t<3>(S.rp, S.ci, S.av, S.n, q, X, Y, Bsub); break;
        default: spmm_t<4>(S.rp, S.ci, S.av, S.n, q, X, Y, Bsub); break;
    }
}

// Z = U^{-1} L^{-1} V; St: shared staging of the sweeps (in scratch that is dead here)
template <int CPL, typename TF>
__device__ __forceinline__ void prec_apply_t(const Sys &S, int q, const double *V, double *Z, SweepStage<TF> &St) {
    trsv_t<CPL, TF>(S.L, q, V, Z, St);
    trsv_t<CPL, TF>(S.U, q, Z, Z, St);
}

template <typename TF>
__device__ __noinline__ void prec_apply(const Sys &S, int q, const double *V, double *Z, SweepStage<TF> &St) {
    switch ((q + kG - 1) / kG) {
        case 1: prec_apply_t<1, TF>(S, q, V, Z, St); break;
        case 2: prec_apply_t<2, TF>(S, q, V, Z, St); break;
        case 3: prec_apply_t<3, TF>(S, q, V, Z, St); break;
        default: prec_apply_t<4, TF>(S, q, V, Z, St); break;
    }
}

// ---------------------------------------------------------------------------------------
// Cholesky-QR
// ---------------------------------------------------------------------------------------
// Warp 0: the diagonally scaled Gram matrix C = D^{-1} G D^{-1} + shift I (G in `G`, destroyed)
// is factored C = R'^T R'; R = R' D and Rinv = D^{-1} R'^{-1} (upper, ld kLd).  Returns (to all
// threads) whether every pivot was positive.
__device__ bool chol_inv(int q, double *G, double *R, double *Rinv, double *dsc, double shift, int *flag) {
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < 32) {
        for (int c = lane; c < q; c += 32) {
            const double d = G[c * kLd + c];
            dsc[c] = d > 0.0 ? sqrt(d) : 1.0;
        }
        __syncwarp();
        for (int idx = lane; idx < q * q; idx += 32) {
            const int a = idx / q, b = idx - a * q;
            G[a * kLd + b] = G[a * kLd + b] / (dsc[a] * dsc[b]) + (a == b ? shift : 0.0);
        }
        __syncwarp();
        int ok = 1;
        for (int k = 0; k < q; k++) {
            const double piv = G[k * kLd + k];
            if (!(piv > 1e-15)) {
                ok = 0;
                break;
            }
            const double rk = sqrt(piv);
            for (int b = lane; b < q; b += 32)
                R[k * kLd + b] = b < k ? 0.0 : (b == k ? rk : G[k * kLd + b] / rk);
            __syncwarp();
            for (int b = lane; b < q; b += 32)
                if (b > k) {
                    const double rkb = R[k * kLd + b];
                    for (int a = k + 1; a <= b; a++) G[a * kLd + b] -= R[k * kLd + a] * rkb;
                }
            __syncwarp();
        }
        if (ok) {
            // column b of R'^{-1} by back substitution (lane b), then the scalings
            for (int b = lane; b < q; b += 32) {
                for (int a = b + 1; a < q; a++) Rinv[a * kLd + b] = 0.0;
                Rinv[b * kLd + b] = 1.0 / R[b * kLd + b];
                for (int a = b - 1; a >= 0; a--) {
                    double s = 0.0;
                    for (int k = a + 1; k <= b; k++) s += R[a * kLd + k] * Rinv[k * kLd + b];
                    Rinv[a * kLd + b] = -s / R[a * kLd + a];
                }
            }
            __syncwarp();
            for (int b = lane; b < q; b += 32)
                for (int a = 0; a <= b; a++) {
                    R[a * kLd + b] *= dsc[b];
                    Rinv[a * kLd + b] /= dsc[a];
                }
        }
        if (lane == 0) *flag = ok;
    }
    __syncthreads();
    return *flag != 0;
}

// C = A B for upper-triangular q x q matrices (ld kLd); C must not alias A or B.
__device__ void upper_mul(int q, const double *A, const double *B, double *C) {
    for (int idx = threadIdx.x; idx < q * q; idx += kT) {
        const int a = idx / q, b = idx - a * q;
        double s = 0.0;
        for (int k = a; k <= b; k++) s += A[a * kLd + k] * B[k * kLd + b];
        C[a * kLd + b] = a <= b ? s : 0.0;
    }
}

// W (n x q) -> Q in place with W = Q R, R left in sm.racc.  Two passes (three when the first
// needed a shift).  Returns false if even the shifted factorization failed.
__device__ bool cholqr(double *W, int n, int q, Smem &sm) {
    int passes = 2;
    bool shifted = false;
    for (int pass = 0; pass < passes; pass++) {
        gram(W, 0, 1, W, n, q, sm.red, sm.gm, 0, kLd);
        if (!chol_inv(q, sm.gm, sm.r0, sm.rinv, sm.dsc, 0.0, &sm.ival[0])) {
            if (shifted) return false;
            // Shifted Cholesky-QR (Fukaya et al., 2020): shift 11 (n q + q (q + 1)) u ||C||_2,
            // ||C||_2 <= q for the scaled Gram matrix; two unshifted passes follow.
            const double shift = 11.0 * ((double)n * q + (double)q * (q + 1)) * 1.1102230246251565e-16 * q;
            gram(W, 0, 1, W, n, q, sm.red, sm.gm, 0, kLd);
            if (!chol_inv(q, sm.gm, sm.r0, sm.rinv, sm.dsc, shift, &sm.ival[0])) return false;
            shifted = true;
            passes = pass + 3;
        }
        update(W, W, 0, sm.rinv, 0, kLd, 1, n, q, 1.0, false);
        if (pass == 0) {
            for (int idx = threadIdx.x; idx < kLd * kLd; idx += kT) sm.racc[idx] = sm.r0[idx];
        } else {
            upper_mul(q, sm.r0, sm.racc, sm.gm);
            __syncthreads();
            for (int idx = threadIdx.x; idx < kLd * kLd; idx += kT) sm.racc[idx] = sm.gm[idx];
        }
        __syncthreads();
    }
    return true;
}

// ---------------------------------------------------------------------------------------
// Hessenberg QR (per-column Householder on a 2q x q window: top = rows [iq, (i+1)q), bottom =
// rows [(i+1)q, (i+2)q) of the column block).  Lanes: column b = tid / tpc, tpc = kT / 2^ceil(log2 q).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int col_tpc(int q) {
    int p2 = 8;
    while (p2 < q) p2 <<= 1;
    return kT / p2;
}

__device__ __forceinline__ double &win_at(double *top, double *bot, int q, int row, int b) {
    return row < q ? top[row * kLd + b] : bot[(row - q) * kLd + b];
}

__device__ __forceinline__ unsigned group_mask(int tpc) {
    const int lane = threadIdx.x & 31;
    return tpc >= 32 ? 0xffffffffu : (((1u << tpc) - 1u) << (lane / tpc * tpc));
}

// Apply reflector c (v in refl[t * kLd + c], t = 0..q; tau at refl[(kQ + 1) * kLd + c]) to column
// b of the window, by the tpc lanes of the column's group.
__device__ __forceinline__ void refl_one(double *top, double *bot, const double *refl, int q, int c, int b,
                                         int sub, int tpc, unsigned gmask) {
    const double tau = refl[(kQ + 1) * kLd + c];
    if (tau == 0.0) return;
    double w = 0.0;
    for (int t = sub; t <= q; t += tpc) w += refl[t * kLd + c] * win_at(top, bot, q, c + t, b);
    for (int o = tpc >> 1; o > 0; o >>= 1) w += __shfl_xor_sync(gmask, w, o);
    w *= tau;
    for (int t = sub; t <= q; t += tpc) win_at(top, bot, q, c + t, b) -= refl[t * kLd + c] * w;
}

// All q reflectors of `refl`, in order, to the q columns of the window.  No barrier inside the
// loop: a column's rows are touched only by its own group.
__device__ void refl_apply_all(double *top, double *bot, const double *refl, int q) {
    const int tpc = col_tpc(q);
    const int b = threadIdx.x / tpc, sub = threadIdx.x % tpc;
    if (b < q) {
        const unsigned gmask = group_mask(tpc);
        for (int c = 0; c < q; c++) {
            refl_one(top, bot, refl, q, c, b, sub, tpc, gmask);
            __syncwarp(gmask);
        }
    }
    __syncthreads();
}

// Householder QR of the window whose bottom block is upper triangular (reflector c has support
// rows c .. c + q); reflectors into `refl`, R in the top block.
__device__ void house_window(double *top, double *bot, double *refl, int q) {
    const int tpc = col_tpc(q);
    const int b = threadIdx.x / tpc, sub = threadIdx.x % tpc;
    const unsigned gmask = b < q ? group_mask(tpc) : 0u;
    for (int c = 0; c < q; c++) {
        if (b == c) {
            const double alpha = top[c * kLd + c];
            double sg = 0.0;   // sum of squares below the diagonal (t = 1 .. q)
            for (int t = (sub == 0 ? tpc : sub); t <= q; t += tpc) {
                const double x = win_at(top, bot, q, c + t, c);
                sg += x * x;
            }
            for (int o = tpc >> 1; o > 0; o >>= 1) sg += __shfl_xor_sync(gmask, sg, o);
            double tau = 0.0, beta = alpha, scale = 0.0;
            if (sg > 0.0) {
                beta = -copysign(sqrt(alpha * alpha + sg), alpha);
                tau = (beta - alpha) / beta;
                scale = 1.0 / (alpha - beta);
            }
            for (int t = sub; t <= q; t += tpc) {
                if (t == 0) {
                    refl[c] = 1.0;
                    top[c * kLd + c] = beta;
                } else {
                    double &x = win_at(top, bot, q, c + t, c);
                    refl[t * kLd + c] = x * scale;
                    x = 0.0;
                }
            }
            if (sub == 0) refl[(kQ + 1) * kLd + c] = tau;
        }
        __syncthreads();
        if (b > c && b < q) refl_one(top, bot, refl, q, c, b, sub, tpc, gmask);
        __syncthreads();
    }
}

__device__ __forceinline__ size_t rcol_off(int j, int q) { return (size_t)j * (j + 3) / 2 * q * q; }

__device__ void load_blk(double *dst, const double *src, int q) {
    for (int idx = threadIdx.x; idx < q * q; idx += kT) {
        const int a = idx / q, b = idx - a * q;
        dst[a * kLd + b] = src[idx];
    }
}
__device__ void store_blk(double *dst, const double *src, int q, bool upper_only) {
    for (int idx = threadIdx.x; idx < q * q; idx += kT) {
        const int a = idx / q, b = idx - a * q;
        dst[idx] = (upper_only && a > b) ? 0.0 : src[a * kLd + b];
    }
}

// Compact-WY factor of the window's reflector set (`refl` as house_window leaves it): with
// Y = [v_0 .. v_{q-1}] (v_c on window rows c .. c + q, v_c[0] = 1), H_0 H_1 .. H_{q-1} =
// I - Y T Y^T, T upper triangular: T_cc = tau_c, T[0:c, c] = -tau_c T[0:c, 0:c] (Y^T v_c)[0:c]
// (LAPACK's forward, columnwise larft).  T into `T` (ld kLd); z is q doubles of scratch.
__device__ void wy_factor(const double *refl, int q, double *T, double *z) {
    for (int idx = threadIdx.x; idx < q * kLd; idx += kT) T[idx] = 0.0;
    __syncthreads();
    for (int c = 0; c < q; c++) {
        const double tau = refl[(kQ + 1) * kLd + c];
        // z_r = v_r . v_c over the rows they share, c .. r + q (r < c)
        for (int r = threadIdx.x; r < c; r += kT) {
            double acc = 0.0;
            for (int row = c; row <= r + q; row++) acc += refl[(row - r) * kLd + r] * refl[(row - c) * kLd + c];
            z[r] = acc;
        }
        __syncthreads();
        for (int r = threadIdx.x; r < c; r += kT) {
            double acc = 0.0;
            for (int u = r; u < c; u++) acc += T[r * kLd + u] * z[u];
            T[r * kLd + c] = -tau * acc;
        }
        if (threadIdx.x == 0) T[c * kLd + c] = tau;
        __syncthreads();
    }
}

// The window (top; bot) <- H_{q-1} .. H_0 (top; bot) = (I - Y T^T Y^T)(top; bot) in three
// products (W1 = Y^T X, W2 = T^T W1, X -= Y W2) instead of q reflector steps.
__device__ void wy_apply(double *top, double *bot, const double *refl, const double *T, double *W1, double *W2,
                         int q) {
    for (int idx = threadIdx.x; idx < q * q; idx += kT) {
        const int r = idx / q, b = idx - r * q;
        double acc = 0.0;
        for (int t = 0; t <= q; t++) acc += refl[t * kLd + r] * win_at(top, bot, q, r + t, b);
        W1[r * kLd + b] = acc;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < q * q; idx += kT) {
        const int r = idx / q, b = idx - r * q;
        double acc = 0.0;
        for (int u = 0; u <= r; u++) acc += T[u * kLd + r] * W1[u * kLd + b];
        W2[r * kLd + b] = acc;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < 2 * q * q; idx += kT) {
        const int row = idx / q, b = idx - row * q;
        const int r0 = max(0, row - q), r1 = min(q - 1, row);
        double acc = 0.0;
        for (int r = r0; r <= r1; r++) acc += refl[(row - r) * kLd + r] * W2[r * kLd + b];
        win_at(top, bot, q, row, b) -= acc;
    }
    __syncthreads();
}

// Column j of the block Hessenberg matrix (blocks 0..j+1 in U.R) -> R column j; new reflectors
// into U.HV; g_j, g_{j+1} updated.  Returns ||g_{j+1}||_F, the least-squares residual.
__device__ double hess_update(const Unit &U, int j, Smem &sm) {
    const int q = U.q;
    const size_t qq = (size_t)q * q;
    double *Rc = U.R + rcol_off(j, q);
    double *wa = sm.red, *wb = sm.red + kQ * kLd;
    double *refl = sm.red + 2 * kQ * kLd;
    double *ga = refl + (kQ + 2) * kLd, *gb = ga + kQ * kLd;
    double *Tw = gb + kQ * kLd, *zw = Tw + kQ * kLd;   // WY factor of a window, larft scratch
    const size_t hvs = (size_t)(2 * q + 2) * q;
    load_blk(wa, Rc, q);
    __syncthreads();
    double *top = wa, *bot = wb;
    for (int i = 0; i < j; i++) {
        load_blk(bot, Rc + (i + 1) * qq, q);
        const double *hv = U.HV + (size_t)i * hvs;
        for (int idx = threadIdx.x; idx < (q + 1) * q; idx += kT) {
            const int t = idx / q, c = idx - t * q;
            refl[t * kLd + c] = hv[idx];
        }
        for (int idx = threadIdx.x; idx < q * q; idx += kT) {
            const int r = idx / q, c = idx - r * q;
            Tw[r * kLd + c] = hv[(q + 2) * q + idx];
        }
        __syncthreads();
        wy_apply(top, bot, refl, Tw, ga, gb, q);   // ga / gb are free until the window loop ends
        store_blk(Rc + i * qq, top, q, false);
        __syncthreads();
        double *tmp = top;
        top = bot;
        bot = tmp;
    }
    load_blk(bot, Rc + (j + 1) * qq, q);
    __syncthreads();
    house_window(top, bot, refl, q);
    wy_factor(refl, q, Tw, zw);
    double *hv = U.HV + (size_t)j * hvs;
    for (int idx = threadIdx.x; idx < (q + 1) * q; idx += kT) {
        const int t = idx / q, c = idx - t * q;
        hv[idx] = refl[t * kLd + c];
    }
    for (int c = threadIdx.x; c < q; c += kT) hv[(q + 1) * q + c] = refl[(kQ + 1) * kLd + c];
    for (int idx = threadIdx.x; idx < q * q; idx += kT) {
        const int r = idx / q, c = idx - r * q;
        hv[(q + 2) * q + idx] = Tw[r * kLd + c];
    }
    store_blk(Rc + j * qq, top, q, true);
    load_blk(ga, U.g + j * qq, q);
    for (int idx = threadIdx.x; idx < q * q; idx += kT) {
        const int a = idx / q, b = idx - a * q;
        gb[a * kLd + b] = 0.0;
    }
    __syncthreads();
    refl_apply_all(ga, gb, refl, q);
    store_blk(U.g + j * qq, ga, q, false);
    store_blk(U.g + (j + 1) * qq, gb, q, false);
    double s = 0.0;
    for (int idx = threadIdx.x; idx < q * q; idx += kT) {
        const int a = idx / q, b = idx - a * q;
        const double v = gb[a * kLd + b];
        s += v * v;
    }
    s = cta_sum(s, sm.scal);
    __syncthreads();
    return sqrt(s);
}

// Block back substitution R y = g over J column blocks; y overwrites g's blocks.
__device__ void backsub(const Unit &U, int J, Smem &sm) {
    const int q = U.q;
    const size_t qq = (size_t)q * q;
    double *yk = sm.red, *rk = sm.red + kQ * kLd;
    const int tpc = col_tpc(q);
    const int b = threadIdx.x / tpc, sub = threadIdx.x % tpc;
    for (int k = J - 1; k >= 0; k--) {
        const double *Rck = U.R + rcol_off(k, q);
        load_blk(yk, U.g + k * qq, q);
        load_blk(rk, Rck + k * qq, q);
        __syncthreads();
        if (b < q) {
            const unsigned gmask = group_mask(tpc);
            for (int a = q - 1; a >= 0; a--) {
                double s = 0.0;
                for (int c = a + 1 + sub; c < q; c += tpc) s += rk[a * kLd + c] * yk[c * kLd + b];
                for (int o = tpc >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(gmask, s, o);
                if (sub == 0) yk[a * kLd + b] = (yk[a * kLd + b] - s) / rk[a * kLd + a];
                __syncwarp(gmask);
            }
        }
        __syncthreads();
        store_blk(U.g + k * qq, yk, q, false);
        const int tot = k * q * q;
        for (int idx = threadIdx.x; idx < tot; idx += kT) {
            const int i = idx / (q * q), rem = idx - i * q * q;
            const int a = rem / q, c2 = rem - a * q;
            const double *Rik = Rck + i * qq + a * q;
            double s = 0.0;
            for (int c = 0; c < q; c++) s += Rik[c] * yk[c * kLd + c2];
            U.g[i * qq + rem] -= s;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// one unit
// ---------------------------------------------------------------------------------------
template <typename TF>
__device__ void solve_unit(const Sys &S, const Unit &U, const IO &io, const Cfg &cfg, UnitOut *out, Smem &sm) {
    const int n = S.n, q = U.q, m = U.m;
    const size_t bs = (size_t)n * q, qq = (size_t)q * q;
    PhaseClock pc;
    pc.start();
    const long long t_begin = pc.t;
    // B's slice in A_hat's order; X0 = 0
    double s = 0.0;
    for (size_t idx = threadIdx.x; idx < bs; idx += kT) {
        const int c = (int)(idx / n), r = (int)(idx - (size_t)c * n);
        const double v = io.B[(size_t)(U.col0 + c) * io.ldb + __ldg(S.perm + r)];
        U.Bh[(size_t)r * q + c] = v;
        U.V[(size_t)r * q + c] = v;
        U.Xh[(size_t)r * q + c] = 0.0;
        s += v * v;
    }
    const double rn0 = sqrt(cta_sum(s, sm.scal));
    const double eps = cfg.atol + cfg.rtol * rn0;
    const int itmax = cfg.itmax > 0 ? cfg.itmax : max(2 * (n / q), 50);
    int iter = 0, cycles = 0, status = BPF_SOLVE_UNKNOWN;
    double rn = rn0;
    bool solved = rn0 <= eps;
    if (!solved) {
        // A zero column of B would make the first block rank deficient: it is solved with a
        // stand-in column (X's column is set to zero at the end, the exact solution); the
        // stopping test keeps eps from the caller's B.
        gram(U.Bh, 0, 1, U.Bh, n, q, sm.red, sm.gm, 0, kLd);
        if (threadIdx.x == 0) {
            unsigned mask = 0u;
            double sum = 0.0;
            int cnt = 0;
            for (int c = 0; c < q; c++) {
                const double d = sm.gm[c * kLd + c];
                if (d == 0.0) mask |= 1u << c;
                else {
                    sum += d;
                    cnt++;
                }
            }
            sm.zmask = mask;
            sm.zscale = cnt > 0 ? sqrt(sum / cnt / (double)n) : 1.0;
        }
        __syncthreads();
        if (sm.zmask) {
            const unsigned mask = sm.zmask;
            const double zs = sm.zscale;
            for (size_t idx = threadIdx.x; idx < bs; idx += kT) {
                const int r = (int)(idx / q), c = (int)(idx - (size_t)r * q);
                if ((mask >> c) & 1u) {
                    const double v = zs * standin(r, c);
                    U.Bh[idx] = v;
                    U.V[idx] = v;
                }
            }
        }
        __syncthreads();
    } else if (threadIdx.x == 0) {
        sm.zmask = 0u;
    }
    while (!solved && iter < itmax) {
        cycles++;
        pc.mark(PH_SPMM);
        // V_0 R_0 = residual; g = [R_0; 0]
        if (!cholqr(U.V, n, q, sm)) {
            status = -1;
            break;
        }
        store_blk(U.g, sm.racc, q, true);
        __syncthreads();
        pc.mark(PH_CHOLQR);
        int j = 0;
        bool brk = false;
        while (j < m && iter < itmax) {
            double *Vj = U.V + j * bs, *Zj = U.Z + j * bs, *Vn = U.V + (j + 1) * bs;
            // the Gram / Cholesky / Hessenberg scratch is dead here
            static_assert(sizeof(SweepStage<double>) <= sizeof(Smem::red), "sweep staging fits the scratch");
            prec_apply<TF>(S, q, Vj, Zj, *reinterpret_cast<SweepStage<TF> *>(sm.red));
            pc.mark(PH_PREC);
            spmm(S, q, Zj, Vn, nullptr);
            __syncthreads();
            pc.mark(PH_SPMM);
            double *Rc = U.R + rcol_off(j, q);
            gram(U.V, bs, j + 1, Vn, n, q, sm.red, Rc, qq, q);
            pc.mark(PH_GRAM);
            update_staged(Vn, U.V, bs, Rc, qq, j + 1, n, q, -1.0, true, sm.red, kW * kLd * kLd);
            __syncthreads();
            pc.mark(PH_UPDATE);
            gram(U.V, bs, j + 1, Vn, n, q, sm.red, U.C2, qq, q);
            pc.mark(PH_GRAM);
            update_staged(Vn, U.V, bs, U.C2, qq, j + 1, n, q, -1.0, true, sm.red, kW * kLd * kLd);
            __syncthreads();
            for (size_t idx = threadIdx.x; idx < (size_t)(j + 1) * qq; idx += kT) Rc[idx] += U.C2[idx];
            pc.mark(PH_UPDATE);
            if (!cholqr(Vn, n, q, sm)) {
                // breakdown of the new block: the cycle ends with the j columns built
                brk = true;
                break;
            }
            store_blk(Rc + (j + 1) * qq, sm.racc, q, true);
            __syncthreads();
            pc.mark(PH_CHOLQR);
            rn = hess_update(U, j, sm);
            pc.mark(PH_HESS);
            iter++;
            j++;
            if (!(rn == rn)) {
                status = -1;
                break;
            }
            if (rn <= eps) {
                solved = true;
                break;
            }
        }
        if (status == -1) break;
        if (j > 0) {
            backsub(U, j, sm);
            pc.mark(PH_BACKSUB);
            update_staged(U.Xh, U.Z, bs, U.g, qq, j, n, q, 1.0, true, sm.red, kW * kLd * kLd);
            __syncthreads();
            pc.mark(PH_UPDATE);
        }
        if (brk && j == 0) {
            status = -1;
            break;
        }
        // the true residual: the next cycle's start, and the check of a converged estimate (the
        // least-squares residual can fall below eps while B - A X has not, when rounding has
        // eroded the basis' orthogonality); a failed check refines from the true residual
        spmm(S, q, U.Xh, U.V, U.Bh);
        __syncthreads();
        if (solved) {
            double s2 = 0.0;
            for (size_t idx = threadIdx.x; idx < bs; idx += kT) {
                const double v = U.V[idx];
                s2 += v * v;
            }
            rn = sqrt(cta_sum(s2, sm.scal));
            if (rn <= eps) break;
            solved = false;
        }
        pc.mark(PH_SPMM);
    }
    if (status != -1) status = solved ? BPF_SOLVE_SOLVED : BPF_SOLVE_ITMAX;
    __syncthreads();
    const unsigned zmask = sm.zmask;
    for (size_t idx = threadIdx.x; idx < bs; idx += kT) {
        const int c = (int)(idx / n), r = (int)(idx - (size_t)c * n);
        io.X[(size_t)(U.col0 + c) * io.ldx + __ldg(S.perm + r)] = ((zmask >> c) & 1u) ? 0.0 : U.Xh[(size_t)r * q + c];
    }
    if (threadIdx.x == 0) {
        out->niter = iter;
        out->status = status;
        out->cycles = cycles;
        out->rnorm0 = rn0;
        out->rnorm = rn;
        for (int i = 0; i < PH_COUNT; i++) out->phase_cycles[i] = pc.acc[i];
        out->total_cycles = clock64() - t_begin;
    }
}

__global__ void __launch_bounds__(kT, 1)
batch_solve_kernel(const Sys *__restrict__ sys, const Unit *__restrict__ units, int nunits,
                   const IO *__restrict__ io, const int *__restrict__ sys_err, Cfg cfg, UnitOut *out,
                   int *counter) {
    extern __shared__ __align__(128) unsigned char smraw[];
    Smem &sm = *reinterpret_cast<Smem *>(smraw);
    __shared__ int s_unit;
    for (;;) {
        if (threadIdx.x == 0) s_unit = atomicAdd(counter, 1);
        __syncthreads();
        const int u = s_unit;
        __syncthreads();
        if (u >= nunits) break;
        const Unit U = units[u];
        const Sys &S = sys[U.sys];
        if (sys_err[U.sys] != 0) {
            if (threadIdx.x == 0) {
                out[u].niter = 0;
                out[u].status = -2;
                out[u].cycles = 0;
                out[u].rnorm0 = out[u].rnorm = 0.0;
                for (int i = 0; i < PH_COUNT; i++) out[u].phase_cycles[i] = 0;
                out[u].total_cycles = 0;
            }
            continue;
        }
        if (cfg.f32) solve_unit<float>(S, U, io[U.sys], cfg, out + u, sm);
        else solve_unit<double>(S, U, io[U.sys], cfg, out + u, sm);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// ILU(0) of every system (one CTA per system, a warp per row, __syncthreads between the
// levels of the forward dependencies), then the level-sorted FP64 / FP32 factor copies.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kT) batch_factor_kernel(const Sys *__restrict__ sys, int nsys, int *sys_err) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int s = blockIdx.x; s < nsys; s += gridDim.x) {
        const Sys &S = sys[s];
        if (threadIdx.x == 0) sys_err[s] = 0;
        for (int k = threadIdx.x; k < S.nnz; k += kT) {
            const double v = S.vals[k];
            const int t = __ldg(S.amap + k);
            S.av[t] = v;
            S.fv[t] = v;
        }
        __syncthreads();
        double *fv = S.fv;
        const TriKernelArgs &L = S.L;
        for (int l = 0; l < L.nlev; l++) {
            const int q0 = __ldg(L.lev_ptr + l), q1 = __ldg(L.lev_ptr + l + 1);
            for (int qq = q0 + warp; qq < q1; qq += kW) {
                const int i = __ldg(L.rows + qq);
                const int rs = __ldg(S.rp + i), di = __ldg(S.diag + i);
                for (int e = rs; e < di; e++) {
                    const int k = __ldg(S.ci + e);
                    const int p0 = __ldg(S.pp + e), p1 = __ldg(S.pp + e + 1);
                    double l_ik = 0.0;
                    if (lane == 0) {
                        const double piv = fv[__ldg(S.diag + k)];
                        l_ik = fv[e] / piv;
                        fv[e] = l_ik;
                        if (piv == 0.0) atomicCAS(sys_err + s, 0, k + 1);
                    }
                    l_ik = __shfl_sync(0xffffffffu, l_ik, 0);
                    for (int t = p0 + lane; t < p1; t += 32) {
                        const int d = __ldg(S.pdst + t);
                        fv[d] -= l_ik * fv[__ldg(S.psrc + t)];
                    }
                    __syncwarp();
                }
                if (lane == 0 && fv[di] == 0.0) atomicCAS(sys_err + s, 0, i + 1);
                __syncwarp();
            }
            __syncthreads();
        }
        const TriKernelArgs &U = S.U;
        for (int e = threadIdx.x; e < L.nnz; e += kT) {
            const double v = fv[__ldg(L.map + e)];
            L.val[e] = v;
            L.valf[e] = (float)v;
        }
        for (int e = threadIdx.x; e < U.nnz; e += kT) {
            const double v = fv[__ldg(U.map + e)];
            U.val[e] = v;
            U.valf[e] = (float)v;
        }
        for (int qq = threadIdx.x; qq < U.n; qq += kT) {
            const double d = 1.0 / fv[__ldg(U.dmap + qq)];
            U.dinv[qq] = d;
            U.dinvf[qq] = (float)d;
        }
        __syncthreads();
    }
}

}  // namespace batch
}  // namespace bpf

using namespace bpf;
using namespace bpf::batch;

struct bpf_batch {
    bpf_ctx *ctx = nullptr;
    int nsys = 0, nunits = 0, grid = 0;
    bpf_batch_opts opts{};
    std::vector<int> n, p;
    std::vector<Unit> units;
    unsigned char *dpool = nullptr;   // patterns, orderings, factor storage, device tables
    double *dws = nullptr;            // unit workspaces
    size_t pool_bytes = 0, ws_bytes = 0;
    Sys *d_sys = nullptr;
    Unit *d_units = nullptr;
    IO *d_io = nullptr;
    UnitOut *d_out = nullptr;
    int *d_err = nullptr;
    int *d_counter = nullptr;
    IO *h_io = nullptr;          // pinned
    UnitOut *h_out = nullptr;    // pinned
    int *h_err = nullptr;        // pinned
    cudaStream_t cstream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    std::vector<double> unit_iter_bytes;   // algorithmic bytes of one iteration (without basis reads)
    std::vector<double> unit_basis_bytes;  // basis bytes per block read by one iteration
    double factor_bytes = 0.0;             // algorithmic bytes of one launch of the factor kernel
    double factor_flops = 0.0;
    int factor_grid = 0;
    Cfg cfg{};
};

namespace {

size_t smem_bytes() { return sizeof(bpf::batch::Smem); }

// Basis blocks for a unit of n rows and q columns: the iteration counts of unrestarted ILU(0)
// block-GMRES on power-flow Jacobians grow like (n / q)^0.7 (fitted on 200 - 6,000-unknown grids:
// 31 iterations at n = 568, q = 8; 146 at n = 5,698, q = 8; 36 at n = 5,698, q = 64), and
// restarting a block of <= 32 columns stagnates, so the basis holds twice the fitted count.
int auto_memory(int n, int q) {
    const double est = 1.5 * pow((double)n / (double)q, 0.7);
    return std::max(8, (int)std::ceil(2.0 * est) + 10);
}

size_t unit_doubles(int n, int q, int m) {
    const size_t bs = (size_t)n * q, qq = (size_t)q * q;
    return bs * (2 * (size_t)m + 3) + qq * ((size_t)m * (m + 3) / 2 + 2 * ((size_t)m + 1)) +
           (size_t)m * (2 * q + 2) * q;
}

struct Packer {
    std::vector<unsigned char> host;
    size_t add(const void *src, size_t bytes) {
        size_t off = (host.size() + 255) & ~(size_t)255;
        host.resize(off + bytes);
        if (bytes && src) memcpy(host.data() + off, src, bytes);
        return off;
    }
    template <typename T, typename A>
    size_t add(const std::vector<T, A> &v) { return add(v.data(), v.size() * sizeof(T)); }
    size_t reserve(size_t bytes) { return add(nullptr, bytes); }
};

}  // namespace

extern "C" {

void bpf_batch_opts_default(bpf_batch_opts *o) {
    if (!o) return;
    o->atol = 0.0;
    o->rtol = 1e-8;
    o->itmax = 0;
    o->memory = 0;
    o->factor_dtype = BPF_F32;
    o->ordering = BPF_ORDER_AMD;
    o->slice = 0;
    o->ctas_per_sm = 0;
}

bpf_status bpf_batch_destroy(bpf_batch *b) {
    if (!b) return BPF_SUCCESS;
    if (b->ctx) cudaStreamSynchronize(b->ctx->stream);
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->cstream) cudaStreamDestroy(b->cstream);
    cudaFree(b->dpool);
    cudaFree(b->dws);
    cudaFreeHost(b->h_io);
    cudaFreeHost(b->h_out);
    cudaFreeHost(b->h_err);
    delete b;
    return BPF_SUCCESS;
}

bpf_status bpf_batch_plan(bpf_ctx *ctx, int nsys, const bpf_csr_desc *A, const int *nrhs,
                          const bpf_batch_opts *opts_in, bpf_batch **out) {
    return bpf_batch_plan_sliced(ctx, nsys, A, nrhs, nullptr, opts_in, out);
}

bpf_status bpf_batch_plan_sliced(bpf_ctx *ctx, int nsys, const bpf_csr_desc *A, const int *nrhs,
                                 const int *slices, const bpf_batch_opts *opts_in, bpf_batch **out) {
    if (!ctx || !out) return BPF_ERR_INVALID_VALUE;
    *out = nullptr;
    if (nsys <= 0 || !A || !nrhs) return set_error(ctx, BPF_ERR_INVALID_VALUE, "batch: nsys > 0, A and nrhs required");
    if (slices)
        for (int s = 0; s < nsys; s++)
            if (slices[s] < 0 || slices[s] > kQ)
                return set_error(ctx, BPF_ERR_INVALID_VALUE, "batch: slices[%d] must be 0..%d", s, kQ);
    bpf_batch_opts o;
    if (opts_in) o = *opts_in;
    else bpf_batch_opts_default(&o);
    if (o.factor_dtype != BPF_F64 && o.factor_dtype != BPF_F32)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "batch: factor dtype must be BPF_F64 or BPF_F32");
    if (o.ordering == BPF_ORDER_METIS)
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "batch: ordering :METIS needs a METIS library");
    if (o.ordering < 0 || o.ordering > BPF_ORDER_NATURAL)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "batch: unknown ordering %d", o.ordering);
    if (o.slice < 0 || o.slice > kQ) return set_error(ctx, BPF_ERR_INVALID_VALUE, "batch: slice must be 0..%d", kQ);
    if (o.ctas_per_sm < 0 || o.ctas_per_sm > 2)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "batch: ctas_per_sm must be 0, 1 or 2");
    if (o.memory < 0 || o.itmax < 0 || !(o.atol >= 0.0) || !(o.rtol >= 0.0))
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "batch: negative memory, itmax or tolerance");
    const int qmax = o.slice > 0 ? o.slice : 16;
    const int cps = o.ctas_per_sm > 0 ? o.ctas_per_sm : 2;

    bpf_batch *b = new bpf_batch();
    b->ctx = ctx;
    b->nsys = nsys;
    b->opts = o;
    b->n.resize(nsys);
    b->p.resize(nsys);
    auto fail = [&](bpf_status st) {
        bpf_batch_destroy(b);
        return st;
    };

    // ---- host analysis of every system, packed into one device pool ----
    Packer pk;
    struct Offs {
        size_t rp, ci, diag, amap, pp, pdst, psrc, perm, av, fv;
        size_t l_lev, l_rows, l_rp, l_ci, l_map, l_val, l_valf;
        size_t u_lev, u_rows, u_rp, u_ci, u_map, u_dmap, u_val, u_valf, u_dinv, u_dinvf;
        int lnlev, unlev, lnnz, unnz;
    };
    std::vector<Offs> offs(nsys);
    std::vector<const void *> vals(nsys);
    // the patterns to the host (one system after another: the context's stream and error state)
    std::vector<std::vector<int>> arps(nsys), acis(nsys);
    for (int s = 0; s < nsys; s++) {
        const bpf_csr_desc &D = A[s];
        if (D.dtype != BPF_F64) return fail(set_error(ctx, BPF_ERR_NOT_SUPPORTED, "batch: system %d is not FP64", s));
        if (nrhs[s] < 1) return fail(set_error(ctx, BPF_ERR_INVALID_VALUE, "batch: system %d has nrhs < 1", s));
        bpf_status st = csr_pattern_to_host(ctx, &D, arps[s], acis[s], false, nullptr);
        if (st != BPF_SUCCESS) {
            const std::string msg = ctx->last_error;
            return fail(set_error(ctx, st, "batch: system %d: %s", s, msg.c_str()));
        }
        if (D.n < 1) return fail(set_error(ctx, BPF_ERR_INVALID_VALUE, "batch: system %d is empty", s));
    }
    // the per-system analysis (ordering, permuted pattern, ILU(0) update pairs, level-sorted
    // factors) is independent host work: host threads take systems from a counter
    struct SysHost {
        std::vector<int> rp, ci, diag, amap, perm, pp;
        PairVec pdst, psrc;
        TriHost L, U;
        int bad = -1;        // structurally zero diagonal at this row
        bool pairs_ok = true;
    };
    std::vector<SysHost> sh(nsys);
    {
        std::atomic<int> next{0};
        auto work = [&]() {
            for (int s = next++; s < nsys; s = next++) {
                SysHost &h = sh[s];
                const int n = A[s].n;
                if (o.ordering == BPF_ORDER_NATURAL) {
                    h.perm.resize(n);
                    std::iota(h.perm.begin(), h.perm.end(), 0);
                } else if (o.ordering == BPF_ORDER_RCM) {
                    h.perm = order_rcm(n, arps[s], acis[s]);
                } else {
                    h.perm = order_min_degree(n, arps[s], acis[s]);
                }
                h.bad = permute_pattern(n, arps[s], acis[s], h.perm, h.rp, h.ci, h.amap, h.diag);
                if (h.bad >= 0) continue;
                h.pairs_ok = build_pairs(n, h.rp.data(), h.ci.data(), h.diag.data(), false, h.pp, h.pdst, h.psrc);
                if (!h.pairs_ok) continue;
                h.L = build_tri(n, h.rp.data(), h.ci.data(), h.diag.data(), 0, true);
                h.U = build_tri(n, h.rp.data(), h.ci.data(), h.diag.data(), 1, false);
                std::vector<int>().swap(arps[s]);
                std::vector<int>().swap(acis[s]);
            }
        };
        const int nth = std::max(1, std::min({nsys, 32, (int)std::thread::hardware_concurrency()}));
        std::vector<std::thread> pool;
        for (int t = 1; t < nth; t++) pool.emplace_back(work);
        work();
        for (auto &th : pool) th.join();
    }
    for (int s = 0; s < nsys; s++) {
        const bpf_csr_desc &D = A[s];
        SysHost &h = sh[s];
        if (h.bad >= 0)
            return fail(set_error(ctx, BPF_ERR_SINGULAR, "batch: system %d: structurally zero diagonal at row %d", s, h.bad));
        if (!h.pairs_ok)
            return fail(set_error(ctx, BPF_ERR_NOT_SUPPORTED, "batch: system %d: ILU(0) update pairs exceed 2^31 - 1", s));
        const int n = D.n;
        std::vector<int> &rp = h.rp, &ci = h.ci, &diag = h.diag, &amap = h.amap, &perm = h.perm, &pp = h.pp;
        PairVec &pdst = h.pdst, &psrc = h.psrc;
        TriHost &L = h.L, &U = h.U;
        Offs &f = offs[s];
        f.rp = pk.add(rp);
        f.ci = pk.add(ci);
        f.diag = pk.add(diag);
        f.amap = pk.add(amap);
        f.pp = pk.add(pp);
        f.pdst = pk.add(pdst);
        f.psrc = pk.add(psrc);
        f.perm = pk.add(perm);
        f.l_lev = pk.add(L.lev_ptr);
        f.l_rows = pk.add(L.rows);
        f.l_rp = pk.add(L.rp);
        f.l_ci = pk.add(L.ci);
        f.l_map = pk.add(L.map);
        f.u_lev = pk.add(U.lev_ptr);
        f.u_rows = pk.add(U.rows);
        f.u_rp = pk.add(U.rp);
        f.u_ci = pk.add(U.ci);
        f.u_map = pk.add(U.map);
        f.u_dmap = pk.add(U.dmap);
        const int nnz = D.nnz;
        f.av = pk.reserve(sizeof(double) * nnz);
        f.fv = pk.reserve(sizeof(double) * nnz);
        f.lnnz = (int)L.ci.size();
        f.unnz = (int)U.ci.size();
        f.l_val = pk.reserve(sizeof(double) * f.lnnz);
        f.l_valf = pk.reserve(sizeof(float) * f.lnnz);
        f.u_val = pk.reserve(sizeof(double) * f.unnz);
        f.u_valf = pk.reserve(sizeof(float) * f.unnz);
        f.u_dinv = pk.reserve(sizeof(double) * n);
        f.u_dinvf = pk.reserve(sizeof(float) * n);
        f.lnlev = L.nlev;
        f.unlev = U.nlev;
        // factor kernel, per system: values in (8 + 4 map) and scattered twice (16), the update
        // pairs' indices (8 each), the level-sorted FP64 + FP32 copies (map 4 + read 8 + 12 written)
        // and the inverted diagonal
        b->factor_bytes += 28.0 * nnz + 4.0 * (n + 1) + 8.0 * (double)pdst.size() +
                           24.0 * ((double)f.lnnz + f.unnz) + 16.0 * n;
        b->factor_flops += 2.0 * (double)pdst.size();
        b->n[s] = n;
        b->p[s] = nrhs[s];
        vals[s] = D.vals;
        // work units: ceil(p / q_s) slices of nearly equal width, q_s = min(qmax, n / 24): a block
        // wider than n / 24 exhausts the Krylov space of a small system within a few iterations,
        // where a partial breakdown (directions that have converged) stalls block-GMRES
        const int p = nrhs[s];
        const int qs = std::max(1, std::min(slices && slices[s] > 0 ? slices[s] : qmax, n / 24));
        const int ns = (p + qs - 1) / qs;
        int col = 0;
        for (int k = 0; k < ns; k++) {
            const int q = p / ns + (k < p % ns ? 1 : 0);
            Unit un{};
            un.sys = s;
            un.col0 = col;
            un.q = q;
            un.m = o.memory > 0 ? o.memory : auto_memory(n, q);
            if (o.itmax > 0) un.m = std::min(un.m, o.itmax);
            un.m = std::max(1, std::min(un.m, n / q - 1));   // (m + 1) q <= n: the basis stays in R^n
            // cost: basis traffic ~ iterations^2 n q plus per-iteration level latency
            const double it = std::min((double)un.m, 1.5 * pow((double)n / q, 0.7));
            un.est = it * it * (double)n * q * 8.0 + it * (L.nlev + U.nlev) * 2.0e4;
            b->units.push_back(un);
            col += q;
        }
    }
    const size_t t_sys = pk.reserve(sizeof(Sys) * nsys);
    const int nunits = (int)b->units.size();
    b->nunits = nunits;
    const size_t t_units = pk.reserve(sizeof(Unit) * nunits);
    const size_t t_io = pk.reserve(sizeof(IO) * nsys);
    const size_t t_out = pk.reserve(sizeof(UnitOut) * nunits);
    const size_t t_err = pk.reserve(sizeof(int) * nsys);
    const size_t t_cnt = pk.reserve(sizeof(int) * 4);
    b->pool_bytes = pk.host.size();
    if (cudaMalloc((void **)&b->dpool, b->pool_bytes) != cudaSuccess)
        return fail(set_error(ctx, BPF_ERR_ALLOC, "batch: %zu bytes of analysis storage", b->pool_bytes));
    // unit workspaces, longest first
    std::stable_sort(b->units.begin(), b->units.end(), [](const Unit &x, const Unit &y) { return x.est > y.est; });
    size_t ws = 0;
    std::vector<size_t> wso(nunits);
    for (int u = 0; u < nunits; u++) {
        wso[u] = ws;
        ws += (unit_doubles(b->n[b->units[u].sys], b->units[u].q, b->units[u].m) + 31) & ~(size_t)31;
    }
    b->ws_bytes = ws * sizeof(double);
    if (cudaMalloc((void **)&b->dws, b->ws_bytes) != cudaSuccess)
        return fail(set_error(ctx, BPF_ERR_ALLOC, "batch: %zu bytes of basis storage", b->ws_bytes));
    for (int u = 0; u < nunits; u++) {
        Unit &un = b->units[u];
        const int n = b->n[un.sys], q = un.q, m = un.m;
        const size_t bs = (size_t)n * q, qq = (size_t)q * q;
        double *w = b->dws + wso[u];
        un.V = w;
        w += bs * (m + 1);
        un.Z = w;
        w += bs * m;
        un.Bh = w;
        w += bs;
        un.Xh = w;
        w += bs;
        un.R = w;
        w += qq * ((size_t)m * (m + 3) / 2);
        un.C2 = w;
        w += qq * (m + 1);
        un.g = w;
        w += qq * (m + 1);
        un.HV = w;
    }
    // device tables
    unsigned char *D = b->dpool;
    std::vector<Sys> hs(nsys);
    for (int s = 0; s < nsys; s++) {
        const Offs &f = offs[s];
        Sys &S = hs[s];
        S.n = b->n[s];
        S.nnz = A[s].nnz;
        S.p = b->p[s];
        S.rp = (const int *)(D + f.rp);
        S.ci = (const int *)(D + f.ci);
        S.diag = (const int *)(D + f.diag);
        S.amap = (const int *)(D + f.amap);
        S.pp = (const int *)(D + f.pp);
        S.pdst = (const int *)(D + f.pdst);
        S.psrc = (const int *)(D + f.psrc);
        S.perm = (const int *)(D + f.perm);
        S.vals = (const double *)vals[s];
        S.av = (double *)(D + f.av);
        S.fv = (double *)(D + f.fv);
        TriKernelArgs &L = S.L;
        L.n = S.n;
        L.nlev = f.lnlev;
        L.nnz = f.lnnz;
        L.lev_ptr = (const int *)(D + f.l_lev);
        L.rows = (const int *)(D + f.l_rows);
        L.rp = (const int *)(D + f.l_rp);
        L.ci = (const int *)(D + f.l_ci);
        L.map = (const int *)(D + f.l_map);
        L.dmap = nullptr;
        L.val = (double *)(D + f.l_val);
        L.valf = (float *)(D + f.l_valf);
        L.dinv = nullptr;
        L.dinvf = nullptr;
        TriKernelArgs &U = S.U;
        U.n = S.n;
        U.nlev = f.unlev;
        U.nnz = f.unnz;
        U.lev_ptr = (const int *)(D + f.u_lev);
        U.rows = (const int *)(D + f.u_rows);
        U.rp = (const int *)(D + f.u_rp);
        U.ci = (const int *)(D + f.u_ci);
        U.map = (const int *)(D + f.u_map);
        U.dmap = (const int *)(D + f.u_dmap);
        U.val = (double *)(D + f.u_val);
        U.valf = (float *)(D + f.u_valf);
        U.dinv = (double *)(D + f.u_dinv);
        U.dinvf = (float *)(D + f.u_dinvf);
    }
    memcpy(pk.host.data() + t_sys, hs.data(), sizeof(Sys) * nsys);
    memcpy(pk.host.data() + t_units, b->units.data(), sizeof(Unit) * nunits);
    b->d_sys = (Sys *)(D + t_sys);
    b->d_units = (Unit *)(D + t_units);
    b->d_io = (IO *)(D + t_io);
    b->d_out = (UnitOut *)(D + t_out);
    b->d_err = (int *)(D + t_err);
    b->d_counter = (int *)(D + t_cnt);
    if (cudaMemcpy(b->dpool, pk.host.data(), b->pool_bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(set_error(ctx, BPF_ERR_CUDA, "batch: upload of the analysis failed"));
    if (cudaMallocHost((void **)&b->h_io, sizeof(IO) * nsys) != cudaSuccess ||
        cudaMallocHost((void **)&b->h_out, sizeof(UnitOut) * nunits) != cudaSuccess ||
        cudaMallocHost((void **)&b->h_err, sizeof(int) * nsys) != cudaSuccess)
        return fail(set_error(ctx, BPF_ERR_ALLOC, "batch: pinned host tables"));
    memset(b->h_io, 0, sizeof(IO) * nsys);
    memset(b->h_out, 0, sizeof(UnitOut) * nunits);
    // algorithmic bytes per unit iteration (without the basis reads) and per basis block read
    b->unit_iter_bytes.resize(nunits);
    b->unit_basis_bytes.resize(nunits);
    for (int u = 0; u < nunits; u++) {
        const Unit &un = b->units[u];
        const Offs &f = offs[un.sys];
        const double n = b->n[un.sys], q = un.q, nnz = A[un.sys].nnz;
        const double fsz = b->opts.factor_dtype == BPF_F32 ? 4.0 : 8.0;
        // factors (index + value per entry, row pointers, row ids, 1/diag), the SpMM's matrix,
        // and the new block: read V_j, write and re-read Z_j, write W, ten passes over W
        // (two Gram-Schmidt updates, four Gram products, Cholesky-QR scalings)
        const double fb = (4.0 + fsz) * (f.lnnz + f.unnz) + 8.0 * 2 * (n + 1) + fsz * n;
        b->unit_iter_bytes[u] = fb + 12.0 * nnz + 4.0 * (n + 1) + 8.0 * n * q * 14.0;
        b->unit_basis_bytes[u] = 4.0 * 8.0 * n * q;   // CGS2: four passes over each basis block
    }
    // launch shape
    const size_t smem = smem_bytes();
    if (cudaFuncSetAttribute(batch_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return fail(set_error(ctx, BPF_ERR_CUDA, "batch: %zu bytes of shared memory per CTA not available", smem));
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_solve_kernel, kT, smem) != cudaSuccess || per_sm < 1)
        return fail(set_error(ctx, BPF_ERR_CUDA, "batch: solve kernel does not fit on an SM"));
    b->grid = std::max(1, std::min(nunits, std::min(cps, per_sm) * ctx->num_sms));
    // the graph: tables in, counter reset, factorization, solve
    if (cudaStreamCreateWithFlags(&b->cstream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(set_error(ctx, BPF_ERR_CUDA, "batch: stream creation failed"));
    Cfg cfg;
    cfg.atol = o.atol;
    cfg.rtol = o.rtol;
    cfg.itmax = o.itmax;
    cfg.f32 = o.factor_dtype == BPF_F32;
    b->cfg = cfg;
    b->factor_grid = std::min(nsys, 4 * ctx->num_sms);
    cudaError_t e = cudaStreamBeginCapture(b->cstream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_io, b->h_io, sizeof(IO) * nsys, cudaMemcpyHostToDevice, b->cstream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_counter, 0, sizeof(int), b->cstream);
    if (e == cudaSuccess) {
        batch_factor_kernel<<<b->factor_grid, kT, 0, b->cstream>>>(b->d_sys, nsys, b->d_err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        batch_solve_kernel<<<b->grid, kT, smem, b->cstream>>>(b->d_sys, b->d_units, nunits, b->d_io, b->d_err, cfg,
                                                              b->d_out, b->d_counter);
        e = cudaGetLastError();
    }
    cudaError_t e2 = cudaStreamEndCapture(b->cstream, &b->graph);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->gexec, b->graph, 0);
    if (e != cudaSuccess) return fail(cuda_error(ctx, e, "batch graph capture", __FILE__, __LINE__));
    *out = b;
    return BPF_SUCCESS;
}

bpf_status bpf_batch_solve(bpf_batch *b, const double *const *B, const int *ldb, double *const *X, const int *ldx,
                           bpf_stats *stats) {
    if (!b) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = b->ctx;
    if (!B || !X) return set_error(ctx, BPF_ERR_INVALID_VALUE, "batch solve: B and X pointer arrays required");
    for (int s = 0; s < b->nsys; s++) {
        const int lb = ldb ? ldb[s] : b->n[s], lx = ldx ? ldx[s] : b->n[s];
        if (!B[s] || !X[s]) return set_error(ctx, BPF_ERR_INVALID_VALUE, "batch solve: null block of system %d", s);
        if (lb < b->n[s] || lx < b->n[s])
            return set_error(ctx, BPF_ERR_DIMENSION, "batch solve: leading dimension below n for system %d", s);
        b->h_io[s].B = B[s];
        b->h_io[s].X = X[s];
        b->h_io[s].ldb = lb;
        b->h_io[s].ldx = lx;
    }
    if (!ctx->timing) {
        BPF_CUDA(ctx, cudaGraphLaunch(b->gexec, ctx->stream));
        ctx->launches += 2;
    } else {
        // Per-kernel timing: the graph's four steps issued one by one on the context's stream,
        // so that each kernel gets its own pair of events (same kernels, same arguments).
        BPF_CUDA(ctx, cudaMemcpyAsync(b->d_io, b->h_io, sizeof(IO) * b->nsys, cudaMemcpyHostToDevice, ctx->stream));
        BPF_CUDA(ctx, cudaMemsetAsync(b->d_counter, 0, sizeof(int), ctx->stream));
        {
            KScope ks(ctx, BPF_KC_FACTOR, b->factor_bytes, b->factor_flops);
            batch_factor_kernel<<<b->factor_grid, kT, 0, ctx->stream>>>(b->d_sys, b->nsys, b->d_err);
            BPF_CUDA(ctx, cudaGetLastError());
        }
        {
            KScope ks(ctx, BPF_KC_BATCH, 0.0, 0.0);
            batch_solve_kernel<<<b->grid, kT, smem_bytes(), ctx->stream>>>(b->d_sys, b->d_units, b->nunits, b->d_io,
                                                                          b->d_err, b->cfg, b->d_out, b->d_counter);
            BPF_CUDA(ctx, cudaGetLastError());
        }
        ctx->launches += 2;
    }
    BPF_CUDA(ctx, cudaMemcpyAsync(b->h_out, b->d_out, sizeof(UnitOut) * b->nunits, cudaMemcpyDeviceToHost, ctx->stream));
    BPF_CUDA(ctx, cudaMemcpyAsync(b->h_err, b->d_err, sizeof(int) * b->nsys, cudaMemcpyDeviceToHost, ctx->stream));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    // algorithmic bytes of what ran: per unit, iterations x (fixed part + basis reads)
    double bytes = 0.0, flops = 0.0;
    for (int u = 0; u < b->nunits; u++) {
        const int it = b->h_out[u].niter;
        const double q = b->units[u].q, n = b->n[b->units[u].sys];
        const int m = b->units[u].m;
        // basis blocks read per iteration: j + 1 at inner iteration j (restarts reset j)
        double blocks = 0.0;
        for (int k = 0; k < it; k++) blocks += (k % m) + 1;
        bytes += it * b->unit_iter_bytes[u] + blocks * b->unit_basis_bytes[u];
        flops += blocks * 8.0 * n * q * q;
    }
    if (ctx->timing && !ctx->timed.empty() && ctx->timed.back().kc == BPF_KC_BATCH) {
        ctx->timed.back().bytes = bytes;
        ctx->timed.back().flops = flops;
    }
    int first_bad = -1, first_num = -1;
    for (int s = 0; s < b->nsys; s++)
        if (b->h_err[s] != 0 && first_bad < 0) first_bad = s;
    if (stats) {
        for (int s = 0; s < b->nsys; s++) {
            stats[s].niter = 0;
            stats[s].solved = 1;
            stats[s].status = BPF_SOLVE_SOLVED;
            stats[s].timer = 0.0;
            stats[s].n_residuals = 0;
            stats[s].npass = 0;
        }
    }
    for (int u = 0; u < b->nunits; u++) {
        const UnitOut &r = b->h_out[u];
        const int s = b->units[u].sys;
        if (r.status == -1 && first_num < 0) first_num = s;
        if (stats) {
            bpf_stats &st = stats[s];
            st.niter = std::max(st.niter, r.niter);
            st.npass = std::max(st.npass, r.cycles);
            if (r.status != BPF_SOLVE_SOLVED) {
                st.solved = 0;
                if (st.status == BPF_SOLVE_SOLVED) st.status = r.status == BPF_SOLVE_ITMAX ? BPF_SOLVE_ITMAX : BPF_SOLVE_UNKNOWN;
            }
        }
    }
    if (first_bad >= 0)
        return set_error(ctx, BPF_ERR_SINGULAR, "batch: zero pivot in the ILU(0) of system %d (row %d of its ordering)",
                         first_bad, b->h_err[first_bad] - 1);
    if (first_num >= 0)
        return set_error(ctx, BPF_ERR_NUMERIC, "batch: Cholesky-QR breakdown or non-finite residual in system %d", first_num);
    return BPF_SUCCESS;
}

bpf_status bpf_batch_unit_stats(const bpf_batch *b, int *sys, int *col0, int *q, int *memory, int *niter,
                                int *status, double *rnorm0, double *rnorm) {
    if (!b) return BPF_ERR_INVALID_VALUE;
    for (int u = 0; u < b->nunits; u++) {
        if (sys) sys[u] = b->units[u].sys;
        if (col0) col0[u] = b->units[u].col0;
        if (q) q[u] = b->units[u].q;
        if (memory) memory[u] = b->units[u].m;
        if (niter) niter[u] = b->h_out[u].niter;
        if (status) status[u] = b->h_out[u].status;
        if (rnorm0) rnorm0[u] = b->h_out[u].rnorm0;
        if (rnorm) rnorm[u] = b->h_out[u].rnorm;
    }
    return BPF_SUCCESS;
}

bpf_status bpf_batch_unit_cycles(const bpf_batch *b, long long *cycles) {
    if (!b || !cycles) return BPF_ERR_INVALID_VALUE;
    for (int u = 0; u < b->nunits; u++) {
        for (int i = 0; i < PH_COUNT; i++) cycles[u * (PH_COUNT + 1) + i] = b->h_out[u].phase_cycles[i];
        cycles[u * (PH_COUNT + 1) + PH_COUNT] = b->h_out[u].total_cycles;
    }
    return BPF_SUCCESS;
}

bpf_status bpf_batch_info(const bpf_batch *b, int *nunits, int *grid, long long *device_bytes) {
    if (!b) return BPF_ERR_INVALID_VALUE;
    if (nunits) *nunits = b->nunits;
    if (grid) *grid = b->grid;
    if (device_bytes) *device_bytes = (long long)(b->ws_bytes + b->pool_bytes);
    return BPF_SUCCESS;
}

}  // extern "C"
