// ILU(0) / IC(0) preconditioners: host analysis (level schedules, update lists), device
// numeric factorization, and the multi-RHS triangular solves of ldiv!.
//
// Reference: src/preconditioners_nvidia.jl (ilu0 :42-47 -> csrilu02; ic0 :6-11 -> csric02;
// ldiv! :13-35, :49-71 -> two cusparseSpSM/SpSV per application).
//
// Design (B200):
//  * One host analysis per sparsity pattern: dependency levels of the forward and backward
//    solves, rows stored level by level (so a level's rows are contiguous), and for the
//    numeric factorization the list of (destination, source) update pairs of every L entry.
//  * The numeric factorization is a cooperative persistent kernel: one warp per row, the
//    rows of a level spread over the grid, one bounded grid barrier between levels.
//  * ldiv! is ONE cooperative launch that runs every level of L and then of U (or L'):
//    a group of G lanes per row, lanes over the p right-hand sides of the row-major block,
//    the row's (col, val) pairs broadcast by shuffles.  Values written in earlier levels are
//    read with ld.global.cg (L2, never a stale L1 line).  No scratch vector: the forward
//    solve writes Y and the backward solve updates Y in place.
//  * FP32 factors (factor_dtype = BPF_F32) keep float copies of L, U and 1/diag, read half the
//    factor bytes and compute in FP32; the block stays FP64 in memory.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <numeric>
#include <system_error>
#include <thread>

#include <cstdlib>

#include "bpf_internal.cuh"
#include "prec.cuh"

namespace bpf {

// ------------------------------------------------------------------------------------
// host analysis
// ------------------------------------------------------------------------------------
// Build a triangular factor from a 0-based CSR pattern.
//   part 0: strict lower part of each row (forward solve, dependencies c < i)
//   part 1: strict upper part of each row (backward solve, dependencies c > i)
//   part 2: transpose of the strict lower part (row i of L' holds L(j,i), j > i)
// diag[i] (index of A(i,i) in the pattern) gives the diagonal; unit == true ignores it.
TriHost build_tri(int n, const int *rp, const int *ci, const int *diag, int part, bool unit) {
    TriHost t;
    t.n = n;
    t.unit = unit;
    // rows of the factor as lists of (col, position-in-pattern)
    std::vector<int> cnt(n, 0);
    std::vector<int> frp(n + 1, 0), fci, fpos;
    if (part == 0 || part == 1) {
        for (int i = 0; i < n; i++)
            for (int k = rp[i]; k < rp[i + 1]; k++)
                if ((part == 0 && ci[k] < i) || (part == 1 && ci[k] > i)) cnt[i]++;
        for (int i = 0; i < n; i++) frp[i + 1] = frp[i] + cnt[i];
        fci.resize(frp[n]);
        fpos.resize(frp[n]);
        std::vector<int> fill(frp.begin(), frp.end() - 1);
        for (int i = 0; i < n; i++)
            for (int k = rp[i]; k < rp[i + 1]; k++)
                if ((part == 0 && ci[k] < i) || (part == 1 && ci[k] > i)) {
                    fci[fill[i]] = ci[k];
                    fpos[fill[i]++] = k;
                }
    } else {
        for (int i = 0; i < n; i++)
            for (int k = rp[i]; k < rp[i + 1]; k++)
                if (ci[k] < i) cnt[ci[k]]++;
        for (int i = 0; i < n; i++) frp[i + 1] = frp[i] + cnt[i];
        fci.resize(frp[n]);
        fpos.resize(frp[n]);
        std::vector<int> fill(frp.begin(), frp.end() - 1);
        for (int i = 0; i < n; i++)
            for (int k = rp[i]; k < rp[i + 1]; k++)
                if (ci[k] < i) {
                    int r = ci[k];
                    fci[fill[r]] = i;
                    fpos[fill[r]++] = k;
                }
    }
    // dependency levels
    std::vector<int> lev(n, 0);
    int nlev = 0;
    if (part == 0) {
        for (int i = 0; i < n; i++) {
            int l = 0;
            for (int k = frp[i]; k < frp[i + 1]; k++) l = std::max(l, lev[fci[k]] + 1);
            lev[i] = l;
            nlev = std::max(nlev, l + 1);
        }
    } else {
        for (int i = n - 1; i >= 0; i--) {
            int l = 0;
            for (int k = frp[i]; k < frp[i + 1]; k++) l = std::max(l, lev[fci[k]] + 1);
            lev[i] = l;
            nlev = std::max(nlev, l + 1);
        }
    }
    if (n == 0) nlev = 0;
    t.nlev = nlev;
    t.lev_ptr.assign(nlev + 1, 0);
    for (int i = 0; i < n; i++) t.lev_ptr[lev[i] + 1]++;
    for (int l = 0; l < nlev; l++) t.lev_ptr[l + 1] += t.lev_ptr[l];
    t.rows.resize(n);
    {
        std::vector<int> fill(t.lev_ptr.begin(), t.lev_ptr.end() - 1);
        if (part == 0) {
            for (int i = 0; i < n; i++) t.rows[fill[lev[i]]++] = i;
        } else {
            for (int i = n - 1; i >= 0; i--) t.rows[fill[lev[i]]++] = i;
        }
    }
    t.max_level_rows = 0;
    for (int l = 0; l < nlev; l++)
        t.max_level_rows = std::max(t.max_level_rows, t.lev_ptr[l + 1] - t.lev_ptr[l]);
    // level-sorted row storage
    t.rp.assign(n + 1, 0);
    for (int q = 0; q < n; q++) t.rp[q + 1] = t.rp[q] + (frp[t.rows[q] + 1] - frp[t.rows[q]]);
    t.ci.resize(t.rp[n]);
    t.map.resize(t.rp[n]);
    for (int q = 0; q < n; q++) {
        int i = t.rows[q];
        std::copy(fci.begin() + frp[i], fci.begin() + frp[i + 1], t.ci.begin() + t.rp[q]);
        std::copy(fpos.begin() + frp[i], fpos.begin() + frp[i + 1], t.map.begin() + t.rp[q]);
    }
    if (!unit) {
        t.dmap.resize(n);
        for (int q = 0; q < n; q++) t.dmap[q] = diag[t.rows[q]];
    }
    return t;
}

// ILU(0) update pairs: for the L entry e = (i,k), every j > k with (k,j) and (i,j) both in
// the pattern gives (dst = pos(i,j), src = pos(k,j)); applied as fv[dst] -= fv[e] * fv[src].
// IC(0) pairs: for the L entry e = (i,k), every j < k with (i,j) and (k,j) in the lower
// pattern gives (pos(i,j), pos(k,j)); fv[e] -= sum fv[pos(i,j)] * fv[pos(k,j)].
bool build_pairs(int n, const int *rp, const int *ci, const int *diag, bool ic,
                 std::vector<int> &pp, PairVec &pdst, PairVec &psrc) {
    const int nnz = rp[n];
    pp.assign(nnz + 1, 0);
    // rows [i0, i1): pass 0 counts the pairs of every entry into pp[e + 1]; pass 1 writes them at
    // the entry's prefix offset pp[e].  Every entry belongs to one row, so rows can be taken by
    // any thread in any order and the output is the same.
    auto rows = [&](int pass, int i0, int i1, std::vector<int> &pos) {
        int *dst = pass ? pdst.data() : nullptr, *src = pass ? psrc.data() : nullptr;
        for (int i = i0; i < i1; i++) {
            for (int k = rp[i]; k < rp[i + 1]; k++) pos[ci[k]] = k;
            for (int e = rp[i]; e < rp[i + 1]; e++) {
                const int kc = ci[e];
                const long long base = pass ? pp[e] : 0;
                long long c = 0;
                if (kc < i) {
                    if (!ic) {
                        for (int j = diag[kc] + 1; j < rp[kc + 1]; j++) {
                            const int q = pos[ci[j]];
                            if (q >= 0) {
                                if (pass) {
                                    dst[base + c] = q;
                                    src[base + c] = j;
                                }
                                c++;
                            }
                        }
                    } else {
                        for (int j = rp[kc]; j < diag[kc]; j++) {
                            const int q = pos[ci[j]];
                            if (q >= 0 && ci[j] < kc) {
                                if (pass) {
                                    dst[base + c] = q;
                                    src[base + c] = j;
                                }
                                c++;
                            }
                        }
                    }
                }
                if (!pass) pp[e + 1] = (int)std::min<long long>(c, INT_MAX);
            }
            for (int k = rp[i]; k < rp[i + 1]; k++) pos[ci[k]] = -1;
        }
    };
    // large patterns (the LU patterns of the refactorization) on several host threads, each with
    // its own position array, taking blocks of 64 rows from a shared counter
    const unsigned hw = std::thread::hardware_concurrency();
    const int nthreads = nnz >= 200000 ? (int)std::min(16u, std::max(1u, hw)) : 1;
    auto run = [&](int pass) {
        std::atomic<int> next(0);
        auto work = [&]() {
            std::vector<int> pos(n, -1);
            for (;;) {
                const int b = next.fetch_add(64);
                if (b >= n) break;
                rows(pass, b, std::min(n, b + 64), pos);
            }
        };
        std::vector<std::thread> pool;
        try {
            for (int t = 1; t < nthreads; t++) pool.emplace_back(work);
        } catch (const std::system_error &) {
            // fewer helpers than asked (a thread limit): the calling thread still takes every
            // block the helpers do not
        }
        work();
        for (auto &th : pool) th.join();
    };
    run(0);
    long long total = 0;
    for (int e = 0; e < nnz; e++) {
        total += pp[e + 1];
        if (total > INT_MAX) {   // offsets are int: the caller reports the pattern as too dense
            pp.clear();
            pdst.clear();
            psrc.clear();
            return false;
        }
        pp[e + 1] = (int)total;
    }
    pdst.resize(pp[nnz]);   // left uninitialised (NoInitAlloc): pass 1 writes every entry
    psrc.resize(pp[nnz]);
    run(1);
    return true;
}

// ------------------------------------------------------------------------------------
// device helpers for the TriDev struct
// ------------------------------------------------------------------------------------
template <typename T>
static bpf_status upload(bpf_ctx *ctx, T **dptr, const std::vector<T> &h) {
    *dptr = nullptr;
    if (h.empty()) return BPF_SUCCESS;
    BPF_CUDA(ctx, cudaMalloc((void **)dptr, sizeof(T) * h.size()));
    BPF_CUDA(ctx, cudaMemcpyAsync(*dptr, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice,
                                  ctx->stream));
    return BPF_SUCCESS;
}

bpf_status tri_upload(bpf_ctx *ctx, const TriHost &h, TriDev &d) {
    d.n = h.n;
    d.nlev = h.nlev;
    d.nnz = (int)h.ci.size();
    d.unit = h.unit;
    d.max_level_rows = h.max_level_rows;
    d.lev_ptr_h = h.lev_ptr;
    BPF_TRY(upload(ctx, &d.lev_ptr, h.lev_ptr));
    BPF_TRY(upload(ctx, &d.rows, h.rows));
    BPF_TRY(upload(ctx, &d.rp, h.rp));
    BPF_TRY(upload(ctx, &d.ci, h.ci));
    BPF_TRY(upload(ctx, &d.map, h.map));
    BPF_TRY(upload(ctx, &d.dmap, h.dmap));
    if (d.nnz > 0) {
        BPF_CUDA(ctx, cudaMalloc((void **)&d.val, sizeof(double) * d.nnz));
        BPF_CUDA(ctx, cudaMalloc((void **)&d.valf, sizeof(float) * d.nnz));
    }
    if (!h.unit && h.n > 0) {
        BPF_CUDA(ctx, cudaMalloc((void **)&d.dinv, sizeof(double) * h.n));
        BPF_CUDA(ctx, cudaMalloc((void **)&d.dinvf, sizeof(float) * h.n));
    }
    return BPF_SUCCESS;
}

void tri_free(TriDev &d) {
    cudaFree(d.lev_ptr);
    cudaFree(d.rows);
    cudaFree(d.rp);
    cudaFree(d.ci);
    cudaFree(d.map);
    cudaFree(d.dmap);
    cudaFree(d.val);
    cudaFree(d.valf);
    cudaFree(d.dinv);
    cudaFree(d.dinvf);
    d = TriDev();
}

// Copy factor values (pattern order) into the level-sorted triangular storage.
__global__ void tri_scatter_kernel(TriKernelArgs t, const double *__restrict__ fv) {
    const int stride = gridDim.x * blockDim.x;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < t.nnz; e += stride) {
        double v = fv[t.map[e]];
        t.val[e] = v;
        t.valf[e] = (float)v;
    }
    if (t.dinv) {
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < t.n; q += stride) {
            double d = 1.0 / fv[t.dmap[q]];
            t.dinv[q] = d;
            t.dinvf[q] = (float)d;
        }
    }
}

bpf_status tri_scatter(bpf_ctx *ctx, const TriDev &d, const double *fv) {
    if (d.n == 0) return BPF_SUCCESS;
    int work = std::max(d.nnz, d.n);
    int blocks = std::min(ceil_div(work, 256), ctx->num_sms * 8);
    tri_scatter_kernel<<<blocks, 256, 0, ctx->stream>>>(d.args(), fv);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

// ------------------------------------------------------------------------------------
// numeric factorization (cooperative, level by level, one warp per row)
// ------------------------------------------------------------------------------------
struct FactorArgs {
    int n;
    const int *rp;      // pattern (0-based)
    const int *ci;
    const int *diag;
    const int *pp;      // pair pointer per pattern entry (nnz+1)
    const int *pdst;
    const int *psrc;
    const int *lev_ptr; // level schedule of the forward dependencies
    const int *rows;
    int nlev;
    int ic;             // 0 ILU0, 1 IC0
    double *fv;         // factor values (pattern order), in/out
    DevStatus *ds;
};

__global__ void __launch_bounds__(256) factor_coop_kernel(FactorArgs a) {
    __shared__ unsigned s_gen;
    if (threadIdx.x == 0) s_gen = barrier_gen_start(a.ds);
    __syncthreads();
    unsigned gen = s_gen;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int gw = blockIdx.x * wpb + (threadIdx.x >> 5);
    const int nw = gridDim.x * wpb;
    double *fv = a.fv;
    for (int l = 0; l < a.nlev; l++) {
        const int q0 = a.lev_ptr[l], q1 = a.lev_ptr[l + 1];
        for (int q = q0 + gw; q < q1; q += nw) {
            const int i = a.rows[q];
            const int rs = a.rp[i], di = a.diag[i];
            for (int e = rs; e < di; e++) {
                const int k = a.ci[e];
                const int p0 = a.pp[e], p1 = a.pp[e + 1];
                if (!a.ic) {
                    double l_ik = 0.0;
                    if (lane == 0) {
                        const double piv = __ldcg(fv + a.diag[k]);
                        l_ik = __ldcg(fv + e) / piv;
                        fv[e] = l_ik;
                        if (piv == 0.0) {
                            if (atomicCAS(&a.ds->err, 0, (int)DEV_ZERO_PIVOT) == 0) a.ds->aux = k;
                        }
                    }
                    l_ik = __shfl_sync(0xffffffffu, l_ik, 0);
                    for (int t = p0 + lane; t < p1; t += 32) {
                        const int d = a.pdst[t];
                        fv[d] = __ldcg(fv + d) - l_ik * __ldcg(fv + a.psrc[t]);
                    }
                } else {
                    double s = 0.0;
                    for (int t = p0 + lane; t < p1; t += 32)
                        s += __ldcg(fv + a.pdst[t]) * __ldcg(fv + a.psrc[t]);
                    s = warp_sum(s);
                    if (lane == 0) fv[e] = (__ldcg(fv + e) - s) / __ldcg(fv + a.diag[k]);
                }
                __syncwarp();
            }
            if (a.ic) {
                double s = 0.0;
                for (int e = rs + lane; e < di; e += 32) {
                    double v = __ldcg(fv + e);
                    s += v * v;
                }
                s = warp_sum(s);
                if (lane == 0) {
                    double d = __ldcg(fv + di) - s;
                    if (!(d > 0.0)) {
                        if (atomicCAS(&a.ds->err, 0, (int)DEV_ZERO_PIVOT) == 0) a.ds->aux = i;
                        d = 1.0;
                    }
                    fv[di] = sqrt(d);
                }
            } else if (lane == 0) {
                if (__ldcg(fv + di) == 0.0) {
                    if (atomicCAS(&a.ds->err, 0, (int)DEV_ZERO_PIVOT) == 0) a.ds->aux = i;
                }
            }
            __syncwarp();
        }
        if (l + 1 < a.nlev) {
            if (!grid_barrier(a.ds, gen)) return;
        }
    }
}

// Right-looking LU on a fill pattern by column steps (the RF refactorization).  Level by
// level, a warp per L entry e = (i, k) of the level's steps: l_ik = a_ik / u_kk, then the
// entry's update pairs a_ij -= l_ik u_kj, added atomically (independent steps of one level may
// update the same entry).  Every value a level reads was final before its barrier.
__global__ void __launch_bounds__(256) lu_colstep_kernel(int nlev, const int *__restrict__ lev_ptr,
                                                         const int *__restrict__ ent, const int *__restrict__ ci,
                                                         const int *__restrict__ diag, const int *__restrict__ pp,
                                                         const int *__restrict__ pdst, const int *__restrict__ psrc,
                                                         double *fv, DevStatus *ds) {
    __shared__ unsigned s_gen;
    if (threadIdx.x == 0) s_gen = barrier_gen_start(ds);
    __syncthreads();
    unsigned gen = s_gen;
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (blockDim.x >> 5);
    for (int l = 0; l < nlev; l++) {
        const int q0 = __ldg(lev_ptr + l), q1 = __ldg(lev_ptr + l + 1);
        for (int q = q0 + gw; q < q1; q += nw) {
            const int e = __ldg(ent + q);
            const int k = __ldg(ci + e);
            double lik = 0.0;
            if (lane == 0) {
                const double piv = __ldcg(fv + __ldg(diag + k));
                if (piv == 0.0) {
                    if (atomicCAS(&ds->err, 0, (int)DEV_ZERO_PIVOT) == 0) ds->aux = k;
                } else {
                    lik = __ldcg(fv + e) / piv;
                }
                fv[e] = lik;
            }
            lik = __shfl_sync(0xffffffffu, lik, 0);
            const int t1 = __ldg(pp + e + 1);
            if (lik != 0.0)
                for (int t = __ldg(pp + e) + lane; t < t1; t += 32)
                    atomicAdd(fv + __ldg(pdst + t), -lik * __ldcg(fv + __ldg(psrc + t)));
        }
        if (l + 1 < nlev) {
            if (!grid_barrier(ds, gen)) return;
        }
    }
}

// The same column steps without stored update pairs: for the L entry e = (i, k) (row i from
// erow), every U entry (k, j), j > k, updates (i, j), whose position is found by a binary search
// of column j in row i after e (the fill pattern is closed under elimination, so it is there).
// Used where the pairs would exceed 2^31 - 1 (the 70,000-bus minimum-degree LU).
__global__ void __launch_bounds__(256) lu_colstep_search_kernel(int nlev, const int *__restrict__ lev_ptr,
                                                                const int *__restrict__ ent,
                                                                const int *__restrict__ erow,
                                                                const int *__restrict__ rp,
                                                                const int *__restrict__ ci,
                                                                const int *__restrict__ diag, double *fv,
                                                                DevStatus *ds) {
    __shared__ unsigned s_gen;
    if (threadIdx.x == 0) s_gen = barrier_gen_start(ds);
    __syncthreads();
    unsigned gen = s_gen;
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (blockDim.x >> 5);
    for (int l = 0; l < nlev; l++) {
        const int q0 = __ldg(lev_ptr + l), q1 = __ldg(lev_ptr + l + 1);
        for (int q = q0 + gw; q < q1; q += nw) {
            const int e = __ldg(ent + q);
            const int i = __ldg(erow + q);
            const int k = __ldg(ci + e);
            double lik = 0.0;
            if (lane == 0) {
                const double piv = __ldcg(fv + __ldg(diag + k));
                if (piv == 0.0) {
                    if (atomicCAS(&ds->err, 0, (int)DEV_ZERO_PIVOT) == 0) ds->aux = k;
                } else {
                    lik = __ldcg(fv + e) / piv;
                }
                fv[e] = lik;
            }
            lik = __shfl_sync(0xffffffffu, lik, 0);
            if (lik == 0.0) continue;
            const int u0 = __ldg(diag + k) + 1, u1 = __ldg(rp + k + 1);
            const int r0 = e + 1, r1 = __ldg(rp + i + 1);
            for (int t = u0 + lane; t < u1; t += 32) {
                const int j = __ldg(ci + t);
                int lo = r0, hi = r1;   // first position in [r0, r1) with column >= j
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (__ldg(ci + mid) < j) lo = mid + 1;
                    else hi = mid;
                }
                if (lo < r1 && __ldg(ci + lo) == j) atomicAdd(fv + lo, -lik * __ldcg(fv + t));
            }
        }
        if (l + 1 < nlev) {
            if (!grid_barrier(ds, gen)) return;
        }
    }
}

// LU solve in push form, in place on row-major n x p blocks (p <= 256): forward sweep, level by
// level, a warp per unit-L entry (i, k) whose source row k is final: y_i -= l_ik y_k; backward
// sweep, a warp per U entry (i, k), i < k: y_i -= (u_ik / u_kk) y_k with y_k not yet divided;
// finally y_k /= u_kk.  Rows of a level receive atomic contributions from many entries at once,
// so a level's work is spread over all the factor entries, not over its (few, long) rows.
__global__ void __launch_bounds__(512) lu_push_solve_kernel(int n, int p, int nlev0, const int *__restrict__ ptr0,
                                                            const int *__restrict__ src0, const int *__restrict__ dst0,
                                                            const int *__restrict__ pos0, int nlev1,
                                                            const int *__restrict__ ptr1, const int *__restrict__ src1,
                                                            const int *__restrict__ dst1, const int *__restrict__ pos1,
                                                            const int *__restrict__ diag, const double *__restrict__ fv,
                                                            double *Y, DevStatus *ds) {
    __shared__ unsigned s_gen;
    if (threadIdx.x == 0) s_gen = barrier_gen_start(ds);
    __syncthreads();
    unsigned gen = s_gen;
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (blockDim.x >> 5);
    for (int sweep = 0; sweep < 2; sweep++) {
        const int nlev = sweep == 0 ? nlev0 : nlev1;
        const int *ptr = sweep == 0 ? ptr0 : ptr1, *src = sweep == 0 ? src0 : src1,
                  *dst = sweep == 0 ? dst0 : dst1, *pos = sweep == 0 ? pos0 : pos1;
        for (int l = 0; l < nlev; l++) {
            const int q0 = __ldg(ptr + l), q1 = __ldg(ptr + l + 1);
            for (int q = q0 + gw; q < q1; q += nw) {
                const int k = __ldg(src + q), i = __ldg(dst + q);
                double a = __ldg(fv + __ldg(pos + q));
                if (sweep == 1) a /= __ldg(fv + __ldg(diag + k));
                const double *yk = Y + (size_t)k * p;
                double *yi = Y + (size_t)i * p;
                for (int c = lane; c < p; c += 32) atomicAdd(yi + c, -a * __ldcg(yk + c));
            }
            if (!grid_barrier(ds, gen)) return;
        }
    }
    const size_t total = (size_t)n * p;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x)
        Y[e] = __ldcg(Y + e) / __ldg(fv + __ldg(diag + e / p));
}

// Cooperative grid size: enough blocks for the widest level, capped by co-residency.
template <typename K>
static bpf_status coop_grid(bpf_ctx *ctx, K kernel, int threads, size_t smem, int want,
                            int *grid) {
    int per_sm = 0;
    BPF_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    if (per_sm < 1) return set_error(ctx, BPF_ERR_CUDA, "cooperative kernel does not fit on an SM");
    int cap = per_sm * ctx->num_sms;
    *grid = std::max(1, std::min(want, cap));
    return BPF_SUCCESS;
}

bpf_status factor_numeric(bpf_ctx *ctx, bpf_prec *P) {
    if (P->kind == PREC_LU && P->cl_nlev > 0 && P->pairless) {
        int grid = 1;
        BPF_TRY(coop_grid(ctx, lu_colstep_search_kernel, 256, 0, std::max(1, ceil_div(P->cl_max_level, 8)), &grid));
        int nlev = P->cl_nlev;
        const int *lp = P->cl_lev_ptr, *en = P->cl_ent, *er = P->cl_row, *rp = P->rp, *ci = P->ci, *dg = P->diag;
        double *fv = P->fv;
        DevStatus *ds = ctx->dstat;
        void *args[] = {&nlev, (void *)&lp, (void *)&en, (void *)&er, (void *)&rp, (void *)&ci, (void *)&dg, &fv, &ds};
        // Algorithmic bytes: the factor values read and written once, the entry lists, and per
        // update a column index, a value read and one atomically updated (the search's reads of
        // row i are cached re-reads)
        KScope ks(ctx, BPF_KC_FACTOR, 16.0 * P->nnz + 8.0 * (P->n + 1) + 28.0 * P->npairs, 2.0 * P->npairs);
        BPF_CUDA(ctx, cudaLaunchCooperativeKernel((const void *)lu_colstep_search_kernel, dim3(grid), dim3(256),
                                                  args, 0, ctx->stream));
        BPF_LAUNCHED(ctx);
        return BPF_SUCCESS;
    }
    if (P->kind == PREC_LU && P->cl_nlev > 0) {
        int grid = 1;
        BPF_TRY(coop_grid(ctx, lu_colstep_kernel, 256, 0, std::max(1, ceil_div(P->cl_max_level, 8)), &grid));
        int nlev = P->cl_nlev;
        const int *lp = P->cl_lev_ptr, *en = P->cl_ent, *ci = P->ci, *dg = P->diag, *pp = P->pp,
                  *pd = P->pdst, *ps = P->psrc;
        double *fv = P->fv;
        DevStatus *ds = ctx->dstat;
        void *args[] = {&nlev, (void *)&lp, (void *)&en, (void *)&ci, (void *)&dg, (void *)&pp,
                        (void *)&pd, (void *)&ps, &fv, &ds};
        // Algorithmic bytes: the factor values read and written once, the entry list, and per
        // update pair two indices, one value read and one atomically updated.
        KScope ks(ctx, BPF_KC_FACTOR, 16.0 * P->nnz + 8.0 * (P->n + 1) + 24.0 * P->npairs,
                  2.0 * P->npairs);
        BPF_CUDA(ctx, cudaLaunchCooperativeKernel((const void *)lu_colstep_kernel, dim3(grid), dim3(256),
                                                  args, 0, ctx->stream));
        BPF_LAUNCHED(ctx);
        return BPF_SUCCESS;
    }
    FactorArgs a;
    a.n = P->n;
    a.rp = P->rp;
    a.ci = P->ci;
    a.diag = P->diag;
    a.pp = P->pp;
    a.pdst = P->pdst;
    a.psrc = P->psrc;
    a.lev_ptr = P->lower.lev_ptr;
    a.rows = P->lower.rows;
    a.nlev = P->lower.nlev;
    a.ic = P->kind == PREC_IC0;
    a.fv = P->fv;
    a.ds = ctx->dstat;
    if (P->n == 0) return BPF_SUCCESS;
    int want = ceil_div(P->lower.max_level_rows, 8);
    int grid = 1;
    BPF_TRY(coop_grid(ctx, factor_coop_kernel, 256, 0, want, &grid));
    void *args[] = {&a};
    // Algorithmic bytes: factor values read and written once, the pattern, and the update
    // pairs' two indices; flops: two per update pair.
    KScope ks(ctx, BPF_KC_FACTOR, 16.0 * P->nnz + 4.0 * P->nnz + 8.0 * (P->n + 1) + 8.0 * P->npairs,
              2.0 * P->npairs);
    BPF_CUDA(ctx, cudaLaunchCooperativeKernel((const void *)factor_coop_kernel, dim3(grid),
                                              dim3(256), args, 0, ctx->stream));
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

// ------------------------------------------------------------------------------------
// triangular solves (cooperative; all levels of both factors in one launch)
// ------------------------------------------------------------------------------------
template <int G, int CPL, typename TF, bool IN_F32, bool OUT_F32>
__global__ void __launch_bounds__(512)
trsv2_coop_kernel(TriKernelArgs t0, TriKernelArgs t1, int p, const void *Xv, void *Yv,
                  DevStatus *ds, const int *gate, const int *perm, double *Zv) {
    __shared__ unsigned s_gen;
    __shared__ int s_skip;
    if (threadIdx.x == 0) s_gen = barrier_gen_start(ds);
    __syncthreads();
    unsigned gen = s_gen;
    if (gate) {
        // The gate (st->active) may be cleared by the other stream while the CTAs start, so CTAs
        // reading it themselves could disagree and leave the others waiting at a level barrier.
        // One decision for the grid: CTA 0 snapshots the gate before a barrier, every CTA reads
        // the snapshot after it, and either all CTAs leave or none does.
        if (blockIdx.x == 0 && threadIdx.x == 0) ds->pad[0] = (*gate == 0) ? 1 : 0;
        if (!grid_barrier(ds, gen)) return;
        if (threadIdx.x == 0) s_skip = ld_relaxed_i32(&ds->pad[0]);
        __syncthreads();
        if (s_skip) return;
    }
    using TIn = typename std::conditional<IN_F32, float, double>::type;
    using TOut = typename std::conditional<OUT_F32, float, double>::type;
    const TIn *X = (const TIn *)Xv;
    TOut *Yout = (TOut *)Yv;
    // Reordered factors (perm != null): the forward sweep gathers X's rows through perm and
    // writes the factor-ordered Z; the backward sweep reads Z and scatters Y's rows through
    // perm.  Otherwise both sweeps work in place in Y.
    TOut *Zf = perm ? (TOut *)Zv : Yout;
    const int lane = threadIdx.x & 31;
    const int glane = lane % G;
    const int gpb = blockDim.x / G;
    const int gid = blockIdx.x * gpb + threadIdx.x / G;
    const int ng = gridDim.x * gpb;
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (lane / G * G));
#pragma unroll 1
    for (int phase = 0; phase < 2; phase++) {
        const TriKernelArgs &t = phase == 0 ? t0 : t1;
        const TF *val = std::is_same<TF, float>::value ? (const TF *)t.valf : (const TF *)t.val;
        const TF *dinv = std::is_same<TF, float>::value ? (const TF *)t.dinvf : (const TF *)t.dinv;
        for (int l = 0; l < t.nlev; l++) {
            const int q0 = __ldg(t.lev_ptr + l), q1 = __ldg(t.lev_ptr + l + 1);
            for (int q = q0 + gid; q < q1; q += ng) {
                const int i = __ldg(t.rows + q);
                const int io = perm ? __ldg(perm + i) : i;   // row of i in the caller's order
                TOut *Y = (phase == 0) ? Zf : Yout;          // the sweep's solved rows
                TF acc[CPL];
#pragma unroll
                for (int j = 0; j < CPL; j++) {
                    const int col = glane + j * G;
                    if (col < p) {
                        if (phase == 0) acc[j] = (TF)X[(size_t)io * p + col];
                        else acc[j] = (TF)__ldcg(Zf + (size_t)i * p + col);
                    } else {
                        acc[j] = (TF)0;
                    }
                }
                const int rs = __ldg(t.rp + q), re = __ldg(t.rp + q + 1);
                for (int kb = rs; kb < re; kb += G) {
                    const int k = kb + glane;
                    int c = 0;
                    TF a = (TF)0;
                    if (k < re) {
                        c = __ldg(t.ci + k);
                        a = __ldg(val + k);
                    }
                    const int cnt = min(G, re - kb);
                    int co = 0;
                    if (k < re && perm && phase == 1) co = __ldg(perm + c);
                    #pragma unroll 4   // several entries' loads in flight; same summation order
                    for (int s = 0; s < cnt; s++) {
                        const int cs = __shfl_sync(gmask, (perm && phase == 1) ? co : c, s, G);
                        const TF as = __shfl_sync(gmask, a, s, G);
                        const TOut *yr = Y + (size_t)cs * p;
#pragma unroll
                        for (int j = 0; j < CPL; j++) {
                            const int col = glane + j * G;
                            if (col < p) acc[j] -= as * (TF)__ldcg(yr + col);
                        }
                    }
                }
                TF dv = (TF)1;
                if (dinv) dv = __ldg(dinv + q);
                TOut *yi = Y + (size_t)((phase == 1) ? io : i) * p;
#pragma unroll
                for (int j = 0; j < CPL; j++) {
                    const int col = glane + j * G;
                    if (col < p) yi[col] = (TOut)(acc[j] * dv);
                }
            }
            const bool last = (phase == 1 && l + 1 == t.nlev);
            if (!last) {
                if (!grid_barrier(ds, gen)) return;
            }
        }
    }
}

template <int G, int CPL, typename TF, bool IN_F32, bool OUT_F32>
static bpf_status launch_trsv2(bpf_ctx *ctx, const TriDev &t0, const TriDev &t1, int p,
                               const void *X, void *Y, const int *gate, const int *perm,
                               double *Z) {
    auto kern = trsv2_coop_kernel<G, CPL, TF, IN_F32, OUT_F32>;
    const int maxrows = std::max(t0.max_level_rows, t1.max_level_rows);
    int threads, grid;
    // Small levels: one block of 512 threads, barriers are __syncthreads.
    if (maxrows <= 2 * (512 / G)) {
        threads = 512;
        grid = 1;
    } else {
        // At most one CTA of 512 threads per SM: the level barriers cost one arrival per CTA,
        // so fewer, wider CTAs make every level cheaper (the widest levels still get a group
        // of lanes per row).
        threads = 512;
        BPF_TRY(coop_grid(ctx, kern, threads, 0,
                          std::min(ceil_div(maxrows, threads / G), ctx->num_sms), &grid));
    }
    TriKernelArgs a0 = t0.args(), a1 = t1.args();
    DevStatus *ds = ctx->dstat;
    void *args[] = {&a0, &a1, &p, (void *)&X, &Y, &ds, (void *)&gate, (void *)&perm, &Z};
    // Algorithmic bytes: (4 + sizeof(TF)) per off-diagonal entry of both factors, the
    // diagonal inverses, row pointers and row ids, and 4 n p vector values (read X, write Y,
    // read and write Y in the backward sweep).
    const double fb = (4.0 + sizeof(TF)) * ((double)t0.nnz + t1.nnz) + sizeof(TF) * (double)t0.n +
                      16.0 * (t0.n + 1) + 8.0 * t0.n;
    const double vb = (double)t0.n * p * ((IN_F32 ? 4.0 : 8.0) + 2.0 * (OUT_F32 ? 4.0 : 8.0) +
                                          (OUT_F32 ? 4.0 : 8.0));
    KScope ks(ctx, BPF_KC_TRSV, fb + vb, 2.0 * ((double)t0.nnz + t1.nnz + t0.n) * p);
    BPF_CUDA(ctx, cudaLaunchCooperativeKernel((const void *)kern, dim3(grid), dim3(threads), args, 0,
                                              ctx->stream));
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

// ------------------------------------------------------------------------------------
// Sync-free triangular solves (p >= 17: a warp per row, lanes over the right-hand sides).
//
// The level-scheduled kernel above separates every dependency level by a grid barrier (~5 us
// each, 26 + 26 of them on the 9,000-bus minimum-degree factors).  Here the rows of a sweep are
// taken in level order, position q by warp q mod W (W = all warps of the co-resident grid), and
// a row waits only for the rows it reads: lane l polls the ready word of the row of entry l
// (acquire), the warp proceeds when all its lanes have seen theirs.  A producer writes its row,
// then publishes it (warp barrier + release store of the word).  No deadlock: the pending row of
// smallest position has all its inputs done (they sit at smaller positions), and its warp is
// resident (cooperative launch) and has finished its earlier positions, so it runs.  Every poll
// is bounded by the context's wait limit; a warp that gives up records the timeout and returns,
// so the rows waiting on it give up too.  One grid barrier separates the two sweeps (the
// backward sweep overwrites in place what forward rows may still read when the pattern is not
// symmetric).  Ready words: 2e after the forward sweep of launch e, 2e + 1 after the backward
// sweep, so they are monotone and never reset.  Same arithmetic, summation order and
// permutation handling as trsv2_coop_kernel, so the results are bit-identical.
// ------------------------------------------------------------------------------------
template <int CPL, typename TF>
__global__ void __launch_bounds__(512)
trsv_sf_kernel(TriKernelArgs t0, TriKernelArgs t1, int p, const double *X, double *Yout,
               DevStatus *ds, const int *gate, const int *perm, double *Zv, unsigned *flags,
               unsigned epoch) {
    __shared__ unsigned s_gen;
    __shared__ int s_skip;
    if (threadIdx.x == 0) s_gen = barrier_gen_start(ds);
    __syncthreads();
    unsigned gen = s_gen;
    if (gate) {   // one decision for the grid, as in trsv2_coop_kernel
        if (blockIdx.x == 0 && threadIdx.x == 0) ds->pad[0] = (*gate == 0) ? 1 : 0;
        if (!grid_barrier(ds, gen)) return;
        if (threadIdx.x == 0) s_skip = ld_relaxed_i32(&ds->pad[0]);
        __syncthreads();
        if (s_skip) return;
    }
    double *Zf = perm ? Zv : Yout;
    const int lane = threadIdx.x & 31;
    const int wid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int nw = gridDim.x * (blockDim.x >> 5);
    const long long lim = ds->wait_limit > 0 ? ds->wait_limit : kSpinLimit;
    bool alive = true;
#pragma unroll 1
    for (int phase = 0; phase < 2; phase++) {
        const TriKernelArgs &t = phase == 0 ? t0 : t1;
        const TF *val = std::is_same<TF, float>::value ? (const TF *)t.valf : (const TF *)t.val;
        const TF *dinv = std::is_same<TF, float>::value ? (const TF *)t.dinvf : (const TF *)t.dinv;
        const unsigned want = 2u * epoch + (unsigned)phase;   // ready word of a row this sweep reads
        double *Y = phase == 0 ? Zf : Yout;                     // the sweep's solved rows
        // the next position's row id, entry range and first 32 entries are loaded while the
        // current row waits and gathers (they do not depend on any row's result)
        int nx_i = 0, nx_rs = 0, nx_re = 0, nx_c = 0;
        TF nx_a = (TF)0;
        if (wid < t.n) {
            nx_i = __ldg(t.rows + wid);
            nx_rs = __ldg(t.rp + wid);
            nx_re = __ldg(t.rp + wid + 1);
            if (nx_rs + lane < nx_re) {
                nx_c = __ldg(t.ci + nx_rs + lane);
                nx_a = __ldg(val + nx_rs + lane);
            }
        }
        for (int q = wid; alive && q < t.n; q += nw) {
            const int i = nx_i, rs = nx_rs, re = nx_re;
            const int c0 = nx_c;
            const TF a0 = nx_a;
            if (q + nw < t.n) {
                nx_i = __ldg(t.rows + q + nw);
                nx_rs = __ldg(t.rp + q + nw);
                nx_re = __ldg(t.rp + q + nw + 1);
                nx_c = 0;
                nx_a = (TF)0;
                if (nx_rs + lane < nx_re) {
                    nx_c = __ldg(t.ci + nx_rs + lane);
                    nx_a = __ldg(val + nx_rs + lane);
                }
            }
            const int io = perm ? __ldg(perm + i) : i;   // row of i in the caller's order
            TF acc[CPL];
#pragma unroll
            for (int j = 0; j < CPL; j++) {
                const int col = lane + j * 32;
                if (col < p) {
                    if (phase == 0) acc[j] = (TF)X[(size_t)io * p + col];
                    else acc[j] = (TF)__ldcg(Zf + (size_t)i * p + col);
                } else {
                    acc[j] = (TF)0;
                }
            }
            for (int kb = rs; kb < re; kb += 32) {
                const int k = kb + lane;
                int c = 0;
                TF a = (TF)0;
                bool ok = true;
                if (k < re) {
                    c = kb == rs ? c0 : __ldg(t.ci + k);
                    a = kb == rs ? a0 : __ldg(val + k);
                    // bounded wait for row c of this sweep (acquire polls: measured faster than
                    // relaxed polls followed by one acquire fence, 92 vs 105 us at 9,000 buses)
                    long long it = 0;
                    while (ld_acquire_u32(flags + c) < want) {
                        if (++it > lim || ld_relaxed_i32(&ds->err) != 0) {
                            ok = false;
                            break;
                        }
                        __nanosleep(32);
                    }
                }
                __syncwarp();   // orders every lane's acquire before the warp's reads of those rows
                if (!__all_sync(0xffffffffu, ok)) {
                    if (!ok) atomicCAS(&ds->err, 0, (int)DEV_BARRIER_TIMEOUT);
                    alive = false;
                    break;
                }
                const int cnt = min(32, re - kb);
                int co = 0;
                if (k < re && perm && phase == 1) co = __ldg(perm + c);
#pragma unroll 4   // several entries' loads in flight; same summation order as the level kernel
                for (int s = 0; s < cnt; s++) {
                    const int cs = __shfl_sync(0xffffffffu, (perm && phase == 1) ? co : c, s);
                    const TF as = __shfl_sync(0xffffffffu, a, s);
                    const double *yr = Y + (size_t)cs * p;
#pragma unroll
                    for (int j = 0; j < CPL; j++) {
                        const int col = lane + j * 32;
                        if (col < p) acc[j] -= as * (TF)__ldcg(yr + col);
                    }
                }
            }
            if (!alive) break;
            TF dv = (TF)1;
            if (dinv) dv = __ldg(dinv + q);
            double *yi = Y + (size_t)((phase == 1) ? io : i) * p;
#pragma unroll
            for (int j = 0; j < CPL; j++) {
                const int col = lane + j * 32;
                if (col < p) yi[col] = (double)(acc[j] * dv);
            }
            // publish: the warp barrier orders every lane's row stores before lane 0's release
            // store, whose gpu-scope release makes them visible to a reader that acquires the
            // word (happens-before is transitive through the barrier), so no separate fence
            __syncwarp();
            if (lane == 0) st_release_u32(flags + i, 2u * epoch + (unsigned)phase);
        }
        if (phase == 0) {
            // every CTA reaches this barrier: a warp that gave up still arrives (its CTA's
            // threads all call it), and the barrier itself sees the pending error
            if (!grid_barrier(ds, gen)) return;
            if (!alive) return;
        }
    }
}

template <int CPL, typename TF>
static bpf_status launch_trsv_sf(bpf_ctx *ctx, const TriDev &t0, const TriDev &t1, int p, const void *X,
                                 void *Y, const int *gate, const int *perm, double *Z, unsigned *flags,
                                 unsigned epoch) {
    auto kern = trsv_sf_kernel<CPL, TF>;
    int per_sm = 0;
    BPF_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 512, 0));
    if (per_sm < 1) return set_error(ctx, BPF_ERR_CUDA, "sync-free triangular solve does not fit on an SM");
    // every warp resident; no more warps than rows of the larger sweep
    const int grid = std::max(1, std::min(per_sm * ctx->num_sms, ceil_div(std::max(t0.n, 1), 16)));
    TriKernelArgs a0 = t0.args(), a1 = t1.args();
    DevStatus *ds = ctx->dstat;
    void *args[] = {&a0, &a1, &p, (void *)&X, &Y, &ds, (void *)&gate, (void *)&perm, &Z, &flags, &epoch};
    const double fb = (4.0 + sizeof(TF)) * ((double)t0.nnz + t1.nnz) + sizeof(TF) * (double)t0.n +
                      16.0 * (t0.n + 1) + 8.0 * t0.n;
    const double vb = (double)t0.n * p * 32.0;
    KScope ks(ctx, BPF_KC_TRSV, fb + vb, 2.0 * ((double)t0.nnz + t1.nnz + t0.n) * p);
    BPF_CUDA(ctx, cudaLaunchCooperativeKernel((const void *)kern, dim3(grid), dim3(512), args, 0, ctx->stream));
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

template <typename TF, bool IN_F32, bool OUT_F32>
static bpf_status trsv2_dispatch(bpf_ctx *ctx, const TriDev &t0, const TriDev &t1, int p,
                                 const void *X, void *Y, const int *gate, const int *perm,
                                 double *Z, unsigned *flags = nullptr, unsigned epoch = 0) {
    // sync-free for blocks of 17..256 columns whose level-scheduled launch would span several CTAs
    static const bool levels_only = getenv("BPF_TRSV_LEVELS") && atoi(getenv("BPF_TRSV_LEVELS")) != 0;
    if (!IN_F32 && !OUT_F32 && flags && !levels_only && p > 16 && p <= 256 &&
        std::max(t0.max_level_rows, t1.max_level_rows) > 2 * (512 / 32)) {
        if (p <= 32) return launch_trsv_sf<1, TF>(ctx, t0, t1, p, X, Y, gate, perm, Z, flags, epoch);
        if (p <= 64) return launch_trsv_sf<2, TF>(ctx, t0, t1, p, X, Y, gate, perm, Z, flags, epoch);
        if (p <= 128) return launch_trsv_sf<4, TF>(ctx, t0, t1, p, X, Y, gate, perm, Z, flags, epoch);
        return launch_trsv_sf<8, TF>(ctx, t0, t1, p, X, Y, gate, perm, Z, flags, epoch);
    }
    if (p <= 4) return launch_trsv2<4, 1, TF, IN_F32, OUT_F32>(ctx, t0, t1, p, X, Y, gate, perm, Z);
    if (p <= 8) return launch_trsv2<8, 1, TF, IN_F32, OUT_F32>(ctx, t0, t1, p, X, Y, gate, perm, Z);
    if (p <= 16) return launch_trsv2<16, 1, TF, IN_F32, OUT_F32>(ctx, t0, t1, p, X, Y, gate, perm, Z);
    if (p <= 32) return launch_trsv2<32, 1, TF, IN_F32, OUT_F32>(ctx, t0, t1, p, X, Y, gate, perm, Z);
    if (p <= 64) return launch_trsv2<32, 2, TF, IN_F32, OUT_F32>(ctx, t0, t1, p, X, Y, gate, perm, Z);
    if (p <= 128) return launch_trsv2<32, 4, TF, IN_F32, OUT_F32>(ctx, t0, t1, p, X, Y, gate, perm, Z);
    if (p <= 256) return launch_trsv2<32, 8, TF, IN_F32, OUT_F32>(ctx, t0, t1, p, X, Y, gate, perm, Z);
    return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "triangular solve: p=%d > 256 per call", p);
}

// Y = P \ X on row-major n x p blocks (FP64 in/out).  Blocks wider than 256 columns are
// solved in 256-column slices by the caller.
bpf_status prec_apply_rowmajor(bpf_ctx *ctx, const bpf_prec *P, int p, const double *X,
                               double *Y, const int *gate) {
    if (P->n == 0 || p == 0) return BPF_SUCCESS;
    if (P->kind == PREC_BJ) return bj_apply_rowmajor(ctx, P, p, X, Y);   // mul! semantics
    if (P->perm && p > P->zcols)
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED,
                         "reordered preconditioner: %d right-hand sides exceed the %d-column scratch "
                         "reserved for it", p, P->zcols);
    if (P->fdtype == BPF_F32)
        return trsv2_dispatch<float, false, false>(ctx, P->lower, P->upper, p, X, Y, gate, P->perm, P->zbuf,
                                                   P->sf_flags, ++P->sf_epoch);
    return trsv2_dispatch<double, false, false>(ctx, P->lower, P->upper, p, X, Y, gate, P->perm, P->zbuf,
                                                P->sf_flags, ++P->sf_epoch);
}

bpf_status prec_reserve_z(bpf_ctx *ctx, bpf_prec *P, int p) {
    if (!P->perm || p <= P->zcols) return BPF_SUCCESS;
    const int cols = std::min(std::max(p, 1), 256);
    double *z = nullptr;
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    BPF_CUDA(ctx, cudaMalloc((void **)&z, sizeof(double) * (size_t)P->n * cols));
    if (P->zbuf) cudaFree(P->zbuf);
    P->zbuf = z;
    P->zcols = cols;
    return BPF_SUCCESS;
}

__global__ void scatter_map_kernel(int nnz, const double *__restrict__ vals, const int *__restrict__ map,
                                   double *__restrict__ out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x)
        out[__ldg(map + k)] = vals[k];
}

bpf_status prec_load_values(bpf_ctx *ctx, bpf_prec *P, const double *vals) {
    if (P->nnz == 0) return BPF_SUCCESS;
    if (!P->amap) {
        BPF_CUDA(ctx, cudaMemcpyAsync(P->fv, vals, sizeof(double) * P->nnz, cudaMemcpyDeviceToDevice,
                                      ctx->stream));
        return BPF_SUCCESS;
    }
    const int blocks = std::max(1, std::min(ceil_div(P->nnz, 256), ctx->num_sms * 8));
    scatter_map_kernel<<<blocks, 256, 0, ctx->stream>>>(P->nnz, vals, P->amap, P->fv);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

bpf_status lu_solve_push_rowmajor(bpf_ctx *ctx, const bpf_prec *P, int p, double *Y) {
    if (P->n == 0 || p == 0) return BPF_SUCCESS;
    if (p > 256) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "LU solve: p=%d > 256 per call", p);
    int grid = 1;
    BPF_TRY(coop_grid(ctx, lu_push_solve_kernel, 512, 0,
                      std::min(ctx->num_sms * 2, std::max(1, ceil_div(P->ps_max_level, 16))), &grid));
    int n = P->n, nl0 = P->ps_nlev[0], nl1 = P->ps_nlev[1];
    const int *p0 = P->ps_ptr[0], *s0 = P->ps_src[0], *d0 = P->ps_dst[0], *q0 = P->ps_pos[0];
    const int *p1 = P->ps_ptr[1], *s1 = P->ps_src[1], *d1 = P->ps_dst[1], *q1 = P->ps_pos[1];
    const int *dg = P->diag;
    const double *fv = P->fv;
    DevStatus *ds = ctx->dstat;
    void *args[] = {&n, &p, &nl0, (void *)&p0, (void *)&s0, (void *)&d0, (void *)&q0, &nl1, (void *)&p1,
                    (void *)&s1, (void *)&d1, (void *)&q1, (void *)&dg, (void *)&fv, &Y, &ds};
    // Algorithmic bytes: per factor entry 3 indices and its value, the block read once per
    // entry's source row and target row updated (atomics), read and written once at the end.
    const double nnz_off = (double)P->nnz - P->n;
    KScope ks(ctx, BPF_KC_TRSV, 20.0 * nnz_off + 8.0 * P->n + 32.0 * (double)P->n * p,
              2.0 * (nnz_off + P->n) * p);
    BPF_CUDA(ctx, cudaLaunchCooperativeKernel((const void *)lu_push_solve_kernel, dim3(grid), dim3(512), args, 0,
                                              ctx->stream));
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

}  // namespace bpf
