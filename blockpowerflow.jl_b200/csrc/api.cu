// C ABI: context, errors, workspace, SpMM and preconditioner entry points.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bpf_internal.cuh"
#include "ordering.cuh"
#include "prec.cuh"

namespace bpf {

bpf_status set_error(bpf_ctx *ctx, bpf_status st, const char *fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return st;
}

bpf_status cuda_error(bpf_ctx *ctx, cudaError_t e, const char *what, const char *file, int line) {
    bpf_status st = (e == cudaErrorMemoryAllocation) ? BPF_ERR_ALLOC : BPF_ERR_CUDA;
    return set_error(ctx, st, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
}

void *ws_get(bpf_ctx *ctx, int slot, size_t bytes, bpf_status *st) {
    *st = BPF_SUCCESS;
    if (bytes == 0) bytes = 16;
    if (ctx->ws_bytes[slot] >= bytes) return ctx->ws[slot];
    if (ctx->ws[slot]) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->ws[slot]);
        ctx->ws[slot] = nullptr;
        ctx->ws_bytes[slot] = 0;
    }
    size_t want = bytes + bytes / 4;
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *st = set_error(ctx, BPF_ERR_ALLOC, "workspace allocation of %zu bytes failed: %s", want,
                        cudaGetErrorString(e));
        return nullptr;
    }
    ctx->ws[slot] = p;
    ctx->ws_bytes[slot] = want;
    return p;
}

cudaEvent_t timing_event(bpf_ctx *ctx) {
    if (ctx->event_next >= ctx->event_pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        ctx->event_pool.push_back(e);
    }
    return ctx->event_pool[ctx->event_next++];
}

bpf_status reset_dev_status(bpf_ctx *ctx) {
    // the error word and the barrier state; the wait limit stays as the caller set it
    BPF_CUDA(ctx, cudaMemsetAsync(ctx->dstat, 0, offsetof(DevStatus, wait_limit), ctx->stream));
    return BPF_SUCCESS;
}

bpf_status check_dev_status(bpf_ctx *ctx, const char *where) {
    BPF_CUDA(ctx, cudaMemcpyAsync(ctx->hstat, ctx->dstat, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    int err = ctx->hstat->err, aux = ctx->hstat->aux;
    if (err == DEV_OK) return BPF_SUCCESS;
    // Clear the word (and the barrier state a timed-out barrier may have left) for the next call.
    BPF_TRY(reset_dev_status(ctx));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    switch (err) {
        case DEV_ZERO_PIVOT:
            return set_error(ctx, BPF_ERR_SINGULAR, "%s: zero pivot at row %d", where, aux);
        case DEV_BARRIER_TIMEOUT:
            return set_error(ctx, BPF_ERR_TIMEOUT, "%s: a device-side wait timed out", where);
        case DEV_NONFINITE:
            return set_error(ctx, BPF_ERR_NUMERIC, "%s: non-finite value at %d", where, aux);
        case DEV_CHOL_FAIL:
            return set_error(ctx, BPF_ERR_NUMERIC, "%s: Cholesky-QR breakdown", where);
        default:
            return set_error(ctx, BPF_ERR_CUDA, "%s: device error %d", where, err);
    }
}

// Validate a CSR descriptor and copy its pattern to the host (0-based).
bpf_status csr_pattern_to_host(bpf_ctx *ctx, const bpf_csr_desc *A, std::vector<int> &rp,
                               std::vector<int> &ci, bool need_diag, std::vector<int> *diag) {
    if (!A) return set_error(ctx, BPF_ERR_INVALID_VALUE, "null CSR descriptor");
    if (A->n < 0 || A->nnz < 0 || (A->n > 0 && (!A->rowptr || (A->nnz > 0 && (!A->colind || !A->vals)))))
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "invalid CSR descriptor");
    if (A->index_base != 0 && A->index_base != 1)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "index_base must be 0 or 1");
    int n = A->n, nnz = A->nnz, b = A->index_base;
    rp.resize(n + 1);
    ci.resize(nnz);
    if (n > 0)
        BPF_CUDA(ctx, cudaMemcpyAsync(rp.data(), A->rowptr, sizeof(int) * (n + 1),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    if (nnz > 0)
        BPF_CUDA(ctx, cudaMemcpyAsync(ci.data(), A->colind, sizeof(int) * nnz,
                                      cudaMemcpyDeviceToHost, ctx->stream));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (b) {
        for (auto &v : rp) v -= b;
        for (auto &v : ci) v -= b;
    }
    if (n > 0 && (rp[0] != 0 || rp[n] != nnz))
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "rowptr inconsistent with nnz=%d", nnz);
    for (int i = 0; i < n; i++) {
        if (rp[i + 1] < rp[i]) return set_error(ctx, BPF_ERR_INVALID_VALUE, "rowptr not monotone");
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            if (ci[k] < 0 || ci[k] >= n)
                return set_error(ctx, BPF_ERR_INVALID_VALUE, "column index out of range in row %d", i);
            if (k > rp[i] && ci[k] <= ci[k - 1])
                return set_error(ctx, BPF_ERR_INVALID_VALUE, "columns of row %d not sorted/unique", i);
        }
    }
    if (need_diag) {
        diag->assign(n, -1);
        for (int i = 0; i < n; i++) {
            for (int k = rp[i]; k < rp[i + 1]; k++)
                if (ci[k] == i) { (*diag)[i] = k; break; }
            if ((*diag)[i] < 0)
                return set_error(ctx, BPF_ERR_SINGULAR, "structural zero pivot: A(%d,%d) missing", i, i);
        }
    }
    return BPF_SUCCESS;
}

// Analyse a 0-based host pattern (sorted rows, diagonal present) and upload everything the
// numeric factorization and the triangular solves need.  P->fv is allocated, not filled.
// kind PREC_ILU0 / PREC_LU: unit L + U on the pattern; PREC_IC0: L and L' (lower part).
bpf_status prec_setup(bpf_ctx *ctx, int kind, int n, const std::vector<int> &rp,
                      const std::vector<int> &ci, const std::vector<int> &diag, bpf_prec **out) {
    *out = nullptr;
    const int nnz = n > 0 ? rp[n] : 0;
    bpf_prec *P = new bpf_prec();
    P->ctx = ctx;
    P->kind = kind;
    P->n = n;
    P->nnz = nnz;
    const bool ic = (kind == PREC_IC0);
    TriHost lo = build_tri(n, rp.data(), ci.data(), diag.data(), 0, !ic);
    TriHost up = ic ? build_tri(n, rp.data(), ci.data(), diag.data(), 2, false)
                    : build_tri(n, rp.data(), ci.data(), diag.data(), 1, false);
    std::vector<int> pp;
    PairVec pdst, psrc;
    const char *env_pl = getenv("BPF_LU_PAIRLESS");
    const bool force_pairless = kind == PREC_LU && env_pl && atoi(env_pl) != 0;
    const bool pairs_ok = !force_pairless && build_pairs(n, rp.data(), ci.data(), diag.data(), ic, pp, pdst, psrc);
    P->npairs = (long long)pdst.size();
    auto fail = [&](bpf_status s) {
        cudaStreamSynchronize(ctx->stream);
        bpf_prec_destroy(P);
        return s;
    };
    if (!pairs_ok && kind != PREC_LU)
        return fail(set_error(ctx, BPF_ERR_NOT_SUPPORTED,
                              "factorization update pairs exceed 2^31 - 1 (pattern of %d entries too dense)", nnz));
    if (!pairs_ok) {
        // the LU refactorization finds each L entry's updates by a search in its row instead
        P->pairless = true;
        long long upd = 0;
        for (int i = 0; i < n; i++)
            for (int q = rp[i]; q < diag[i]; q++) upd += rp[ci[q] + 1] - diag[ci[q]] - 1;
        P->npairs = upd;
    }
    bpf_status s;
    if ((s = tri_upload(ctx, lo, P->lower)) != BPF_SUCCESS) return fail(s);
    if ((s = tri_upload(ctx, up, P->upper)) != BPF_SUCCESS) return fail(s);
    cudaError_t e = cudaSuccess;
    auto up_i = [&](int **d, const auto &h) {   // std::vector<int> or PairVec
        if (e != cudaSuccess || h.empty()) return;
        e = cudaMalloc((void **)d, sizeof(int) * h.size());
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(*d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, ctx->stream);
    };
    if (kind != PREC_LU && n > 0) {
        if (e == cudaSuccess) e = cudaMalloc((void **)&P->sf_flags, sizeof(unsigned) * n);
        if (e == cudaSuccess) e = cudaMemsetAsync(P->sf_flags, 0, sizeof(unsigned) * n, ctx->stream);
    }
    up_i(&P->rp, rp);
    up_i(&P->ci, ci);
    up_i(&P->diag, diag);
    up_i(&P->pp, pp);
    up_i(&P->pdst, pdst);
    up_i(&P->psrc, psrc);
    if (kind == PREC_LU && n > 0) {
        // column-step levels: step k depends on the steps j < k with L(k, j) != 0 (they update
        // row k) or U(j, k) != 0 (they update column k)
        std::vector<int> lev(n, 0);
        std::vector<std::vector<int>> ucol(n);   // ucol[k]: rows j < k with U(j, k) != 0
        for (int j = 0; j < n; j++)
            for (int q = diag[j] + 1; q < rp[j + 1]; q++) ucol[ci[q]].push_back(j);
        int nlev = 0;
        for (int k = 0; k < n; k++) {
            int l = 0;
            for (int q = rp[k]; q < diag[k]; q++) l = std::max(l, lev[ci[q]] + 1);
            for (int j : ucol[k]) l = std::max(l, lev[j] + 1);
            lev[k] = l;
            nlev = std::max(nlev, l + 1);
            std::vector<int>().swap(ucol[k]);
        }
        std::vector<int> lptr(nlev + 1, 0), ent;
        for (int i = 0; i < n; i++)
            for (int q = rp[i]; q < diag[i]; q++) lptr[lev[ci[q]] + 1]++;
        for (int l = 0; l < nlev; l++) lptr[l + 1] += lptr[l];
        ent.resize(lptr[nlev]);
        std::vector<int> fill(lptr.begin(), lptr.end() - 1);
        for (int i = 0; i < n; i++)
            for (int q = rp[i]; q < diag[i]; q++) ent[fill[lev[ci[q]]]++] = q;
        int mx = 0;
        for (int l = 0; l < nlev; l++) mx = std::max(mx, lptr[l + 1] - lptr[l]);
        P->cl_nlev = nlev;
        P->cl_max_level = mx;
        up_i(&P->cl_lev_ptr, lptr);
        up_i(&P->cl_ent, ent);
        if (P->pairless) {
            std::vector<int> erow(ent.size());
            std::vector<int> rowof(nnz > 0 ? nnz : 1);
            for (int i = 0; i < n; i++)
                for (int q = rp[i]; q < rp[i + 1]; q++) rowof[q] = i;
            for (size_t t = 0; t < ent.size(); t++) erow[t] = rowof[ent[t]];
            up_i(&P->cl_row, erow);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        }
        // push lists of the two sweeps: forward, L entry (i, k) leaves row k (level of k in
        // the forward sweep) for row i; backward, U entry (i, k), i < k, leaves row k for row i
        int pmx = 0;
        for (int sweep = 0; sweep < 2; sweep++) {
            const TriHost &t = sweep == 0 ? lo : up;
            std::vector<int> lv(n, 0);
            for (int l = 0; l < t.nlev; l++)
                for (int q = t.lev_ptr[l]; q < t.lev_ptr[l + 1]; q++) lv[t.rows[q]] = l;
            std::vector<int> ptr(t.nlev + 1, 0);
            for (int i = 0; i < n; i++)
                for (int q = rp[i]; q < rp[i + 1]; q++) {
                    const int k = ci[q];
                    if (sweep == 0 ? (k < i) : (k > i)) ptr[lv[k] + 1]++;
                }
            for (int l = 0; l < t.nlev; l++) {
                pmx = std::max(pmx, ptr[l + 1]);
                ptr[l + 1] += ptr[l];
            }
            std::vector<int> src(ptr[t.nlev]), dst(ptr[t.nlev]), pos(ptr[t.nlev]);
            std::vector<int> fl(ptr.begin(), ptr.end() - 1);
            for (int i = 0; i < n; i++)
                for (int q = rp[i]; q < rp[i + 1]; q++) {
                    const int k = ci[q];
                    if (sweep == 0 ? (k < i) : (k > i)) {
                        const int w = fl[lv[k]]++;
                        src[w] = k;
                        dst[w] = i;
                        pos[w] = q;
                    }
                }
            P->ps_nlev[sweep] = t.nlev;
            up_i(&P->ps_ptr[sweep], ptr);
            up_i(&P->ps_src[sweep], src);
            up_i(&P->ps_dst[sweep], dst);
            up_i(&P->ps_pos[sweep], pos);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        }
        P->ps_max_level = pmx;
    }
    if (e == cudaSuccess && nnz > 0) e = cudaMalloc((void **)&P->fv, sizeof(double) * nnz);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // host vectors die on return
    if (e != cudaSuccess) return fail(cuda_error(ctx, e, "preconditioner setup", __FILE__, __LINE__));
    *out = P;
    return BPF_SUCCESS;
}

// Self-test of the bounded grid barrier: every block except `absent` (-1: none) meets at
// one grid barrier; if a block never arrives the others give up after the context's wait limit,
// record DEV_BARRIER_TIMEOUT and return.  `arrived` counts the blocks that passed the barrier.
__global__ void barrier_selftest_kernel(DevStatus *ds, int absent, int *arrived) {
    __shared__ unsigned s_gen;
    if (threadIdx.x == 0) s_gen = barrier_gen_start(ds);
    __syncthreads();
    unsigned gen = s_gen;
    if ((int)blockIdx.x == absent) return;
    if (!grid_barrier(ds, gen)) return;
    if (threadIdx.x == 0) atomicAdd(arrived, 1);
}

}  // namespace bpf

using namespace bpf;

extern "C" {

bpf_status bpf_ctx_create(bpf_ctx **out, void *stream) {
    if (!out) return BPF_ERR_INVALID_VALUE;
    *out = nullptr;
    bpf_ctx *ctx = new bpf_ctx();
    ctx->stream = (cudaStream_t)stream;
    if (const char *env = getenv("BPF_FP64_MMA")) ctx->fp64_mma = atoi(env) != 0;
    cudaError_t e = cudaGetDevice(&ctx->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&ctx->max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
    if (e == cudaSuccess) e = cudaMalloc((void **)&ctx->dstat, sizeof(DevStatus));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&ctx->hstat, sizeof(DevStatus));
    if (e == cudaSuccess) e = cudaMemset(ctx->dstat, 0, sizeof(DevStatus));
    if (const char *env = getenv("BPF_OVERLAP")) ctx->overlap = atoi(env) != 0;
    if (e == cudaSuccess) {
        int least = 0, greatest = 0;
        e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&ctx->hstream, cudaStreamNonBlocking, greatest);
    }
    for (int i = 0; i < 2 && e == cudaSuccess; i++) {
        e = cudaEventCreateWithFlags(&ctx->ev_a[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_b[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) noalloc_forget_device(ctx->device);
    if (e != cudaSuccess) {
        cudaGetLastError();
        for (int i = 0; i < 2; i++) {
            if (ctx->ev_a[i]) cudaEventDestroy(ctx->ev_a[i]);
            if (ctx->ev_b[i]) cudaEventDestroy(ctx->ev_b[i]);
        }
        if (ctx->hstream) cudaStreamDestroy(ctx->hstream);
        if (ctx->dstat) cudaFree(ctx->dstat);
        if (ctx->hstat) cudaFreeHost(ctx->hstat);
        delete ctx;
        return e == cudaErrorMemoryAllocation ? BPF_ERR_ALLOC : BPF_ERR_CUDA;
    }
    *out = ctx;
    return BPF_SUCCESS;
}

bpf_status bpf_ctx_set_stream(bpf_ctx *ctx, void *stream) {
    if (!ctx) return BPF_ERR_INVALID_VALUE;
    ctx->stream = (cudaStream_t)stream;
    return BPF_SUCCESS;
}

bpf_status bpf_ctx_destroy(bpf_ctx *ctx) {
    if (!ctx) return BPF_SUCCESS;
    cudaStreamSynchronize(ctx->stream);
    if (ctx->hstream) cudaStreamSynchronize(ctx->hstream);
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    for (int i = 0; i < 2; i++) {
        if (ctx->ev_a[i]) cudaEventDestroy(ctx->ev_a[i]);
        if (ctx->ev_b[i]) cudaEventDestroy(ctx->ev_b[i]);
    }
    if (ctx->hstream) cudaStreamDestroy(ctx->hstream);
    for (int s = 0; s < WS_COUNT; s++)
        if (ctx->ws[s]) cudaFree(ctx->ws[s]);
    cudaFree(ctx->dstat);
    cudaFreeHost(ctx->hstat);
    delete ctx;
    return BPF_SUCCESS;
}

const char *bpf_last_error(const bpf_ctx *ctx) {
    if (!ctx) return "null context";
    return ctx->last_error.c_str();
}

long long bpf_ctx_kernel_launches(const bpf_ctx *ctx) { return ctx ? ctx->launches : 0; }

bpf_status bpf_ctx_set_wait_limit(bpf_ctx *ctx, long long polls) {
    if (!ctx) return BPF_ERR_INVALID_VALUE;
    if (polls < 0) return set_error(ctx, BPF_ERR_INVALID_VALUE, "wait limit must be >= 0");
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->hstat->wait_limit = polls;
    BPF_CUDA(ctx, cudaMemcpyAsync(&ctx->dstat->wait_limit, &ctx->hstat->wait_limit, sizeof(long long),
                                  cudaMemcpyHostToDevice, ctx->stream));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BPF_SUCCESS;
}

bpf_status bpf_selftest_grid_barrier(bpf_ctx *ctx, int nblocks, int absent_block, int *arrived) {
    if (!ctx) return BPF_ERR_INVALID_VALUE;
    if (nblocks < 2 || absent_block < -1 || absent_block >= nblocks)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "selftest: nblocks >= 2 and -1 <= absent_block < nblocks");
    int per_sm = 0;
    BPF_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, barrier_selftest_kernel, 128, 0));
    if (nblocks > per_sm * ctx->num_sms)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "selftest: at most %d co-resident blocks", per_sm * ctx->num_sms);
    bpf_status st = BPF_SUCCESS;
    int *d_arrived = (int *)ws_get(ctx, WS_SMALL, sizeof(int), &st);
    if (!d_arrived) return st;
    BPF_CUDA(ctx, cudaMemsetAsync(d_arrived, 0, sizeof(int), ctx->stream));
    DevStatus *ds = ctx->dstat;
    void *args[] = {&ds, &absent_block, &d_arrived};
    BPF_CUDA(ctx, cudaLaunchCooperativeKernel((const void *)barrier_selftest_kernel, dim3(nblocks), dim3(128),
                                              args, 0, ctx->stream));
    BPF_LAUNCHED(ctx);
    int h = 0;
    BPF_CUDA(ctx, cudaMemcpyAsync(&h, d_arrived, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    st = check_dev_status(ctx, "selftest_grid_barrier");   // synchronizes the stream
    if (arrived) *arrived = h;
    return st;
}

bpf_status bpf_ctx_set_timing(bpf_ctx *ctx, int on) {
    if (!ctx) return BPF_ERR_INVALID_VALUE;
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->timed.clear();
    ctx->event_next = 0;
    ctx->timing = on != 0;
    return BPF_SUCCESS;
}

bpf_status bpf_ctx_kernel_time(bpf_ctx *ctx, int kc, double *total_ms, long long *launches,
                               double *bytes, double *flops) {
    if (!ctx || kc < 0 || kc >= BPF_KC_COUNT) return BPF_ERR_INVALID_VALUE;
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    double t = 0.0, by = 0.0, fl = 0.0;
    long long c = 0;
    for (const auto &r : ctx->timed) {
        if (r.kc != kc) continue;
        float ms = 0.f;
        BPF_CUDA(ctx, cudaEventElapsedTime(&ms, r.a, r.b));
        t += ms;
        by += r.bytes;
        fl += r.flops;
        c++;
    }
    if (total_ms) *total_ms = t;
    if (launches) *launches = c;
    if (bytes) *bytes = by;
    if (flops) *flops = fl;
    return BPF_SUCCESS;
}

const char *bpf_solve_status_string(int status) {
    switch (status) {
        case BPF_SOLVE_SOLVED: return "solution good enough given atol and rtol";
        case BPF_SOLVE_ITMAX: return "maximum number of iterations exceeded";
        case BPF_SOLVE_TIMEMAX: return "time limit exceeded";
        default: return "unknown";
    }
}

bpf_status bpf_spmm(bpf_ctx *ctx, const bpf_csr_desc *A, int p, double alpha, const double *X,
                    int ldx, double beta, double *Y, int ldy) {
    if (!ctx) return BPF_ERR_INVALID_VALUE;
    if (!A || p < 0 || (p > 0 && A->n > 0 && (!X || !Y)))
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "bpf_spmm: invalid argument");
    if (A->dtype != BPF_F64) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "bpf_spmm: FP64 matrices only");
    int n = A->n;
    if (ldx < std::max(1, n) || ldy < std::max(1, n))
        return set_error(ctx, BPF_ERR_DIMENSION, "bpf_spmm: leading dimension < n");
    if (n == 0 || p == 0) return BPF_SUCCESS;
    bpf_status st;
    const int chunk = 256;
    size_t cols = std::min(p, chunk);
    double *xr = (double *)ws_get(ctx, WS_A, sizeof(double) * (size_t)n * cols, &st);
    if (!xr) return st;
    double *yr = (double *)ws_get(ctx, WS_B, sizeof(double) * (size_t)n * cols, &st);
    if (!yr) return st;
    for (int c0 = 0; c0 < p; c0 += chunk) {
        int pc = std::min(chunk, p - c0);
        BPF_TRY(colmajor_to_rowmajor(ctx, n, pc, X + (size_t)c0 * ldx, ldx, xr));
        if (beta != 0.0) BPF_TRY(colmajor_to_rowmajor(ctx, n, pc, Y + (size_t)c0 * ldy, ldy, yr));
        BPF_TRY(spmm_rowmajor(ctx, n, A->nnz, A->rowptr, A->colind, (const double *)A->vals, A->index_base,
                              pc, alpha, xr, beta, yr, nullptr));
        BPF_TRY(rowmajor_to_colmajor(ctx, n, pc, yr, Y + (size_t)c0 * ldy, ldy));
    }
    return BPF_SUCCESS;
}

static bpf_status prec_create(bpf_ctx *ctx, const bpf_csr_desc *A, int nrhs, int fdtype,
                              int kind, int ordering, bpf_prec **out) {
    if (!ctx || !out) return BPF_ERR_INVALID_VALUE;
    *out = nullptr;
    if (!A) return set_error(ctx, BPF_ERR_INVALID_VALUE, "null matrix");
    if (A->dtype != BPF_F64) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "FP64 matrices only");
    if (fdtype != BPF_F64 && fdtype != BPF_F32)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "factor dtype must be BPF_F64 or BPF_F32");
    if (ordering == BPF_ORDER_METIS)
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED,
                         "ordering :METIS needs a METIS library, which this build does not link");
    if (ordering < 0 || ordering > BPF_ORDER_NATURAL)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "unknown ordering %d", ordering);
    std::vector<int> rp, ci, diag;
    int n = A->n, nnz = A->nnz;
    std::vector<int> perm, amap;
    if (ordering == BPF_ORDER_NATURAL) {
        BPF_TRY(csr_pattern_to_host(ctx, A, rp, ci, true, &diag));
    } else {
        // A_hat = A(perm, perm): row i of A_hat is A's row perm[i], columns renumbered by the
        // inverse permutation and sorted; amap sends A's entry k to its A_hat position.
        std::vector<int> arp, aci;
        BPF_TRY(csr_pattern_to_host(ctx, A, arp, aci, false, nullptr));
        perm = ordering == BPF_ORDER_RCM ? order_rcm(n, arp, aci) : order_min_degree(n, arp, aci);
        const int bad = permute_pattern(n, arp, aci, perm, rp, ci, amap, diag);
        if (bad >= 0) return set_error(ctx, BPF_ERR_SINGULAR, "structurally zero diagonal at row %d", bad);
    }
    bpf_prec *P = nullptr;
    BPF_TRY(prec_setup(ctx, kind, n, rp, ci, diag, &P));
    P->nrhs = nrhs;
    P->fdtype = fdtype;
    P->ordering = ordering;
    bool ic = (kind == PREC_IC0);
    auto fail = [&](bpf_status s) {
        cudaStreamSynchronize(ctx->stream);
        bpf_prec_destroy(P);
        return s;
    };
    bpf_status s;
    if (!perm.empty()) {
        cudaError_t e = cudaMalloc((void **)&P->perm, sizeof(int) * n);
        if (e == cudaSuccess && nnz > 0) e = cudaMalloc((void **)&P->amap, sizeof(int) * nnz);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(P->perm, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess && nnz > 0)
            e = cudaMemcpyAsync(P->amap, amap.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);   // host vectors die on return
        if (e != cudaSuccess) return fail(cuda_error(ctx, e, "preconditioner setup", __FILE__, __LINE__));
        P->perm_host = perm;
        if ((s = prec_reserve_z(ctx, P, std::max(nrhs, 1))) != BPF_SUCCESS) return fail(s);
    }
    if ((s = prec_load_values(ctx, P, (const double *)A->vals)) != BPF_SUCCESS) return fail(s);
    if ((s = factor_numeric(ctx, P)) != BPF_SUCCESS) return fail(s);
    if ((s = tri_scatter(ctx, P->lower, P->fv)) != BPF_SUCCESS) return fail(s);
    if ((s = tri_scatter(ctx, P->upper, P->fv)) != BPF_SUCCESS) return fail(s);
    if ((s = check_dev_status(ctx, ic ? "ic0" : "ilu0")) != BPF_SUCCESS) return fail(s);
    *out = P;
    return BPF_SUCCESS;
}

bpf_status bpf_ilu0_create(bpf_ctx *ctx, const bpf_csr_desc *A, int nrhs, int factor_dtype,
                           bpf_prec **prec) {
    return prec_create(ctx, A, nrhs, factor_dtype, PREC_ILU0, BPF_ORDER_NATURAL, prec);
}

bpf_status bpf_ic0_create(bpf_ctx *ctx, const bpf_csr_desc *A, int nrhs, int factor_dtype,
                          bpf_prec **prec) {
    return prec_create(ctx, A, nrhs, factor_dtype, PREC_IC0, BPF_ORDER_NATURAL, prec);
}

bpf_status bpf_ilu0_create_ordered(bpf_ctx *ctx, const bpf_csr_desc *A, int nrhs, int factor_dtype,
                                   int ordering, bpf_prec **prec) {
    return prec_create(ctx, A, nrhs, factor_dtype, PREC_ILU0, ordering, prec);
}

bpf_status bpf_ic0_create_ordered(bpf_ctx *ctx, const bpf_csr_desc *A, int nrhs, int factor_dtype,
                                  int ordering, bpf_prec **prec) {
    return prec_create(ctx, A, nrhs, factor_dtype, PREC_IC0, ordering, prec);
}

bpf_status bpf_prec_permutation(const bpf_prec *P, int *perm) {
    if (!P || (P->n > 0 && !perm)) return BPF_ERR_INVALID_VALUE;
    for (int i = 0; i < P->n; i++) perm[i] = P->perm_host.empty() ? i : P->perm_host[i];
    return BPF_SUCCESS;
}

bpf_status bpf_prec_refactor(bpf_prec *P, const double *vals) {
    if (!P) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = P->ctx;
    if (P->nnz > 0 && !vals) return set_error(ctx, BPF_ERR_INVALID_VALUE, "null values");
    BPF_TRY(prec_load_values(ctx, P, vals));
    if (P->kind == PREC_BJ) {
        BPF_TRY(bj_setup(ctx, P));
        return check_dev_status(ctx, "block-Jacobi (singular diagonal block)");
    }
    BPF_TRY(factor_numeric(ctx, P));
    BPF_TRY(tri_scatter(ctx, P->lower, P->fv));
    BPF_TRY(tri_scatter(ctx, P->upper, P->fv));
    return check_dev_status(ctx, P->kind == PREC_IC0 ? "ic0 refactor" : "ilu0 refactor");
}

bpf_status bpf_prec_apply(bpf_prec *P, int p, const double *X, int ldx, double *Y, int ldy) {
    if (!P) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = P->ctx;
    int n = P->n;
    if (p < 0 || (p > 0 && n > 0 && (!X || !Y)))
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "bpf_prec_apply: invalid argument");
    if (ldx < std::max(1, n) || ldy < std::max(1, n))
        return set_error(ctx, BPF_ERR_DIMENSION, "bpf_prec_apply: leading dimension < n");
    if (n == 0 || p == 0) return BPF_SUCCESS;
    const int chunk = 256;
    bpf_status st;
    double *buf = (double *)ws_get(ctx, WS_A, sizeof(double) * (size_t)n * std::min(p, chunk), &st);
    if (!buf) return st;
    BPF_TRY(prec_reserve_z(ctx, P, std::min(p, chunk)));
    for (int c0 = 0; c0 < p; c0 += chunk) {
        int pc = std::min(chunk, p - c0);
        BPF_TRY(colmajor_to_rowmajor(ctx, n, pc, X + (size_t)c0 * ldx, ldx, buf));
        BPF_TRY(prec_apply_rowmajor(ctx, P, pc, buf, buf));
        BPF_TRY(rowmajor_to_colmajor(ctx, n, pc, buf, Y + (size_t)c0 * ldy, ldy));
    }
    return BPF_SUCCESS;
}

bpf_status bpf_prec_factor_values(const bpf_prec *P, double *vals) {
    if (!P || (P->nnz > 0 && !vals)) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = P->ctx;
    if (P->kind == PREC_BJ)
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "block-Jacobi holds dense block inverses, not factors on A's pattern");
    if (P->nnz > 0)
        BPF_CUDA(ctx, cudaMemcpyAsync(vals, P->fv, sizeof(double) * P->nnz, cudaMemcpyDeviceToDevice,
                                      ctx->stream));
    return BPF_SUCCESS;
}

bpf_status bpf_prec_levels(const bpf_prec *P, int *lo, int *up) {
    if (!P) return BPF_ERR_INVALID_VALUE;
    if (lo) *lo = P->lower.nlev;
    if (up) *up = P->upper.nlev;
    return BPF_SUCCESS;
}

bpf_status bpf_prec_destroy(bpf_prec *P) {
    if (!P) return BPF_SUCCESS;
    if (P->ctx) cudaStreamSynchronize(P->ctx->stream);
    tri_free(P->lower);
    tri_free(P->upper);
    cudaFree(P->rp);
    cudaFree(P->ci);
    cudaFree(P->diag);
    cudaFree(P->pp);
    cudaFree(P->pdst);
    cudaFree(P->psrc);
    cudaFree(P->fv);
    cudaFree(P->perm);
    cudaFree(P->amap);
    cudaFree(P->zbuf);
    cudaFree(P->sf_flags);
    cudaFree(P->cl_lev_ptr);
    cudaFree(P->cl_ent);
    cudaFree(P->cl_row);
    cudaFree(P->bj_rows);
    cudaFree(P->bj_blk);
    cudaFree(P->bj_loc);
    cudaFree(P->bj_inv);
    for (int w = 0; w < 2; w++) {
        cudaFree(P->ps_ptr[w]);
        cudaFree(P->ps_src[w]);
        cudaFree(P->ps_dst[w]);
        cudaFree(P->ps_pos[w]);
    }
    delete P;
    return BPF_SUCCESS;
}

}  // extern "C"
