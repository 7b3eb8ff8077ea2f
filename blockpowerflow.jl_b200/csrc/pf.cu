// Power-flow mismatch and Jacobian assembly on the device: the caller of the multi-RHS solve
// path.  A Newton power-flow step needs F(x) = S(V(x)) - S_spec, the Jacobian Gx = dF/dx on a
// fixed sparsity pattern (refactored and solved by the path every step) and, at the solution,
// Gu = dF/du for the sensitivities Gx^{-1} Gu (one multi-RHS solve).  The reference's benchmark
// reads Gx and Gu that ExaPF assembled (benchmarks/benchmarks_nvidia.jl:29-39) and refactors Gx
// once per Newton step (src/cusolverRF.jl:304-314); assembling them here keeps the whole loop
// on the device, with only the mismatch norm crossing to the host.
//
// Polar form, S = V conj(Ybus V), I = Ybus V (the standard complex derivatives):
//   dS/dtheta = j diag(V) conj(diag(I) - Ybus diag(V)),
//   dS/d|V|   = diag(V) conj(Ybus diag(V / |V|)) + conj(diag(I)) diag(V / |V|).
// Unknowns x = [theta(non-slack buses); |V|(PQ buses)] in bus order, equations
// F = [P(non-slack); Q(PQ)] in the same order, controls u = |V| of the slack bus then the PV
// buses in bus order.  Every Ybus entry (i, k) gives the four Jacobian entries (P_i or Q_i,
// theta_k or |V|_k) that exist, so the assembly is one thread per bus row writing through a
// position map built once on the host: no atomics, every Gx position written at most once.
#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "bpf_internal.cuh"
#include "prec.cuh"

struct bpf_pf {
    bpf_ctx *ctx = nullptr;
    int nb = 0, n = 0, ny = 0, nctrl = 0, njac = 0;
    bool covered = false;               // every Gx position is written by the assembly
    int *yrp = nullptr, *yci = nullptr; // Ybus, with the diagonal of every nonempty row
    double2 *yv = nullptr;
    double2 *sspec = nullptr;           // specified injections
    double2 *vfix = nullptr;            // (|V|, theta) used where they are not unknowns
    int *ia = nullptr, *im = nullptr;   // per bus: index of theta / P (ia), |V| / Q (im) or -1
    int *ctrl = nullptr;                // per bus: control column or -1
    int *map = nullptr;                 // 4 per Ybus entry: Gx positions or -1
    double2 *V = nullptr;               // bus voltages of the last evaluation
    unsigned long long *dnorm = nullptr;
    unsigned long long *hnorm = nullptr;  // pinned
};

namespace bpf {

constexpr int kPfThreads = 256;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// V_i = |V_i| e^{j theta_i} at x + alpha dx (dx nullable); x_out (nullable, may be x) gets that
// point.  x + alpha dx is rounded as a product then a sum, as a host axpy would be.
__global__ void __launch_bounds__(kPfThreads) pf_voltage_kernel(int nb, const double *x, const double *dx,
                                                               double alpha, double *x_out,
                                                               const int *__restrict__ ia,
                                                               const int *__restrict__ im,
                                                               const double2 *__restrict__ vfix, double2 *V) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const int a = ia[i], m = im[i];
    const double2 f = vfix[i];
    double vm = f.x, va = f.y;
    if (a >= 0) {
        va = x[a];
        if (dx) va = __dadd_rn(va, __dmul_rn(alpha, dx[a]));
        if (x_out) x_out[a] = va;
    }
    if (m >= 0) {
        vm = x[m];
        if (dx) vm = __dadd_rn(vm, __dmul_rn(alpha, dx[m]));
        if (x_out) x_out[m] = vm;
    }
    double s, c;
    sincos(va, &s, &c);
    V[i] = make_double2(vm * c, vm * s);
}

__device__ __forceinline__ double2 row_current(int i, const int *__restrict__ yrp, const int *__restrict__ yci,
                                               const double2 *__restrict__ yv, const double2 *__restrict__ V) {
    double2 acc = make_double2(0.0, 0.0);
    const int e1 = yrp[i + 1];
    for (int e = yrp[i]; e < e1; e++) {
        const double2 t = cmul(yv[e], V[yci[e]]);
        acc.x += t.x;
        acc.y += t.y;
    }
    return acc;
}

// F = [Re(S - S_spec) at non-slack buses; Im(S - S_spec) at PQ buses]; *norm = max |F| as the
// bits of a non-negative double (a NaN entry makes the maximum a NaN).
__global__ void __launch_bounds__(kPfThreads) pf_mismatch_kernel(int nb, const int *__restrict__ yrp,
                                                                const int *__restrict__ yci,
                                                                const double2 *__restrict__ yv,
                                                                const double2 *__restrict__ V,
                                                                const double2 *__restrict__ sspec,
                                                                const int *__restrict__ ia,
                                                                const int *__restrict__ im, double *F,
                                                                unsigned long long *norm) {
    __shared__ unsigned long long red[kPfThreads / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long loc = 0;
    if (i < nb) {
        const double2 I = row_current(i, yrp, yci, yv, V);
        const double2 Vi = V[i];
        const double2 S = cmul(Vi, cconj(I));
        const double2 sp = sspec[i];
        const int a = ia[i], m = im[i];
        if (a >= 0) {
            const double f = S.x - sp.x;
            F[a] = f;
            loc = (unsigned long long)__double_as_longlong(fabs(f));
        }
        if (m >= 0) {
            const double f = S.y - sp.y;
            F[m] = f;
            const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(f));
            loc = b > loc ? b : loc;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long b = __shfl_xor_sync(0xffffffffu, loc, o);
        loc = b > loc ? b : loc;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = loc;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kPfThreads / 32; w++) loc = red[w] > loc ? red[w] : loc;
        atomicMax(norm, loc);
    }
}

// Gx values through the position map; Gu (nullable, column-major, ld ldgu, zeroed before) at the
// control columns.
__global__ void __launch_bounds__(kPfThreads) pf_jacobian_kernel(int nb, const int *__restrict__ yrp,
                                                                const int *__restrict__ yci,
                                                                const double2 *__restrict__ yv,
                                                                const double2 *__restrict__ V,
                                                                const int *__restrict__ ia,
                                                                const int *__restrict__ im,
                                                                const int *__restrict__ ctrl,
                                                                const int *__restrict__ map, double *gx,
                                                                double *gu, long long ldgu) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const double2 I = row_current(i, yrp, yci, yv, V);
    const double2 Ic = cconj(I);
    const double2 Vi = V[i];
    const double ri = hypot(Vi.x, Vi.y);
    const double2 Vni = make_double2(Vi.x / ri, Vi.y / ri);
    const int a = ia[i], m = im[i];
    const int e1 = yrp[i + 1];
    for (int e = yrp[i]; e < e1; e++) {
        const int k = yci[e];
        const double2 y = yv[e];
        const double2 Vk = V[k];
        // dS_i/dtheta_k = j V_i ([i == k] conj(I_i) - conj(Y_ik V_k))
        const double2 yvk = cmul(y, Vk);
        double2 t = make_double2(-yvk.x, yvk.y);
        if (k == i) {
            t.x += Ic.x;
            t.y += Ic.y;
        }
        const double2 vt = cmul(Vi, t);
        const double2 dth = make_double2(-vt.y, vt.x);
        // dS_i/d|V_k| = V_i conj(Y_ik V_k / |V_k|) + [i == k] conj(I_i) V_i / |V_i|
        const double rk = hypot(Vk.x, Vk.y);
        const double2 yvn = cmul(y, make_double2(Vk.x / rk, Vk.y / rk));
        double2 dm = cmul(Vi, cconj(yvn));
        if (k == i) {
            const double2 c = cmul(Ic, Vni);
            dm.x += c.x;
            dm.y += c.y;
        }
        const int4 p = *reinterpret_cast<const int4 *>(map + 4 * (size_t)e);
        if (p.x >= 0) gx[p.x] = dth.x;
        if (p.y >= 0) gx[p.y] = dm.x;
        if (p.z >= 0) gx[p.z] = dth.y;
        if (p.w >= 0) gx[p.w] = dm.y;
        if (gu) {
            const int c = ctrl[k];
            if (c >= 0) {
                if (a >= 0) gu[c * ldgu + a] = dm.x;
                if (m >= 0) gu[c * ldgu + m] = dm.y;
            }
        }
    }
}

static bpf_status pf_voltages(bpf_pf *pf, const double *x, const double *dx, double alpha, double *x_out) {
    bpf_ctx *ctx = pf->ctx;
    pf_voltage_kernel<<<ceil_div(pf->nb, kPfThreads), kPfThreads, 0, ctx->stream>>>(
        pf->nb, x, dx, alpha, x_out, pf->ia, pf->im, pf->vfix, pf->V);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

}  // namespace bpf

using namespace bpf;

extern "C" bpf_status bpf_pf_destroy(bpf_pf *pf) {
    if (!pf) return BPF_SUCCESS;
    void *d[] = {pf->yrp, pf->yci, pf->yv, pf->sspec, pf->vfix, pf->ia, pf->im, pf->ctrl, pf->map, pf->V, pf->dnorm};
    for (void *p : d)
        if (p) cudaFree(p);
    if (pf->hnorm) cudaFreeHost(pf->hnorm);
    delete pf;
    return BPF_SUCCESS;
}

extern "C" bpf_status bpf_pf_create(bpf_ctx *ctx, int n_bus, const int *ybus_rowptr, const int *ybus_colind,
                                    const double *ybus_vals, const int *bus_type, const double *vm_fixed,
                                    const double *va_fixed, const double *s_spec, const bpf_csr_desc *jac,
                                    bpf_pf **out) {
    if (!ctx || !out) return BPF_ERR_INVALID_VALUE;
    *out = nullptr;
    if (n_bus < 1 || !ybus_rowptr || !bus_type || !vm_fixed || !va_fixed || !s_spec || !jac)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "power flow: null argument or no bus");
    const int nb = n_bus;
    // Ybus (host, 0-based, sorted unique columns per row)
    const int ny0 = ybus_rowptr[nb];
    if (ybus_rowptr[0] != 0 || ny0 < 0 || (ny0 > 0 && (!ybus_colind || !ybus_vals)))
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "power flow: invalid Ybus row pointers");
    for (int i = 0; i < nb; i++) {
        if (ybus_rowptr[i + 1] < ybus_rowptr[i])
            return set_error(ctx, BPF_ERR_INVALID_VALUE, "power flow: Ybus row pointers not monotone");
        for (int e = ybus_rowptr[i]; e < ybus_rowptr[i + 1]; e++) {
            const int k = ybus_colind[e];
            if (k < 0 || k >= nb)
                return set_error(ctx, BPF_ERR_INVALID_VALUE, "power flow: Ybus column out of range in row %d", i);
            if (e > ybus_rowptr[i] && k <= ybus_colind[e - 1])
                return set_error(ctx, BPF_ERR_INVALID_VALUE, "power flow: Ybus columns of row %d not sorted/unique", i);
        }
    }
    // bus roles: exactly one slack (3), PV (2), PQ (1)
    std::vector<int> ia(nb, -1), im(nb, -1), ctrl(nb, -1);
    int nslack = 0, nnon = 0, npq = 0, slack = -1;
    for (int i = 0; i < nb; i++) {
        const int t = bus_type[i];
        if (t != 1 && t != 2 && t != 3)
            return set_error(ctx, BPF_ERR_INVALID_VALUE, "power flow: bus %d has type %d (1 PQ, 2 PV, 3 slack)", i, t);
        if (t == 3) {
            nslack++;
            slack = i;
        }
    }
    if (nslack != 1) return set_error(ctx, BPF_ERR_INVALID_VALUE, "power flow: %d slack buses (one needed)", nslack);
    for (int i = 0; i < nb; i++)
        if (i != slack) ia[i] = nnon++;
    for (int i = 0; i < nb; i++)
        if (bus_type[i] == 1) im[i] = nnon + npq++;
    int nctrl = 0;
    ctrl[slack] = nctrl++;
    for (int i = 0; i < nb; i++)
        if (bus_type[i] == 2) ctrl[i] = nctrl++;
    const int n = nnon + npq;
    if (jac->n != n)
        return set_error(ctx, BPF_ERR_DIMENSION, "power flow: Jacobian is %d x %d, the buses give %d unknowns",
                         jac->n, jac->n, n);
    std::vector<int> jrp, jci;
    BPF_TRY(csr_pattern_to_host(ctx, jac, jrp, jci, false, nullptr));
    // Ybus with the diagonal of every nonempty row present (the diagonal carries the I_i terms)
    std::vector<int> yrp(nb + 1, 0), yci;
    std::vector<double2> yv;
    yci.reserve(ny0 + nb);
    yv.reserve(ny0 + nb);
    std::vector<char> expl_zero;
    for (int i = 0; i < nb; i++) {
        const int e0 = ybus_rowptr[i], e1 = ybus_rowptr[i + 1];
        bool has_diag = false;
        for (int e = e0; e < e1; e++) has_diag |= ybus_colind[e] == i;
        bool placed = has_diag || e0 == e1;
        for (int e = e0; e < e1; e++) {
            const int k = ybus_colind[e];
            if (!placed && k > i) {
                yci.push_back(i);
                yv.push_back(make_double2(0.0, 0.0));
                expl_zero.push_back(0);   // the diagonal's I_i terms are not zero
                placed = true;
            }
            yci.push_back(k);
            yv.push_back(make_double2(ybus_vals[2 * (size_t)e], ybus_vals[2 * (size_t)e + 1]));
            expl_zero.push_back(k != i && ybus_vals[2 * (size_t)e] == 0.0 && ybus_vals[2 * (size_t)e + 1] == 0.0);
        }
        if (!placed) {
            yci.push_back(i);
            yv.push_back(make_double2(0.0, 0.0));
            expl_zero.push_back(0);
        }
        yrp[i + 1] = (int)yci.size();
    }
    const int ny = yrp[nb];
    // position map: Ybus entry (i, k) -> Gx positions (P_i, theta_k), (P_i, |V|_k), (Q_i, theta_k), (Q_i, |V|_k)
    std::vector<int> map(4 * (size_t)ny, -1);
    std::vector<char> hit(jci.size(), 0);
    size_t nhit = 0;
    for (int i = 0; i < nb; i++) {
        const int rows[2] = {ia[i], im[i]};
        for (int e = yrp[i]; e < yrp[i + 1]; e++) {
            if (expl_zero[e]) continue;   // an explicit zero admittance contributes nothing
            const int k = yci[e];
            const int cols[2] = {ia[k], im[k]};
            for (int r = 0; r < 2; r++)
                for (int c = 0; c < 2; c++) {
                    const int row = rows[r], col = cols[c];
                    if (row < 0 || col < 0) continue;
                    const int *b = jci.data() + jrp[row], *en = jci.data() + jrp[row + 1];
                    const int *f = std::lower_bound(b, en, col);
                    if (f == en || *f != col)
                        return set_error(ctx, BPF_ERR_INVALID_VALUE,
                                         "power flow: the Jacobian pattern lacks entry (%d, %d) of bus pair (%d, %d)",
                                         row, col, i, k);
                    const int pos = (int)(f - jci.data());
                    map[4 * (size_t)e + 2 * r + c] = pos;
                    if (!hit[pos]) {
                        hit[pos] = 1;
                        nhit++;
                    }
                }
        }
    }
    std::vector<double2> sspec(nb), vfix(nb);
    for (int i = 0; i < nb; i++) {
        sspec[i] = make_double2(s_spec[2 * i], s_spec[2 * i + 1]);
        vfix[i] = make_double2(vm_fixed[i], va_fixed[i]);
    }
    bpf_pf *pf = new bpf_pf();
    pf->ctx = ctx;
    pf->nb = nb;
    pf->n = n;
    pf->ny = ny;
    pf->nctrl = nctrl;
    pf->njac = (int)jci.size();
    pf->covered = nhit == jci.size();
    cudaError_t err = cudaSuccess;
    auto up = [&](auto **d, const auto &h) {
        using T = typename std::decay_t<decltype(h)>::value_type;
        if (err == cudaSuccess) err = cudaMalloc((void **)d, sizeof(T) * std::max<size_t>(1, h.size()));
        if (err == cudaSuccess && !h.empty())
            err = cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
    };
    up(&pf->yrp, yrp);
    up(&pf->yci, yci);
    up(&pf->yv, yv);
    up(&pf->sspec, sspec);
    up(&pf->vfix, vfix);
    up(&pf->ia, ia);
    up(&pf->im, im);
    up(&pf->ctrl, ctrl);
    up(&pf->map, map);
    if (err == cudaSuccess) err = cudaMalloc((void **)&pf->V, sizeof(double2) * nb);
    if (err == cudaSuccess) err = cudaMalloc((void **)&pf->dnorm, sizeof(unsigned long long));
    if (err == cudaSuccess) err = cudaMallocHost((void **)&pf->hnorm, sizeof(unsigned long long));
    if (err != cudaSuccess) {
        bpf_status s = cuda_error(ctx, err, "power flow setup", __FILE__, __LINE__);
        bpf_pf_destroy(pf);
        return s;
    }
    *out = pf;
    return BPF_SUCCESS;
}

extern "C" bpf_status bpf_pf_info(const bpf_pf *pf, int *n, int *n_ctrl, int *n_bus) {
    if (!pf) return BPF_ERR_INVALID_VALUE;
    if (n) *n = pf->n;
    if (n_ctrl) *n_ctrl = pf->nctrl;
    if (n_bus) *n_bus = pf->nb;
    return BPF_SUCCESS;
}

extern "C" bpf_status bpf_pf_mismatch(bpf_pf *pf, const double *x, const double *dx, double alpha, double *x_out,
                                      double *F, double *norm_inf) {
    if (!pf) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = pf->ctx;
    if (!x || !F) return set_error(ctx, BPF_ERR_INVALID_VALUE, "power flow: null x or F");
    BPF_TRY(pf_voltages(pf, x, dx, alpha, x_out));
    BPF_CUDA(ctx, cudaMemsetAsync(pf->dnorm, 0, sizeof(unsigned long long), ctx->stream));
    {
        KScope ks(ctx, BPF_KC_PF, 40.0 * pf->ny + 16.0 * pf->nb + 8.0 * pf->n, 8.0 * pf->ny);
        pf_mismatch_kernel<<<ceil_div(pf->nb, kPfThreads), kPfThreads, 0, ctx->stream>>>(
            pf->nb, pf->yrp, pf->yci, pf->yv, pf->V, pf->sspec, pf->ia, pf->im, F, pf->dnorm);
        BPF_LAUNCHED(ctx);
    }
    if (norm_inf) {
        BPF_CUDA(ctx, cudaMemcpyAsync(pf->hnorm, pf->dnorm, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                      ctx->stream));
        BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        const unsigned long long b = *pf->hnorm;
        double v;
        static_assert(sizeof(v) == sizeof(b), "double is 64-bit");
        memcpy(&v, &b, sizeof(v));
        *norm_inf = v;
    }
    return BPF_SUCCESS;
}

extern "C" bpf_status bpf_pf_jacobian(bpf_pf *pf, const double *x, double *jac_vals, double *gu, int ldgu) {
    if (!pf) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = pf->ctx;
    if (!x || !jac_vals) return set_error(ctx, BPF_ERR_INVALID_VALUE, "power flow: null x or Jacobian values");
    if (gu && ldgu < std::max(1, pf->n))
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "power flow: ldgu %d < %d", ldgu, pf->n);
    BPF_TRY(pf_voltages(pf, x, nullptr, 0.0, nullptr));
    if (!pf->covered && pf->njac > 0)
        BPF_CUDA(ctx, cudaMemsetAsync(jac_vals, 0, sizeof(double) * pf->njac, ctx->stream));
    if (gu && pf->n > 0)
        BPF_CUDA(ctx, cudaMemset2DAsync(gu, sizeof(double) * (size_t)ldgu, 0, sizeof(double) * pf->n, pf->nctrl,
                                        ctx->stream));
    KScope ks(ctx, BPF_KC_PF, 72.0 * pf->ny + 16.0 * pf->nb + 8.0 * pf->njac, 40.0 * pf->ny);
    pf_jacobian_kernel<<<ceil_div(pf->nb, kPfThreads), kPfThreads, 0, ctx->stream>>>(
        pf->nb, pf->yrp, pf->yci, pf->yv, pf->V, pf->ia, pf->im, pf->ctrl, pf->map, jac_vals, gu, (long long)ldgu);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}
