// Restarted GMRES with left and right preconditioners
// (boost/numeric/itl/krylov/gmres.hpp:37-137).
//
// Same control flow as the reference: each restart cycle runs k_max =
// min(n, max_iter - i) Arnoldi steps regardless of the residual, solves the
// small upper-triangular system, updates x, and tests the true residual
// ||b - A x||.  Two deliberate differences:
//  * orthogonalization is classical Gram-Schmidt applied twice (one batched
//    multi-dot and one batched multi-axpy per pass) instead of modified
//    Gram-Schmidt plus a re-orthogonalization pass: the same orthogonality to
//    working precision with 4 vector passes per step instead of 2(k+1);
//  * the Givens rotations of earlier columns are the stored (c_i, s_i)
//    applied to column k; the reference rebuilds them from column k-1
//    (gmres.hpp:84-85) and stalls for restart >= 20.
// The Hessenberg matrix and the rotations live on the host in FP64.
#pragma once

namespace mtlg {

// dots[j] = sum_i V_j[i] * w[i] for j < m; per-block partials then a fixed-
// order final sum (deterministic).
template <typename T>
__global__ void k_mdot(long long n, const T* __restrict__ V, long long ldv, int m, const T* __restrict__ w,
                       double* __restrict__ partials)
{
    __shared__ double s_red[kMaxDots * 32];
    for (int j0 = 0; j0 < m; j0 += kMaxDots) {
        double acc[kMaxDots] = {0.0, 0.0, 0.0, 0.0};
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
            const double wi = double(w[i]);
#pragma unroll
            for (int q = 0; q < kMaxDots; ++q)
                if (j0 + q < m) acc[q] += double(V[(j0 + q) * ldv + i]) * wi;
        }
        block_reduce<kMaxDots>(acc, s_red);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int q = 0; q < kMaxDots; ++q)
                if (j0 + q < m) partials[(long long)blockIdx.x * m + j0 + q] = acc[q];
        }
        __syncthreads();
    }
}

__global__ void k_mdot_final(int nblocks, int m, const double* __restrict__ partials, double* __restrict__ out)
{
    const int j = blockIdx.x;
    __shared__ double s_red[kMaxDots * 32];
    double acc[kMaxDots] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) acc[0] += partials[(long long)b * m + j];
    block_reduce<kMaxDots>(acc, s_red);
    if (threadIdx.x == 0) out[j] = acc[0];
}

// w[i] += sign * sum_{j<m} coef[j] * V_j[i]; optionally y = w * scale after.
template <typename T>
__global__ void k_maxpy(long long n, const T* __restrict__ V, long long ldv, int m, const double* __restrict__ coef,
                        double sign, T* __restrict__ w)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        T acc = w[i];
        for (int j = 0; j < m; ++j) acc = fma(T(sign * coef[j]), V[j * ldv + i], acc);
        w[i] = acc;
    }
}

template <typename T>
__global__ void k_scale(long long n, const T* __restrict__ in, double s, T* __restrict__ out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = T(double(in[i]) * s);
}

struct GmresWork {
    mtlg_ctx* c = nullptr;
    long long n = 0;
    int blocks = 0;
    DBuf<unsigned char> V, tmp0, tmp1;
    DBuf<double> partials, dots;
    std::vector<double> hdots;
};

template <typename T>
inline int gm_mdot(GmresWork& W, const T* V, int m, const T* w, double* out_host)
{
    mtlg_ctx* c = W.c;
    k_mdot<T><<<W.blocks, kBlock, 0, c->stream>>>(W.n, V, W.n, m, w, W.partials.p);
    k_mdot_final<<<m, kBlock, 0, c->stream>>>(W.blocks, m, W.partials.p, W.dots.p);
    c->launches += 2;
    MTLG_CUDA(cudaGetLastError());
    MTLG_CUDA(cudaMemcpyAsync(out_host, W.dots.p, sizeof(double) * m, cudaMemcpyDeviceToHost, c->stream));
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    return MTLG_OK;
}

template <typename T>
inline int gm_maxpy(GmresWork& W, const T* V, int m, const double* coef_host, double sign, T* w)
{
    mtlg_ctx* c = W.c;
    MTLG_CUDA(cudaMemcpyAsync(W.dots.p, coef_host, sizeof(double) * m, cudaMemcpyHostToDevice, c->stream));
    k_maxpy<T><<<W.blocks, kBlock, 0, c->stream>>>(W.n, V, W.n, m, W.dots.p, sign, w);
    c->launches++;
    MTLG_CUDA(cudaGetLastError());
    return MTLG_OK;
}

int pc_apply_raw(mtlg_ctx* c, mtlg_pc* P, int dtype, int64_t n, const void* x, void* y);
int spmv_raw(mtlg_ctx* c, mtlg_csr* A, int dtype, const void* x, void* y, const void* w, int asg);

struct HostIter {
    int i = 0, max_iter = 0, error = 0;
    double norm_r0 = 0, rtol = 0, atol = 0, resid = 0;
    bool converged(double r)
    {
        resid = r;
        return norm_r0 == 0 ? r <= atol : (r <= rtol * norm_r0 || r <= atol);
    }
    bool finished(double r)
    {
        if (converged(r)) return true;
        if (i >= max_iter) { error = 1; return true; }
        return false;
    }
};

template <typename T>
int gmres_run(mtlg_ctx* c, mtlg_csr* A, mtlg_pc* L, mtlg_pc* R, mtlg_vec* x, const mtlg_vec* b,
              const mtlg_iter_params* p, mtlg_iter_result* res)
{
    const int dt = x->dtype;
    const long long n = A->n_rows;
    const int restart = p->restart > 0 ? p->restart : 8;
    GmresWork W;
    W.c = c;
    W.n = n;
    W.blocks = int(std::max<long long>(1, std::min<long long>((n + kBlock - 1) / kBlock, 4LL * c->sm_count)));
    MTLG_TRY(W.V.alloc(c, size_t(restart + 1) * size_t(std::max<long long>(n, 1)) * sizeof(T)));
    MTLG_TRY(W.tmp0.alloc(c, size_t(std::max<long long>(n, 1)) * sizeof(T)));
    MTLG_TRY(W.tmp1.alloc(c, size_t(std::max<long long>(n, 1)) * sizeof(T)));
    MTLG_TRY(W.partials.alloc(c, size_t(W.blocks) * (restart + 2)));
    MTLG_TRY(W.dots.alloc(c, restart + 2));
    T* V = reinterpret_cast<T*>(W.V.p);
    T* t0 = reinterpret_cast<T*>(W.tmp0.p);
    T* t1 = reinterpret_cast<T*>(W.tmp1.p);
    T* xp = static_cast<T*>(x->p);
    const T* bp = static_cast<const T*>(b->p);
    auto Vk = [&](int k) { return V + (long long)k * n; };

    cudaEvent_t e0, e1;
    MTLG_CUDA(cudaEventCreate(&e0));
    MTLG_CUDA(cudaEventCreate(&e1));
    MTLG_CUDA(cudaEventRecord(e0, c->stream));

    HostIter it;
    it.max_iter = p->max_iter;
    it.rtol = p->rtol;
    it.atol = p->atol;
    if (p->norm_r0 >= 0) {
        it.norm_r0 = p->norm_r0;
    } else {
        double nb = 0;
        MTLG_TRY(gm_mdot<T>(W, bp, 1, bp, &nb));
        it.norm_r0 = sqrt(fabs(nb));
    }
    const int grid = W.blocks;
    bool outer_done = false;
    int status = MTLG_ST_RUNNING;
    std::vector<double> H((restart + 1) * restart), cs(restart), sn(restart), g(restart + 1), y(restart);
    std::vector<double> h(restart + 2), h2(restart + 2);
    while (!outer_done) {
        // ---- gmres_full on an inner iteration with max = min(i + restart, max_iter)
        HostIter inner = it;
        inner.max_iter = std::min(it.i + restart, it.max_iter);
        const int kmax = int(std::min<long long>(n, std::max(0, inner.max_iter - inner.i)));
        MTLG_TRY(spmv_raw(c, A, dt, xp, t0, bp, ASG_WMINUS));                   // r0 = b - A x
        MTLG_TRY(pc_apply_raw(c, L, dt, n, t0, Vk(0)));                        // r = solve(L, r0)
        double rr = 0;
        MTLG_TRY(gm_mdot<T>(W, Vk(0), 1, Vk(0), &rr));
        double rho = sqrt(fabs(rr));
        int k = 0;
        bool early = inner.finished(rho);
        if (!early) {
            std::fill(H.begin(), H.end(), 0.0);
            std::fill(g.begin(), g.end(), 0.0);
            g[0] = rho;
            k_scale<T><<<grid, kBlock, 0, c->stream>>>(n, Vk(0), 1.0 / rho, Vk(0));
            c->launches++;
            auto hh = [&](int i, int j) -> double& { return H[i * restart + j]; };
            for (k = 0; k < kmax; ++k, ++inner.i) {
                MTLG_TRY(pc_apply_raw(c, R, dt, n, Vk(k), t1));                // solve(R, V_k)
                MTLG_TRY(spmv_raw(c, A, dt, t1, t0, nullptr, ASG_SET));        // A * .
                MTLG_TRY(pc_apply_raw(c, L, dt, n, t0, Vk(k + 1)));            // solve(L, .)
                // two classical Gram-Schmidt passes
                MTLG_TRY(gm_mdot<T>(W, V, k + 1, Vk(k + 1), h.data()));
                MTLG_TRY(gm_maxpy<T>(W, V, k + 1, h.data(), -1.0, Vk(k + 1)));
                MTLG_TRY(gm_mdot<T>(W, V, k + 1, Vk(k + 1), h2.data()));
                MTLG_TRY(gm_maxpy<T>(W, V, k + 1, h2.data(), -1.0, Vk(k + 1)));
                for (int j = 0; j <= k; ++j) hh(j, k) = h[j] + h2[j];
                double ww = 0;
                MTLG_TRY(gm_mdot<T>(W, Vk(k + 1), 1, Vk(k + 1), &ww));
                hh(k + 1, k) = sqrt(fabs(ww));
                if (hh(k + 1, k) != 0.0) {
                    k_scale<T><<<grid, kBlock, 0, c->stream>>>(n, Vk(k + 1), 1.0 / hh(k + 1, k), Vk(k + 1));
                    c->launches++;
                }
                for (int i = 0; i < k; ++i) {
                    const double a0 = hh(i, k), a1 = hh(i + 1, k);
                    hh(i, k) = cs[i] * a0 - sn[i] * a1;
                    hh(i + 1, k) = sn[i] * a0 + cs[i] * a1;
                }
                const double nu = sqrt(hh(k, k) * hh(k, k) + hh(k + 1, k) * hh(k + 1, k));
                if (nu != 0.0) {
                    cs[k] = hh(k, k) / nu;
                    sn[k] = -hh(k + 1, k) / nu;
                    hh(k, k) = cs[k] * hh(k, k) - sn[k] * hh(k + 1, k);
                    hh(k + 1, k) = 0.0;
                    const double g0 = g[k], g1 = g[k + 1];
                    g[k] = cs[k] * g0 - sn[k] * g1;
                    g[k + 1] = sn[k] * g0 + cs[k] * g1;
                }
                rho = fabs(g[k + 1]);
            }
            // reduce k to get a regular matrix, then back-substitute
            int kk = k;
            while (kk > 0 && fabs(g[kk - 1]) <= inner.atol) --kk;
            int range = kk;
            for (; range > 0; --range) {
                bool singular = false;
                for (int i = 0; i < range; ++i) singular |= (hh(i, i) == 0.0);
                if (!singular) break;
            }
            if (range == 0) {
                inner.error = 2;   // "GMRES did not find any direction to correct x" (gmres.hpp:114)
            } else {
                for (int i = range - 1; i >= 0; --i) {
                    double s2 = g[i];
                    for (int j = i + 1; j < range; ++j) s2 -= hh(i, j) * y[j];
                    y[i] = s2 / hh(i, i);
                }
                // x += solve(R, V y)
                MTLG_CUDA(cudaMemsetAsync(t0, 0, size_t(n) * sizeof(T), c->stream));
                MTLG_TRY(gm_maxpy<T>(W, V, range, y.data(), 1.0, t0));
                MTLG_TRY(pc_apply_raw(c, R, dt, n, t0, t1));
                const double one = 1.0;
                MTLG_TRY(gm_maxpy<T>(W, t1, 1, &one, 1.0, xp));
                MTLG_TRY(spmv_raw(c, A, dt, xp, t0, bp, ASG_WMINUS));           // r = b - A x
                double r2 = 0;
                MTLG_TRY(gm_mdot<T>(W, t0, 1, t0, &r2));
                inner.finished(sqrt(fabs(r2)));                                // iter.terminate(r)
            }
        }
        // iter.update_progress(inner) (basic_iteration.hpp:145-155)
        it.i = inner.i;
        it.resid = inner.resid;
        if (inner.error > 1) {
            it.error = inner.error;
            status = MTLG_ST_NO_DIRECTION;
            outer_done = true;
        } else if (it.finished(it.resid)) {
            outer_done = true;
            status = it.error == 0 ? MTLG_ST_CONVERGED : MTLG_ST_MAXIT;
        }
        if (!outer_done && kmax == 0) {   // no progress possible
            it.error = 1;
            status = MTLG_ST_MAXIT;
            outer_done = true;
        }
    }
    MTLG_CUDA(cudaEventRecord(e1, c->stream));
    MTLG_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    MTLG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (res) {
        res->iterations = it.i;
        res->error_code = it.error;
        res->status = status;
        res->outer_iterations = 0;
        res->resid = it.resid;
        res->norm_r0 = it.norm_r0;
        res->relresid = it.norm_r0 != 0 ? it.resid / it.norm_r0 : it.resid;
        res->seconds = ms * 1e-3;
    }
    return MTLG_OK;
}

}  // namespace mtlg

extern "C" int mtlg_gmres_impl(mtlg_ctx* c, mtlg_csr* A, mtlg_pc* L, mtlg_pc* R, mtlg_vec* x, const mtlg_vec* b,
                               const mtlg_iter_params* p, mtlg_iter_result* r)
{
    if (x->dtype == MTLG_F32) return mtlg::gmres_run<float>(c, A, L, R, x, b, p, r);
    return mtlg::gmres_run<double>(c, A, L, R, x, b, p, r);
}
