// Host-driven Krylov bodies on device vectors: the reference's bicg, cgs,
// tfqmr, qmr, bicgstab_2, bicgstab_ell and idr_s (itl/krylov/*.hpp), and cg /
// bicgstab for operators the graph-captured engine does not take (the
// matrix-free Poisson operator).  Each step is one device pass (SpMV,
// preconditioner apply, vector update) and every scalar the reference
// computes (dots, norms, the small dense systems of bicgstab_ell and idr_s)
// is read back to the host, where the reference's scalar recurrences run as
// written.  Vector updates follow the reference's expressions term by term
// (fused multiply-adds where the expression is a*x + y).  Dots and norms are
// the library's reductions (the reference's summation order under
// reduction_order 1).
#pragma once

namespace mtlg {

// ---------------------------------------------------------------- vector passes
enum KVec : int {
    KV_COPY = 0,    // y = x
    KV_FILL,        // y = a
    KV_AXPY,        // y = y + a x
    KV_XPAY,        // y = x + a y
    KV_AXPBY,       // y = a x + b y
    KV_SCAL,        // y = a y
    KV_DIV,         // y = x / a
    KV_XMY,         // y = x - z
    KV_XPAYPBZ,     // y = x + a (z + b y)        (cgs: p = u + beta (q + beta p); tfqmr's v)
    KV_XPAZ,        // y = x + a z
    KV_XPAYPBZ2,    // y = x + a (y + b z)        (bicgstab: p = r + beta (p - omega v))
    KV_AXPBZ,       // y = y + (a x + b z)        (bicgstab: x += omega shat + alpha phat)
    KV_AX,          // y = a x                    (y is not read)
};

__global__ void __launch_bounds__(kBlock) k_kvec(int op, long long n, double* __restrict__ y,
                                                 const double* __restrict__ x, const double* __restrict__ z,
                                                 double a, double b)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        switch (op) {
        case KV_COPY: y[i] = x[i]; break;
        case KV_FILL: y[i] = a; break;
        case KV_AXPY: y[i] = fma(a, x[i], y[i]); break;
        case KV_XPAY: y[i] = fma(a, y[i], x[i]); break;
        case KV_AXPBY: y[i] = fma(a, x[i], b * y[i]); break;
        case KV_SCAL: y[i] = a * y[i]; break;
        case KV_DIV: y[i] = x[i] / a; break;
        case KV_XMY: y[i] = x[i] - z[i]; break;
        case KV_XPAYPBZ: y[i] = fma(a, fma(b, y[i], z[i]), x[i]); break;
        case KV_XPAZ: y[i] = fma(a, z[i], x[i]); break;
        case KV_XPAYPBZ2: y[i] = fma(a, fma(b, z[i], y[i]), x[i]); break;
        case KV_AXPBZ: y[i] = y[i] + fma(a, x[i], b * z[i]); break;
        case KV_AX: y[i] = a * x[i]; break;
        default: break;
        }
    }
}

int dot_raw(mtlg_ctx* c, int64_t n, const double* x, const double* y, int rk, double* out);
int spmv_raw(mtlg_ctx* c, mtlg_csr* A, int dtype, const void* x, void* y, const void* w, int asg);
int pc_apply_raw(mtlg_ctx* c, mtlg_pc* P, int dtype, int64_t n, const void* x, void* y);
int pc_adjoint_raw(mtlg_ctx* c, mtlg_pc* P, int64_t n, const double* x, double* y);

// The linear operator of a host-driven solve: a CSR matrix (and its
// transpose, made on first need) or the matrix-free 2D Poisson stencil.
struct KOp {
    mtlg_ctx* c = nullptr;
    mtlg_csr* A = nullptr;
    int pm = 0, pn = 0;   // poisson2D_dirichlet(m, n) when A is null
    int64_t n = 0;
    int apply(const double* x, double* y);
    int apply_t(const double* x, double* y);
};

struct KWork {
    mtlg_ctx* c;
    int64_t n;
    int grid;
    std::vector<std::unique_ptr<DBuf<double>>> bufs;
    // a zeroed work vector (no pass ever reads leftover device memory)
    double* vec()
    {
        bufs.emplace_back(new DBuf<double>());
        const size_t len = static_cast<size_t>(std::max<int64_t>(n, 1));
        if (bufs.back()->alloc(c, len) != MTLG_OK) return nullptr;
        if (cudaMemsetAsync(bufs.back()->p, 0, len * sizeof(double), c->stream) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return bufs.back()->p;
    }
    int kv(int op, double* y, const double* x = nullptr, const double* z = nullptr, double a = 0.0, double b = 0.0)
    {
        if (n == 0) return MTLG_OK;
        k_kvec<<<grid, kBlock, 0, c->stream>>>(op, n, y, x, z, a, b);
        c->launches++;
        MTLG_CUDA(cudaGetLastError());
        return MTLG_OK;
    }
    double dot(const double* x, const double* y, int& st)
    {
        double r = 0.0;
        st = dot_raw(c, n, x, y, RK_DOT4, &r);
        return r;
    }
    double norm(const double* x, int& st)
    {
        double r = 0.0;
        st = dot_raw(c, n, x, x, RK_NORM4, &r);
        return std::sqrt(std::fabs(r));
    }
};

// basic_iteration on the host (basic_iteration.hpp:43-65).
struct KIter {
    int i = 0, max_iter = 0, error = 0;
    double norm_r0 = 0, rtol = 0, atol = 0, resid = 0;
    bool finished(double r)
    {
        resid = r;
        if (norm_r0 == 0 ? r <= atol : (r <= rtol * norm_r0 || r <= atol)) return true;
        if (i >= max_iter) { error = 1; return true; }
        return false;
    }
    bool first() const { return i <= 1; }
    int fail(int code) { error = code; return code; }
};

#define KTRY(expr)                          \
    do {                                    \
        const int _s = (expr);              \
        if (_s != MTLG_OK) return _s;       \
    } while (0)
#define KDOT(var, a, b)                     \
    do {                                    \
        int _s;                             \
        var = W.dot(a, b, _s);              \
        if (_s != MTLG_OK) return _s;       \
    } while (0)
#define KNORM(var, a)                       \
    do {                                    \
        int _s;                             \
        var = W.norm(a, _s);                \
        if (_s != MTLG_OK) return _s;       \
    } while (0)

inline int kpc(mtlg_ctx* c, mtlg_pc* P, int64_t n, const double* x, double* y)
{
    return pc_apply_raw(c, P, MTLG_F64, n, x, y);
}

// r = b - A x
inline int kresid(KOp& A, KWork& W, const double* b, const double* x, double* r)
{
    KTRY(A.apply(x, r));
    return W.kv(KV_XMY, r, b, r);
}

// ---- bicg (itl/krylov/bicg.hpp:28-72)
inline int k_bicg(KOp& A, KWork& W, double* x, const double* b, mtlg_pc* M, KIter& it)
{
    const int64_t n = W.n;
    double *r = W.vec(), *z = W.vec(), *p = W.vec(), *q = W.vec(), *rt = W.vec(), *zt = W.vec(), *pt = W.vec(),
           *qt = W.vec();
    if (!qt) return MTLG_ERR_OOM;
    KTRY(kresid(A, W, b, x, r));
    KTRY(W.kv(KV_COPY, rt, r));
    double rho_1 = 0, rho_2 = 0, alpha = 0, beta = 0, nr;
    for (;;) {
        KNORM(nr, r);
        if (it.finished(nr)) break;
        ++it.i;
        KTRY(kpc(W.c, M, n, r, z));
        KTRY(pc_adjoint_raw(W.c, M, n, rt, zt));
        KDOT(rho_1, zt, z);
        if (rho_1 == 0.0) return it.fail(2), MTLG_OK;
        if (it.first()) {
            KTRY(W.kv(KV_COPY, p, z));
            KTRY(W.kv(KV_COPY, pt, zt));
        } else {
            beta = rho_1 / rho_2;
            KTRY(W.kv(KV_XPAY, p, z, nullptr, beta));
            KTRY(W.kv(KV_XPAY, pt, zt, nullptr, beta));
        }
        KTRY(A.apply(p, q));
        KTRY(A.apply_t(pt, qt));
        double ptq;
        KDOT(ptq, pt, q);
        alpha = rho_1 / ptq;
        KTRY(W.kv(KV_AXPY, x, p, nullptr, alpha));
        KTRY(W.kv(KV_AXPY, r, q, nullptr, -alpha));
        KTRY(W.kv(KV_AXPY, rt, qt, nullptr, -alpha));
        rho_2 = rho_1;
    }
    return MTLG_OK;
}

// ---- cgs (itl/krylov/cgs.hpp:28-72)
inline int k_cgs(KOp& A, KWork& W, double* x, const double* b, mtlg_pc* M, KIter& it)
{
    const int64_t n = W.n;
    double *p = W.vec(), *phat = W.vec(), *q = W.vec(), *qhat = W.vec(), *vhat = W.vec(), *u = W.vec(),
           *uhat = W.vec(), *r = W.vec(), *rt = W.vec(), *tmp = W.vec();
    if (!tmp) return MTLG_ERR_OOM;
    KTRY(kresid(A, W, b, x, r));
    KTRY(W.kv(KV_COPY, rt, r));
    double rho_1 = 0, rho_2 = 0, alpha = 0, beta = 0, nr, g;
    for (;;) {
        KNORM(nr, r);
        if (it.finished(nr)) break;
        ++it.i;
        KDOT(rho_1, rt, r);
        if (rho_1 == 0.0) it.fail(2);   // the reference flags the breakdown and goes on
        if (it.first()) {
            KTRY(W.kv(KV_COPY, u, r));
            KTRY(W.kv(KV_COPY, p, r));
        } else {
            beta = rho_1 / rho_2;
            KTRY(W.kv(KV_XPAZ, u, r, q, beta));                 // u = r + beta q
            KTRY(W.kv(KV_XPAYPBZ, p, u, q, beta, beta));        // p = u + beta (q + beta p)
        }
        KTRY(kpc(W.c, M, n, p, phat));
        KTRY(A.apply(phat, vhat));
        KDOT(g, rt, vhat);
        alpha = rho_1 / g;
        KTRY(W.kv(KV_XPAZ, q, u, vhat, -alpha));                // q = u - alpha vhat
        KTRY(W.kv(KV_AXPY, u, q, nullptr, 1.0));                // u += q
        KTRY(kpc(W.c, M, n, u, uhat));
        KTRY(W.kv(KV_AXPY, x, uhat, nullptr, alpha));
        KTRY(A.apply(uhat, qhat));
        KTRY(W.kv(KV_AXPY, r, qhat, nullptr, -alpha));
        rho_2 = rho_1;
    }
    return MTLG_OK;
}

// ---- tfqmr (itl/krylov/tfqmr.hpp:30-98), left preconditioner L, right R
inline int k_tfqmr(KOp& A, KWork& W, double* x, const double* b, mtlg_pc* L, mtlg_pc* R, KIter& it)
{
    const int64_t n = W.n;
    double *rt = W.vec(), *r = W.vec(), *u1 = W.vec(), *u2 = W.vec(), *y1 = W.vec(), *y2 = W.vec(), *w = W.vec(),
           *d = W.vec(), *v = W.vec(), *t = W.vec();
    if (!t) return MTLG_ERR_OOM;
    double theta = 0, eta = 0, tau, rho, rhon, sigma, alpha, beta, cc, nrt;
    KTRY(kpc(W.c, R, n, x, t));                 // shift x = R x
    KTRY(kresid(A, W, b, t, rt));               // rt = b - A solve(R, x)
    KTRY(kpc(W.c, L, n, rt, r));
    KTRY(W.kv(KV_FILL, d, nullptr, nullptr, 0.0));
    KNORM(nrt, rt);
    if (it.finished(nrt)) return MTLG_OK;
    KTRY(W.kv(KV_COPY, y1, r));
    KTRY(W.kv(KV_COPY, w, r));
    KTRY(kpc(W.c, R, n, y1, t));
    KTRY(A.apply(t, rt));
    KTRY(kpc(W.c, L, n, rt, u1));
    KTRY(W.kv(KV_COPY, v, u1));
    KNORM(tau, r);
    rho = tau * tau;
    while (!it.finished(tau)) {
        ++it.i;
        KDOT(sigma, r, v);
        if (sigma == 0.0) return it.fail(1), MTLG_OK;
        alpha = rho / sigma;
        for (int j = 1; j < 3; ++j) {
            if (j == 1) {
                KTRY(W.kv(KV_AXPY, w, u1, nullptr, -alpha));
                KTRY(W.kv(KV_XPAY, d, y1, nullptr, theta * theta * eta / alpha));
            } else {
                KTRY(W.kv(KV_XPAZ, y2, y1, v, -alpha));
                KTRY(kpc(W.c, R, n, y2, t));
                KTRY(A.apply(t, rt));
                KTRY(kpc(W.c, L, n, rt, u2));
                KTRY(W.kv(KV_AXPY, w, u2, nullptr, -alpha));
                KTRY(W.kv(KV_XPAY, d, y2, nullptr, theta * theta * eta / alpha));
            }
            double nw;
            KNORM(nw, w);
            theta = nw / tau;
            cc = 1.0 / std::sqrt(1.0 + theta * theta);
            tau *= theta * cc;
            eta = cc * cc * alpha;
            KTRY(W.kv(KV_AXPY, x, d, nullptr, eta));
        }
        if (rho == 0.0) return it.fail(1), MTLG_OK;
        KDOT(rhon, r, w);
        beta = rhon / rho;
        rho = rhon;
        KTRY(W.kv(KV_XPAZ, y1, w, y2, beta));                 // y1 = w + beta y2
        KTRY(kpc(W.c, R, n, y1, t));
        KTRY(A.apply(t, rt));
        KTRY(kpc(W.c, L, n, rt, u1));
        KTRY(W.kv(KV_XPAYPBZ, v, u1, u2, beta, beta));        // v = u1 + beta (u2 + beta v)
    }
    KTRY(kpc(W.c, R, n, x, t));
    return W.kv(KV_COPY, x, t);
}

// ---- qmr (itl/krylov/qmr.hpp:31-116), left L, right R
inline int k_qmr(KOp& A, KWork& W, double* x, const double* b, mtlg_pc* L, mtlg_pc* R, KIter& it)
{
    const int64_t n = W.n;
    double *r = W.vec(), *vt = W.vec(), *y = W.vec(), *wt = W.vec(), *z = W.vec(), *v = W.vec(), *w = W.vec(),
           *yt = W.vec(), *zt = W.vec(), *p = W.vec(), *q = W.vec(), *pt = W.vec(), *d = W.vec(), *s = W.vec(),
           *t = W.vec();
    if (!t) return MTLG_ERR_OOM;
    double beta, gamma = 1.0, gamma_1, delta, eta = -1.0, ep = 1.0, rho_1, theta = 0.0, theta_1, nr;
    KTRY(kresid(A, W, b, x, r));
    KTRY(W.kv(KV_COPY, vt, r));
    KTRY(kpc(W.c, L, n, vt, y));
    KTRY(W.kv(KV_COPY, wt, r));
    KTRY(pc_adjoint_raw(W.c, R, n, wt, z));
    KNORM(nr, r);
    if (it.finished(nr)) return MTLG_OK;
    double rho, xi;
    KNORM(rho, y);
    KNORM(xi, z);
    while (!it.finished(rho)) {
        ++it.i;
        if (rho == 0.0) return it.fail(1), MTLG_OK;
        if (xi == 0.0) return it.fail(2), MTLG_OK;
        KTRY(W.kv(KV_DIV, v, vt, nullptr, rho));
        KTRY(W.kv(KV_DIV, y, y, nullptr, rho));
        KTRY(W.kv(KV_DIV, w, wt, nullptr, xi));
        KTRY(W.kv(KV_DIV, z, z, nullptr, xi));
        KDOT(delta, z, y);
        if (delta == 0.0) return it.fail(3), MTLG_OK;
        KTRY(kpc(W.c, R, n, y, yt));
        KTRY(pc_adjoint_raw(W.c, L, n, z, zt));
        if (it.first()) {
            KTRY(W.kv(KV_COPY, p, yt));
            KTRY(W.kv(KV_COPY, q, zt));
        } else {
            KTRY(W.kv(KV_XPAY, p, yt, nullptr, -((xi * delta) / ep)));
            KTRY(W.kv(KV_XPAY, q, zt, nullptr, -((rho * delta) / ep)));
        }
        KTRY(A.apply(p, pt));
        KDOT(ep, q, pt);
        if (ep == 0.0) return it.fail(4), MTLG_OK;
        beta = ep / delta;
        if (beta == 0.0) return it.fail(5), MTLG_OK;
        KTRY(W.kv(KV_XPAZ, vt, pt, v, -beta));               // v_tld = p_tld - beta v
        KTRY(kpc(W.c, L, n, vt, y));
        rho_1 = rho;
        KNORM(rho, y);
        KTRY(A.apply_t(q, t));
        KTRY(W.kv(KV_XPAZ, wt, t, w, -beta));                // w_tld = trans(A) q - beta w
        KTRY(pc_adjoint_raw(W.c, R, n, wt, z));
        KNORM(xi, z);
        gamma_1 = gamma;
        theta_1 = theta;
        theta = rho / (gamma_1 * beta);
        gamma = 1.0 / std::sqrt(1.0 + theta * theta);
        if (gamma == 0.0) return it.fail(6), MTLG_OK;
        eta = -eta * rho_1 * gamma * gamma / (beta * gamma_1 * gamma_1);
        if (it.first()) {
            KTRY(W.kv(KV_AX, d, p, nullptr, eta));
            KTRY(W.kv(KV_AX, s, pt, nullptr, eta));
        } else {
            const double f = theta_1 * theta_1 * gamma * gamma;
            KTRY(W.kv(KV_AXPBY, d, p, nullptr, eta, f));
            KTRY(W.kv(KV_AXPBY, s, pt, nullptr, eta, f));
        }
        KTRY(W.kv(KV_AXPY, x, d, nullptr, 1.0));
        KTRY(W.kv(KV_AXPY, r, s, nullptr, -1.0));
    }
    return MTLG_OK;
}

// Modified Gram-Schmidt of the vectors v[0..k) with the factors (the
// reference's orthogonalize_factors, itl/krylov/bicgstab_ell.hpp via
// mtl/operation/orth.hpp): tau(i, j) = <v_i, v_j> / tau(i, i) for i < j,
// tau(j, j) = <v_j, v_j> before normalizing... here as in the reference: for
// each j, for i < j: tau(i,j) = dot(v_i, v_j) / tau(i,i); v_j -= tau(i,j) v_i;
// then tau(j,j) = dot(v_j, v_j), and v_j keeps its length.
inline int k_orth_factors(KWork& W, std::vector<double*>& v, std::vector<std::vector<double>>& tau)
{
    const int k = int(v.size());
    for (int j = 0; j < k; ++j) {
        for (int i = 0; i < j; ++i) {
            double d;
            KDOT(d, v[i], v[j]);
            tau[i][j] = d / tau[i][i];
            KTRY(W.kv(KV_AXPY, v[j], v[i], nullptr, -tau[i][j]));
        }
        double d;
        KDOT(d, v[j], v[j]);
        tau[j][j] = d;
    }
    return MTLG_OK;
}

// ---- bicgstab_ell (itl/krylov/bicgstab_ell.hpp:29-132); bicgstab_2 is l = 2
// with the right preconditioner the identity (bicgstab_2.hpp:29-125)
inline int k_bicgstab_ell(KOp& A, KWork& W, double* x, const double* b, mtlg_pc* L, mtlg_pc* R, KIter& it, int l)
{
    const int64_t n = W.n;
    l = std::max(l, 1);
    double *x0 = W.vec(), *y = W.vec(), *r0t = W.vec(), *t = W.vec();
    std::vector<double*> rh(static_cast<size_t>(l) + 1), uh(static_cast<size_t>(l) + 1);
    for (int i = 0; i <= l; ++i) { rh[i] = W.vec(); uh[i] = W.vec(); }
    if (!uh[l]) return MTLG_ERR_OOM;
    KTRY(W.kv(KV_FILL, x0, nullptr, nullptr, 0.0));
    KTRY(W.kv(KV_COPY, rh[0], b));
    double nx;
    KNORM(nx, x);
    if (nx != 0.0) {
        KTRY(A.apply(x, t));
        KTRY(W.kv(KV_AXPY, rh[0], t, nullptr, -1.0));
        KTRY(W.kv(KV_COPY, x0, x));
        KTRY(W.kv(KV_FILL, x, nullptr, nullptr, 0.0));
    }
    double nr0;
    KNORM(nr0, rh[0]);
    KTRY(W.kv(KV_DIV, r0t, rh[0], nullptr, nr0));
    KTRY(kpc(W.c, L, n, rh[0], y));
    KTRY(W.kv(KV_COPY, rh[0], y));
    KTRY(W.kv(KV_FILL, uh[0], nullptr, nullptr, 0.0));
    double rho_0 = 1.0, rho_1 = 0.0, alpha = 0.0, Gamma = 0.0, beta = 0.0, omega = 1.0;
    std::vector<std::vector<double>> tau(static_cast<size_t>(l) + 1, std::vector<double>(static_cast<size_t>(l) + 1, 0.0));
    std::vector<double> gamma(static_cast<size_t>(l) + 1), gamma_a(static_cast<size_t>(l) + 1), gamma_aa(static_cast<size_t>(l) + 1);
    for (;;) {
        double nr;
        KNORM(nr, rh[0]);
        if (it.finished(nr)) break;
        ++it.i;
        rho_0 = -omega * rho_0;
        for (int j = 0; j < l; ++j) {
            KDOT(rho_1, r0t, rh[j]);
            beta = alpha * rho_1 / rho_0;
            rho_0 = rho_1;
            for (int i = 0; i <= j; ++i) KTRY(W.kv(KV_XPAY, uh[i], rh[i], nullptr, -beta));   // u = r - beta u
            KTRY(kpc(W.c, R, n, uh[j], t));
            KTRY(A.apply(t, y));
            KTRY(kpc(W.c, L, n, y, uh[j + 1]));
            KDOT(Gamma, r0t, uh[j + 1]);
            alpha = rho_0 / Gamma;
            for (int i = 0; i <= j; ++i) KTRY(W.kv(KV_AXPY, rh[i], uh[i + 1], nullptr, -alpha));
            KNORM(nr, rh[j]);
            if (it.finished(nr)) {
                KTRY(kpc(W.c, R, n, x, t));
                KTRY(W.kv(KV_COPY, x, t));
                return W.kv(KV_AXPY, x, x0, nullptr, 1.0);
            }
            KTRY(kpc(W.c, R, n, rh[j], t));
            KTRY(A.apply(t, y));
            KTRY(kpc(W.c, L, n, y, rh[j + 1]));
            KTRY(W.kv(KV_AXPY, x, uh[0], nullptr, alpha));
        }
        std::vector<double*> tail(rh.begin() + 1, rh.end());
        std::vector<std::vector<double>> tt(static_cast<size_t>(l), std::vector<double>(static_cast<size_t>(l), 0.0));
        KTRY(k_orth_factors(W, tail, tt));
        for (int i = 1; i <= l; ++i)
            for (int j = 1; j <= l; ++j) tau[i][j] = tt[i - 1][j - 1];
        for (int j = 1; j <= l; ++j) {
            double d;
            KDOT(d, rh[j], rh[0]);
            gamma_a[j] = d / tau[j][j];
        }
        gamma[l] = gamma_a[l];
        omega = gamma[l];
        if (omega == 0.0) return it.fail(3), MTLG_OK;
        for (int j = l - 1; j > 0; --j) {
            double sum = 0.0;
            for (int i = j + 1; i <= l; ++i) sum += tau[j][i] * gamma[i];
            gamma[j] = gamma_a[j] - sum;
        }
        // gamma_aa[1..l) = strict_upper(tau[1..l)[1..l)) * gamma[2..l] + gamma[2..l]
        for (int j = 1; j < l; ++j) {
            double sum = 0.0;
            for (int i = j + 1; i < l; ++i) sum += tau[j][i] * gamma[i + 1];
            gamma_aa[j] = sum + gamma[j + 1];
        }
        KTRY(W.kv(KV_AXPY, x, rh[0], nullptr, gamma[1]));
        KTRY(W.kv(KV_AXPY, rh[0], rh[l], nullptr, -gamma_a[l]));
        KTRY(W.kv(KV_AXPY, uh[0], uh[l], nullptr, -gamma[l]));
        for (int j = 1; j < l; ++j) {
            KTRY(W.kv(KV_AXPY, uh[0], uh[j], nullptr, -gamma[j]));
            KTRY(W.kv(KV_AXPY, x, rh[j], nullptr, gamma_aa[j]));
            KTRY(W.kv(KV_AXPY, rh[0], rh[j], nullptr, -gamma_a[j]));
        }
    }
    KTRY(kpc(W.c, R, n, x, t));
    KTRY(W.kv(KV_COPY, x, t));
    return W.kv(KV_AXPY, x, x0, nullptr, 1.0);
}

// Small dense LU solve with partial pivoting (the reference's lu_solve on
// the s x s system of idr_s).
inline std::vector<double> small_lu_solve(std::vector<std::vector<double>> M, std::vector<double> rhs)
{
    const int s = int(rhs.size());
    std::vector<int> piv(static_cast<size_t>(s));
    for (int k = 0; k < s; ++k) {
        int p = k;
        for (int i = k + 1; i < s; ++i)
            if (std::fabs(M[i][k]) > std::fabs(M[p][k])) p = i;
        std::swap(M[k], M[p]);
        std::swap(rhs[k], rhs[p]);
        for (int i = k + 1; i < s; ++i) {
            const double f = M[i][k] / M[k][k];
            for (int j = k; j < s; ++j) M[i][j] -= f * M[k][j];
            rhs[i] -= f * rhs[k];
        }
    }
    std::vector<double> xs(static_cast<size_t>(s));
    for (int i = s - 1; i >= 0; --i) {
        double sum = rhs[i];
        for (int j = i + 1; j < s; ++j) sum -= M[i][j] * xs[j];
        xs[i] = sum / M[i][i];
    }
    return xs;
}

// ---- idr_s (itl/krylov/idr_s.hpp:31-109).  The shadow space P is s random
// vectors (the first replaced by r), orthonormalized; its random part is
// drawn from a fixed seed here, so runs repeat but differ from the
// reference's generator (iteration counts agree to the scatter a new random
// space gives).
__global__ void k_fill_random(long long n, double* v, unsigned long long seed)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        v[i] = double(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;
    }
}

inline int k_idr_s(KOp& A, KWork& W, double* x, const double* b, KIter& it, int s)
{
    const int64_t n = W.n;
    s = std::max(s, 1);
    double *y = W.vec(), *v = W.vec(), *t = W.vec(), *q = W.vec(), *r = W.vec();
    std::vector<double*> dR(static_cast<size_t>(s)), dX(static_cast<size_t>(s)), P(static_cast<size_t>(s));
    for (int k = 0; k < s; ++k) { dR[k] = W.vec(); dX[k] = W.vec(); P[k] = W.vec(); }
    if (!P[s - 1]) return MTLG_ERR_OOM;
    KTRY(kresid(A, W, b, x, r));
    for (int k = 0; k < s; ++k) {
        KTRY(W.kv(KV_FILL, dR[k], nullptr, nullptr, 0.0));
        KTRY(W.kv(KV_FILL, dX[k], nullptr, nullptr, 0.0));
        k_fill_random<<<W.grid, kBlock, 0, W.c->stream>>>(n, P[k], 0x5EEDull + 7919ull * k);
        W.c->launches++;
    }
    KTRY(W.kv(KV_COPY, P[0], r));
    // orth(P): Gram-Schmidt with normalization
    for (int j = 0; j < s; ++j) {
        for (int i = 0; i < j; ++i) {
            double d;
            KDOT(d, P[i], P[j]);
            KTRY(W.kv(KV_AXPY, P[j], P[i], nullptr, -d));
        }
        double nj;
        KNORM(nj, P[j]);
        KTRY(W.kv(KV_DIV, P[j], P[j], nullptr, nj));
    }
    std::vector<std::vector<double>> M(static_cast<size_t>(s), std::vector<double>(static_cast<size_t>(s), 0.0));
    std::vector<double> m(static_cast<size_t>(s)), c(static_cast<size_t>(s)), dm(static_cast<size_t>(s));
    double omega = 0.0, nr;
    for (int k = 0; k < s; ++k) {
        KTRY(A.apply(r, v));
        double vr, vv;
        KDOT(vr, v, r);
        KDOT(vv, v, v);
        omega = vr / vv;
        KTRY(W.kv(KV_AX, dX[k], r, nullptr, omega));
        KTRY(W.kv(KV_AX, dR[k], v, nullptr, -omega));
        KTRY(W.kv(KV_AXPY, x, dX[k], nullptr, 1.0));
        KTRY(W.kv(KV_AXPY, r, dR[k], nullptr, 1.0));
        ++it.i;
        KNORM(nr, r);
        if (it.finished(nr)) return MTLG_OK;
        for (int i = 0; i < s; ++i) KDOT(M[i][k], P[i], dR[k]);
    }
    int oldest = 0;
    for (int i = 0; i < s; ++i) KDOT(m[i], P[i], r);
    for (;;) {
        KNORM(nr, r);
        if (it.finished(nr)) break;
        for (int k = 0; k < s; ++k) {
            c = small_lu_solve(M, m);
            KTRY(W.kv(KV_FILL, q, nullptr, nullptr, 0.0));
            for (int i = 0; i < s; ++i) KTRY(W.kv(KV_AXPY, q, dR[i], nullptr, -c[i]));   // q = dR * -c
            KTRY(W.kv(KV_XPAZ, v, r, q, 1.0));                                         // v = r + q
            if (k == 0) {
                KTRY(A.apply(v, t));
                double tv, tt;
                KDOT(tv, t, v);
                KDOT(tt, t, t);
                omega = tv / tt;
                KTRY(W.kv(KV_XPAZ, dR[oldest], q, t, -omega));                        // q - omega t
            }
            // dX[oldest] = omega v - dX * c, every column of dX (the oldest one
            // included) read before the update
            KTRY(W.kv(KV_AX, y, dX[0], nullptr, -c[0]));
            for (int i = 1; i < s; ++i) KTRY(W.kv(KV_AXPY, y, dX[i], nullptr, -c[i]));
            KTRY(W.kv(KV_AXPY, y, v, nullptr, omega));
            KTRY(W.kv(KV_COPY, dX[oldest], y));
            if (k != 0) {
                KTRY(A.apply(dX[oldest], dR[oldest]));                                 // A * -dX
                KTRY(W.kv(KV_SCAL, dR[oldest], nullptr, nullptr, -1.0));
            }
            KTRY(W.kv(KV_AXPY, r, dR[oldest], nullptr, 1.0));
            KTRY(W.kv(KV_AXPY, x, dX[oldest], nullptr, 1.0));
            ++it.i;
            KNORM(nr, r);
            if (it.finished(nr)) return MTLG_OK;
            for (int i = 0; i < s; ++i) KDOT(dm[i], P[i], dR[oldest]);
            for (int i = 0; i < s; ++i) {
                M[i][oldest] = dm[i];
                m[i] += dm[i];
            }
            oldest = (oldest + 1) % s;
        }
    }
    return MTLG_OK;
}

// ---- cg and bicgstab, host-driven (cg.hpp:40-111, bicgstab.hpp:29-77), for
// operators outside the graph-captured engine
inline int k_cg(KOp& A, KWork& W, double* x, const double* b, mtlg_pc* M, KIter& it)
{
    const int64_t n = W.n;
    double *p = W.vec(), *q = W.vec(), *r = W.vec(), *z = W.vec();
    if (!z) return MTLG_ERR_OOM;
    KTRY(kresid(A, W, b, x, r));
    double rho = 0, rho_1 = 0, rr, alpha, pq;
    KDOT(rr, r, r);
    while (!it.finished(std::sqrt(std::fabs(rr)))) {
        ++it.i;
        KTRY(kpc(W.c, M, n, r, z));
        KDOT(rho, r, z);
        if (it.first()) KTRY(W.kv(KV_COPY, p, z));
        else KTRY(W.kv(KV_XPAY, p, z, nullptr, rho / rho_1));
        KTRY(A.apply(p, q));
        KDOT(pq, p, q);
        alpha = rho / pq;
        KTRY(W.kv(KV_AXPY, x, p, nullptr, alpha));
        rho_1 = rho;
        KTRY(W.kv(KV_AXPY, r, q, nullptr, -alpha));
        KDOT(rr, r, r);
    }
    return MTLG_OK;
}

inline int k_bicgstab(KOp& A, KWork& W, double* x, const double* b, mtlg_pc* M, KIter& it)
{
    const int64_t n = W.n;
    double *p = W.vec(), *phat = W.vec(), *s = W.vec(), *shat = W.vec(), *t = W.vec(), *v = W.vec(), *r = W.vec(),
           *rt = W.vec();
    if (!rt) return MTLG_ERR_OOM;
    KTRY(W.kv(KV_FILL, p, nullptr, nullptr, 0.0));
    KTRY(W.kv(KV_FILL, v, nullptr, nullptr, 0.0));
    KTRY(kresid(A, W, b, x, r));
    KTRY(W.kv(KV_COPY, rt, r));
    double rho_1 = 0, rho_2 = 0, alpha = 0, beta = 0, omega = 0, nr, g;
    for (;;) {
        KNORM(nr, r);
        if (it.finished(nr)) break;
        ++it.i;
        KDOT(rho_1, rt, r);
        if (rho_1 == 0.0) return MTLG_ERR_BREAKDOWN;
        if (it.first()) {
            KTRY(W.kv(KV_COPY, p, r));
        } else {
            if (omega == 0.0) return MTLG_ERR_BREAKDOWN;
            beta = (rho_1 / rho_2) * (alpha / omega);
            KTRY(W.kv(KV_XPAYPBZ2, p, r, v, beta, -omega));   // p = r + beta (p - omega v)
        }
        KTRY(kpc(W.c, M, n, p, phat));
        KTRY(A.apply(phat, v));
        KDOT(g, rt, v);
        if (g == 0.0) return MTLG_ERR_BREAKDOWN;
        alpha = rho_1 / g;
        KTRY(W.kv(KV_XPAZ, s, r, v, -alpha));
        KNORM(nr, s);
        if (it.finished(nr)) {
            KTRY(W.kv(KV_AXPY, x, phat, nullptr, alpha));
            break;
        }
        KTRY(kpc(W.c, M, n, s, shat));
        KTRY(A.apply(shat, t));
        double ts, tt;
        KDOT(ts, t, s);
        KDOT(tt, t, t);
        omega = ts / tt;
        KTRY(W.kv(KV_AXPBZ, x, phat, shat, alpha, omega));   // x += omega shat + alpha phat
        KTRY(W.kv(KV_XPAZ, r, s, t, -omega));
        rho_2 = rho_1;
    }
    return MTLG_OK;
}

}  // namespace mtlg

namespace mtlg {

// poisson2D_dirichlet(m, n) * v (matrix/poisson2D_dirichlet.hpp:24-80): the
// 5-point stencil 4 v_k - (neighbours) on an m x n grid (k = i n + j), each
// region's terms subtracted in the reference's order (inner points: up,
// down, left, right; borders and corners as written there).  4 v is exact,
// so the results are bitwise the reference's.
template <int ASG>
__global__ void __launch_bounds__(kBlock) k_poisson2d(int m, int n, const double* __restrict__ v, double* __restrict__ w)
{
    const long long s = (long long)m * n;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < s; k += (long long)gridDim.x * blockDim.x) {
        const int i = int(k / n), j = int(k % n);
        const bool top = i == 0, bot = i == m - 1, lef = j == 0, rig = j == n - 1;
        double t = 4.0 * v[k];
        if (!top && !bot && !lef && !rig) {
            t = t - v[k - n]; t = t - v[k + n]; t = t - v[k - 1]; t = t - v[k + 1];
        } else if (top && !lef && !rig) {
            t = t - v[k + n]; t = t - v[k - 1]; t = t - v[k + 1];
        } else if (bot && !lef && !rig) {
            t = t - v[k - n]; t = t - v[k - 1]; t = t - v[k + 1];
        } else if (lef && !top && !bot) {
            t = t - v[k - n]; t = t - v[k + n]; t = t - v[k + 1];
        } else if (rig && !top && !bot) {
            t = t - v[k - n]; t = t - v[k + n]; t = t - v[k - 1];
        } else if (top && lef) {
            t = t - v[1]; t = t - v[n];
        } else if (top && rig) {
            t = t - v[n - 2]; t = t - v[2 * n - 1];
        } else if (bot && lef) {
            t = t - v[(long long)(m - 2) * n]; t = t - v[(long long)(m - 1) * n + 1];
        } else {   // bottom right
            t = t - v[(long long)m * n - 2]; t = t - v[(long long)m * n - n - 1];
        }
        if (ASG == ASG_SET) w[k] = t;
        else if (ASG == ASG_ADD) w[k] = w[k] + t;
        else w[k] = w[k] - t;
    }
}

inline int poisson2d_apply(mtlg_ctx* c, int m, int n, const double* x, double* y, int asg)
{
    const long long s = (long long)m * n;
    if (s == 0) return MTLG_OK;
    const int g = int(std::max<long long>(1, std::min<long long>((s + kBlock - 1) / kBlock, 148LL * 16)));
    if (asg == ASG_SET) k_poisson2d<ASG_SET><<<g, kBlock, 0, c->stream>>>(m, n, x, y);
    else if (asg == ASG_ADD) k_poisson2d<ASG_ADD><<<g, kBlock, 0, c->stream>>>(m, n, x, y);
    else k_poisson2d<ASG_SUB><<<g, kBlock, 0, c->stream>>>(m, n, x, y);
    c->launches++;
    MTLG_CUDA(cudaGetLastError());
    return MTLG_OK;
}

// Transposed CSR of A (values from the device), made once per matrix.
inline int ensure_transpose(mtlg_csr* A)
{
    if (A->AT) return MTLG_OK;
    mtlg_ctx* c = A->ctx;
    const int64_t nr = A->n_rows, nc = A->n_cols, nz = A->nnz;
    std::vector<double> v(static_cast<size_t>(std::max<int64_t>(nz, 1)));
    if (nz) MTLG_CUDA(cudaMemcpy(v.data(), A->v64.p, static_cast<size_t>(nz) * 8, cudaMemcpyDeviceToHost));
    std::vector<int64_t> rp(static_cast<size_t>(nc) + 1, 0);
    for (int64_t e = 0; e < nz; ++e) rp[static_cast<size_t>(A->h_ci[static_cast<size_t>(e)]) + 1]++;
    for (int64_t j = 0; j < nc; ++j) rp[static_cast<size_t>(j) + 1] += rp[static_cast<size_t>(j)];
    std::vector<int32_t> ci(static_cast<size_t>(std::max<int64_t>(nz, 1)));
    std::vector<double> tv(static_cast<size_t>(std::max<int64_t>(nz, 1)));
    std::vector<int64_t> pos(rp.begin(), rp.end() - 1);
    for (int64_t i = 0; i < nr; ++i)
        for (int64_t e = A->h_rp[static_cast<size_t>(i)]; e < A->h_rp[static_cast<size_t>(i) + 1]; ++e) {
            const int64_t o = pos[static_cast<size_t>(A->h_ci[static_cast<size_t>(e)])]++;
            ci[static_cast<size_t>(o)] = int32_t(i);
            tv[static_cast<size_t>(o)] = v[static_cast<size_t>(e)];
        }
    return mtlg_csr_create(c, nc, nr, nz, rp.data(), ci.data(), tv.data(), MTLG_F64, &A->AT);
}

inline int KOp::apply(const double* x, double* y)
{
    if (A) return spmv_raw(c, A, MTLG_F64, x, y, nullptr, ASG_SET);
    return poisson2d_apply(c, pm, pn, x, y, ASG_SET);
}

inline int KOp::apply_t(const double* x, double* y)
{
    if (!A) return poisson2d_apply(c, pm, pn, x, y, ASG_SET);   // symmetric
    MTLG_TRY(ensure_transpose(A));
    return spmv_raw(c, A->AT, MTLG_F64, x, y, nullptr, ASG_SET);
}

// Runs a host-driven body; params and result as mtlg_solve's.
inline int krylov_run(mtlg_ctx* c, int solver, KOp& A, mtlg_pc* L, mtlg_pc* R, double* x, const double* b,
                      const mtlg_iter_params* p, mtlg_iter_result* res)
{
    KWork W;
    W.c = c;
    W.n = A.n;
    W.grid = int(std::max<int64_t>(1, std::min<int64_t>((A.n + kBlock - 1) / kBlock, int64_t(c->sm_count) * 8)));
    KIter it;
    it.max_iter = p->max_iter;
    it.rtol = p->rtol;
    it.atol = p->atol;
    if (p->norm_r0 >= 0) {
        it.norm_r0 = p->norm_r0;
    } else {
        int s;
        it.norm_r0 = W.norm(b, s);   // basic_iteration from b: two_norm(b)
        if (s != MTLG_OK) return s;
    }
    cudaEvent_t e0, e1;
    MTLG_CUDA(cudaEventCreate(&e0));
    MTLG_CUDA(cudaEventCreate(&e1));
    MTLG_CUDA(cudaEventRecord(e0, c->stream));
    int st;
    switch (solver) {
    case MTLG_CG: st = k_cg(A, W, x, b, L, it); break;
    case MTLG_BICGSTAB: st = k_bicgstab(A, W, x, b, L, it); break;
    case MTLG_BICG: st = k_bicg(A, W, x, b, L, it); break;
    case MTLG_CGS: st = k_cgs(A, W, x, b, L, it); break;
    case MTLG_TFQMR: st = k_tfqmr(A, W, x, b, L, R, it); break;
    case MTLG_QMR: st = k_qmr(A, W, x, b, L, R, it); break;
    case MTLG_BICGSTAB_2: st = k_bicgstab_ell(A, W, x, b, L, nullptr, it, 2); break;
    case MTLG_BICGSTAB_ELL: st = k_bicgstab_ell(A, W, x, b, L, R, it, p->restart > 0 ? p->restart : 2); break;
    case MTLG_IDR_S: st = k_idr_s(A, W, x, b, it, p->restart > 0 ? p->restart : 4); break;
    default: st = MTLG_ERR_NOT_SUPPORTED;
    }
    MTLG_CUDA(cudaEventRecord(e1, c->stream));
    MTLG_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (res) {
        memset(res, 0, sizeof *res);
        res->iterations = it.i;
        res->error_code = st == MTLG_ERR_BREAKDOWN ? 1 : it.error;
        res->resid = it.resid;
        res->norm_r0 = it.norm_r0;
        res->relresid = it.norm_r0 != 0 ? it.resid / it.norm_r0 : it.resid;
        res->status = st == MTLG_ERR_BREAKDOWN ? MTLG_ST_BREAKDOWN
                      : it.error == 0          ? MTLG_ST_CONVERGED
                      : it.error == 1          ? MTLG_ST_MAXIT
                                               : MTLG_ST_BREAKDOWN;
        res->seconds = ms * 1e-3;
    }
    if (st == MTLG_ERR_BREAKDOWN) set_error("%s breakdown (zero rho, gamma or omega)", "BiCGSTAB");
    return st;
}

}  // namespace mtlg
