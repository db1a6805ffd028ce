// Test infrastructure only (the checker, never the product): a CPU
// restatement of MTL4's sparse-solve hot path in plain C++ with a C ABI.
// Each function names the reference file:line whose algorithm it follows;
// paths are relative to the MTL4 tree (boost/numeric/...).  The restatement
// is pinned against the reference-built library (oracle/_ref) and against the
// known-answer vectors of the reference's own tests by tests/test_oracle.py.
//
// Index types: int64 row pointers, int32 columns; values double or float.
//
// Built with -ffp-contract=off: every fused multiply-add below is an explicit
// std::fma, placed where the reference's FMA-contracted build fuses (FP64
// triangular sweeps, the ILU(0) update).  SpMV row sums, the IC(0) pivot
// update and sweeps with FP32 factors or vectors round each product before
// the addition, as the reference build does.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <type_traits>

namespace {

struct Csr {
    int64_t n;
    const int64_t* rp;
    const int32_t* ci;
};

// w (=|+=|-=) A*v: per row an accumulator started at zero, entries in
// storage order, tmp += a * v[col] (mtl/operation/mat_vec_mult.hpp:614-683);
// Assign::first_update then assigns, adds or subtracts.  The reference build
// (g++ -O3 -march=x86-64-v3 -ffp-contract=fast) evaluates the FP64 row loop
// in groups of four entries that add the rounded product, and the row's last
// (L mod 4) entries as fused multiply-adds; FP32 rows add rounded products
// throughout.  Determined against the build's outputs, where this rule
// reproduces every row bitwise (rows of 1 to 4096 entries).
template <typename V, typename T>
void spmv(const Csr& A, const V* val, const T* x, T* y, int assign)
{
    for (int64_t i = 0; i < A.n; ++i) {
        T tmp = T(0);
        const int64_t a = A.rp[i], e = A.rp[i + 1], tail = a + (e - a) / 4 * 4;
        for (int64_t k = a; k < tail; ++k) tmp = tmp + T(val[k]) * x[A.ci[k]];
        for (int64_t k = tail; k < e; ++k)
            tmp = std::is_same<T, double>::value ? T(std::fma(double(val[k]), double(x[A.ci[k]]), double(tmp)))
                                                 : T(tmp + T(val[k]) * x[A.ci[k]]);
        if (assign == 0) y[i] = tmp;
        else if (assign == 1) y[i] += tmp;
        else y[i] -= tmp;
    }
}

// One step of a triangular row sweep, rr -= a * w.  The reference's build
// fuses it only when factor and vector are both double; with float factors or
// float vectors the product is rounded before the subtraction.
template <typename T, typename S>
inline T sweep_step(T rr, S a, T w)
{
    if (std::is_same<T, double>::value && std::is_same<S, double>::value) return std::fma(-T(a), w, rr);
    return rr - T(a) * w;
}

template <typename T>
double dot(int64_t n, const T* a, const T* b)
{
    double s = 0;
    for (int64_t i = 0; i < n; ++i) s += double(a[i]) * double(b[i]);
    return s;
}

// Reductions in the reference build's order (FP64).  Each keeps four partial
// sums t[k] over the entries i = k (mod 4) of the first 4*floor(n/4), the
// remaining entries go to t[0].  Determined against the build's outputs (the
// unrolled loops are vectorized with rounded products; scalar tails are
// contracted or not as listed):
//   dot4   mtl::dot (operation/dot.hpp:99-145, Unroll 4): rounded products
//          throughout; (t0 + t1) + (t2 + t3).
//   norm4  mtl::two_norm squared (operation/two_norm.hpp:35-56,
//          vector/reduction.hpp:85-175): rounded products, fused tail;
//          t0 + (t1 + (t2 + t3)) (reduction<>::finish).
//   ldot4  lazy_dot in a fused expression (vector/dot_index_evaluator.hpp:
//          20-45, operation/fused_expr.hpp:60-75): rounded products;
//          ((t0 + t1) + t2) + t3.
//   udot4  lazy_unary_dot in a fused expression
//          (vector/reduction_index_evaluator.hpp:31-34): fused products
//          throughout; (t0 + t1) + (t2 + t3).
inline double rprod(double a, double b) { return a * b; }   // -ffp-contract=off: rounded
template <int Kind>
double red4(int64_t n, const double* a, const double* b)
{
    double t[4] = {0.0, 0.0, 0.0, 0.0};
    const int64_t nb = n / 4 * 4;
    const bool fused_main = Kind == 3, fused_tail = Kind == 1 || Kind == 3;
    for (int64_t i = 0; i < nb; i += 4)
        for (int k = 0; k < 4; ++k)
            t[k] = fused_main ? std::fma(a[i + k], b[i + k], t[k]) : t[k] + rprod(a[i + k], b[i + k]);
    for (int64_t i = nb; i < n; ++i) t[0] = fused_tail ? std::fma(a[i], b[i], t[0]) : t[0] + rprod(a[i], b[i]);
    if (Kind == 1) return t[0] + (t[1] + (t[2] + t[3]));
    if (Kind == 2) return ((t[0] + t[1]) + t[2]) + t[3];
    return (t[0] + t[1]) + (t[2] + t[3]);
}
inline double dot4(int64_t n, const double* a, const double* b) { return red4<0>(n, a, b); }
inline double norm4(int64_t n, const double* a) { return red4<1>(n, a, a); }
inline double ldot4(int64_t n, const double* a, const double* b) { return red4<2>(n, a, b); }
inline double udot4(int64_t n, const double* a) { return red4<3>(n, a, a); }
// FP32 vectors: dots accumulate in double in storage order (the GPU's FP32
// inner solves accumulate in double as well)
inline double dot4(int64_t n, const float* a, const float* b) { return dot(n, a, b); }
inline double norm4(int64_t n, const float* a) { return dot(n, a, a); }
inline double ldot4(int64_t n, const float* a, const float* b) { return dot(n, a, b); }
inline double udot4(int64_t n, const float* a) { return dot(n, a, a); }

// itl::basic_iteration (itl/iteration/basic_iteration.hpp:32-93).
struct Iter {
    int i = 0, max_iter = 0, error = 0;
    double norm_r0 = 0, rtol = 0, atol = 0, resid = 0;
    bool finished(double r)
    {
        resid = r;
        bool conv = norm_r0 == 0 ? r <= atol : (r <= rtol * norm_r0 || r <= atol);
        if (conv) return true;
        if (i >= max_iter) { error = 1; return true; }
        return false;
    }
    bool first() const { return i <= 1; }
};

// Preconditioners ------------------------------------------------------------
// Stored factors in CSR with the reference's in-row layout.
template <typename S>
struct Tri {
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    std::vector<S> v;
};

template <typename S>
struct PC {
    int kind = 0;                // 0 identity, 1 diagonal, 2 ilu_0, 3 ic_0
    int64_t n = 0;
    std::vector<S> inv_diag;     // diagonal
    Tri<S> L, U;

    // itl/pc/diagonal.hpp:57-64, itl/pc/ilu.hpp:84-91, itl/pc/ic_0.hpp:80-87
    template <typename T>
    void apply(const T* x, T* y) const
    {
        if (kind == 0) { std::copy(x, x + n, y); return; }
        if (kind == 1) { for (int64_t i = 0; i < n; ++i) y[i] = T(inv_diag[i]) * x[i]; return; }
        std::vector<T> y0(n);
        if (kind == 2) {
            // lower_trisolve_t<L, unit_diagonal, compact> (operation/lower_trisolve.hpp:174-189)
            for (int64_t r = 0; r < n; ++r) {
                T rr = x[r];
                for (int64_t k = L.rp[r]; k < L.rp[r + 1]; ++k) rr = sweep_step(rr, L.v[k], y0[L.ci[k]]);
                y0[r] = rr;
            }
        } else {
            // lower_trisolve_t<L, inverse_diagonal, compact>, diagonal last
            // (operation/lower_trisolve.hpp:193-209)
            for (int64_t r = 0; r < n; ++r) {
                int64_t j0 = L.rp[r], j1 = L.rp[r + 1] - 1;
                const S dia = L.v[j1];
                T rr = x[r];
                for (; j0 != j1; ++j0) rr = sweep_step(rr, L.v[j0], y0[L.ci[j0]]);
                y0[r] = rr * T(dia);
            }
        }
        // upper_trisolve_t<U, inverse_diagonal, compact>, diagonal first
        // (operation/upper_trisolve.hpp:161-176)
        for (int64_t r = n; r-- > 0;) {
            int64_t j0 = U.rp[r];
            const int64_t j1 = U.rp[r + 1];
            const S dia = U.v[j0++];
            T rr = y0[r];
            for (; j0 != j1; ++j0) rr = sweep_step(rr, U.v[j0], y[U.ci[j0]]);
            y[r] = rr * T(dia);
        }
    }
};

inline int64_t find(const Csr& A, int64_t r, int64_t c)
{
    const int32_t* b = A.ci + A.rp[r];
    const int32_t* e = A.ci + A.rp[r + 1];
    const int32_t* p = std::lower_bound(b, e, int32_t(c));
    return (p != e && *p == c) ? (p - A.ci) : -1;
}

// ILU(0), Saad's IKJ variant (itl/pc/ilu_0.hpp:45-82) followed by
// invert_diagonal, strict_lower and upper (ilu_0.hpp:79-81).
template <typename S>
void ilu0(const Csr& A, const double* a, PC<S>& P)
{
    const int64_t n = A.n;
    std::vector<double> lu(a, a + A.rp[n]);
    std::vector<double> inv_dia(n);
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t kc = A.rp[i]; kc < A.rp[i + 1]; ++kc) {
            const int64_t k = A.ci[kc];
            if (k == i) break;
            const double aik = lu[kc] * inv_dia[k];
            lu[kc] = aik;
            for (int64_t jc = kc + 1; jc < A.rp[i + 1]; ++jc) {
                const int64_t pos = find(A, k, A.ci[jc]);
                const double lkj = pos >= 0 ? lu[pos] : 0.0;
                lu[jc] = std::fma(-aik, lkj, lu[jc]);
            }
        }
        const int64_t d = find(A, i, i);
        inv_dia[i] = 1.0 / (d >= 0 ? lu[d] : 0.0);
    }
    P.L.rp.assign(1, 0);
    P.U.rp.assign(1, 0);
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
            const int64_t c = A.ci[k];
            if (c < i) { P.L.ci.push_back(int32_t(c)); P.L.v.push_back(S(lu[k])); }
            else if (c == i) { P.U.ci.push_back(int32_t(c)); P.U.v.push_back(S(1.0 / lu[k])); }
            else { P.U.ci.push_back(int32_t(c)); P.U.v.push_back(S(lu[k])); }
        }
        P.L.rp.push_back(int64_t(P.L.ci.size()));
        P.U.rp.push_back(int64_t(P.U.ci.size()));
    }
}

// IC(0) (itl/pc/ic_0.hpp:136-186): U = upper(A); per row k the diagonal
// becomes 1/sqrt(u_kk), the row is scaled by it, and for every entry (k, i)
// the nonzeros of row i with column in (k, i] -- the diagonal -- are reduced
// by d * U[k][i].  L = trans(U) with the diagonal last (ic_0.hpp:57).
template <typename S>
void ic0(const Csr& A, const double* a, PC<S>& P)
{
    const int64_t n = A.n;
    std::vector<int64_t> urp(1, 0);
    std::vector<int32_t> uci;
    std::vector<double> uv;
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
            if (A.ci[k] >= i) { uci.push_back(A.ci[k]); uv.push_back(a[k]); }
        urp.push_back(int64_t(uci.size()));
    }
    for (int64_t k = 0; k < n; ++k) {
        int64_t ic = urp[k];
        const double inv_dia = 1.0 / std::sqrt(uv[ic]);
        uv[ic] = inv_dia;
        for (++ic; ic < urp[k + 1]; ++ic) {
            const double d = uv[ic] * inv_dia;
            uv[ic] = d;
            const int64_t i = uci[ic];
            // row i of U holds columns >= i; the range (k, i] is its diagonal
            for (int64_t jc = urp[i]; jc < urp[i + 1]; ++jc) {
                const int64_t j = uci[jc];
                if (j <= k || j > i) continue;
                // U[k][j] with j == i is d; the reference rounds the
                // product before the subtraction (no fused multiply-add)
                uv[jc] = uv[jc] - d * d;
            }
        }
    }
    P.U.rp = urp;
    P.U.ci = uci;
    P.U.v.assign(uv.begin(), uv.end());
    // L = trans(U): row r holds U[k][r] for k <= r (diagonal last)
    std::vector<int64_t> cnt(n + 1, 0);
    for (size_t e = 0; e < uci.size(); ++e) cnt[uci[e] + 1]++;
    for (int64_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
    P.L.rp = cnt;
    P.L.ci.resize(uci.size());
    P.L.v.resize(uci.size());
    std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
    for (int64_t k = 0; k < n; ++k)
        for (int64_t e = urp[k]; e < urp[k + 1]; ++e) {
            const int64_t r = uci[e], o = pos[r]++;
            P.L.ci[o] = int32_t(k);
            P.L.v[o] = S(uv[e]);
        }
}

template <typename S>
void make_pc(const Csr& A, const double* a, int kind, PC<S>& P)
{
    P.kind = kind;
    P.n = A.n;
    if (kind == 1) {
        P.inv_diag.resize(A.n);
        for (int64_t i = 0; i < A.n; ++i) {
            const int64_t d = find(A, i, i);
            P.inv_diag[i] = S(1) / S(d >= 0 ? a[d] : 0.0);
        }
    } else if (kind == 2) {
        ilu0(A, a, P);
    } else if (kind == 3) {
        ic0(A, a, P);
    }
}

// Conjugate gradients (itl/krylov/cg.hpp:76-111; identity: cg.hpp:40-71).
// r = b - A x; rr = dot(r, r); per iteration z = solve(L, r) and
// rho = dot(r, z) (the fused pair evaluates as two passes, the preconditioner
// not being index-evaluatable), p = z + (rho / rho_1) p, the fused
// q = A p || lazy_dot(p, q), x += alpha p, the fused r -= alpha q ||
// lazy_unary_dot(r).  The identity preconditioner runs the reference's
// unpreconditioned body, where rho is the fused unary dot itself.
template <typename V, typename T, typename S>
int cg(const Csr& A, const V* val, T* x, const T* b, const PC<S>& P, Iter& it)
{
    const int64_t n = A.n;
    const bool ident = P.kind == 0;
    std::vector<T> p(n, T(0)), q(n), r(n), z(n);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i];
    spmv(A, val, x, r.data(), 2);
    double rho = 0, rho_1 = 0, rr = dot4(n, r.data(), r.data());
    if (ident) rho = rr;
    while (!it.finished(std::sqrt(std::fabs(ident ? rho : rr)))) {
        ++it.i;
        const T* zz = r.data();
        if (!ident) {
            P.apply(r.data(), z.data());
            rho = dot4(n, r.data(), z.data());
            zz = z.data();
        }
        if (it.first()) for (int64_t i = 0; i < n; ++i) p[i] = zz[i];
        else {
            const T beta = T(rho / rho_1);
            for (int64_t i = 0; i < n; ++i) p[i] = std::fma(beta, p[i], zz[i]);
        }
        spmv(A, val, p.data(), q.data(), 0);
        const T alpha = T(rho / ldot4(n, p.data(), q.data()));
        for (int64_t i = 0; i < n; ++i) x[i] = std::fma(alpha, p[i], x[i]);
        rho_1 = rho;
        for (int64_t i = 0; i < n; ++i) r[i] = std::fma(-alpha, q[i], r[i]);
        if (ident) rho = udot4(n, r.data());
        else rr = udot4(n, r.data());
    }
    return it.error;
}

// BiCGSTAB (itl/krylov/bicgstab.hpp:29-77).  Returns -2 on the breakdowns
// for which the reference throws unexpected_orthogonality.  Norms are
// two_norm (iter.finished(r), finished(s)), the scalars mtl::dot; the update
// x += omega shat + alpha phat is evaluated x + fma(alpha, phat, omega shat)
// as the reference build does.
template <typename V, typename T, typename S>
int bicgstab(const Csr& A, const V* val, T* x, const T* b, const PC<S>& P, Iter& it)
{
    const int64_t n = A.n;
    std::vector<T> p(n, T(0)), phat(n), s(n), shat(n), t(n), v(n, T(0)), r(n), rt(n);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i];
    spmv(A, val, x, r.data(), 2);
    rt = r;
    double rho_1 = 0, rho_2 = 0, alpha = 0, beta = 0, omega = 0;
    while (!it.finished(std::sqrt(norm4(n, r.data())))) {
        ++it.i;
        rho_1 = dot4(n, rt.data(), r.data());
        if (rho_1 == 0.0) return -2;
        if (it.first()) p = r;
        else {
            if (omega == 0.0) return -2;
            beta = (rho_1 / rho_2) * (alpha / omega);
            for (int64_t i = 0; i < n; ++i) p[i] = std::fma(T(beta), std::fma(-T(omega), v[i], p[i]), r[i]);
        }
        P.apply(p.data(), phat.data());
        spmv(A, val, phat.data(), v.data(), 0);
        const double gamma = dot4(n, rt.data(), v.data());
        if (gamma == 0.0) return -2;
        alpha = rho_1 / gamma;
        for (int64_t i = 0; i < n; ++i) s[i] = std::fma(-T(alpha), v[i], r[i]);
        if (it.finished(std::sqrt(norm4(n, s.data())))) {
            for (int64_t i = 0; i < n; ++i) x[i] = std::fma(T(alpha), phat[i], x[i]);
            break;
        }
        P.apply(s.data(), shat.data());
        spmv(A, val, shat.data(), t.data(), 0);
        omega = dot4(n, t.data(), s.data()) / dot4(n, t.data(), t.data());
        for (int64_t i = 0; i < n; ++i) {
            x[i] = x[i] + std::fma(T(alpha), phat[i], T(omega) * shat[i]);
            r[i] = std::fma(-T(omega), t[i], s[i]);
        }
        rho_2 = rho_1;
    }
    return it.error;
}

// Restarted GMRES (itl/krylov/gmres.hpp:37-137): modified Gram-Schmidt with
// one re-orthogonalization pass, Givens QR of H, back substitution on the
// leading k x k block, x += V y, restart until finished.  The reference
// rebuilds the rotations of column k from column k-1 (gmres.hpp:84-85); this
// restatement applies the stored rotations (c_i, s_i) to column k, the
// standard update, and is the iteration-count oracle for GMRES.
template <typename V, typename T, typename S>
int gmres(const Csr& A, const V* val, T* x, const T* b, const PC<S>& Lp, Iter& it, int restart)
{
    const int64_t n = A.n;
    std::vector<T> r(n), w(n), tmp(n);
    while (true) {
        const int kmax = int(std::min<int64_t>(n, std::max(0, std::min(restart, it.max_iter - it.i))));
        for (int64_t i = 0; i < n; ++i) tmp[i] = b[i];
        spmv(A, val, x, tmp.data(), 2);
        Lp.apply(tmp.data(), r.data());
        double rho = std::sqrt(dot(n, r.data(), r.data()));
        if (it.finished(rho) || kmax == 0) break;
        std::vector<std::vector<T>> Vb(kmax + 1, std::vector<T>(n));
        std::vector<double> H((kmax + 1) * kmax, 0.0), cs(kmax, 0), sn(kmax, 0), g(kmax + 1, 0);
        auto h = [&](int i, int j) -> double& { return H[i * kmax + j]; };
        g[0] = rho;
        for (int64_t i = 0; i < n; ++i) Vb[0][i] = T(r[i] / rho);
        int k = 0;
        for (; k < kmax; ++k) {
            ++it.i;
            spmv(A, val, Vb[k].data(), tmp.data(), 0);
            Lp.apply(tmp.data(), w.data());
            for (int j = 0; j <= k; ++j) {
                h(j, k) = dot(n, Vb[j].data(), w.data());
                for (int64_t i = 0; i < n; ++i) w[i] = std::fma(-T(h(j, k)), Vb[j][i], w[i]);
            }
            for (int j = 0; j <= k; ++j) {
                const double hr = dot(n, w.data(), Vb[j].data());
                h(j, k) += hr;
                for (int64_t i = 0; i < n; ++i) w[i] = std::fma(-T(hr), Vb[j][i], w[i]);
            }
            h(k + 1, k) = std::sqrt(dot(n, w.data(), w.data()));
            if (h(k + 1, k) != 0.0)
                for (int64_t i = 0; i < n; ++i) Vb[k + 1][i] = T(w[i] / h(k + 1, k));
            for (int i = 0; i < k; ++i) {
                const double a0 = h(i, k), a1 = h(i + 1, k);
                h(i, k) = cs[i] * a0 - sn[i] * a1;
                h(i + 1, k) = sn[i] * a0 + cs[i] * a1;
            }
            const double nu = std::sqrt(h(k, k) * h(k, k) + h(k + 1, k) * h(k + 1, k));
            if (nu != 0.0) {
                cs[k] = h(k, k) / nu;
                sn[k] = -h(k + 1, k) / nu;
                h(k, k) = cs[k] * h(k, k) - sn[k] * h(k + 1, k);
                h(k + 1, k) = 0.0;
                const double g0 = g[k], g1 = g[k + 1];
                g[k] = cs[k] * g0 - sn[k] * g1;
                g[k + 1] = sn[k] * g0 + cs[k] * g1;
            }
            if (it.i >= it.max_iter) { ++k; break; }
        }
        int kk = std::min(k, kmax);
        while (kk > 0 && std::fabs(g[kk - 1]) <= it.atol) --kk;
        std::vector<double> y(kk, 0.0);
        for (int i = kk - 1; i >= 0; --i) {
            double s2 = g[i];
            for (int j = i + 1; j < kk; ++j) s2 -= h(i, j) * y[j];
            y[i] = h(i, i) != 0.0 ? s2 / h(i, i) : 0.0;
        }
        for (int j = 0; j < kk; ++j)
            for (int64_t i = 0; i < n; ++i) x[i] = std::fma(T(y[j]), Vb[j][i], x[i]);
        for (int64_t i = 0; i < n; ++i) tmp[i] = b[i];
        spmv(A, val, x, tmp.data(), 2);
        const double res = std::sqrt(dot(n, tmp.data(), tmp.data()));
        if (it.finished(res)) break;
    }
    return it.error;
}

template <typename V, typename T, typename S>
int run(int solver, const Csr& A, const V* val, T* x, const T* b, const PC<S>& P, Iter& it, int restart)
{
    if (solver == 0) return cg(A, val, x, b, P, it);
    if (solver == 1) return bicgstab(A, val, x, b, P, it);
    return gmres(A, val, x, b, P, it, restart);
}

}  // namespace

extern "C" {

struct mtlo_result {
    int iterations;
    int error;
    double resid;
    double relresid;
    int outer;
    int pad;
};

void mtlo_spmv(int64_t n, const int64_t* rp, const int32_t* ci, const double* val, const double* x, double* y,
               int assign)
{
    spmv(Csr{n, rp, ci}, val, x, y, assign);
}

// w (=|+=|-=) E v for MTL4's ELL layout (operation/mat_vec_mult.hpp:686-700):
// per row the slots in order, entry (r, i) at k = r + i * stride, padding
// included (value 0); the reference build adds rounded products throughout.
void mtlo_ell_spmv(int64_t n, int64_t stride, int64_t slots, const int64_t* minor, const double* data,
                   const double* x, double* y, int assign)
{
    for (int64_t r = 0; r < n; ++r) {
        double s = 0.0;
        for (int64_t i = 0, k = r; i < slots; ++i, k += stride) s = s + data[k] * x[minor[k]];
        if (assign == 0) y[r] = s;
        else if (assign == 1) y[r] += s;
        else y[r] -= s;
    }
}

// Rows of sparse_banded's product loop (operation/mat_vec_mult.hpp:704-803)
// run in 4-row blocks or singly: the row range is cut where a band starts or
// ends; in each piece [from, to) rows from .. from + 4 floor((to-from)/4) go
// in blocks, the rest singly.  flags[r] = 1 for a blocked row; rows outside
// every band's range get 2 (no active band).
void mtlo_banded_row_kinds(int64_t nr, int64_t nc, int64_t nb, const int64_t* bands, unsigned char* flags)
{
    for (int64_t r = 0; r < nr; ++r) flags[r] = 2;
    if (nb == 0) return;
    std::vector<int64_t> begin_rows(nb), end_rows(nb);
    for (int64_t b = 0; b < nb; ++b) {
        begin_rows[b] = std::max<int64_t>(0, -bands[b]);
        end_rows[b] = std::min<int64_t>(nr, nc - bands[b]);
    }
    int64_t bp = 0, ep = nb - 1;
    while (bp < nb && begin_rows[bp] > 0) bp++;
    if (bp == nb) --bp;
    int64_t from = begin_rows[bp];
    while (bp > 0 && begin_rows[bp - 1] == from) bp--;
    for (bool active = true; active;) {
        const int64_t to = bp > 0 && begin_rows[bp - 1] <= end_rows[ep] ? begin_rows[bp - 1] : end_rows[ep];
        const int64_t blocked_to = ((to - from) & -4) + from;
        for (int64_t r = from; r < to; ++r) flags[r] = r < blocked_to ? 1 : 0;
        if (bp > 0) {
            if (begin_rows[bp - 1] == to) bp--;
            if (end_rows[ep] == to) ep--;
        } else {
            if (end_rows[0] == to) active = false;
            else ep--;
        }
        from = to;
    }
}

// w (=|+=|-=) S v for MTL4's sparse_banded layout (values row by row, one
// per band): per row the bands inside the matrix in increasing order; the
// reference build adds rounded products in groups of 2 (blocked rows) or 4
// (single rows of at least 4 bands; shorter single rows round every product)
// and fuses the rest.  Rows with no band inside the matrix get
// 0 for '=' and stay as they are for '+=' / '-='.
void mtlo_banded_spmv(int64_t nr, int64_t nc, int64_t nb, const int64_t* bands, const double* data,
                      const double* x, double* y, int assign)
{
    std::vector<unsigned char> kind(size_t(nr), 2);
    mtlo_banded_row_kinds(nr, nc, nb, bands, kind.data());
    for (int64_t r = 0; r < nr; ++r) {
        if (kind[r] == 2) {
            if (assign == 0) y[r] = 0.0;
            continue;
        }
        int64_t lo = 0, hi = nb;
        while (lo < nb && r + bands[lo] < 0) ++lo;
        while (hi > lo && r + bands[hi - 1] >= nc) --hi;
        // blocked rows: groups of 2, the odd last band fused; single rows:
        // groups of 4 and the rest fused when the row has 4 bands or more,
        // else every product rounded
        const int64_t cnt = hi - lo;
        const int64_t q = kind[r] == 1 ? lo + cnt / 2 * 2 : (cnt >= 4 ? lo + cnt / 4 * 4 : hi);
        double s = 0.0;
        for (int64_t b = lo; b < hi; ++b) {
            const double a = data[r * nb + b], v = x[r + bands[b]];
            s = b < q ? s + a * v : std::fma(a, v, s);
        }
        if (assign == 0) y[r] = s;
        else if (assign == 1) y[r] += s;
        else y[r] -= s;
    }
}

void mtlo_spmv_f32(int64_t n, const int64_t* rp, const int32_t* ci, const float* val, const float* x, float* y,
                   int assign)
{
    spmv(Csr{n, rp, ci}, val, x, y, assign);
}

double mtlo_dot(int64_t n, const double* a, const double* b) { return dot(n, a, b); }
// mtl::dot and two_norm squared in the reference build's summation order
double mtlo_dot4(int64_t n, const double* a, const double* b) { return dot4(n, a, b); }
double mtlo_norm4(int64_t n, const double* a) { return norm4(n, a); }

/// y = solve(P, x); storage_f32 selects the stored factor precision.
void mtlo_pc_apply(int64_t n, const int64_t* rp, const int32_t* ci, const double* a, int kind, int storage_f32,
                   const double* x, double* y)
{
    Csr A{n, rp, ci};
    if (storage_f32) { PC<float> P; make_pc(A, a, kind, P); P.apply(x, y); }
    else { PC<double> P; make_pc(A, a, kind, P); P.apply(x, y); }
}

void mtlo_pc_apply_f32(int64_t n, const int64_t* rp, const int32_t* ci, const double* a, int kind, const float* x,
                       float* y)
{
    Csr A{n, rp, ci};
    PC<float> P;
    if (kind == 1) {
        // pc::diagonal of the FP32 matrix: 1/float(a_ii) in FP32
        P.kind = 1; P.n = n; P.inv_diag.resize(n);
        for (int64_t i = 0; i < n; ++i) { int64_t d = find(A, i, i); P.inv_diag[i] = 1.0f / float(d >= 0 ? a[d] : 0.0); }
    } else {
        make_pc(A, a, kind, P);
    }
    P.apply(x, y);
}

/// Factor export in the reference's layout; null arrays query the sizes.
int mtlo_pc_factor(int64_t n, const int64_t* rp, const int32_t* ci, const double* a, int kind, int which,
                   int64_t* nnz, int64_t* out_rp, int32_t* out_ci, double* out_v)
{
    Csr A{n, rp, ci};
    PC<double> P;
    make_pc(A, a, kind, P);
    const Tri<double>& T = which == 0 ? P.L : P.U;
    if (nnz) *nnz = int64_t(T.ci.size());
    if (out_rp) std::copy(T.rp.begin(), T.rp.end(), out_rp);
    if (out_ci) std::copy(T.ci.begin(), T.ci.end(), out_ci);
    if (out_v) std::copy(T.v.begin(), T.v.end(), out_v);
    return 0;
}

/// FP64 solve; norm_r0 < 0 takes ||b||.  solver 0 cg, 1 bicgstab, 2 gmres.
int mtlo_solve(int64_t n, const int64_t* rp, const int32_t* ci, const double* a, int solver, int kind, const double* b,
               double* x, int max_iter, double rtol, double atol, int restart, double norm_r0, mtlo_result* out)
{
    Csr A{n, rp, ci};
    PC<double> P;
    make_pc(A, a, kind, P);
    Iter it;
    it.max_iter = max_iter; it.rtol = rtol; it.atol = atol;
    it.norm_r0 = norm_r0 >= 0 ? norm_r0 : std::sqrt(norm4(n, b));   // two_norm(b)
    int err = run(solver, A, a, x, b, P, it, restart);
    if (out) { *out = mtlo_result{it.i, err, it.resid, it.norm_r0 ? it.resid / it.norm_r0 : it.resid, 0, 0}; }
    return err;
}

/// FP64 iterative refinement around an FP32 inner solve (no reference
/// counterpart): r = b - A x in FP64; stop when ||r|| <= rtol ||b||; inner
/// solve of A_f32 d = float(r / ||r||) to inner_rtol with the FP32 values
/// and a PC factorized in FP64 and stored in FP32; x += ||r|| d.
int mtlo_refine_solve(int64_t n, const int64_t* rp, const int32_t* ci, const double* a, int solver, int kind,
                      const double* b, double* x, int max_outer, int max_inner, double rtol, double inner_rtol,
                      mtlo_result* out)
{
    Csr A{n, rp, ci};
    std::vector<float> af(a, a + rp[n]);
    PC<float> P;
    if (kind == 1) {
        P.kind = 1; P.n = n; P.inv_diag.resize(n);
        for (int64_t i = 0; i < n; ++i) { int64_t d = find(A, i, i); P.inv_diag[i] = 1.0f / float(d >= 0 ? a[d] : 0.0); }
    } else {
        make_pc(A, a, kind, P);
    }
    std::vector<double> r(n);
    std::vector<float> rf(n), d(n);
    const double nb = std::sqrt(dot(n, b, b));
    int inner = 0, outer = 0, err = 1;
    double rn = 0;
    for (outer = 0; outer <= max_outer; ++outer) {
        for (int64_t i = 0; i < n; ++i) r[i] = b[i];
        spmv(A, a, x, r.data(), 2);
        rn = std::sqrt(dot(n, r.data(), r.data()));
        if (rn <= rtol * nb) { err = 0; break; }
        if (outer == max_outer) break;
        for (int64_t i = 0; i < n; ++i) rf[i] = float(r[i] / rn);
        std::fill(d.begin(), d.end(), 0.0f);
        Iter it;
        it.max_iter = max_inner; it.rtol = inner_rtol; it.atol = 0;
        it.norm_r0 = std::sqrt(dot(n, rf.data(), rf.data()));
        run(solver, A, af.data(), d.data(), rf.data(), P, it, 0);
        inner += it.i;
        for (int64_t i = 0; i < n; ++i) x[i] = std::fma(rn, double(d[i]), x[i]);
    }
    if (out) *out = mtlo_result{inner, err, rn, nb ? rn / nb : rn, outer, 0};
    return err;
}

}  // extern "C"
