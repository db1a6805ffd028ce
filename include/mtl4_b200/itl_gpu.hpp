// C++ front end over the mtl4_b200 C ABI: the reference's call surface for
// the sparse-solve hot path, on GPU-resident types.
//
//   mtl::gpu::compressed2D<T>   like mtl::compressed2D<T>  (matrix/compressed2D.hpp:259,355)
//   mtl::gpu::dense_vector<T>   like mtl::dense_vector<T>  (vector/dense_vector.hpp:52,122)
//   y = A * x; y += A * x; y -= A * x; dot(x, y); two_norm(x)
//   itl::basic_iteration<Real>  (itl/iteration/basic_iteration.hpp:24-164)
//   itl::pc::identity / diagonal / ilu_0 / ic_0 <gpu matrix, Value>   (itl/pc/*.hpp)
//   solve(P, x), adjoint_solve(P, x)
//   itl::cg(A, x, b, P, iter)                 (itl/krylov/cg.hpp:76)
//   itl::bicgstab(A, x, b, P, iter)           (itl/krylov/bicgstab.hpp:29)
//   itl::gmres(A, x, b, L, R, iter, restart)  (itl/krylov/gmres.hpp:124)
//   itl::refine_cg / refine_bicgstab          (FP64 refinement around FP32; new)
//
// User code written against MTL4 keeps its solver calls; only the matrix
// and vector types change.  If MTL4's own ITL headers are used in the same
// translation unit, include them before this header: then their
// itl::basic_iteration is used and the preconditioner templates below are
// added as specializations of theirs.  Errors become exceptions named after
// the reference's (mtl::gpu::matrix_not_square, ...,
// itl::gpu::unexpected_orthogonality).
#ifndef MTL4_B200_ITL_GPU_HPP
#define MTL4_B200_ITL_GPU_HPP

#include <cmath>
#include <cstdint>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "mtlg.h"

namespace mtl {
namespace gpu {

struct runtime_error : std::runtime_error {
    int status;
    runtime_error(int s, const std::string& what) : std::runtime_error(what), status(s) {}
};
struct matrix_not_square : runtime_error { using runtime_error::runtime_error; };
struct missing_diagonal : runtime_error { using runtime_error::runtime_error; };
struct incompatible_size : runtime_error { using runtime_error::runtime_error; };
struct device_timeout : runtime_error { using runtime_error::runtime_error; };

}  // namespace gpu
}  // namespace mtl

namespace itl {
namespace gpu {
struct unexpected_orthogonality : mtl::gpu::runtime_error { using runtime_error::runtime_error; };
}  // namespace gpu
}  // namespace itl

namespace mtl {
namespace gpu {

inline void check(int s, const char* what)
{
    if (s == MTLG_OK) return;
    std::string msg = std::string(what) + ": " + mtlg_status_string(s);
    const char* d = mtlg_last_error_message();
    if (d && *d) msg += std::string(" (") + d + ")";
    switch (s) {
    case MTLG_ERR_NOT_SQUARE: throw matrix_not_square(s, msg);
    case MTLG_ERR_MISSING_DIAGONAL: throw missing_diagonal(s, msg);
    case MTLG_ERR_INCOMPATIBLE_SIZE: throw incompatible_size(s, msg);
    case MTLG_ERR_BREAKDOWN: throw itl::gpu::unexpected_orthogonality(s, msg);
    case MTLG_ERR_TIMEOUT: throw device_timeout(s, msg);
    default: throw runtime_error(s, msg);
    }
}

template <typename T> struct dtype_of;
template <> struct dtype_of<double> { static const mtlg_dtype value = MTLG_F64; };
template <> struct dtype_of<float> { static const mtlg_dtype value = MTLG_F32; };

/// One device and its stream; objects keep a reference to their context.
class context {
  public:
    explicit context(int device = 0, std::size_t hbm_budget = 0)
    {
        mtlg_ctx* c = nullptr;
        check(mtlg_ctx_create(device, hbm_budget, &c), "context");
        h_.reset(c, [](mtlg_ctx* p) { mtlg_ctx_destroy(p); });
    }
    mtlg_ctx* get() const { return h_.get(); }
    void synchronize() const { check(mtlg_ctx_synchronize(get()), "synchronize"); }
    /// Device residual log of at least `tests` termination tests (grown, never shrunk).
    void ensure_residual_log(int tests)
    {
        if (tests > log_cap_) {
            check(mtlg_ctx_set_residual_log(get(), tests), "residual log");
            log_cap_ = tests;
        }
    }
    int residual_log_capacity() const { return log_cap_; }
    int64_t kernel_launches() const { return mtlg_ctx_kernel_launches(get()); }
    static context& default_context()
    {
        static context c(0);
        return c;
    }

  private:
    std::shared_ptr<mtlg_ctx> h_;
    int log_cap_ = 0;
};

template <typename T> struct mat_cvec_times;

template <typename T>
class dense_vector {
  public:
    typedef T value_type;
    typedef std::size_t size_type;

    explicit dense_vector(size_type n = 0, context& ctx = context::default_context()) : ctx_(ctx), n_(n)
    {
        mtlg_vec* v = nullptr;
        check(mtlg_vec_create(ctx_.get(), int64_t(n), dtype_of<T>::value, &v), "dense_vector");
        h_.reset(v, [](mtlg_vec* p) { mtlg_vec_destroy(p); });
    }
    dense_vector(const std::vector<T>& host, context& ctx = context::default_context()) : dense_vector(host.size(), ctx)
    {
        upload(host.data());
    }
    dense_vector(size_type n, const T* host, context& ctx = context::default_context()) : dense_vector(n, ctx)
    {
        upload(host);
    }
    void upload(const T* host) { check(mtlg_vec_upload(get(), host, int64_t(n_)), "upload"); }
    void download(T* host) const { check(mtlg_vec_download(get(), host, int64_t(n_)), "download"); }
    std::vector<T> to_host() const
    {
        std::vector<T> out(n_);
        download(out.data());
        return out;
    }
    dense_vector& operator=(T value)
    {
        check(mtlg_vec_fill(get(), double(value)), "fill");
        return *this;
    }
    /// w = A * v  (vector/crtp_base_vector.hpp:94-101)
    dense_vector& operator=(const mat_cvec_times<T>& e);
    size_type size() const { return n_; }
    mtlg_vec* get() const { return h_.get(); }
    context& ctx() const { return ctx_; }

  private:
    context& ctx_;
    size_type n_;
    std::shared_ptr<mtlg_vec> h_;
};

template <typename T>
inline std::size_t size(const dense_vector<T>& v) { return v.size(); }

/// CSR matrix: built from raw CSR arrays like compressed2D(m, n, nnz,
/// Major, Minor, Entries), with std::size_t or int64 row starts.
template <typename T>
class compressed2D {
  public:
    typedef T value_type;
    typedef std::size_t size_type;

    template <typename Major, typename Minor>
    compressed2D(size_type m, size_type n, size_type nnz, const Major* starts, const Minor* indices, const T* entries,
                 context& ctx = context::default_context())
        : ctx_(ctx), m_(m), n_(n), nnz_(nnz)
    {
        std::vector<int64_t> rp(starts, starts + m + 1);
        std::vector<int32_t> ci(indices, indices + nnz);
        mtlg_csr* a = nullptr;
        check(mtlg_csr_create(ctx_.get(), int64_t(m), int64_t(n), int64_t(nnz), rp.data(), ci.data(), entries,
                              dtype_of<T>::value, &a),
              "compressed2D");
        h_.reset(a, [](mtlg_csr* p) { mtlg_csr_destroy(p); });
    }
    size_type num_rows() const { return m_; }
    size_type num_cols() const { return n_; }
    size_type nnz() const { return nnz_; }
    mtlg_csr* get() const { return h_.get(); }
    context& ctx() const { return ctx_; }

  private:
    context& ctx_;
    size_type m_, n_, nnz_;
    std::shared_ptr<mtlg_csr> h_;
};

template <typename T> inline std::size_t num_rows(const compressed2D<T>& A) { return A.num_rows(); }
template <typename T> inline std::size_t num_cols(const compressed2D<T>& A) { return A.num_cols(); }

/// 2D 5-point Laplacian on an m x n grid (matrix/laplacian_setup.hpp:26-41).
template <typename T>
compressed2D<T> laplacian_setup(unsigned m, unsigned n, context& ctx = context::default_context())
{
    std::vector<int64_t> rp(1, 0);
    std::vector<int32_t> ci;
    std::vector<T> v;
    for (unsigned i = 0; i < m; ++i)
        for (unsigned j = 0; j < n; ++j) {
            const int64_t row = int64_t(i) * n + j;
            if (i > 0) { ci.push_back(int32_t(row - n)); v.push_back(T(-1)); }
            if (j > 0) { ci.push_back(int32_t(row - 1)); v.push_back(T(-1)); }
            ci.push_back(int32_t(row)); v.push_back(T(4));
            if (j + 1 < n) { ci.push_back(int32_t(row + 1)); v.push_back(T(-1)); }
            if (i + 1 < m) { ci.push_back(int32_t(row + n)); v.push_back(T(-1)); }
            rp.push_back(int64_t(ci.size()));
        }
    return compressed2D<T>(std::size_t(m) * n, std::size_t(m) * n, ci.size(), rp.data(), ci.data(), v.data(), ctx);
}

template <typename T>
struct mat_cvec_times {
    const compressed2D<T>& A;
    const dense_vector<T>& v;
};

template <typename T>
inline mat_cvec_times<T> operator*(const compressed2D<T>& A, const dense_vector<T>& v) { return {A, v}; }

template <typename T>
inline void mult(const compressed2D<T>& A, const dense_vector<T>& v, dense_vector<T>& w, int assign = MTLG_ASSIGN)
{
    check(mtlg_spmv(A.ctx().get(), A.get(), v.get(), w.get(), assign), "mult");
}

template <typename T>
inline dense_vector<T>& dense_vector<T>::operator=(const mat_cvec_times<T>& e)
{
    mult(e.A, e.v, *this, MTLG_ASSIGN);
    return *this;
}
template <typename T>
inline dense_vector<T>& operator+=(dense_vector<T>& w, const mat_cvec_times<T>& e)
{
    mult(e.A, e.v, w, MTLG_PLUS);
    return w;
}
template <typename T>
inline dense_vector<T>& operator-=(dense_vector<T>& w, const mat_cvec_times<T>& e)
{
    mult(e.A, e.v, w, MTLG_MINUS);
    return w;
}

template <typename T>
inline double dot(const dense_vector<T>& x, const dense_vector<T>& y)
{
    double r = 0;
    check(mtlg_dot(x.ctx().get(), x.get(), y.get(), &r), "dot");
    return r;
}
template <typename T>
inline double two_norm(const dense_vector<T>& x)
{
    double r = 0;
    check(mtlg_two_norm(x.ctx().get(), x.get(), &r), "two_norm");
    return r;
}

}  // namespace gpu

#ifdef MTL_COLLECTION_INCLUDE
// With MTL4's headers included first, its templates take their defaults from
// mtl::Collection (concept/collection.hpp:43-55), e.g. the Value argument of
// itl::pc::diagonal<Matrix, Value>: the GPU types are collections of T.
template <typename T>
struct Collection<gpu::compressed2D<T> > {
    typedef T value_type;
    typedef const T& const_reference;
    typedef std::size_t size_type;
};
template <typename T>
struct Collection<gpu::dense_vector<T> > {
    typedef T value_type;
    typedef const T& const_reference;
    typedef std::size_t size_type;
};
#endif
}  // namespace mtl

namespace itl {

#ifndef ITL_BASIC_ITERATION_INCLUDE
#define ITL_BASIC_ITERATION_INCLUDE
/// Termination control with the reference's members (basic_iteration.hpp).
template <class Real>
class basic_iteration {
  public:
    typedef Real real;
    template <class Vector>
    basic_iteration(const Vector& r0, int max_iter, Real rtol, Real atol = Real(0))
        : error_(0), i_(0), norm_r0_(std::abs(two_norm(r0))), max_iter_(max_iter), rtol_(rtol), atol_(atol), resid_(0)
    {}
    basic_iteration(Real nb, int max_iter, Real rtol, Real atol = Real(0))
        : error_(0), i_(0), norm_r0_(nb), max_iter_(max_iter), rtol_(rtol), atol_(atol), resid_(0)
    {}
    bool finished(const Real& r)
    {
        resid_ = r;
        if (norm_r0_ == 0 ? r <= atol_ : (r <= rtol_ * norm_r0_ || r <= atol_)) return true;
        if (i_ >= max_iter_) { error_ = 1; return true; }
        return false;
    }
    basic_iteration& operator+=(int n) { i_ += n; return *this; }
    basic_iteration& operator++() { ++i_; return *this; }
    int iterations() const { return i_; }
    int max_iterations() const { return max_iter_; }
    int error_code() const { return error_; }
    operator int() const { return error_; }
    bool is_converged() const { return error_ == 0 && resid_ <= std::max(rtol_ * norm_r0_, atol_); }
    Real resid() const { return resid_; }
    Real relresid() const { return norm_r0_ ? resid_ / norm_r0_ : resid_; }
    Real norm_r0() const { return norm_r0_; }
    Real tol() const { return rtol_; }
    Real atol() const { return atol_; }
    int fail(int code) { error_ = code; return error_; }

  private:
    int error_, i_;
    Real norm_r0_;
    int max_iter_;
    Real rtol_, atol_, resid_;
};
#endif

#ifndef ITL_CYCLIC_ITERATION_INCLUDE
#define ITL_CYCLIC_ITERATION_INCLUDE
/// Termination control that prints the residual every `cycle` iterations
/// and a summary from error_code(), as the reference's cyclic_iteration
/// (itl/iteration/cyclic_iteration.hpp:22-95) does.  On the GPU the tests run
/// on the device; their (iteration, residual) log is replayed through
/// finished() after the solve, so the output is the same lines.
template <class Real, class OStream = std::ostream>
class cyclic_iteration : public basic_iteration<Real> {
    typedef basic_iteration<Real> super;

  public:
    template <class Vector>
    cyclic_iteration(const Vector& r0, int max_iter, Real tol, Real atol = Real(0), int cycle = 100,
                     OStream& out = std::cout)
        : super(r0, max_iter, tol, atol), cycle_(cycle), last_print_(-1), multi_print_(false), out_(out)
    {}
    cyclic_iteration(Real r0, int max_iter, Real tol, Real atol = Real(0), int cycle = 100, OStream& out = std::cout)
        : super(r0, max_iter, tol, atol), cycle_(cycle), last_print_(-1), multi_print_(false), out_(out)
    {}
    bool finished(const Real& r)
    {
        const bool ret = super::finished(r);
        print_resid();
        return ret;
    }
    cyclic_iteration& operator++() { super::operator++(); return *this; }
    cyclic_iteration& operator+=(int n) { super::operator+=(n); return *this; }
    operator int() const { return error_code(); }
    bool is_multi_print() const { return multi_print_; }
    void set_multi_print(bool m) { multi_print_ = m; }
    void set_cycle(int c) { cycle_ = c; }
    /// Error code with the final summary (printed on every call, as the reference does).
    int error_code() const
    {
        out_ << "finished! error code = " << super::error_code() << '\n'
             << this->iterations() << " iterations\n"
             << this->resid() << " is actual final residual. \n"
             << this->relresid() << " is actual relative tolerance achieved. \n"
             << "Relative tol: " << this->tol() << "  Absolute tol: " << this->atol() << '\n'
             << "Convergence:  " << std::pow(this->relresid(), 1.0 / double(this->iterations())) << std::endl;
        return super::error_code();
    }

  private:
    void print_resid()
    {
        if (this->iterations() % cycle_ == 0 && (multi_print_ || this->iterations() != last_print_)) {
            out_ << "iteration " << this->iterations() << ": resid " << this->resid() << std::endl;
            last_print_ = this->iterations();
        }
    }
    int cycle_, last_print_;
    bool multi_print_;
    OStream& out_;
};
#endif

#ifndef ITL_NOISY_ITERATION_INCLUDE
#define ITL_NOISY_ITERATION_INCLUDE
/// cyclic_iteration printing every iteration (itl/iteration/noisy_iteration.hpp:22-35).
template <class Real, class OStream = std::ostream>
class noisy_iteration : public cyclic_iteration<Real, OStream> {
  public:
    template <class Vector>
    noisy_iteration(const Vector& r0, int max_iter, Real tol, Real atol = Real(0), OStream& out = std::cout)
        : cyclic_iteration<Real, OStream>(r0, max_iter, tol, atol, 1, out)
    {}
};
#endif

namespace gpu {
/// Takes a device result into any iteration object with the reference's
/// members (iterations via +=, resid via finished(), error via fail()).
/// With a residual log, every device-side termination test is replayed
/// through finished() in order, so iteration objects that act on each test
/// (cyclic_iteration, noisy_iteration, the reference's own) see the same
/// sequence as in the reference's loop.  error_code() is not read here: the
/// reference's cyclic_iteration prints its summary on each call, and the
/// solver's return reads it once.
template <class Iteration>
inline int take_result(Iteration& iter, const mtlg_iter_result& r, const std::vector<double>* log = nullptr)
{
    typedef typename Iteration::real Real;
    if (log && !log->empty()) {
        for (std::size_t k = 0; k + 1 < log->size(); k += 2) {
            const int add = int((*log)[k]) - iter.iterations();
            if (add > 0) iter += add;
            iter.finished(Real((*log)[k + 1]));
        }
        const int add = r.iterations - iter.iterations();
        if (add > 0) iter += add;
    } else {
        const int add = r.iterations - iter.iterations();
        if (add > 0) iter += add;
        iter.finished(Real(r.resid));
    }
    if (r.error_code > 1) iter.fail(r.error_code);
    return r.error_code;
}

/// The residual log of the context's last solve (empty when it holds more
/// tests than the capacity, or none).
inline std::vector<double> residual_log(const mtl::gpu::context& c)
{
    int count = 0;
    mtl::gpu::check(mtlg_ctx_residual_log(c.get(), nullptr, 0, &count), "residual log");
    std::vector<double> out;
    if (count > 0 && count <= c.residual_log_capacity()) {
        out.resize(std::size_t(2 * count));
        mtl::gpu::check(mtlg_ctx_residual_log(c.get(), out.data(), count, &count), "residual log");
    }
    return out;
}

template <class Iteration>
inline mtlg_iter_params params_of(const Iteration& iter, int restart = 0)
{
    mtlg_iter_params p;
    p.max_iter = iter.max_iterations();
    p.restart = restart;
    p.rtol = double(iter.tol());
    p.atol = double(iter.atol());
    p.norm_r0 = double(iter.norm_r0());
    return p;
}
}  // namespace gpu

namespace pc {

#ifndef ITL_PC_IDENTITY_INCLUDE
template <typename Matrix, typename Value = typename Matrix::value_type> class identity;
#endif
#ifndef ITL_PC_DIAGONAL_INCLUDE
template <typename Matrix, typename Value = typename Matrix::value_type> class diagonal;
#endif
#ifndef ITL_PC_ILU_0_INCLUDE
template <typename Matrix, typename Value = typename Matrix::value_type> class ilu_0;
#endif
#ifndef ITL_PC_IC_0_INCLUDE
template <typename Matrix, typename Value = typename Matrix::value_type> class ic_0;
#endif

namespace detail {
/// Device preconditioner of a given kind over a GPU matrix.
template <typename T, typename Value, int Kind>
class gpu_pc {
  public:
    typedef Value value_type;
    explicit gpu_pc(const mtl::gpu::compressed2D<T>& A) : ctx_(&A.ctx())
    {
        mtlg_pc* p = nullptr;
        mtl::gpu::check(mtlg_pc_create(A.ctx().get(), A.get(), Kind, mtl::gpu::dtype_of<Value>::value, &p), "pc");
        h_.reset(p, [](mtlg_pc* q) { mtlg_pc_destroy(q); });
    }
    mtlg_pc* get() const { return h_.get(); }
    mtl::gpu::context& ctx() const { return *ctx_; }
    template <typename V>
    mtl::gpu::dense_vector<V> solve(const mtl::gpu::dense_vector<V>& x) const
    {
        mtl::gpu::dense_vector<V> y(x.size(), x.ctx());
        mtl::gpu::check(mtlg_pc_apply(ctx_->get(), get(), x.get(), y.get()), "solve");
        return y;
    }
    template <typename V>
    mtl::gpu::dense_vector<V> adjoint_solve(const mtl::gpu::dense_vector<V>& x) const
    {
        mtl::gpu::dense_vector<V> y(x.size(), x.ctx());
        mtl::gpu::check(mtlg_pc_adjoint_apply(ctx_->get(), get(), x.get(), y.get()), "adjoint_solve");
        return y;
    }

  private:
    mtl::gpu::context* ctx_;
    std::shared_ptr<mtlg_pc> h_;
};
}  // namespace detail

template <typename T, typename Value>
class identity<mtl::gpu::compressed2D<T>, Value> : public detail::gpu_pc<T, Value, MTLG_PC_IDENTITY> {
  public:
    explicit identity(const mtl::gpu::compressed2D<T>& A) : detail::gpu_pc<T, Value, MTLG_PC_IDENTITY>(A) {}
};
template <typename T, typename Value>
class diagonal<mtl::gpu::compressed2D<T>, Value> : public detail::gpu_pc<T, Value, MTLG_PC_DIAGONAL> {
  public:
    explicit diagonal(const mtl::gpu::compressed2D<T>& A) : detail::gpu_pc<T, Value, MTLG_PC_DIAGONAL>(A) {}
};
template <typename T, typename Value>
class ilu_0<mtl::gpu::compressed2D<T>, Value> : public detail::gpu_pc<T, Value, MTLG_PC_ILU0> {
  public:
    explicit ilu_0(const mtl::gpu::compressed2D<T>& A) : detail::gpu_pc<T, Value, MTLG_PC_ILU0>(A) {}
};
template <typename T, typename Value>
class ic_0<mtl::gpu::compressed2D<T>, Value> : public detail::gpu_pc<T, Value, MTLG_PC_IC0> {
  public:
    explicit ic_0(const mtl::gpu::compressed2D<T>& A) : detail::gpu_pc<T, Value, MTLG_PC_IC0>(A) {}
};

template <typename T, typename Value, int Kind, typename V>
inline mtl::gpu::dense_vector<V> solve(const detail::gpu_pc<T, Value, Kind>& P, const mtl::gpu::dense_vector<V>& x)
{
    return P.solve(x);
}
template <typename T, typename Value, int Kind, typename V>
inline mtl::gpu::dense_vector<V> adjoint_solve(const detail::gpu_pc<T, Value, Kind>& P,
                                               const mtl::gpu::dense_vector<V>& x)
{
    return P.adjoint_solve(x);
}

}  // namespace pc

namespace gpu {
template <typename T, typename PC, typename Iteration>
inline int run(int solver, const mtl::gpu::compressed2D<T>& A, mtl::gpu::dense_vector<T>& x,
               const mtl::gpu::dense_vector<T>& b, const PC* L, const PC* R, Iteration& iter, int restart = 0)
{
    mtlg_iter_params p = params_of(iter, restart);
    mtlg_iter_result r;
    // BiCGSTAB tests twice per iteration: room for every test of the solve
    A.ctx().ensure_residual_log(2 * iter.max_iterations() + 8);
    const int s = mtlg_solve(A.ctx().get(), solver, A.get(), L ? L->get() : nullptr, R ? R->get() : nullptr,
                             x.get(), b.get(), &p, &r);
    const std::vector<double> log = residual_log(A.ctx());
    take_result(iter, r, &log);
    mtl::gpu::check(s, solver == MTLG_CG ? "cg" : solver == MTLG_BICGSTAB ? "bicgstab" : "gmres");
    return iter.error_code();
}
}  // namespace gpu

/// Conjugate gradients (itl/krylov/cg.hpp:76-111).
template <typename T, typename Preconditioner, typename Iteration>
inline int cg(const mtl::gpu::compressed2D<T>& A, mtl::gpu::dense_vector<T>& x, const mtl::gpu::dense_vector<T>& b,
              const Preconditioner& L, Iteration& iter)
{
    return gpu::run(MTLG_CG, A, x, b, &L, static_cast<const Preconditioner*>(nullptr), iter);
}

/// BiCGSTAB (itl/krylov/bicgstab.hpp:29-77); breakdown throws
/// itl::gpu::unexpected_orthogonality.
template <typename T, typename Preconditioner, typename Iteration>
inline int bicgstab(const mtl::gpu::compressed2D<T>& A, mtl::gpu::dense_vector<T>& x,
                    const mtl::gpu::dense_vector<T>& b, const Preconditioner& L, Iteration& iter)
{
    return gpu::run(MTLG_BICGSTAB, A, x, b, &L, static_cast<const Preconditioner*>(nullptr), iter);
}

/// Restarted GMRES (itl/krylov/gmres.hpp:124-137).
template <typename T, typename Left, typename Right, typename Iteration>
inline int gmres(const mtl::gpu::compressed2D<T>& A, mtl::gpu::dense_vector<T>& x, const mtl::gpu::dense_vector<T>& b,
                 Left& L, Right& R, Iteration& iter, std::size_t restart)
{
    mtlg_iter_params p = gpu::params_of(iter, int(restart));
    mtlg_iter_result r;
    const int s = mtlg_solve(A.ctx().get(), MTLG_GMRES, A.get(), L.get(), R.get(), x.get(), b.get(), &p, &r);
    gpu::take_result(iter, r);
    mtl::gpu::check(s, "gmres");
    return iter.error_code();
}

/// The reference's other Krylov bodies (itl/krylov/*.hpp), host-driven on
/// device vectors (FP64): bicg, cgs and bicgstab_2 with one preconditioner,
/// tfqmr and qmr with left and right ones, bicgstab_ell and idr_s with both
/// and their ell / s.
namespace gpu {
template <typename T, typename Left, typename Right, typename Iteration>
inline int run2(int solver, const mtl::gpu::compressed2D<T>& A, mtl::gpu::dense_vector<T>& x,
                const mtl::gpu::dense_vector<T>& b, const Left* L, const Right* R, Iteration& iter, int param = 0)
{
    mtlg_iter_params p = params_of(iter, param);
    mtlg_iter_result r;
    const int s = mtlg_solve(A.ctx().get(), solver, A.get(), L ? L->get() : nullptr, R ? R->get() : nullptr, x.get(),
                             b.get(), &p, &r);
    take_result(iter, r);
    mtl::gpu::check(s, "krylov");
    return iter.error_code();
}
}  // namespace gpu

template <typename T, typename PC, typename Iteration>
inline int bicg(const mtl::gpu::compressed2D<T>& A, mtl::gpu::dense_vector<T>& x, const mtl::gpu::dense_vector<T>& b,
                const PC& M, Iteration& iter)
{
    return gpu::run2(MTLG_BICG, A, x, b, &M, static_cast<const PC*>(nullptr), iter);
}
template <typename T, typename PC, typename Iteration>
inline int cgs(const mtl::gpu::compressed2D<T>& A, mtl::gpu::dense_vector<T>& x, const mtl::gpu::dense_vector<T>& b,
               const PC& M, Iteration& iter)
{
    return gpu::run2(MTLG_CGS, A, x, b, &M, static_cast<const PC*>(nullptr), iter);
}
template <typename T, typename PC, typename Iteration>
inline int bicgstab_2(const mtl::gpu::compressed2D<T>& A, mtl::gpu::dense_vector<T>& x,
                      const mtl::gpu::dense_vector<T>& b, const PC& L, Iteration& iter)
{
    return gpu::run2(MTLG_BICGSTAB_2, A, x, b, &L, static_cast<const PC*>(nullptr), iter);
}
template <typename T, typename Left, typename Right, typename Iteration>
inline int tfqmr(const mtl::gpu::compressed2D<T>& A, mtl::gpu::dense_vector<T>& x, const mtl::gpu::dense_vector<T>& b,
                 const Left& L, const Right& R, Iteration& iter)
{
    return gpu::run2(MTLG_TFQMR, A, x, b, &L, &R, iter);
}
template <typename T, typename Left, typename Right, typename Iteration>
inline int qmr(const mtl::gpu::compressed2D<T>& A, mtl::gpu::dense_vector<T>& x, const mtl::gpu::dense_vector<T>& b,
               Left& L, const Right& R, Iteration& iter)
{
    return gpu::run2(MTLG_QMR, A, x, b, &L, &R, iter);
}
template <typename T, typename Left, typename Right, typename Iteration>
inline int bicgstab_ell(const mtl::gpu::compressed2D<T>& A, mtl::gpu::dense_vector<T>& x,
                        const mtl::gpu::dense_vector<T>& b, const Left& L, const Right& R, Iteration& iter,
                        std::size_t l)
{
    return gpu::run2(MTLG_BICGSTAB_ELL, A, x, b, &L, &R, iter, int(l));
}
template <typename T, typename Left, typename Right, typename Iteration>
inline int idr_s(const mtl::gpu::compressed2D<T>& A, mtl::gpu::dense_vector<T>& x, const mtl::gpu::dense_vector<T>& b,
                 const Left& L, const Right& R, Iteration& iter, std::size_t s)
{
    return gpu::run2(MTLG_IDR_S, A, x, b, &L, &R, iter, int(s));
}

/// FP64 iterative refinement around an FP32 inner CG / BiCGSTAB (no
/// reference counterpart): x, b FP64; P an FP32-stored preconditioner of A.
template <typename PC>
inline mtlg_iter_result refine(int solver, const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
                               const mtl::gpu::dense_vector<double>& b, const PC& P, double rtol = 1e-8,
                               double inner_rtol = 1e-4, int max_outer = 20, int max_inner = 2000)
{
    mtlg_refine_params rp;
    rp.max_outer = max_outer;
    rp.max_inner = max_inner;
    rp.restart = 0;
    rp.pad = 0;
    rp.rtol = rtol;
    rp.inner_rtol = inner_rtol;
    mtlg_iter_result r;
    mtl::gpu::check(mtlg_refine_solve(A.ctx().get(), solver, A.get(), P.get(), x.get(), b.get(), &rp, &r), "refine");
    return r;
}
template <typename PC>
inline mtlg_iter_result refine_cg(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
                                  const mtl::gpu::dense_vector<double>& b, const PC& P, double rtol = 1e-8)
{
    return refine(MTLG_CG, A, x, b, P, rtol);
}
template <typename PC>
inline mtlg_iter_result refine_bicgstab(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
                                        const mtl::gpu::dense_vector<double>& b, const PC& P, double rtol = 1e-8)
{
    return refine(MTLG_BICGSTAB, A, x, b, P, rtol);
}

}  // namespace itl

#endif  // MTL4_B200_ITL_GPU_HPP
