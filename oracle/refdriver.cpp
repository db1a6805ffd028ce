// Test infrastructure only: a C-ABI driver around the UNCHANGED MTL4 headers
// (compiled from the reference tree by oracle/Makefile, output in oracle/_ref/).
// It is the checker for the GPU library and the timed CPU baseline; nothing in
// the product links or calls it.
//
// Entry points wrap raw CSR arrays into mtl::compressed2D through the
// raw-array constructor (boost/numeric/mtl/matrix/compressed2D.hpp:355-364)
// and run the reference's own kernels and solvers:
//   SpMV      w = A*v, w += A*v, w -= A*v  (operation/mat_vec_mult.hpp:614-683)
//   dot       (operation/dot.hpp:228)
//   PCs       itl::pc::diagonal / ilu_0 / ic_0 / identity  (itl/pc/*.hpp)
//   solvers   itl::cg (itl/krylov/cg.hpp:76), itl::bicgstab
//             (itl/krylov/bicgstab.hpp:29), itl::gmres (itl/krylov/gmres.hpp:124)
//   iteration itl::basic_iteration<double>(b, max_iter, rtol, atol)
//             (itl/iteration/basic_iteration.hpp:32-34), norm_r0 = ||b||.
// The mixed-precision refinement loop is not in the reference; it is stated
// here around the reference's FP32 inner solvers so the GPU's refinement has
// a reference-built checker.
#include <boost/numeric/mtl/mtl.hpp>
#include <boost/numeric/mtl/io/matrix_market.hpp>
#include <boost/numeric/itl/itl.hpp>
#include <boost/numeric/mtl/matrix/poisson2D_dirichlet.hpp>

#include <chrono>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <memory>
#include <sstream>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef mtl::mat::parameters<mtl::row_major, mtl::index::c_index, mtl::non_fixed::dimensions, false, std::size_t> para_t;
typedef mtl::compressed2D<double, para_t> dmat;
typedef mtl::compressed2D<float, para_t> fmat;
typedef mtl::dense_vector<double> dvec;
typedef mtl::dense_vector<float> fvec;

typedef mtl::mat::ell_matrix<double> dell;
typedef mtl::mat::sparse_banded<double> dband;

struct RefCsr {
    std::unique_ptr<dmat> A;
    std::unique_ptr<fmat> Af;   // lazily built FP32 copy (values rounded once)
    std::unique_ptr<dell> E;    // lazily built ELL copy (E = A)
    std::unique_ptr<dband> S;   // lazily built sparse_banded copy (S = A)
    std::size_t n_rows = 0, n_cols = 0, nnz = 0;
};

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename T>
std::unique_ptr<mtl::compressed2D<T, para_t> >
make_matrix(std::size_t m, std::size_t n, std::size_t nnz, const int64_t* rp, const int32_t* ci, const T* v)
{
    std::vector<std::size_t> major(rp, rp + m + 1), minor(ci, ci + nnz);
    std::vector<T> entries(v, v + nnz);
    return std::unique_ptr<mtl::compressed2D<T, para_t> >(
        new mtl::compressed2D<T, para_t>(m, n, nnz, major.data(), minor.data(), entries.data()));
}

fmat& fp32_copy(RefCsr* h)
{
    if (!h->Af) {
        std::vector<float> vf(h->nnz);
        const double* d = h->A->address_data();
        for (std::size_t k = 0; k < h->nnz; ++k) vf[k] = float(d[k]);
        std::vector<int64_t> rp(h->n_rows + 1);
        std::vector<int32_t> ci(h->nnz);
        for (std::size_t i = 0; i <= h->n_rows; ++i) rp[i] = int64_t(h->A->address_major()[i]);
        for (std::size_t k = 0; k < h->nnz; ++k) ci[k] = int32_t(h->A->address_minor()[k]);
        h->Af = make_matrix<float>(h->n_rows, h->n_cols, h->nnz, rp.data(), ci.data(), vf.data());
    }
    return *h->Af;
}

template <typename Mat, typename Vec>
void spmv_impl(const Mat& A, const Vec& v, Vec& w, int assign)
{
    if (assign == 0) w = A * v;
    else if (assign == 1) w += A * v;
    else w -= A * v;
}

template <typename M>
void export_csr(const M& L, int64_t* nnz, int64_t* rp, int32_t* ci, double* val)
{
    std::size_t m = num_rows(L), z = L.nnz();
    if (nnz) *nnz = int64_t(z);
    if (rp) for (std::size_t i = 0; i <= m; ++i) rp[i] = int64_t(L.address_major()[i]);
    if (ci) for (std::size_t k = 0; k < z; ++k) ci[k] = int32_t(L.address_minor()[k]);
    if (val) for (std::size_t k = 0; k < z; ++k) val[k] = double(L.address_data()[k]);
}

} // namespace

extern "C" {

struct mtlref_result {
    int iterations;
    int error;
    double resid;
    double relresid;
    double setup_s;
    double solve_s;
    int outer_iterations;   // refinement steps (refine_solve only)
    int pad;
};

void* mtlref_csr_create(int64_t n_rows, int64_t n_cols, int64_t nnz, const int64_t* row_ptr, const int32_t* col,
                        const double* val)
{
    RefCsr* h = new RefCsr;
    h->n_rows = std::size_t(n_rows); h->n_cols = std::size_t(n_cols); h->nnz = std::size_t(nnz);
    h->A = make_matrix<double>(h->n_rows, h->n_cols, h->nnz, row_ptr, col, val);
    return h;
}

void mtlref_csr_destroy(void* p) { delete static_cast<RefCsr*>(p); }

int mtlref_openmp_threads()
{
#ifdef MTL_WITH_OPENMP
    int t = 1;
#   pragma omp parallel
    {
#       pragma omp master
        t = omp_get_num_threads();
    }
    return t;
#else
    return 1;
#endif
}

/// w (=|+=|-=) A*v in FP64; assign 0: '=', 1: '+=', 2: '-='.
int mtlref_spmv(void* p, const double* x, double* y, int assign)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    dvec v(h->n_cols, const_cast<double*>(x)), w(h->n_rows, y);
    spmv_impl(*h->A, v, w, assign);
    return 0;
}

/// Same on the FP32 copy of the matrix with FP32 vectors.
int mtlref_spmv_f32(void* p, const float* x, float* y, int assign)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    fmat& Af = fp32_copy(h);
    fvec v(h->n_cols, const_cast<float*>(x)), w(h->n_rows, y);
    spmv_impl(Af, v, w, assign);
    return 0;
}

/// Repeated SpMV for the CPU baseline; returns seconds for `reps` products.
double mtlref_spmv_timed(void* p, const double* x, double* y, int reps)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    dvec v(h->n_cols, const_cast<double*>(x)), w(h->n_rows, y);
    double t0 = now_s();
    for (int r = 0; r < reps; ++r) w = (*h->A) * v;
    return now_s() - t0;
}

double mtlref_dot(int64_t n, const double* a, const double* b)
{
    dvec va(std::size_t(n), const_cast<double*>(a)), vb(std::size_t(n), const_cast<double*>(b));
    return mtl::dot(va, vb);
}

double mtlref_two_norm(int64_t n, const double* a)
{
    dvec va(std::size_t(n), const_cast<double*>(a));
    return mtl::two_norm(va);
}

// A = mtl::io::matrix_market(path) through matrix_market_istream >> A
// (io/matrix_market.hpp:44-214) into compressed2D<double>; the CSR arrays
// out (call with null arrays for the sizes).  Returns 0, 1 when the
// reference throws file_not_found, 2 for any other exception.
int mtlref_mm_read(const char* path, int64_t* n_rows, int64_t* n_cols, int64_t* nnz, int64_t* rp, int32_t* ci,
                   double* val)
{
    try {
        dmat A;
        mtl::io::matrix_market_istream ms(path);
        ms >> A;
        *n_rows = int64_t(num_rows(A));
        *n_cols = int64_t(num_cols(A));
        *nnz = int64_t(A.nnz());
        if (rp)
            for (std::size_t i = 0; i <= num_rows(A); ++i) rp[i] = int64_t(A.address_major()[i]);
        if (ci)
            for (std::size_t k = 0; k < A.nnz(); ++k) ci[k] = int32_t(A.address_minor()[k]);
        if (val)
            for (std::size_t k = 0; k < A.nnz(); ++k) val[k] = A.address_data()[k];
        return 0;
    } catch (const mtl::file_not_found&) {
        return 1;
    } catch (const std::exception& e) {
        fprintf(stderr, "mtlref_mm_read(%s): %s\n", path, e.what());
        return 2;
    } catch (...) {
        return 2;
    }
}

} // extern "C"

// pc kinds: 0 identity, 1 diagonal, 2 ilu_0, 3 ic_0.  pc_f32 selects the
// preconditioner's Value type (float) as in pc::ic_0<Matrix, float>.  The
// reference's free solve(P, x) exists only for pc::diagonal<Matrix> with the
// matrix's own value type (itl/pc/diagonal.hpp:85-90), so a diagonal PC
// always stores the matrix's precision.
template <typename PC, typename Vec>
static void apply_pc(const PC& P, const Vec& x, Vec& y) { y = solve(P, x); }

extern "C" {

int mtlref_pc_apply(void* p, int kind, int pc_f32, const double* x, double* y)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    const dmat& A = *h->A;
    dvec vx(h->n_rows, const_cast<double*>(x)), vy(h->n_rows, y);
    switch (kind * 2 + (pc_f32 ? 1 : 0)) {
    case 0: case 1: { itl::pc::identity<dmat> P(A); apply_pc(P, vx, vy); break; }
    case 2: { itl::pc::diagonal<dmat> P(A); apply_pc(P, vx, vy); break; }
    case 3: { itl::pc::diagonal<dmat> P(A); apply_pc(P, vx, vy); break; }
    case 4: { itl::pc::ilu_0<dmat> P(A); apply_pc(P, vx, vy); break; }
    case 5: { itl::pc::ilu_0<dmat, float> P(A); apply_pc(P, vx, vy); break; }
    case 6: { itl::pc::ic_0<dmat> P(A); apply_pc(P, vx, vy); break; }
    case 7: { itl::pc::ic_0<dmat, float> P(A); apply_pc(P, vx, vy); break; }
    default: return -1;
    }
    return 0;
}

/// y = adjoint_solve(P, x) of pc::ilu_0<M> / pc::ilu_0<M, float>
/// (itl/pc/ilu.hpp:94-115): U^H then L^H through the transposed views.
int mtlref_pc_adjoint_apply(void* p, int kind, int pc_f32, const double* x, double* y)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    const dmat& A = *h->A;
    dvec vx(h->n_rows, const_cast<double*>(x)), vy(h->n_rows, y);
    if (kind != 2) return -1;
    if (pc_f32) { itl::pc::ilu_0<dmat, float> P(A); vy = adjoint_solve(P, vx); }
    else { itl::pc::ilu_0<dmat> P(A); vy = adjoint_solve(P, vx); }
    return 0;
}

/// FP32 vectors through a preconditioner factorized from the FP64 matrix
/// and stored in FP32 (pc::ilu_0<M,float> / pc::ic_0<M,float>).
int mtlref_pc_apply_f32(void* p, int kind, const float* x, float* y)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    const dmat& A = *h->A;
    fvec vx(h->n_rows, const_cast<float*>(x)), vy(h->n_rows, y);
    switch (kind) {
    case 0: { itl::pc::identity<dmat> P(A); apply_pc(P, vx, vy); break; }
    case 1: { itl::pc::diagonal<fmat> P(fp32_copy(h)); apply_pc(P, vx, vy); break; }
    case 2: { itl::pc::ilu_0<dmat, float> P(A); apply_pc(P, vx, vy); break; }
    case 3: { itl::pc::ic_0<dmat, float> P(A); apply_pc(P, vx, vy); break; }
    default: return -1;
    }
    return 0;
}

/// Factor export (FP64 factorization, values as stored): ILU(0) -> L (strict
/// lower, unit diagonal implied) and U (upper, diagonal inverted first in
/// each row); IC(0) -> U (diagonal stored as 1/sqrt, first in each row) and
/// L = trans(U).  Pass null arrays to query the nnz counts first.
int mtlref_pc_factors(void* p, int kind, int64_t* nnzL, int64_t* L_rp, int32_t* L_ci, double* L_v,
                      int64_t* nnzU, int64_t* U_rp, int32_t* U_ci, double* U_v)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    const dmat& A = *h->A;
    if (kind == 2) {
        itl::pc::ilu_0<dmat> P(A);
        export_csr(P.get_L(), nnzL, L_rp, L_ci, L_v);
        export_csr(P.get_U(), nnzU, U_rp, U_ci, U_v);
    } else if (kind == 3) {
        itl::pc::ic_0<dmat> P(A);
        export_csr(P.get_L(), nnzL, L_rp, L_ci, L_v);
        export_csr(P.get_U(), nnzU, U_rp, U_ci, U_v);
    } else {
        return -1;
    }
    return 0;
}

} // extern "C"

template <typename Mat, typename Vec, typename PC>
static int run_solver(int solver, const Mat& A, Vec& x, const Vec& b, const PC& P, itl::basic_iteration<double>& iter,
                      int restart)
{
    if (solver == 0) return itl::cg(A, x, b, P, iter);
    if (solver == 1) return itl::bicgstab(A, x, b, P, iter);
    itl::pc::identity<Mat> R(A);
    PC& Pm = const_cast<PC&>(P);
    typedef typename mtl::Collection<Vec>::value_type T;
    if constexpr (std::is_same<T, double>::value) {
        return itl::gmres(A, x, b, Pm, R, iter, std::size_t(restart));
    } else {
        // gmres_full passes its scalar type to iter.finished(), so an FP32
        // GMRES needs basic_iteration<float> (itl/krylov/gmres.hpp:57).
        itl::basic_iteration<T> it(T(iter.norm_r0()), iter.max_iterations(), T(iter.tol()), T(iter.atol()));
        itl::gmres(A, x, b, Pm, R, it, std::size_t(restart));
        iter += it.iterations();
        iter.finished(double(it.resid()));
        if (it.error_code() > 1) iter.fail(it.error_code());
        return iter.error_code();
    }
}

template <typename Mat, typename Vec, typename Factor>
static int solve_typed(int solver, int kind, int pc_f32, const Mat& A, const Factor& Afac, Vec& x, const Vec& b,
                       itl::basic_iteration<double>& iter, int restart, double& setup_s)
{
    typedef typename mtl::Collection<Vec>::value_type T;
    double t0 = now_s();
    switch (kind * 2 + (pc_f32 ? 1 : 0)) {
    case 0: case 1: { itl::pc::identity<Mat> P(A); setup_s = now_s() - t0; return run_solver(solver, A, x, b, P, iter, restart); }
    case 2: case 3: { itl::pc::diagonal<Mat> P(A); setup_s = now_s() - t0; return run_solver(solver, A, x, b, P, iter, restart); }
    case 4: { itl::pc::ilu_0<Factor, T> P(Afac); setup_s = now_s() - t0; return run_solver(solver, A, x, b, P, iter, restart); }
    case 5: { itl::pc::ilu_0<Factor, float> P(Afac); setup_s = now_s() - t0; return run_solver(solver, A, x, b, P, iter, restart); }
    case 6: { itl::pc::ic_0<Factor, T> P(Afac); setup_s = now_s() - t0; return run_solver(solver, A, x, b, P, iter, restart); }
    case 7: { itl::pc::ic_0<Factor, float> P(Afac); setup_s = now_s() - t0; return run_solver(solver, A, x, b, P, iter, restart); }
    default: return -1;
    }
}

template <typename PC>
static int run_krylov(int solver, const dmat& A, dvec& x, const dvec& b, const PC& P, itl::basic_iteration<double>& iter,
                      int param)
{
    itl::pc::identity<dmat> I(A);
    PC& Pm = const_cast<PC&>(P);
    switch (solver) {
    case 3: return itl::bicg(A, x, b, P, iter);
    case 4: return itl::cgs(A, x, b, P, iter);
    case 5: return itl::tfqmr(A, x, b, P, I, iter);
    case 6: return itl::qmr(A, x, b, Pm, I, iter);
    case 7: return itl::bicgstab_2(A, x, b, P, iter);
    case 8: return itl::bicgstab_ell(A, x, b, P, I, iter, std::size_t(param > 0 ? param : 2));
    case 9: return itl::idr_s(A, x, b, P, I, iter, std::size_t(param > 0 ? param : 4));
    default: return -1;
    }
}

template <typename PC>
static int run_cyclic(int solver, const dmat& A, dvec& x, const dvec& b, const PC& P,
                      itl::cyclic_iteration<double>& iter)
{
    if (solver == 0) return itl::cg(A, x, b, P, iter);
    return itl::bicgstab(A, x, b, P, iter);
}

extern "C" {

static dell& ell_copy(RefCsr* h)
{
    if (!h->E) {
        h->E.reset(new dell(h->n_rows, h->n_cols));
        *h->E = *h->A;
    }
    return *h->E;
}

static dband& band_copy(RefCsr* h)
{
    if (!h->S) {
        h->S.reset(new dband(h->n_rows, h->n_cols));
        *h->S = *h->A;
    }
    return *h->S;
}

/// The ELL form of A as MTL4 builds it (ell_matrix = compressed2D,
/// matrix/ell_matrix.hpp:127-170): entry j of row i at k = i + j * stride,
/// stride = n_rows rounded up to 32, slots = longest row; padding repeats the
/// row's last column with value 0.  Null arrays: sizes only.
void mtlref_ell_export(void* p, int64_t* stride, int64_t* slots, int64_t* minor, double* data)
{
    dell& E = ell_copy(static_cast<RefCsr*>(p));
    *stride = int64_t(E.stride());
    *slots = int64_t(E.slots());
    const std::size_t m = E.stride() * E.slots();
    if (minor)
        for (std::size_t k = 0; k < m; ++k) minor[k] = int64_t(E.ref_minor()[k]);
    if (data)
        for (std::size_t k = 0; k < m; ++k) data[k] = E.ref_data()[k];
}

/// w (=|+=|-=) E * v (operation/mat_vec_mult.hpp:686-700)
void mtlref_ell_spmv(void* p, const double* x, double* y, int assign)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    dvec vx(h->n_cols, const_cast<double*>(x)), vy(h->n_rows, y);
    spmv_impl(ell_copy(h), vx, vy, assign);
}

/// The sparse_banded form of A (sparse_banded = compressed2D,
/// matrix/sparse_banded.hpp:168-260): the diagonal offsets in increasing
/// order and the values row by row, one per band (0 outside the matrix).
void mtlref_banded_export(void* p, int64_t* nb, int64_t* bands, double* data)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    dband& S = band_copy(h);
    *nb = int64_t(S.ref_bands().size());
    if (bands)
        for (std::size_t b = 0; b < S.ref_bands().size(); ++b) bands[b] = int64_t(S.ref_bands()[b]);
    if (data)
        for (std::size_t k = 0; k < h->n_rows * S.ref_bands().size(); ++k) data[k] = S.ref_data()[k];
}

/// w (=|+=|-=) S * v (operation/mat_vec_mult.hpp:704-803)
void mtlref_banded_spmv(void* p, const double* x, double* y, int assign)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    dvec vx(h->n_cols, const_cast<double*>(x)), vy(h->n_rows, y);
    spmv_impl(band_copy(h), vx, vy, assign);
}

/// FP64 bicg (3), cgs (4), tfqmr (5), qmr (6), bicgstab_2 (7),
/// bicgstab_ell (8, ell = param), idr_s (9, s = param) with a left
/// preconditioner of `kind` (right: identity), basic_iteration from b.
int mtlref_solve_krylov(void* p, int solver, int kind, const double* b, double* x, int max_iter, double rtol, int param,
                        mtlref_result* out)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    dvec vb(h->n_rows, const_cast<double*>(b)), vx(h->n_rows, x);
    itl::basic_iteration<double> iter(vb, max_iter, rtol);
    int err = -1;
    try {
        const dmat& A = *h->A;
        if (kind == 0) { itl::pc::identity<dmat> P(A); err = run_krylov(solver, A, vx, vb, P, iter, param); }
        else if (kind == 1) { itl::pc::diagonal<dmat> P(A); err = run_krylov(solver, A, vx, vb, P, iter, param); }
        else if (kind == 2) { itl::pc::ilu_0<dmat> P(A); err = run_krylov(solver, A, vx, vb, P, iter, param); }
        else if (kind == 3) { itl::pc::ic_0<dmat> P(A); err = run_krylov(solver, A, vx, vb, P, iter, param); }
    } catch (const itl::unexpected_orthogonality&) {
        err = -2;
    }
    if (out) {
        out->iterations = iter.iterations(); out->error = err; out->resid = iter.resid();
        out->relresid = iter.relresid(); out->setup_s = 0; out->solve_s = 0;
        out->outer_iterations = 0; out->pad = 0;
    }
    return err;
}

/// poisson2D_dirichlet(m, n) times x (matrix/poisson2D_dirichlet.hpp), and a
/// CG solve on it without preconditioning (the tutorial's use).
void mtlref_poisson2d_mult(int m, int n, const double* x, double* y, int assign)
{
    mtl::mat::poisson2D_dirichlet A(m, n);
    dvec vx(std::size_t(m) * n, const_cast<double*>(x)), vy(std::size_t(m) * n, y);
    if (assign == 0) vy = A * vx;
    else if (assign == 1) vy += A * vx;
    else vy -= A * vx;
}

int mtlref_poisson2d_cg(int m, int n, const double* b, double* x, int max_iter, double rtol, mtlref_result* out)
{
    mtl::mat::poisson2D_dirichlet A(m, n);
    dvec vb(std::size_t(m) * n, const_cast<double*>(b)), vx(std::size_t(m) * n, x);
    itl::basic_iteration<double> iter(vb, max_iter, rtol);
    itl::pc::identity<mtl::mat::poisson2D_dirichlet> P(A);
    const int err = itl::cg(A, vx, vb, P, iter);
    if (out) {
        out->iterations = iter.iterations(); out->error = err; out->resid = iter.resid();
        out->relresid = iter.relresid(); out->setup_s = 0; out->solve_s = 0;
        out->outer_iterations = 0; out->pad = 0;
    }
    return err;
}

/// FP64 CG (solver 0) or BiCGSTAB (1) with itl::cyclic_iteration<double>
/// (itl/iteration/cyclic_iteration.hpp:22-95) printing into a string: the
/// per-cycle residual lines and the final summary that the solver's return
/// (iter converted to int, error_code()) prints.  text receives at most cap
/// bytes (NUL-terminated); needed gets the full length + 1.
int mtlref_solve_cyclic(void* p, int solver, int kind, const double* b, double* x, int max_iter, double rtol,
                        int cycle, int multi_print, char* text, size_t cap, size_t* needed)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    dvec vb(h->n_rows, const_cast<double*>(b)), vx(h->n_rows, x);
    std::ostringstream os;
    itl::cyclic_iteration<double> iter(vb, max_iter, rtol, 0.0, cycle, os);
    iter.set_multi_print(multi_print != 0);
    int err = -1;
    try {
        const dmat& A = *h->A;
        if (kind == 0) { itl::pc::identity<dmat> P(A); err = run_cyclic(solver, A, vx, vb, P, iter); }
        else if (kind == 1) { itl::pc::diagonal<dmat> P(A); err = run_cyclic(solver, A, vx, vb, P, iter); }
        else if (kind == 2) { itl::pc::ilu_0<dmat> P(A); err = run_cyclic(solver, A, vx, vb, P, iter); }
        else if (kind == 3) { itl::pc::ic_0<dmat> P(A); err = run_cyclic(solver, A, vx, vb, P, iter); }
    } catch (const itl::unexpected_orthogonality&) {
        err = -2;
    }
    const std::string t = os.str();
    if (needed) *needed = t.size() + 1;
    if (text && cap) {
        const size_t k = std::min(cap - 1, t.size());
        std::memcpy(text, t.data(), k);
        text[k] = 0;
    }
    return err;
}

/// FP64 solve: solver 0 cg, 1 bicgstab, 2 gmres(restart) with right PC = identity.
/// x is in/out (initial guess on entry).  BiCGSTAB breakdown
/// (itl::unexpected_orthogonality) is reported as error -2.
int mtlref_solve(void* p, int solver, int kind, int pc_f32, const double* b, double* x, int max_iter, double rtol,
                 double atol, int restart, mtlref_result* out)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    dvec vb(h->n_rows, const_cast<double*>(b)), vx(h->n_rows, x);
    itl::basic_iteration<double> iter(vb, max_iter, rtol, atol);
    double setup_s = 0, t0 = now_s();
    int err;
    try {
        err = solve_typed(solver, kind, pc_f32, *h->A, *h->A, vx, vb, iter, restart, setup_s);
    } catch (const itl::unexpected_orthogonality&) {
        err = -2;
    }
    double total = now_s() - t0;
    if (out) {
        out->iterations = iter.iterations(); out->error = err; out->resid = iter.resid();
        out->relresid = iter.relresid(); out->setup_s = setup_s; out->solve_s = total - setup_s;
        out->outer_iterations = 0; out->pad = 0;
    }
    return err;
}

/// FP32 solve on the FP32 copy of A with FP32 vectors; the preconditioner is
/// factorized from the FP64 matrix and stored in FP32.
int mtlref_solve_f32(void* p, int solver, int kind, const float* b, float* x, int max_iter, double rtol, double atol,
                     int restart, mtlref_result* out)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    fmat& Af = fp32_copy(h);
    fvec vb(h->n_rows, const_cast<float*>(b)), vx(h->n_rows, x);
    itl::basic_iteration<double> iter(vb, max_iter, rtol, atol);
    double setup_s = 0, t0 = now_s();
    int err;
    try {
        err = solve_typed(solver, kind, 1, Af, *h->A, vx, vb, iter, restart, setup_s);
    } catch (const itl::unexpected_orthogonality&) {
        err = -2;
    }
    double total = now_s() - t0;
    if (out) {
        out->iterations = iter.iterations(); out->error = err; out->resid = iter.resid();
        out->relresid = iter.relresid(); out->setup_s = setup_s; out->solve_s = total - setup_s;
        out->outer_iterations = 0; out->pad = 0;
    }
    return err;
}

/// FP64 iterative refinement around the reference's FP32 inner solver:
///   r = b - A x (FP64);  stop when ||r|| <= rtol * ||b||;
///   solve A_f32 d = float(r / ||r||) to inner_rtol;  x += ||r|| * d (FP64).
/// The preconditioner is built once (FP64 factorization, FP32 storage).
int mtlref_refine_solve(void* p, int solver, int kind, const double* b, double* x, int max_outer, int max_inner,
                        double rtol, double inner_rtol, int restart, mtlref_result* out)
{
    RefCsr* h = static_cast<RefCsr*>(p);
    const dmat& A = *h->A;
    fmat& Af = fp32_copy(h);
    std::size_t n = h->n_rows;
    dvec vb(n, const_cast<double*>(b)), vx(n, x), r(n);
    fvec rf(n), df(n);
    double nb = mtl::two_norm(vb), t0 = now_s(), setup_s = 0, relres = 0, rn = 0;
    int inner_total = 0, outer = 0, err = 1;

    auto body = [&](auto& P) {
        for (outer = 0; outer <= max_outer; ++outer) {
            r = vb - A * vx;
            rn = mtl::two_norm(r);
            relres = nb > 0 ? rn / nb : rn;
            if (rn <= rtol * nb) { err = 0; break; }
            if (outer == max_outer) break;
            for (std::size_t i = 0; i < n; ++i) rf[i] = float(r[i] / rn);
            df = 0.0f;
            itl::basic_iteration<double> it(rf, max_inner, inner_rtol, 0.0);
            try {
                run_solver(solver, Af, df, rf, P, it, restart);
            } catch (const itl::unexpected_orthogonality&) {}
            inner_total += it.iterations();
            for (std::size_t i = 0; i < n; ++i) vx[i] += rn * double(df[i]);
        }
    };
    double s0 = now_s();
    if (kind == 0) { itl::pc::identity<fmat> P(Af); setup_s = now_s() - s0; body(P); }
    else if (kind == 1) { itl::pc::diagonal<fmat> P(Af); setup_s = now_s() - s0; body(P); }
    else if (kind == 2) { itl::pc::ilu_0<dmat, float> P(A); setup_s = now_s() - s0; body(P); }
    else if (kind == 3) { itl::pc::ic_0<dmat, float> P(A); setup_s = now_s() - s0; body(P); }
    else return -1;
    double total = now_s() - t0;
    if (out) {
        out->iterations = inner_total; out->error = err; out->resid = rn; out->relresid = relres;
        out->setup_s = setup_s; out->solve_s = total - setup_s; out->outer_iterations = outer; out->pad = 0;
    }
    return err;
}

/// Reference 2D Laplacian (matrix/laplacian_setup.hpp:26-41) exported as CSR,
/// so generated stencils can be checked against the reference's own setup.
int mtlref_laplacian_setup(int m, int n, int64_t* nnz, int64_t* rp, int32_t* ci, double* val)
{
    dmat A(std::size_t(m) * n, std::size_t(m) * n);
    mtl::mat::laplacian_setup(A, unsigned(m), unsigned(n));
    export_csr(A, nnz, rp, ci, val);
    return 0;
}

} // extern "C"
