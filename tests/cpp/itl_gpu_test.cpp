// Reference-style use of the C++ front end: the solver calls read as they do
// against MTL4 (itl::cg(A, x, b, P, iter) with itl::basic_iteration<double>),
// only the matrix and vector types are the GPU ones.  Exit code 0 = pass.
#include <cmath>
#include <cstdio>
#include <sstream>
#include <string>
#include <vector>

#include "mtl4_b200/itl_gpu.hpp"

static double relres(const mtl::gpu::compressed2D<double>& A, const mtl::gpu::dense_vector<double>& x,
                     const mtl::gpu::dense_vector<double>& b)
{
    mtl::gpu::dense_vector<double> r(b.size());
    r = A * x;
    std::vector<double> rh = r.to_host(), bh = b.to_host();
    double num = 0, den = 0;
    for (size_t i = 0; i < rh.size(); ++i) { num += (bh[i] - rh[i]) * (bh[i] - rh[i]); den += bh[i] * bh[i]; }
    return std::sqrt(num / den);
}

#define REQUIRE(c, msg)                                  \
    do {                                                 \
        if (!(c)) { std::printf("FAIL: %s\n", msg); return 1; } \
    } while (0)

int main()
{
    typedef mtl::gpu::compressed2D<double> matrix_type;
    const unsigned m = 64;
    matrix_type A = mtl::gpu::laplacian_setup<double>(m, m);
    const std::size_t N = A.num_rows();
    std::vector<double> xt(N);
    for (std::size_t i = 0; i < N; ++i) xt[i] = std::sin(0.1 * double(i));
    mtl::gpu::dense_vector<double> x_true(xt), b(N), x(N);
    b = A * x_true;

    // the KAT of libs/numeric/mtl/test/matrix_vector_product_test.cpp on a 5x5 grid
    {
        matrix_type L5 = mtl::gpu::laplacian_setup<double>(5, 5);
        std::vector<double> col12(25, 0.0);
        col12[12] = 4; col12[7] = col12[11] = col12[13] = col12[17] = -1;
        mtl::gpu::dense_vector<double> v(col12), w(25);
        w = L5 * v;
        std::vector<double> wh = w.to_host();
        REQUIRE(wh[12] == 20 && wh[13] == -8 && wh[14] == 1 && wh[18] == 2, "SpMV stencil");
        w += L5 * v;
        REQUIRE(w.to_host()[12] == 40, "w += A*v");
        w -= L5 * v;
        REQUIRE(w.to_host()[12] == 20, "w -= A*v");
    }
    {
        itl::pc::diagonal<matrix_type> P(A);
        itl::basic_iteration<double> iter(b, 2000, 1.e-8);
        x = 0.0;
        itl::cg(A, x, b, P, iter);
        std::printf("cg+diagonal: %d iterations, relres %.3e\n", iter.iterations(), relres(A, x, b));
        REQUIRE(iter.error_code() == 0 && relres(A, x, b) <= 1.05e-8, "cg+diagonal");
    }
    {
        itl::pc::ic_0<matrix_type, float> P(A);   // as in libs/numeric/itl/test/ic_0_test.cpp
        itl::basic_iteration<double> iter(b, 2000, 1.e-8);
        x = 0.0;
        itl::cg(A, x, b, P, iter);
        std::printf("cg+ic_0<float>: %d iterations, relres %.3e\n", iter.iterations(), relres(A, x, b));
        REQUIRE(iter.error_code() == 0 && relres(A, x, b) <= 1.05e-8, "cg+ic_0");
    }
    {
        itl::pc::ilu_0<matrix_type> P(A);
        itl::basic_iteration<double> iter(b, 2000, 1.e-8);
        x = 0.0;
        itl::bicgstab(A, x, b, P, iter);
        std::printf("bicgstab+ilu_0: %d iterations, relres %.3e\n", iter.iterations(), relres(A, x, b));
        REQUIRE(iter.error_code() == 0 && relres(A, x, b) <= 1.05e-8, "bicgstab+ilu_0");
    }
    {
        // itl::cyclic_iteration: one line per cycle of the device-side tests,
        // then the summary the solver's return prints
        itl::pc::diagonal<matrix_type> P(A);
        std::ostringstream out;
        itl::cyclic_iteration<double> iter(b, 2000, 1.e-8, 0.0, 25, out);
        x = 0.0;
        itl::cg(A, x, b, P, iter);
        const std::string t = out.str();
        int lines = 0;
        for (std::size_t k = 0; (k = t.find("iteration ", k)) != std::string::npos; ++k) ++lines;
        std::printf("cg+diagonal, cyclic_iteration(25): %d iterations, %d residual lines\n", iter.iterations(), lines);
        REQUIRE(t.rfind("iteration 0: resid ", 0) == 0, "cyclic first line");
        REQUIRE(lines == iter.iterations() / 25 + 1, "cyclic line count");
        REQUIRE(t.find("finished! error code = 0") != std::string::npos, "cyclic summary");
    }
    {
        // the other Krylov bodies with the reference's call shapes
        itl::pc::ilu_0<matrix_type> P(A);
        itl::pc::identity<matrix_type> I(A);
        const char* names[] = {"cgs", "bicgstab_2", "tfqmr", "bicgstab_ell(2)", "idr_s(4)"};
        for (int k = 0; k < 5; ++k) {
            itl::basic_iteration<double> iter(b, 2000, 1.e-8);
            x = 0.0;
            if (k == 0) itl::cgs(A, x, b, P, iter);
            else if (k == 1) itl::bicgstab_2(A, x, b, P, iter);
            else if (k == 2) itl::tfqmr(A, x, b, I, I, iter);
            else if (k == 3) itl::bicgstab_ell(A, x, b, P, I, iter, 2);
            else itl::idr_s(A, x, b, I, I, iter, 4);
            std::printf("%s: %d iterations, relres %.3e\n", names[k], iter.iterations(), relres(A, x, b));
            REQUIRE(iter.error_code() == 0, names[k]);
        }
    }
    {
        itl::pc::identity<matrix_type> L(A), R(A);
        itl::basic_iteration<double> iter(b, 5000, 1.e-8);
        x = 0.0;
        itl::gmres(A, x, b, L, R, iter, 30);
        std::printf("gmres(30): %d iterations, relres %.3e\n", iter.iterations(), relres(A, x, b));
        REQUIRE(iter.error_code() == 0 && relres(A, x, b) <= 1.05e-8, "gmres");
    }
    {
        itl::pc::ic_0<matrix_type, float> P(A);
        x = 0.0;
        mtlg_iter_result r = itl::refine_cg(A, x, b, P, 1e-10);
        std::printf("refine_cg: %d inner iterations, %d outer, relres %.3e\n", r.iterations, r.outer_iterations,
                    relres(A, x, b));
        REQUIRE(r.error_code == 0 && relres(A, x, b) <= 1.05e-10, "refine_cg");
    }
    {
        bool thrown = false;
        try {
            std::vector<int64_t> rp = {0, 1, 2};
            std::vector<int32_t> ci = {1, 0};
            std::vector<double> v = {1.0, 1.0};
            matrix_type B(2, 2, 2, rp.data(), ci.data(), v.data());
            itl::pc::ic_0<matrix_type> P(B);
        } catch (const mtl::gpu::missing_diagonal&) {
            thrown = true;
        }
        REQUIRE(thrown, "missing_diagonal exception");
    }
    std::printf("PASS (%lld kernels)\n", (long long)mtl::gpu::context::default_context().kernel_launches());
    return 0;
}
