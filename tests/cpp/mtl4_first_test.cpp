// The C++ front end next to MTL4 itself: the reference's headers are
// included first, so itl::basic_iteration, itl::cyclic_iteration and the
// preconditioner templates are the reference's own; the GPU types plug into
// them, and itl::cg / itl::bicgstab pick the GPU overloads for GPU matrices.
// The same systems are solved through MTL4 on the CPU and through the GPU in
// the reference summation order ("reduction_order" 1); the programs' printed
// outputs (cyclic_iteration lines and summaries) and the solutions must be
// identical.  Built by oracle/Makefile (target mtl4first) against the MTL4
// tree; exit code 0 = pass.
#include <boost/numeric/mtl/mtl.hpp>
#include <boost/numeric/itl/itl.hpp>

#include "mtl4_b200/itl_gpu.hpp"

#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

typedef mtl::mat::parameters<mtl::row_major, mtl::index::c_index, mtl::non_fixed::dimensions, false, std::size_t> para_t;
typedef mtl::compressed2D<double, para_t> cpu_matrix;
typedef mtl::dense_vector<double> cpu_vector;
typedef mtl::gpu::compressed2D<double> gpu_matrix;
typedef mtl::gpu::dense_vector<double> gpu_vector;

#define REQUIRE(c, msg)                                                 \
    do {                                                                \
        if (!(c)) { std::printf("FAIL: %s\n", msg); return 1; }         \
    } while (0)

int main()
{
    const int m = 40;
    cpu_matrix Ac;
    mtl::mat::laplacian_setup(Ac, m, m);
    const std::size_t n = num_rows(Ac);
    // CSR arrays of the CPU matrix for the GPU one
    std::vector<int64_t> rp(n + 1);
    std::vector<int32_t> ci(Ac.nnz());
    std::vector<double> va(Ac.nnz());
    for (std::size_t i = 0; i <= n; ++i) rp[i] = int64_t(Ac.address_major()[i]);
    for (std::size_t k = 0; k < Ac.nnz(); ++k) {
        ci[k] = int32_t(Ac.address_minor()[k]);
        va[k] = Ac.address_data()[k];
    }
    gpu_matrix Ag(int64_t(n), int64_t(n), int64_t(Ac.nnz()), rp.data(), ci.data(), va.data());
    mtlg_ctx_set_tuning(Ag.ctx().get(), "reduction_order", 1);

    std::vector<double> bh(n);
    for (std::size_t i = 0; i < n; ++i) bh[i] = std::sin(0.37 * double(i)) + 0.25;
    cpu_vector bc(n), xc(n);
    for (std::size_t i = 0; i < n; ++i) bc[i] = bh[i];
    gpu_vector bg(bh), xg(n);

    int fails = 0;
    for (int solver = 0; solver < 2; ++solver) {
        for (int pck = 0; pck < 3; ++pck) {
            std::ostringstream oc, og;
            xc = 0.0;
            xg = 0.0;
            itl::cyclic_iteration<double> ic(bc, 2000, 1.e-8, 0.0, 7, oc);
            itl::cyclic_iteration<double> ig(bg, 2000, 1.e-8, 0.0, 7, og);
            if (pck == 0) {
                itl::pc::diagonal<cpu_matrix> Pc(Ac);
                itl::pc::diagonal<gpu_matrix> Pg(Ag);
                if (solver == 0) { itl::cg(Ac, xc, bc, Pc, ic); itl::cg(Ag, xg, bg, Pg, ig); }
                else { itl::bicgstab(Ac, xc, bc, Pc, ic); itl::bicgstab(Ag, xg, bg, Pg, ig); }
            } else if (pck == 1) {
                itl::pc::ic_0<cpu_matrix> Pc(Ac);
                itl::pc::ic_0<gpu_matrix> Pg(Ag);
                if (solver == 0) { itl::cg(Ac, xc, bc, Pc, ic); itl::cg(Ag, xg, bg, Pg, ig); }
                else { itl::bicgstab(Ac, xc, bc, Pc, ic); itl::bicgstab(Ag, xg, bg, Pg, ig); }
            } else {
                itl::pc::ilu_0<cpu_matrix> Pc(Ac);
                itl::pc::ilu_0<gpu_matrix> Pg(Ag);
                if (solver == 0) { itl::cg(Ac, xc, bc, Pc, ic); itl::cg(Ag, xg, bg, Pg, ig); }
                else { itl::bicgstab(Ac, xc, bc, Pc, ic); itl::bicgstab(Ag, xg, bg, Pg, ig); }
            }
            const std::vector<double> xh = xg.to_host();
            bool same_x = true;
            for (std::size_t i = 0; i < n; ++i) same_x = same_x && xh[i] == xc[i];
            const bool same_text = oc.str() == og.str();
            std::printf("%s + %s: CPU %d / GPU %d iterations, output %s, x %s\n", solver ? "bicgstab" : "cg",
                        pck == 0 ? "diagonal" : pck == 1 ? "ic_0" : "ilu_0", ic.iterations(), ig.iterations(),
                        same_text ? "identical" : "DIFFERS", same_x ? "bitwise equal" : "DIFFERS");
            if (!same_text) std::printf("--- CPU\n%s--- GPU\n%s", oc.str().c_str(), og.str().c_str());
            fails += !(same_text && same_x);
        }
    }
    REQUIRE(fails == 0, "CPU and GPU runs differ");
    std::printf("PASS\n");
    return 0;
}
