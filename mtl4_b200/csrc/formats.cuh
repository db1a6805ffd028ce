// ELL and sparse_banded matrices and their products (the reference's
// mtl::mat::ell_matrix and mtl::mat::sparse_banded with
// operation/mat_vec_mult.hpp:686-803).
//
// ELL: the reference's layout as it is -- entry j of row r at
// k = r + j * stride (stride >= rows, the reference rounds it up to 32), the
// slots of short rows padded with value 0 -- which is already the GPU's
// coalesced layout: one thread per row, a warp reads 32 consecutive k per
// slot.  Row sums add the rounded products slot by slot, padding included,
// as the reference build does, so FP64 results are bitwise the reference's.
//
// sparse_banded: the reference stores one value per band and row, row by
// row; here the values are kept band by band (value of band b, row r at
// b * rows + r) so that a warp's threads (consecutive rows) read
// consecutive addresses.  A row sums its bands that fall inside the matrix
// in increasing order.  The reference's product runs the rows in 4-row
// blocks or singly (row ranges cut where a band starts or ends,
// mat_vec_mult.hpp:727-795) and its build contracts those loops
// differently: blocked rows add rounded products in pairs and fuse an odd
// last band; single rows of 4 bands or more add rounded products in groups
// of four and fuse the rest, shorter single rows round every product.  The
// row kinds are computed once on the host and the kernel follows them, so
// FP64 results are bitwise the reference's; FP32 rounds every product.
#pragma once
#include "kernels.cuh"

struct mtlg_ell {
    mtlg_ctx* ctx = nullptr;
    int64_t n_rows = 0, n_cols = 0, slots = 0, stride = 0;
    mtlg::DBuf<int> minor;
    mtlg::DBuf<double> v64;
    mtlg::DBuf<float> v32;
};

struct mtlg_banded {
    mtlg_ctx* ctx = nullptr;
    int64_t n_rows = 0, n_cols = 0, nb = 0;
    std::vector<int64_t> h_bands;
    mtlg::DBuf<int> bands;
    mtlg::DBuf<unsigned char> kind;   // per row: 1 blocked, 0 single, 2 no band inside the matrix
    mtlg::DBuf<double> v64;            // band-major
    mtlg::DBuf<float> v32;
};

namespace mtlg {

template <typename T, int ASG>
__global__ void __launch_bounds__(kBlock) k_ell_spmv(int n, int stride, int slots, const int* __restrict__ minor,
                                                     const T* __restrict__ val, const T* __restrict__ x,
                                                     T* __restrict__ y)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        T acc = T(0);
        int j = 0;
        for (; j + 4 <= slots; j += 4) {
            T av[4], xv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const long long k = (long long)(j + u) * stride + r;
                av[u] = val[k];
                xv[u] = x[minor[k]];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) acc = mac(acc, av[u], xv[u]);
        }
        for (; j < slots; ++j) {
            const long long k = (long long)j * stride + r;
            acc = mac(acc, val[k], x[minor[k]]);
        }
        const T base = (ASG == ASG_SET) ? T(0) : y[r];
        y[r] = assign_out<T, ASG>(base, acc);
    }
}

template <typename T, int ASG>
__global__ void __launch_bounds__(kBlock) k_banded_spmv(int n, int nc, int nb, const int* __restrict__ bands,
                                                        const unsigned char* __restrict__ kind,
                                                        const T* __restrict__ val, const T* __restrict__ x,
                                                        T* __restrict__ y)
{
    extern __shared__ int s_bands[];
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s_bands[b] = bands[b];
    __syncthreads();
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int kd = kind[r];
        if (kd == 2) {   // no band inside the matrix: '=' gives 0, '+=' / '-=' leave the row
            if (ASG == ASG_SET) y[r] = T(0);
            continue;
        }
        int lo = 0, hi = nb;
        while (lo < nb && r + s_bands[lo] < 0) ++lo;
        while (hi > lo && r + s_bands[hi - 1] >= nc) --hi;
        const int cnt = hi - lo;
        const int q = kd == 1 ? lo + cnt / 2 * 2 : (cnt >= 4 ? lo + cnt / 4 * 4 : hi);
        T acc = T(0);
        for (int b = lo; b < hi; ++b) {
            const T a = val[(long long)b * n + r], v = x[r + s_bands[b]];
            acc = (sizeof(T) == 8 && b >= q) ? T(__fma_rn(double(a), double(v), double(acc))) : mac(acc, a, v);
        }
        const T base = (ASG == ASG_SET) ? T(0) : y[r];
        y[r] = assign_out<T, ASG>(base, acc);
    }
}

// Row kinds of the reference's banded product loop: the rows are cut where a
// band starts (row max(0, -band)) or ends (row min(rows, cols - band)); in
// each piece [from, to) the rows from .. from + 4 floor((to - from) / 4) run
// in 4-row blocks (1), the rest singly (0); rows outside every band get 2.
inline void banded_row_kinds(int64_t nr, int64_t nc, const std::vector<int64_t>& bands, std::vector<unsigned char>& kind)
{
    kind.assign(size_t(nr), 2);
    const int64_t nb = int64_t(bands.size());
    if (nb == 0) return;
    std::vector<int64_t> begin_rows(size_t(nb), 0), end_rows(size_t(nb), 0);
    for (int64_t b = 0; b < nb; ++b) {
        begin_rows[size_t(b)] = std::max<int64_t>(0, -bands[size_t(b)]);
        end_rows[size_t(b)] = std::min<int64_t>(nr, nc - bands[size_t(b)]);
    }
    int64_t bp = 0, ep = nb - 1;
    while (bp < nb && begin_rows[size_t(bp)] > 0) bp++;
    if (bp == nb) --bp;
    int64_t from = begin_rows[size_t(bp)];
    while (bp > 0 && begin_rows[size_t(bp - 1)] == from) bp--;
    for (bool active = true; active;) {
        const int64_t to = bp > 0 && begin_rows[size_t(bp - 1)] <= end_rows[size_t(ep)] ? begin_rows[size_t(bp - 1)]
                                                                                         : end_rows[size_t(ep)];
        const int64_t blocked_to = ((to - from) & -4) + from;
        for (int64_t r = std::max<int64_t>(0, from); r < std::min(to, nr); ++r) kind[size_t(r)] = r < blocked_to ? 1 : 0;
        if (bp > 0) {
            if (begin_rows[size_t(bp - 1)] == to) bp--;
            if (end_rows[size_t(ep)] == to) ep--;
        } else {
            if (end_rows[0] == to) active = false;
            else ep--;
        }
        if (ep < 0) break;
        from = to;
    }
}

inline int spmv_grid(int64_t n) { return int(std::max<int64_t>(1, std::min<int64_t>((n + kBlock - 1) / kBlock, 148 * 16))); }

}  // namespace mtlg

extern "C" {

int mtlg_ell_create(mtlg_ctx* c, int64_t n_rows, int64_t n_cols, int64_t slots, int64_t stride, const int64_t* minor,
                    const void* data, mtlg_dtype dt, mtlg_ell** out)
{
    using namespace mtlg;
    MTLG_TRACE(9010, "ell_create");
    MTLG_CHECK_ARG(c && out && n_rows >= 0 && n_cols >= 0 && slots >= 0 && stride >= n_rows, "ctx/out/sizes");
    MTLG_CHECK_ARG(dt == MTLG_F64 || dt == MTLG_F32, "dtype");
    const int64_t m = slots * stride;
    MTLG_CHECK_ARG(m == 0 || (minor && data), "arrays");
    if (m > INT32_MAX || n_rows > INT32_MAX || n_cols > INT32_MAX) {
        set_error("ELL of %lld x %lld slots exceeds int32 indexing", (long long)stride, (long long)slots);
        return MTLG_ERR_TOO_LARGE;
    }
    std::vector<int> mi(static_cast<size_t>(m), 0);
    for (int64_t k = 0; k < m; ++k) {
        if (minor[k] < 0 || minor[k] >= std::max<int64_t>(n_cols, 1)) {
            set_error("ELL column %lld at %lld out of range", (long long)minor[k], (long long)k);
            return MTLG_ERR_UNSORTED;
        }
        mi[size_t(k)] = int(minor[k]);
    }
    std::unique_ptr<mtlg_ell> E(new mtlg_ell);
    E->ctx = c;
    E->n_rows = n_rows;
    E->n_cols = n_cols;
    E->slots = slots;
    E->stride = stride;
    MTLG_TRY(E->minor.upload(c, mi.data(), size_t(std::max<int64_t>(m, 1))));
    std::vector<double> v(size_t(std::max<int64_t>(m, 1)), 0.0);
    for (int64_t k = 0; k < m; ++k) v[size_t(k)] = dt == MTLG_F64 ? static_cast<const double*>(data)[k]
                                                                  : double(static_cast<const float*>(data)[k]);
    MTLG_TRY(E->v64.upload(c, v.data(), v.size()));
    std::vector<float> vf(v.size());
    for (size_t k = 0; k < v.size(); ++k) vf[k] = float(v[k]);
    MTLG_TRY(E->v32.upload(c, vf.data(), vf.size()));
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    *out = E.release();
    return MTLG_OK;
}

int mtlg_ell_destroy(mtlg_ell* E)
{
    if (E) {
        cudaStreamSynchronize(E->ctx->stream);
        delete E;
    }
    return MTLG_OK;
}

int mtlg_ell_spmv(mtlg_ctx* c, mtlg_ell* E, const mtlg_vec* x, mtlg_vec* y, int assign)
{
    using namespace mtlg;
    MTLG_TRACE(3050, "ell_cvec_mult");
    MTLG_CHECK_ARG(c && E && x && y, "null handle");
    MTLG_CHECK_ARG(x->dtype == y->dtype, "x and y dtypes differ");
    MTLG_CHECK_ARG(assign >= MTLG_ASSIGN && assign <= MTLG_MINUS, "assign");
    if (x->n != E->n_cols || y->n != E->n_rows) {
        set_error("ELL %lldx%lld times %lld -> %lld", (long long)E->n_rows, (long long)E->n_cols, (long long)x->n,
                  (long long)y->n);
        return MTLG_ERR_INCOMPATIBLE_SIZE;
    }
    if (E->n_rows == 0) return MTLG_OK;
    const int g = spmv_grid(E->n_rows);
    const int n = int(E->n_rows), st = int(E->stride), sl = int(E->slots);
#define MTLG_ELL_CASE(T, V, ASG) \
    k_ell_spmv<T, ASG><<<g, kBlock, 0, c->stream>>>(n, st, sl, E->minor.p, V, static_cast<const T*>(x->p), static_cast<T*>(y->p))
    const int asg = assign == MTLG_ASSIGN ? ASG_SET : (assign == MTLG_PLUS ? ASG_ADD : ASG_SUB);
    if (x->dtype == MTLG_F64) {
        if (asg == ASG_SET) MTLG_ELL_CASE(double, E->v64.p, ASG_SET);
        else if (asg == ASG_ADD) MTLG_ELL_CASE(double, E->v64.p, ASG_ADD);
        else MTLG_ELL_CASE(double, E->v64.p, ASG_SUB);
    } else {
        if (asg == ASG_SET) MTLG_ELL_CASE(float, E->v32.p, ASG_SET);
        else if (asg == ASG_ADD) MTLG_ELL_CASE(float, E->v32.p, ASG_ADD);
        else MTLG_ELL_CASE(float, E->v32.p, ASG_SUB);
    }
#undef MTLG_ELL_CASE
    c->launches++;
    MTLG_CUDA(cudaGetLastError());
    return MTLG_OK;
}

int mtlg_banded_create(mtlg_ctx* c, int64_t n_rows, int64_t n_cols, int64_t nbands, const int64_t* bands,
                       const void* data, mtlg_dtype dt, mtlg_banded** out)
{
    using namespace mtlg;
    MTLG_TRACE(9011, "banded_create");
    MTLG_CHECK_ARG(c && out && n_rows >= 0 && n_cols >= 0 && nbands >= 0 && nbands <= 4096, "ctx/out/sizes");
    MTLG_CHECK_ARG(dt == MTLG_F64 || dt == MTLG_F32, "dtype");
    MTLG_CHECK_ARG(nbands == 0 || (bands && data), "arrays");
    if (n_rows * std::max<int64_t>(nbands, 1) > INT32_MAX || n_rows > INT32_MAX || n_cols > INT32_MAX) {
        set_error("banded matrix exceeds int32 indexing");
        return MTLG_ERR_TOO_LARGE;
    }
    for (int64_t b = 0; b < nbands; ++b) {
        if ((b > 0 && bands[b] <= bands[b - 1]) || bands[b] <= -n_rows || bands[b] >= n_cols) {
            set_error("bands must increase strictly and meet the matrix (band %lld = %lld)", (long long)b,
                      (long long)bands[b]);
            return MTLG_ERR_UNSORTED;
        }
    }
    std::unique_ptr<mtlg_banded> S(new mtlg_banded);
    S->ctx = c;
    S->n_rows = n_rows;
    S->n_cols = n_cols;
    S->nb = nbands;
    S->h_bands.assign(bands, bands + nbands);
    std::vector<int> bi(size_t(std::max<int64_t>(nbands, 1)), 0);
    for (int64_t b = 0; b < nbands; ++b) bi[size_t(b)] = int(bands[b]);
    MTLG_TRY(S->bands.upload(c, bi.data(), bi.size()));
    std::vector<unsigned char> kind;
    banded_row_kinds(n_rows, n_cols, S->h_bands, kind);
    kind.resize(size_t(std::max<int64_t>(n_rows, 1)), 2);
    MTLG_TRY(S->kind.upload(c, kind.data(), kind.size()));
    // row-major (reference) -> band-major
    const size_t m = size_t(std::max<int64_t>(n_rows * nbands, 1));
    std::vector<double> v(m, 0.0);
    std::vector<float> vf(m, 0.0f);
    for (int64_t r = 0; r < n_rows; ++r)
        for (int64_t b = 0; b < nbands; ++b) {
            const double a = dt == MTLG_F64 ? static_cast<const double*>(data)[r * nbands + b]
                                            : double(static_cast<const float*>(data)[r * nbands + b]);
            v[size_t(b * n_rows + r)] = a;
            vf[size_t(b * n_rows + r)] = float(a);
        }
    MTLG_TRY(S->v64.upload(c, v.data(), v.size()));
    MTLG_TRY(S->v32.upload(c, vf.data(), vf.size()));
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    *out = S.release();
    return MTLG_OK;
}

int mtlg_banded_destroy(mtlg_banded* S)
{
    if (S) {
        cudaStreamSynchronize(S->ctx->stream);
        delete S;
    }
    return MTLG_OK;
}

int mtlg_banded_spmv(mtlg_ctx* c, mtlg_banded* S, const mtlg_vec* x, mtlg_vec* y, int assign)
{
    using namespace mtlg;
    MTLG_TRACE(3069, "sparse_banded_cvec_mult");
    MTLG_CHECK_ARG(c && S && x && y, "null handle");
    MTLG_CHECK_ARG(x->dtype == y->dtype, "x and y dtypes differ");
    MTLG_CHECK_ARG(assign >= MTLG_ASSIGN && assign <= MTLG_MINUS, "assign");
    if (x->n != S->n_cols || y->n != S->n_rows) {
        set_error("banded %lldx%lld times %lld -> %lld", (long long)S->n_rows, (long long)S->n_cols, (long long)x->n,
                  (long long)y->n);
        return MTLG_ERR_INCOMPATIBLE_SIZE;
    }
    if (S->n_rows == 0) return MTLG_OK;
    const int g = spmv_grid(S->n_rows);
    const int n = int(S->n_rows), nc = int(S->n_cols), nb = int(S->nb);
    const size_t smem = size_t(std::max(nb, 1)) * sizeof(int);
#define MTLG_BAND_CASE(T, V, ASG) \
    k_banded_spmv<T, ASG><<<g, kBlock, smem, c->stream>>>(n, nc, nb, S->bands.p, S->kind.p, V, static_cast<const T*>(x->p), static_cast<T*>(y->p))
    const int asg = assign == MTLG_ASSIGN ? ASG_SET : (assign == MTLG_PLUS ? ASG_ADD : ASG_SUB);
    if (x->dtype == MTLG_F64) {
        if (asg == ASG_SET) MTLG_BAND_CASE(double, S->v64.p, ASG_SET);
        else if (asg == ASG_ADD) MTLG_BAND_CASE(double, S->v64.p, ASG_ADD);
        else MTLG_BAND_CASE(double, S->v64.p, ASG_SUB);
    } else {
        if (asg == ASG_SET) MTLG_BAND_CASE(float, S->v32.p, ASG_SET);
        else if (asg == ASG_ADD) MTLG_BAND_CASE(float, S->v32.p, ASG_ADD);
        else MTLG_BAND_CASE(float, S->v32.p, ASG_SUB);
    }
#undef MTLG_BAND_CASE
    c->launches++;
    MTLG_CUDA(cudaGetLastError());
    return MTLG_OK;
}

}  // extern "C"
