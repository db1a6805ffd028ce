// Host side: preconditioner structure (factor patterns, dependency levels,
// level-ordered layout) and the device factorization launches.
#pragma once
#include "host_core.cuh"

namespace mtlg {

// Off-diagonal entries of a triangular factor in natural row order, each with
// the source of its value (index into a value array) and the row whose
// inverse pivot multiplies it (-1: none).
struct RowLists {
    std::vector<int> rp;   // n + 1
    std::vector<int> col, src, mul;
};

// Level-ordered, warp-padded triangular factor.
struct TriDev {
    int n = 0, npad = 0, nnz = 0, nlev = 0;
    bool lower = true;
    std::vector<int> h_row_of;         // npad
    std::vector<int> h_rp;             // npad + 1
    std::vector<int> h_ci, h_src, h_mul;
    std::vector<int> lev_task_begin;   // nlev + 1, in units of tasks
    DBuf<int> row_of, rp, ci, src, mul;
    DBuf<unsigned char> val, dia;      // storage type S
    DBuf<SweepTask> tasks;             // single-system task list (sys = 0)
};

inline void compute_levels(const RowLists& F, int n, bool lower, std::vector<int>& lev, int& nlev)
{
    lev.assign(n, 0);
    int mx = -1;
    if (lower) {
        for (int i = 0; i < n; ++i) {
            int l = 0;
            for (int e = F.rp[i]; e < F.rp[i + 1]; ++e) l = std::max(l, lev[F.col[e]] + 1);
            lev[i] = l;
            mx = std::max(mx, l);
        }
    } else {
        for (int i = n - 1; i >= 0; --i) {
            int l = 0;
            for (int e = F.rp[i]; e < F.rp[i + 1]; ++e) l = std::max(l, lev[F.col[e]] + 1);
            lev[i] = l;
            mx = std::max(mx, l);
        }
    }
    nlev = mx + 1;
}

inline int build_tri(mtlg_ctx* c, const RowLists& F, int n, bool lower, TriDev& T)
{
    T.n = n;
    T.lower = lower;
    std::vector<int> lev;
    compute_levels(F, n, lower, lev, T.nlev);
    std::vector<int> cnt(T.nlev + 1, 0);
    for (int i = 0; i < n; ++i) cnt[lev[i]]++;
    // padded level starts
    std::vector<int> start(T.nlev + 1, 0);
    T.lev_task_begin.assign(T.nlev + 1, 0);
    for (int l = 0; l < T.nlev; ++l) {
        const int padded = (cnt[l] + kSweepRows - 1) / kSweepRows * kSweepRows;
        start[l + 1] = start[l] + padded;
        T.lev_task_begin[l + 1] = T.lev_task_begin[l] + padded / kSweepRows;
    }
    T.npad = start[T.nlev];
    T.h_row_of.assign(T.npad, -1);
    std::vector<int> fill(start.begin(), start.end() - 1);
    // rows ascending within a level (lower) / descending (upper)
    if (lower) {
        for (int i = 0; i < n; ++i) T.h_row_of[fill[lev[i]]++] = i;
    } else {
        for (int i = n - 1; i >= 0; --i) T.h_row_of[fill[lev[i]]++] = i;
    }
    T.h_rp.assign(T.npad + 1, 0);
    for (int k = 0; k < T.npad; ++k) {
        const int r = T.h_row_of[k];
        T.h_rp[k + 1] = T.h_rp[k] + (r >= 0 ? F.rp[r + 1] - F.rp[r] : 0);
    }
    T.nnz = T.h_rp[T.npad];
    T.h_ci.resize(T.nnz);
    T.h_src.resize(T.nnz);
    T.h_mul.resize(T.nnz);
    for (int k = 0; k < T.npad; ++k) {
        const int r = T.h_row_of[k];
        if (r < 0) continue;
        int o = T.h_rp[k];
        for (int e = F.rp[r]; e < F.rp[r + 1]; ++e, ++o) {
            T.h_ci[o] = F.col[e];
            T.h_src[o] = F.src[e];
            T.h_mul[o] = F.mul[e];
        }
    }
    std::vector<SweepTask> tasks(T.npad / kSweepRows);
    for (size_t t = 0; t < tasks.size(); ++t) tasks[t] = {0, int(t) * kSweepRows};
    MTLG_TRY(T.row_of.upload(c, T.h_row_of.data(), T.h_row_of.size()));
    MTLG_TRY(T.rp.upload(c, T.h_rp.data(), T.h_rp.size()));
    MTLG_TRY(T.ci.upload(c, T.h_ci.data(), T.h_ci.size()));
    MTLG_TRY(T.src.upload(c, T.h_src.data(), T.h_src.size()));
    MTLG_TRY(T.mul.upload(c, T.h_mul.data(), T.h_mul.size()));
    MTLG_TRY(T.tasks.upload(c, tasks.data(), tasks.size()));
    return MTLG_OK;
}

}  // namespace mtlg

struct mtlg_pc {
    mtlg_ctx* ctx = nullptr;
    mtlg_csr* A = nullptr;
    int kind = MTLG_PC_IDENTITY;
    int storage = MTLG_F64;
    int n = 0;
    DBuf<unsigned char> inv_diag;   // Jacobi, storage type
    TriDev L, U;
    DBuf<double> inv_dia;           // FP64 pivots (ILU: 1/u_ii, IC: 1/sqrt(u_ii))
    DBuf<unsigned char> tmp;        // sentinel-filled temporary (n x 8 bytes)
    DBuf<int> tickets;              // self-resetting work tickets
    DBuf<SysDesc> desc;
    DBuf<SysState> st;
    DBuf<int> misc;
    RowLists lt;                    // IC(0): transposed upper pattern (natural order)
    DBuf<int> lt_rp, lt_row, lt_src;
    bool has_factors() const { return kind == MTLG_PC_ILU0 || kind == MTLG_PC_IC0; }
    size_t ssize() const { return storage == MTLG_F64 ? 8 : 4; }
};

namespace mtlg {

inline int fill_sentinel(mtlg_ctx* c, void* p, size_t bytes)
{
    if (!bytes) return MTLG_OK;
    MTLG_CUDA(cudaMemsetAsync(p, 0xFF, bytes, c->stream));
    return MTLG_OK;
}

inline int sweep_grid(mtlg_ctx* c) { return c->sweep_grid; }

inline int pc_setup_single_set(mtlg_pc* P)
{
    mtlg_ctx* c = P->ctx;
    MTLG_TRY(P->desc.alloc(c, 1));
    MTLG_TRY(P->st.alloc(c, 1));
    MTLG_CUDA(cudaMemsetAsync(P->st.p, 0, sizeof(SysState), c->stream));
    MTLG_TRY(P->misc.alloc(c, 4));
    MTLG_CUDA(cudaMemsetAsync(P->misc.p, 0, 4 * sizeof(int), c->stream));
    MTLG_TRY(P->tickets.alloc(c, 8));
    MTLG_CUDA(cudaMemsetAsync(P->tickets.p, 0, 8 * sizeof(int), c->stream));
    MTLG_TRY(P->tmp.alloc(c, size_t(std::max(P->n, 1)) * 8));
    MTLG_TRY(fill_sentinel(c, P->tmp.p, size_t(P->n) * 8));
    return MTLG_OK;
}

inline int launch_grid(int64_t n, int maxg = 8192) { return int(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, maxg))); }

// Structure + device factorization.
inline int pc_build(mtlg_pc* P)
{
    mtlg_csr* A = P->A;
    mtlg_ctx* c = P->ctx;
    const int n = P->n;
    const int64_t* rp = A->h_rp.data();
    const int* ci = A->h_ci.data();
    if (P->kind == MTLG_PC_DIAGONAL) {
        MTLG_TRY(P->inv_diag.alloc(c, size_t(n) * P->ssize()));
        if (n) {
            k_inv_diag<<<launch_grid(n), 256, 0, c->stream>>>(n, A->v64.p, A->dpos.p, P->inv_diag.p, P->storage == MTLG_F32);
            c->launches++;
            MTLG_CUDA(cudaGetLastError());
        }
        // trivial factors so the batched sweep path can apply Jacobi too:
        // L: no entries, dia = 1/a_ii; U: no entries, dia = 1.
        RowLists E;
        E.rp.assign(n + 1, 0);
        MTLG_TRY(build_tri(c, E, n, true, P->L));
        MTLG_TRY(build_tri(c, E, n, false, P->U));
        MTLG_TRY(P->L.val.alloc(c, 16));
        MTLG_TRY(P->U.val.alloc(c, 16));
        MTLG_TRY(P->L.dia.alloc(c, size_t(P->L.npad) * P->ssize()));
        MTLG_TRY(P->U.dia.alloc(c, size_t(P->U.npad) * P->ssize()));
        MTLG_TRY(P->inv_dia.alloc(c, std::max(n, 1)));
        if (n) {
            // inv_dia (FP64) = 1 / a_ii for the trivial L's diagonal multiplier
            k_inv_diag<<<launch_grid(n), 256, 0, c->stream>>>(n, A->v64.p, A->dpos.p, P->inv_dia.p, 0);
            k_fill_dia<<<launch_grid(P->L.npad), 256, 0, c->stream>>>(P->L.npad, P->L.row_of.p, P->inv_dia.p, 0,
                                                                       P->L.dia.p, P->storage == MTLG_F32);
            k_fill_dia<<<launch_grid(P->U.npad), 256, 0, c->stream>>>(P->U.npad, P->U.row_of.p, P->inv_dia.p, 1,
                                                                       P->U.dia.p, P->storage == MTLG_F32);
            c->launches += 3;
            MTLG_CUDA(cudaGetLastError());
        }
        return pc_setup_single_set(P);
    }
    if (!P->has_factors()) return pc_setup_single_set(P);

    for (int i = 0; i < n; ++i) {
        if (A->h_dpos[i] < 0) {
            set_error("row %d has no diagonal entry", i);
            return MTLG_ERR_MISSING_DIAGONAL;
        }
    }
    RowLists Lr, Ur;
    Lr.rp.assign(n + 1, 0);
    Ur.rp.assign(n + 1, 0);
    if (P->kind == MTLG_PC_ILU0) {
        // L = strict_lower(LU) (unit diagonal), U = upper(LU) with the
        // inverted diagonal first (ilu_0.hpp:79-81, ilu.hpp:84-91)
        for (int i = 0; i < n; ++i) {
            for (int64_t e = rp[i]; e < rp[i + 1]; ++e) {
                if (ci[e] < i) { Lr.col.push_back(ci[e]); Lr.src.push_back(int(e)); Lr.mul.push_back(-1); }
                else if (ci[e] > i) { Ur.col.push_back(ci[e]); Ur.src.push_back(int(e)); Ur.mul.push_back(-1); }
            }
            Lr.rp[i + 1] = int(Lr.col.size());
            Ur.rp[i + 1] = int(Ur.col.size());
        }
    } else {
        // U = upper(A) scaled by its row's inverse pivot; L = trans(U) with
        // the diagonal last (ic_0.hpp:47-57, 80-87)
        std::vector<int> cntT(n + 1, 0);
        for (int i = 0; i < n; ++i)
            for (int64_t e = rp[i]; e < rp[i + 1]; ++e)
                if (ci[e] > i) cntT[ci[e] + 1]++;
        for (int i = 0; i < n; ++i) cntT[i + 1] += cntT[i];
        Lr.rp = cntT;
        Lr.col.resize(cntT[n]);
        Lr.src.resize(cntT[n]);
        Lr.mul.resize(cntT[n]);
        std::vector<int> pos(cntT.begin(), cntT.end() - 1);
        for (int i = 0; i < n; ++i) {
            for (int64_t e = rp[i]; e < rp[i + 1]; ++e) {
                if (ci[e] > i) {
                    const int j = ci[e], o = pos[j]++;
                    Lr.col[o] = i; Lr.src[o] = int(e); Lr.mul[o] = i;
                    Ur.col.push_back(j); Ur.src.push_back(int(e)); Ur.mul.push_back(i);
                }
            }
            Ur.rp[i + 1] = int(Ur.col.size());
        }
        MTLG_TRY(P->lt_rp.upload(c, Lr.rp.data(), Lr.rp.size()));
        MTLG_TRY(P->lt_row.upload(c, Lr.col.data(), std::max<size_t>(1, Lr.col.size())));
        MTLG_TRY(P->lt_src.upload(c, Lr.src.data(), std::max<size_t>(1, Lr.src.size())));
    }
    MTLG_TRY(build_tri(c, Lr, n, true, P->L));
    MTLG_TRY(build_tri(c, Ur, n, false, P->U));
    MTLG_TRY(pc_setup_single_set(P));

    // ---- numeric factorization on the device (FP64)
    MTLG_TRY(P->inv_dia.alloc(c, std::max(n, 1)));
    MTLG_TRY(fill_sentinel(c, P->inv_dia.p, size_t(n) * 8));
    DBuf<double> lu;
    const double* srcvals = A->v64.p;
    FactorOp op;
    memset(&op, 0, sizeof op);
    op.tasks = P->L.tasks.p;
    op.ntasks = int(P->L.tasks.n);
    op.ticket = P->tickets.p + 7;
    op.row_of = P->L.row_of.p;
    op.rp = A->rp.p;
    op.ci = A->ci.p;
    op.inv_dia = P->inv_dia.p;
    op.dpos = A->dpos.p;
    op.err = P->misc.p + 1;
    if (P->kind == MTLG_PC_ILU0) {
        MTLG_TRY(lu.alloc(c, size_t(std::max<int64_t>(1, A->nnz))));
        MTLG_CUDA(cudaMemcpyAsync(lu.p, A->v64.p, size_t(A->nnz) * 8, cudaMemcpyDeviceToDevice, c->stream));
        op.lu = lu.p;
        if (op.ntasks) {
            k_ilu0_factor<<<sweep_grid(c), kBlock, 0, c->stream>>>(op);
            c->launches++;
        }
        srcvals = lu.p;
    } else {
        op.lt_rp = P->lt_rp.p;
        op.lt_row = P->lt_row.p;
        op.lt_src = P->lt_src.p;
        op.a = A->v64.p;
        if (op.ntasks) {
            k_ic0_factor<<<sweep_grid(c), kBlock, 0, c->stream>>>(op);
            c->launches++;
        }
    }
    MTLG_CUDA(cudaGetLastError());
    const int f32 = P->storage == MTLG_F32;
    for (TriDev* T : {&P->L, &P->U}) {
        MTLG_TRY(T->val.alloc(c, size_t(std::max(T->nnz, 1)) * P->ssize()));
        MTLG_TRY(T->dia.alloc(c, size_t(std::max(T->npad, 1)) * P->ssize()));
        if (T->nnz) {
            k_fill_factor<<<launch_grid(T->nnz), 256, 0, c->stream>>>(T->nnz, T->src.p, T->mul.p, srcvals, P->inv_dia.p,
                                                                      T->val.p, f32);
            c->launches++;
        }
        const int unit = (P->kind == MTLG_PC_ILU0 && T == &P->L);
        if (T->npad) {
            k_fill_dia<<<launch_grid(T->npad), 256, 0, c->stream>>>(T->npad, T->row_of.p, P->inv_dia.p, unit, T->dia.p, f32);
            c->launches++;
        }
        MTLG_CUDA(cudaGetLastError());
    }
    int err = 0;
    MTLG_CUDA(cudaMemcpyAsync(&err, P->misc.p + 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    if (err) {
        set_error("factorization dependency wait expired");
        return MTLG_ERR_TIMEOUT;
    }
    return MTLG_OK;
}

}  // namespace mtlg
