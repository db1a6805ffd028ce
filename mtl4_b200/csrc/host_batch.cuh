// Batched solves: many independent systems advanced together by one set of
// kernels per iteration (see SolveSet).
#pragma once

struct mtlg_batch {
    mtlg_ctx* ctx = nullptr;
    struct Sys {
        mtlg_csr* A = nullptr;
        mtlg_pc* P64 = nullptr;   // plain FP64 solves
        mtlg_pc* P32 = nullptr;   // FP32 inner solves
        int solver = MTLG_CG;
        int pc_kind = MTLG_PC_IDENTITY;
        mtlg_iter_params params{};
        DBuf<double> x, b;
        mtlg_iter_result result{};
    };
    std::vector<std::unique_ptr<Sys>> sys;
    std::map<std::pair<int, int>, std::unique_ptr<SolveSet>> sets;   // (solver, precision)
    ~mtlg_batch()
    {
        sets.clear();
        for (auto& s : sys) {
            mtlg_pc_destroy(s->P64);
            mtlg_pc_destroy(s->P32);
            mtlg_csr_destroy(s->A);
        }
    }
};

extern "C" {

int mtlg_batch_create(mtlg_ctx* c, mtlg_batch** out)
{
    MTLG_CHECK_ARG(c && out, "ctx/out");
    *out = new mtlg_batch;
    (*out)->ctx = c;
    return MTLG_OK;
}

int mtlg_batch_destroy(mtlg_batch* B)
{
    if (B) {
        cudaStreamSynchronize(B->ctx->stream);
        delete B;
    }
    return MTLG_OK;
}

int mtlg_batch_add(mtlg_batch* B, int64_t n, int64_t nnz, const int64_t* row_ptr, const int32_t* col,
                   const double* val, const double* b, int solver, int pc_kind, const mtlg_iter_params* params,
                   int* index)
{
    MTLG_TRACE(9121, "batch.add");
    MTLG_CHECK_ARG(B && b && params, "batch/b/params");
    MTLG_CHECK_ARG(solver == MTLG_CG || solver == MTLG_BICGSTAB, "batched solver must be CG or BiCGSTAB");
    MTLG_CHECK_ARG(pc_kind >= MTLG_PC_IDENTITY && pc_kind <= MTLG_PC_IC0, "pc kind");
    std::unique_ptr<mtlg_batch::Sys> s(new mtlg_batch::Sys);
    MTLG_TRY(mtlg_csr_create(B->ctx, n, n, nnz, row_ptr, col, val, MTLG_F64, &s->A));
    s->solver = solver;
    s->pc_kind = pc_kind;
    s->params = *params;
    MTLG_TRY(s->b.upload(B->ctx, b, size_t(std::max<int64_t>(n, 1))));
    MTLG_TRY(s->x.alloc(B->ctx, size_t(std::max<int64_t>(n, 1))));
    MTLG_CUDA(cudaMemsetAsync(s->x.p, 0, size_t(n) * 8, B->ctx->stream));
    B->sets.clear();
    B->sys.push_back(std::move(s));
    if (index) *index = int(B->sys.size()) - 1;
    return MTLG_OK;
}

int mtlg_batch_size(const mtlg_batch* B) { return B ? int(B->sys.size()) : 0; }

// Size-balanced greedy assignment of independent systems to devices (longest
// processing time first): systems in order of decreasing cost (ties by
// index) each go to the part with the least cost so far (ties: lowest part).
// Host only; deterministic, so every rank computes the same assignment.
int mtlg_partition_systems(int64_t n_systems, const int64_t* cost, int n_parts, int32_t* part_of, int64_t* part_cost)
{
    MTLG_CHECK_ARG(n_systems >= 0 && n_parts >= 1, "sizes");
    MTLG_CHECK_ARG(n_systems == 0 || (cost && part_of), "null array");
    for (int64_t i = 0; i < n_systems; ++i) MTLG_CHECK_ARG(cost[i] >= 0, "negative cost");
    std::vector<int64_t> order(static_cast<size_t>(n_systems), 0);
    for (int64_t i = 0; i < n_systems; ++i) order[size_t(i)] = i;
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cost[a] > cost[b]; });
    std::vector<int64_t> load(static_cast<size_t>(n_parts), 0);
    for (int64_t i : order) {
        int best = 0;
        for (int p = 1; p < n_parts; ++p)
            if (load[size_t(p)] < load[size_t(best)]) best = p;
        part_of[i] = best;
        load[size_t(best)] += cost[i];
    }
    if (part_cost)
        for (int p = 0; p < n_parts; ++p) part_cost[p] = load[size_t(p)];
    return MTLG_OK;
}

int mtlg_batch_solve(mtlg_batch* B, int precision, const mtlg_refine_params* refine)
{
    MTLG_TRACE(9120, "batch.solve");
    MTLG_CHECK_ARG(B, "batch");
    MTLG_CHECK_ARG(precision == MTLG_F64 || precision == MTLG_F32, "precision");
    mtlg_ctx* c = B->ctx;
    mtlg_refine_params rp{};
    rp.max_outer = 10; rp.max_inner = 2000; rp.restart = 0; rp.rtol = 1e-8; rp.inner_rtol = 1e-4;
    if (refine) rp = *refine;
    const bool mixed = precision == MTLG_F32;
    // the whole batch must use one PC family for the sweep path; an all-
    // identity batch takes the identity path
    bool any_pc = false;
    for (auto& s : B->sys) any_pc |= s->pc_kind != MTLG_PC_IDENTITY;
    for (auto& s : B->sys) {
        int kind = s->pc_kind;
        if (any_pc && kind == MTLG_PC_IDENTITY) kind = MTLG_PC_DIAGONAL;   // keeps one code path
        mtlg_pc*& P = mixed ? s->P32 : s->P64;
        if (!P) MTLG_TRY(mtlg_pc_create(c, s->A, kind, mixed ? MTLG_F32 : MTLG_F64, &P));
        MTLG_CUDA(cudaMemsetAsync(s->x.p, 0, size_t(s->A->n_rows) * 8, c->stream));
    }
    cudaEvent_t e0, e1;
    MTLG_CUDA(cudaEventCreate(&e0));
    MTLG_CUDA(cudaEventCreate(&e1));
    for (int solver : {MTLG_CG, MTLG_BICGSTAB}) {
        std::vector<int> members;
        for (int i = 0; i < int(B->sys.size()); ++i) if (B->sys[i]->solver == solver) members.push_back(i);
        if (members.empty()) continue;
        auto& slot = B->sets[{solver, precision}];
        if (!slot) {
            std::unique_ptr<SolveSet> ss(new SolveSet);
            ss->solver = solver;
            ss->f32 = mixed ? 1 : 0;
            ss->mixed = mixed ? 1 : 0;
            for (int i : members) {
                auto& s = B->sys[i];
                SysInput si;
                si.A = s->A;
                si.P = mixed ? s->P32 : s->P64;
                si.x = s->x.p;
                si.b = s->b.p;
                ss->in.push_back(si);
            }
            MTLG_TRY(build_set(c, *ss));
            slot = std::move(ss);
        }
        SolveSet& ss = *slot;
        for (size_t k = 0; k < members.size(); ++k) {
            auto& s = B->sys[members[k]];
            ss.in[k].max_iter = s->params.max_iter;
            ss.in[k].rtol = s->params.rtol;
            ss.in[k].atol = s->params.atol;
            ss.in[k].norm_r0 = s->params.norm_r0;
        }
        MTLG_CUDA(cudaEventRecord(e0, c->stream));
        if (mixed) MTLG_TRY(run_refine(ss, rp));
        else MTLG_TRY(run_plain<double>(ss));
        MTLG_CUDA(cudaEventRecord(e1, c->stream));
        MTLG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        MTLG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        std::vector<SysState> h(ss.S);
        MTLG_CUDA(cudaMemcpy(h.data(), ss.st.p, sizeof(SysState) * ss.S, cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < members.size(); ++k) {
            fill_result(h[k], mixed, &B->sys[members[k]]->result);
            B->sys[members[k]]->result.seconds = ms * 1e-3;
        }
        // systems whose FP32-inner refinement stalled or broke down: finished in FP64
        if (mixed) {
            for (size_t k = 0; k < members.size(); ++k) {
                auto& s = B->sys[members[k]];
                if (!needs_fp64_finish(s->result)) continue;
                const int st = fp64_finish(c, solver, s->A, s->P32, s->x.p, s->b.p,
                                           fp64_budget(rp, s->result.iterations), rp.rtol, s->result);
                if (st != MTLG_OK && st != MTLG_ERR_BREAKDOWN) return st;
            }
        }
        int flag = 0;
        MTLG_CUDA(cudaMemcpy(&flag, ss.misc.p + 1, sizeof(int), cudaMemcpyDeviceToHost));
        if (flag) {
            for (auto& si : ss.in) pc_reset_sweep_state(si.P);
            reset_set_sweep_buffers(ss);
            set_error("a device-side wait expired during the batched solve");
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return MTLG_ERR_TIMEOUT;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return MTLG_OK;
}

int mtlg_batch_result(const mtlg_batch* B, int index, double* x_host, mtlg_iter_result* result)
{
    MTLG_CHECK_ARG(B && index >= 0 && index < int(B->sys.size()), "batch/index");
    const auto& s = B->sys[index];
    if (x_host) MTLG_CUDA(cudaMemcpy(x_host, s->x.p, size_t(s->A->n_rows) * 8, cudaMemcpyDeviceToHost));
    if (result) *result = s->result;
    return MTLG_OK;
}

// Serving API: built in host_server.cuh.
}  // extern "C"

#include "host_server.cuh"
