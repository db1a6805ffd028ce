// Served solves: continuous batching on one GPU.
//
// A server owns, per solver family (CG, BiCGSTAB), an engine with a fixed
// pool of `max_active` slots.  A slot holds one request's matrix, factors,
// vectors and device-side iteration state for its whole life, so admitting
// or retiring a request never disturbs the others.  Each engine step runs
// the kernels of every phase (initial / outer residual, inner setup, a
// fixed number of inner iterations, FP64 update) over all active slots; a
// kernel acts only on the slots in its phase.  Requests admitted while
// others run therefore overlap with them in the same launches, and because
// tiles never straddle slots and reductions sum per slot in a fixed order, a
// request's result does not depend on what else is in the mix.
//
// Admission: a queued request enters a free slot when the device memory it
// needs fits the server's budget; requests that could never fit are refused
// at submission.
#pragma once

#include <chrono>
#include <deque>

struct mtlg_server {
    mtlg_ctx* ctx = nullptr;
    mtlg_server_opts o{};
    bool refine = false;

    struct Req {
        int64_t id = 0;
        int state = 0;   // 0 queued, 1 active, 2 done, 3 cancelled, 4 failed
        int64_t n = 0, nnz = 0;
        std::vector<int64_t> rp;
        std::vector<int32_t> ci;
        std::vector<double> val, b;
        int solver = MTLG_CG, pc = MTLG_PC_IC0, max_iter = 1000;
        size_t est = 0;
        int engine = 0, slot = -1;
        double nb = 0;
        mtlg_csr* A = nullptr;
        mtlg_pc* P = nullptr;
        DBuf<double> x, bd, ws64;
        DBuf<unsigned char> ws;
        std::vector<double> xh;
        mtlg_iter_result res{};
        int status_code = MTLG_OK;
        void release()
        {
            mtlg_pc_destroy(P);
            P = nullptr;
            mtlg_csr_destroy(A);
            A = nullptr;
            x.release();
            bd.release();
            ws.release();
            ws64.release();
        }
        ~Req() { release(); }
    };

    struct Engine {
        int solver = MTLG_CG;
        SolveSet ss;
        std::vector<int64_t> slot_req;
        bool dirty = false;
        int nactive = 0;
        cudaGraphExec_t exec = nullptr;
        cudaGraph_t graph = nullptr;
        int body_kernels = 0;
        ~Engine()
        {
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
        }
    };

    std::map<int64_t, std::unique_ptr<Req>> reqs;
    std::deque<int64_t> queue;
    int64_t next_id = 1;
    Engine eng[2];
    mtlg_server_stats stats{};
    size_t bytes_held = 0;
};

namespace mtlg {

inline size_t srv_estimate(int64_t n, int64_t nnz, bool refine)
{
    // CSR (int32 pattern, FP64 + FP32 values), factors with their layouts,
    // x/b, the workspace vectors and the FP64 refinement residual.
    const size_t vb = refine ? 4 : 8;
    return size_t(nnz) * (4 + 8 + 4 + 2 * (4 + 4 + 4 + 4 + vb)) + size_t(n) * (4 * 6 + 16 + kNumVec * vb + 8 + 64);
}

// Admission rule.  With a byte budget: a request fits when the server's
// held bytes plus its estimate stay within the budget, and never fits when
// the estimate alone exceeds it.  Without a budget: the device's free memory
// (cudaMemGetInfo, or the context's "admission_free_bytes" stand-in) less a
// reserve; a request that does not fit now waits while the memory the
// server's active requests hold would make room once they retire, and never
// fits otherwise.  Returns 1 admit, 0 wait, -1 never fits.
inline int admission_decision(size_t need, size_t held, size_t budget, size_t free_bytes, size_t reserve)
{
    if (budget) {
        if (need > budget) return -1;
        return held + need <= budget ? 1 : 0;
    }
    const size_t usable = free_bytes > reserve ? free_bytes - reserve : 0;
    if (need <= usable) return 1;
    return need <= usable + held ? 0 : -1;
}

// Free device memory and the reserve kept out of admission (default: the
// larger of 1 GiB and 2% of the device).  The "admission_free_bytes" stand-in
// is the free memory before this server's own requests, so the bytes it holds
// come off it as they do off cudaMemGetInfo's figure.
inline int free_memory(mtlg_ctx* c, size_t held, size_t& free_bytes, size_t& reserve)
{
    size_t fr = 0, total = 0;
    MTLG_CUDA(cudaMemGetInfo(&fr, &total));
    if (c->pool) {
        // blocks the context's pool holds but no buffer uses are free too
        uint64_t reserved = 0, used = 0;
        if (cudaMemPoolGetAttribute(c->pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
            cudaMemPoolGetAttribute(c->pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
            fr += size_t(reserved - used);
        cudaGetLastError();
    }
    if (c->admission_free_bytes > 0) {
        const size_t f = size_t(c->admission_free_bytes);
        free_bytes = f > held ? f - held : 0;
    } else {
        free_bytes = fr;
    }
    reserve = c->admission_reserve_bytes >= 0 ? size_t(c->admission_reserve_bytes)
                                              : std::max<size_t>(size_t(1) << 30, total / 50);
    return MTLG_OK;
}

inline int srv_engine_init(mtlg_server* S, int e)
{
    mtlg_ctx* c = S->ctx;
    auto& E = S->eng[e];
    E.solver = e == 0 ? MTLG_CG : MTLG_BICGSTAB;
    SolveSet& ss = E.ss;
    ss.ctx = c;
    ss.S = S->o.max_active;
    ss.solver = E.solver;
    ss.f32 = S->refine ? 1 : 0;
    ss.mixed = S->refine ? 1 : 0;
    ss.path = PATH_SWEEP;
    ss.pc_f32 = S->refine ? 1 : 0;
    E.slot_req.assign(ss.S, -1);
    MTLG_TRY(ss.desc.alloc(c, ss.S));
    MTLG_TRY(ss.desc64.alloc(c, ss.S));
    MTLG_TRY(ss.st.alloc(c, ss.S));
    MTLG_TRY(ss.counters.alloc(c, ss.S));
    MTLG_TRY(ss.misc.alloc(c, 4));
    MTLG_TRY(ss.tickets.alloc(c, 8));
    MTLG_CUDA(cudaMemsetAsync(ss.counters.p, 0, sizeof(unsigned) * ss.S, c->stream));
    MTLG_CUDA(cudaMemsetAsync(ss.misc.p, 0, 4 * sizeof(int), c->stream));
    MTLG_CUDA(cudaMemsetAsync(ss.tickets.p, 0, 8 * sizeof(int), c->stream));
    std::vector<SysState> st(ss.S);
    for (auto& s : st) {
        memset(&s, 0, sizeof s);
        s.phase = PH_DONE;
        s.status = -1;
        s.ostatus = -1;
    }
    MTLG_CUDA(cudaMemcpyAsync(ss.st.p, st.data(), sizeof(SysState) * ss.S, cudaMemcpyHostToDevice, c->stream));
    ss.h_desc.assign(ss.S, SysDesc{});
    ss.h_desc64.assign(ss.S, SysDesc{});
    for (auto& d : ss.h_desc) memset(&d, 0, sizeof d);
    for (auto& d : ss.h_desc64) memset(&d, 0, sizeof d);
    return MTLG_OK;
}

// Device objects and slot state of an admitted request.
inline int srv_admit(mtlg_server* S, mtlg_server::Req& R, int e, int slot)
{
    mtlg_ctx* c = S->ctx;
    auto& E = S->eng[e];
    SolveSet& ss = E.ss;
    MTLG_TRY(mtlg_csr_create(c, R.n, R.n, R.nnz, R.rp.data(), R.ci.data(), R.val.data(), MTLG_F64, &R.A));
    MTLG_TRY(mtlg_pc_create(c, R.A, R.pc, S->refine ? MTLG_F32 : MTLG_F64, &R.P));
    MTLG_TRY(R.x.alloc(c, size_t(std::max<int64_t>(1, R.n))));
    MTLG_CUDA(cudaMemsetAsync(R.x.p, 0, size_t(R.n) * 8, c->stream));
    MTLG_TRY(R.bd.upload(c, R.b.data(), size_t(R.n)));
    const long long stride = (long long)round_up(size_t(std::max<int64_t>(1, R.n)), 64);
    const size_t vb = vsize(ss.f32);
    MTLG_TRY(R.ws.alloc(c, size_t(stride) * kNumVec * vb));
    MTLG_CUDA(cudaMemsetAsync(R.ws.p, 0, size_t(stride) * kNumVec * vb, c->stream));
    MTLG_TRY(fill_sentinel(c, R.ws.p + size_t(V_Z0) * stride * vb, size_t(stride) * vb));
    if (S->refine) MTLG_TRY(R.ws64.alloc(c, size_t(stride)));
    if (ss.f32) MTLG_TRY(ensure_f32_values(R.A));

    SysDesc& d = ss.h_desc[slot];
    memset(&d, 0, sizeof d);
    d.n = int(R.n);
    d.nnz = int(R.nnz);
    d.rp = R.A->rp.p;
    d.ci = R.A->ci.p;
    d.val = ss.f32 ? (const void*)R.A->v32.p : (const void*)R.A->v64.p;
    d.val64 = R.A->v64.p;
    d.ws = R.ws.p;
    d.ws_stride = stride;
    d.pc = R.P->kind;
    if (R.P->kind == MTLG_PC_DIAGONAL) d.inv_diag = R.P->inv_diag.p;
    MTLG_TRY(pc_views(R.P, ss.f32, d.L, d.U));
    if (S->refine) {
        d.x = R.ws.p + size_t(V_W1) * stride * vb;
        d.b = R.ws.p + size_t(V_W0) * stride * vb;
        d.x64 = R.x.p;
        d.b64 = R.bd.p;
        d.r64 = R.ws64.p;
        SysDesc& d64 = ss.h_desc64[slot];
        d64 = d;
        d64.val = R.A->v64.p;
        d64.x = R.x.p;
        d64.b = R.bd.p;
        d64.ws = R.ws64.p;
        d64.ws_stride = 0;
    } else {
        d.x = R.x.p;
        d.b = R.bd.p;
    }
    SysState st;
    memset(&st, 0, sizeof st);
    st.max_iter = R.max_iter;
    st.atol = 0.0;
    if (S->refine) {
        st.rtol = S->o.inner_rtol;
        st.outer_rtol = S->o.rtol;
        st.max_outer = 20;
        st.inner_rtol = S->o.inner_rtol;
        st.nb = R.nb;
        st.phase = PH_OUTER;
        st.status = -1;
        st.ostatus = MTLG_ST_RUNNING;
    } else {
        st.rtol = S->o.rtol;
        st.norm_r0 = R.nb;
        st.phase = PH_INIT;
        st.status = MTLG_ST_RUNNING;
        st.ostatus = MTLG_ST_RUNNING;
    }
    MTLG_CUDA(cudaMemcpyAsync(ss.st.p + slot, &st, sizeof st, cudaMemcpyHostToDevice, c->stream));
    E.slot_req[slot] = R.id;
    E.nactive++;
    E.dirty = true;
    R.state = 1;
    R.engine = e;
    R.slot = slot;
    return MTLG_OK;
}

// Tiles and merged sweep schedules of the active slots; the loop body of
// `iters_per_step` iterations captured once per membership.
inline int srv_rebuild(mtlg_server* S, int e)
{
    mtlg_ctx* c = S->ctx;
    auto& E = S->eng[e];
    SolveSet& ss = E.ss;
    std::vector<Tile> tiles;
    std::vector<int> stb(ss.S + 1, 0);
    int maxlev = 0;
    for (int s = 0; s < ss.S; ++s) {
        if (E.slot_req[s] >= 0) {
            auto& R = *S->reqs[E.slot_req[s]];
            plan_tiles(R.A->h_rp.data(), int(R.n), s, tiles);
            maxlev = std::max({maxlev, R.P->L.nlev, R.P->U.nlev});
        }
        stb[s + 1] = int(tiles.size());
    }
    ss.n_tiles = int(tiles.size());
    MTLG_TRY(ss.tiles.upload(c, tiles.data(), std::max<size_t>(1, tiles.size())));
    MTLG_TRY(ss.stb.upload(c, stb.data(), stb.size()));
    MTLG_TRY(ss.partials.alloc(c, size_t(std::max(1, ss.n_tiles)) * kMaxDots));
    std::vector<SweepTask> tl, tu;
    for (int l = 0; l < maxlev; ++l) {
        for (int s = 0; s < ss.S; ++s) {
            if (E.slot_req[s] < 0) continue;
            auto& R = *S->reqs[E.slot_req[s]];
            const TriDev& L = R.P->L;
            if (l < L.nlev)
                for (int t = L.lev_task_begin[l]; t < L.lev_task_begin[l + 1]; ++t) tl.push_back({s, t * kSweepRows});
            const TriDev& U = R.P->U;
            if (l < U.nlev)
                for (int t = U.lev_task_begin[l]; t < U.lev_task_begin[l + 1]; ++t) tu.push_back({s, t * kSweepRows});
        }
    }
    ss.ntl = int(tl.size());
    ss.ntu = int(tu.size());
    MTLG_TRY(ss.tl.upload(c, tl.data(), std::max<size_t>(1, tl.size())));
    MTLG_TRY(ss.tu.upload(c, tu.data(), std::max<size_t>(1, tu.size())));
    {
        std::vector<const mtlg_pc*> pcs(ss.S, nullptr);
        for (int s = 0; s < ss.S; ++s)
            if (E.slot_req[s] >= 0) pcs[s] = S->reqs[E.slot_req[s]]->P;
        MTLG_TRY(plan_set_chunks(ss, pcs));
        if (!ss.cplan.ok) {
            // flat sweeps: every active preconditioner's flat entries, and
            // its views refreshed in both descriptors
            for (int s = 0; s < ss.S; ++s) {
                if (!pcs[s]) continue;
                mtlg_pc* P = const_cast<mtlg_pc*>(pcs[s]);
                MTLG_TRY(ensure_flat(P));
                MTLG_TRY(pc_views(P, ss.f32, ss.h_desc[s].L, ss.h_desc[s].U));
                ss.h_desc64[s].L = ss.h_desc[s].L;
                ss.h_desc64[s].U = ss.h_desc[s].U;
            }
        }
    }
    MTLG_CUDA(cudaMemcpyAsync(ss.desc.p, ss.h_desc.data(), sizeof(SysDesc) * ss.S, cudaMemcpyHostToDevice, c->stream));
    MTLG_CUDA(cudaMemcpyAsync(ss.desc64.p, ss.h_desc64.data(), sizeof(SysDesc) * ss.S, cudaMemcpyHostToDevice,
                              c->stream));
    // capture the inner iterations of one step
    if (E.exec) { cudaGraphExecDestroy(E.exec); E.exec = nullptr; }
    if (E.graph) { cudaGraphDestroy(E.graph); E.graph = nullptr; }
    if (!ss.cap_stream) MTLG_CUDA(cudaStreamCreateWithFlags(&ss.cap_stream, cudaStreamNonBlocking));
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    const int64_t before = c->launches;
    MTLG_CUDA(cudaStreamBeginCapture(ss.cap_stream, cudaStreamCaptureModeThreadLocal));
    const SetView sv = ss.view(false, false);
    int st = MTLG_OK;
    const int bodies = std::max(1, S->o.iters_per_step / iters_per_body(ss));
    for (int k = 0; k < bodies && st == MTLG_OK; ++k)
        st = ss.f32 ? enqueue_body<float>(ss, ss.cap_stream, sv) : enqueue_body<double>(ss, ss.cap_stream, sv);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(ss.cap_stream, &g);
    E.body_kernels = int(c->launches - before);
    c->launches = before;
    if (st != MTLG_OK) return st;
    MTLG_CUDA(ce);
    E.graph = g;
    MTLG_CUDA(cudaGraphInstantiate(&E.exec, g, 0));
    E.dirty = false;
    return MTLG_OK;
}

inline double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace mtlg

extern "C" {

int mtlg_server_create(mtlg_ctx* c, const mtlg_server_opts* opts, mtlg_server** out)
{
    MTLG_CHECK_ARG(c && opts && out, "ctx/opts/out");
    MTLG_CHECK_ARG(opts->max_active > 0 && opts->max_active <= 4096, "max_active in 1..4096");
    MTLG_CHECK_ARG(opts->precision == MTLG_F64 || opts->precision == MTLG_F32, "precision");
    std::unique_ptr<mtlg_server> S(new mtlg_server);
    S->ctx = c;
    S->o = *opts;
    if (S->o.iters_per_step <= 0) S->o.iters_per_step = 16;
    if (S->o.rtol <= 0) S->o.rtol = 1e-8;
    if (S->o.inner_rtol <= 0) S->o.inner_rtol = 1e-4;
    S->refine = opts->precision == MTLG_F32;
    MTLG_TRY(srv_engine_init(S.get(), 0));
    MTLG_TRY(srv_engine_init(S.get(), 1));
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    *out = S.release();
    return MTLG_OK;
}

int mtlg_server_admission(size_t request_bytes, size_t held_bytes, size_t budget, size_t free_bytes,
                          size_t reserve_bytes)
{
    return admission_decision(request_bytes, held_bytes, budget, free_bytes, reserve_bytes);
}

int mtlg_server_destroy(mtlg_server* S)
{
    if (!S) return MTLG_OK;
    cudaStreamSynchronize(S->ctx->stream);
    delete S;
    return MTLG_OK;
}

int mtlg_server_submit(mtlg_server* S, int64_t n, int64_t nnz, const int64_t* row_ptr, const int32_t* col,
                       const double* val, const double* b, int solver, int pc_kind, int max_iter, int64_t* id)
{
    MTLG_TRACE(9132, "server.submit");
    MTLG_CHECK_ARG(S && row_ptr && b && id && n > 0 && nnz >= 0, "server/arrays/id");
    MTLG_CHECK_ARG(solver == MTLG_CG || solver == MTLG_BICGSTAB, "served solver must be CG or BiCGSTAB");
    MTLG_CHECK_ARG(pc_kind == MTLG_PC_DIAGONAL || pc_kind == MTLG_PC_ILU0 || pc_kind == MTLG_PC_IC0,
                   "served preconditioner must be diagonal, ILU(0) or IC(0)");
    S->stats.submitted++;
    const size_t est = srv_estimate(n, nnz, S->refine);
    size_t fr = 0, reserve = 0;
    if (!S->o.hbm_budget) MTLG_TRY(free_memory(S->ctx, S->bytes_held, fr, reserve));
    if (admission_decision(est, S->bytes_held, S->o.hbm_budget, fr, reserve) < 0) {
        S->stats.rejected++;
        if (S->o.hbm_budget) set_error("request needs ~%zu bytes, the server budget is %zu", est, S->o.hbm_budget);
        else set_error("request needs ~%zu bytes, the device has %zu free (%zu reserved) and the server holds %zu",
                       est, fr, reserve, S->bytes_held);
        return MTLG_ERR_ADMISSION;
    }
    std::unique_ptr<mtlg_server::Req> R(new mtlg_server::Req);
    R->id = S->next_id++;
    R->n = n;
    R->nnz = nnz;
    R->rp.assign(row_ptr, row_ptr + n + 1);
    R->ci.assign(col, col + nnz);
    R->val.assign(val, val + nnz);
    R->b.assign(b, b + n);
    double nb = 0;
    for (int64_t i = 0; i < n; ++i) nb += b[i] * b[i];
    R->nb = sqrt(nb);
    R->solver = solver;
    R->pc = pc_kind;
    R->max_iter = max_iter > 0 ? max_iter : 1000;
    R->est = est;
    R->res.iterations = 0;
    *id = R->id;
    S->queue.push_back(R->id);
    S->reqs[R->id] = std::move(R);
    return MTLG_OK;
}

int mtlg_server_step(mtlg_server* S)
{
    MTLG_TRACE(9130, "server.step");
    MTLG_CHECK_ARG(S, "server");
    mtlg_ctx* c = S->ctx;
    S->stats.steps++;
    TracePhases ph;
    ph.next(9133, "server.harvest");
    // 1. harvest finished slots
    for (int e = 0; e < 2; ++e) {
        auto& E = S->eng[e];
        if (E.nactive == 0) continue;
        SolveSet& ss = E.ss;
        std::vector<SysState> st(ss.S);
        MTLG_CUDA(cudaMemcpyAsync(st.data(), ss.st.p, sizeof(SysState) * ss.S, cudaMemcpyDeviceToHost, c->stream));
        int flag = 0;
        MTLG_CUDA(cudaMemcpyAsync(&flag, ss.misc.p + 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        MTLG_CUDA(cudaStreamSynchronize(c->stream));
        for (int s = 0; s < ss.S; ++s) {
            if (E.slot_req[s] < 0 || st[s].phase != PH_DONE) continue;
            auto& R = *S->reqs[E.slot_req[s]];
            if (R.state == 1) {
                fill_result(st[s], S->refine, &R.res);
                if (!S->refine) R.res.norm_r0 = R.nb, R.res.relresid = R.nb ? st[s].resid / R.nb : st[s].resid;
                if (S->refine && needs_fp64_finish(R.res) && !flag) {
                    // the FP32-inner refinement stalled or broke down: finish in FP64
                    mtlg_refine_params rp{};
                    rp.max_outer = 20;
                    rp.max_inner = R.max_iter;
                    rp.rtol = S->o.rtol;
                    MTLG_TRACE(9137, "server.fp64_finish");
                    MTLG_TRY(fp64_finish(c, R.solver, R.A, R.P, R.x.p, R.bd.p, fp64_budget(rp, R.res.iterations),
                                         S->o.rtol, R.res));
                }
                R.xh.resize(size_t(R.n));
                MTLG_CUDA(cudaMemcpy(R.xh.data(), R.x.p, size_t(R.n) * 8, cudaMemcpyDeviceToHost));
                R.res.seconds = 0;
                R.state = 2;
                R.status_code = flag ? MTLG_ERR_TIMEOUT : MTLG_OK;
                S->stats.completed++;
            }
            S->bytes_held -= std::min(S->bytes_held, R.est);
            R.release();
            const int64_t rid = E.slot_req[s];
            E.slot_req[s] = -1;
            E.nactive--;
            E.dirty = true;
            if (R.state == 3) S->reqs.erase(rid);
        }
        if (flag) {
            int z = 0;
            MTLG_CUDA(cudaMemcpy(ss.misc.p + 1, &z, sizeof z, cudaMemcpyHostToDevice));
            MTLG_CUDA(cudaMemset(ss.tickets.p, 0, 8 * sizeof(int)));
            MTLG_TRY(reset_set_sweep_buffers(ss));
        }
    }
    // 2. admit queued requests while slots and memory allow
    ph.next(9134, "server.admit");
    while (!S->queue.empty()) {
        const int64_t id = S->queue.front();
        auto it = S->reqs.find(id);
        if (it == S->reqs.end() || it->second->state != 0) {
            S->queue.pop_front();
            continue;
        }
        auto& R = *it->second;
        const int e = R.solver == MTLG_CG ? 0 : 1;
        auto& E = S->eng[e];
        int slot = -1;
        for (int s = 0; s < E.ss.S; ++s) if (E.slot_req[s] < 0) { slot = s; break; }
        if (slot < 0) break;
        size_t fr = 0, reserve = 0;
        if (!S->o.hbm_budget) MTLG_TRY(free_memory(c, S->bytes_held, fr, reserve));
        const int adm = admission_decision(R.est, S->bytes_held, S->o.hbm_budget, fr, reserve);
        if (adm == 0) break;   // waits for active requests to retire
        S->queue.pop_front();
        if (adm < 0) {
            R.state = 4;
            R.status_code = MTLG_ERR_ADMISSION;
            S->stats.rejected++;
            continue;
        }
        int st = srv_admit(S, R, e, slot);
        if (st != MTLG_OK) {
            R.release();
            E.slot_req[slot] = -1;
            if (st == MTLG_ERR_OOM) {   // not now: back to the queue head
                S->queue.push_front(id);
                break;
            }
            R.state = 4;
            R.status_code = st;
            S->stats.rejected++;
            continue;
        }
        S->bytes_held += R.est;
        S->stats.admitted++;
    }
    // 3. run one step of every active engine
    for (int e = 0; e < 2; ++e) {
        auto& E = S->eng[e];
        if (E.nactive == 0) continue;
        if (E.dirty) {
            ph.next(9135, "server.rebuild");
            MTLG_TRY(srv_rebuild(S, e));
        }
        ph.next(9136, "server.launch");
        SolveSet& ss = E.ss;
        const SetView sv = ss.view(false, false);
        if (S->refine) {
            const SetView v64 = ss.view(false, true);
            SpmvOp r = spmv_op_default();
            r.x = SLOT_X; r.w = SLOT_B; r.y = 0;
            set_dot(r, 0, OPND_Y, OPND_Y);
            r.fin = FIN_REF_OUTER;
            r.skip = SKIP_PH_BASE + PH_OUTER;
            MTLG_TRY(launch_spmv<double>(c, c->stream, v64, r, XF_PLAIN, ASG_WMINUS));
            if (E.solver == MTLG_CG) MTLG_TRY(cg_init<float>(ss, c->stream, sv, true, SKIP_PH_BASE + PH_CAST));
            else MTLG_TRY(bicg_init<float>(ss, c->stream, sv, true, SKIP_PH_BASE + PH_CAST));
        } else {
            if (E.solver == MTLG_CG) MTLG_TRY(cg_init<double>(ss, c->stream, sv, false, SKIP_PH_BASE + PH_INIT));
            else MTLG_TRY(bicg_init<double>(ss, c->stream, sv, false, SKIP_PH_BASE + PH_INIT));
        }
        MTLG_CUDA(cudaGraphLaunch(E.exec, c->stream));
        c->launches += E.body_kernels;
        if (S->refine) {
            VecOp up = vec_op_default(VOP_REF_UPDATE);
            up.a = SLOT_X;
            up.skip = SKIP_PH_BASE + PH_UPDATE;
            up.fin = FIN_PHASE_OUTER;
            MTLG_TRY(launch_vec<float>(c, c->stream, sv, up));
        }
        MTLG_CUDA(cudaGetLastError());
    }
    return MTLG_OK;
}

int mtlg_server_poll(mtlg_server* S, int64_t id, double* x_host, mtlg_iter_result* result)
{
    MTLG_CHECK_ARG(S, "server");
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) {
        set_error("unknown request %lld", (long long)id);
        return MTLG_ERR_NOT_FOUND;
    }
    auto& R = *it->second;
    if (R.state == 0 || R.state == 1) return MTLG_PENDING;
    if (R.state == 3) {
        set_error("request %lld was cancelled", (long long)id);
        return MTLG_ERR_NOT_FOUND;
    }
    if (R.state == 4) return R.status_code;
    if (x_host) memcpy(x_host, R.xh.data(), size_t(R.n) * 8);
    if (result) *result = R.res;
    const int st = R.status_code;
    S->reqs.erase(it);
    return st;
}

int mtlg_server_cancel(mtlg_server* S, int64_t id)
{
    MTLG_CHECK_ARG(S, "server");
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return MTLG_ERR_NOT_FOUND;
    auto& R = *it->second;
    if (R.state == 1) {
        // stop the slot's device work: the next step retires it
        auto& E = S->eng[R.engine];
        const int ph = PH_DONE;
        MTLG_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(E.ss.st.p + R.slot) + offsetof(SysState, phase), &ph,
                                  sizeof ph, cudaMemcpyHostToDevice, S->ctx->stream));
        const int rs = -2;
        MTLG_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(E.ss.st.p + R.slot) + offsetof(SysState, status), &rs,
                                  sizeof rs, cudaMemcpyHostToDevice, S->ctx->stream));
        MTLG_CUDA(cudaStreamSynchronize(S->ctx->stream));
    }
    R.state = 3;
    S->stats.cancelled++;
    return MTLG_OK;
}

int mtlg_server_stats_get(const mtlg_server* S, mtlg_server_stats* st)
{
    MTLG_CHECK_ARG(S && st, "server/stats");
    *st = S->stats;
    int64_t active = 0, queued = 0;
    for (auto& kv : S->reqs) {
        active += kv.second->state == 1;
        queued += kv.second->state == 0;
    }
    st->active = active;
    st->queued = queued;
    st->bytes_in_use = S->bytes_held;
    return MTLG_OK;
}

}  // extern "C"
