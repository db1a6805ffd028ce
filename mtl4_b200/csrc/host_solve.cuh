// Host side: the solver engine.  A SolveSet is a set of independent systems
// advanced together; a single mtlg_solve is a set of one.  The init kernels
// run once; the loop body is captured into a CUDA graph whose WHILE node
// repeats it until no system is running, so a whole solve costs one graph
// launch and no host round trip per iteration.
#pragma once
#include "host_pc.cuh"

namespace mtlg {

enum Path : int { PATH_IDENTITY = 0, PATH_JACOBI = 1, PATH_SWEEP = 2 };

struct SysInput {
    mtlg_csr* A = nullptr;
    mtlg_pc* P = nullptr;        // null: identity
    void* x = nullptr;           // plain: T vector; refinement: FP64
    const void* b = nullptr;
    int max_iter = 0;
    double rtol = 0, atol = 0, norm_r0 = -1;
    double* log = nullptr;       // device residual log (2 * log_cap doubles) or null
    int log_cap = 0;
};

struct SolveSet {
    mtlg_ctx* ctx = nullptr;
    int S = 0;
    int solver = MTLG_CG;
    int f32 = 0;          // inner vectors are FP32
    int mixed = 0;        // FP64 refinement around the inner solve
    int path = PATH_IDENTITY;
    int pc_f32 = 0;       // storage type of the factors (sweep path)
    std::vector<SysInput> in;
    std::vector<SysDesc> h_desc, h_desc64;
    DBuf<SysDesc> desc, desc64;
    DBuf<SysState> st;
    int n_tiles = 0;
    DBuf<Tile> tiles;
    DBuf<int> stb;
    DBuf<double> partials;
    DBuf<unsigned> counters;
    DBuf<int> misc;       // [0] running, [1] timeout flag, [2] body runs, [3] body cap
    DBuf<SweepTask> tl, tu;
    int ntl = 0, ntu = 0;
    // chunked sweeps: groups of chunks of all systems
    ChunkPlan cplan;
    DBuf<int> tickets;
    DBuf<unsigned char> ws, ws64;
    long long stride = 0;
    // graph of the loop body
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long cond = 0;
    int body_kernels = 0;
    int iters_per_body = 1;
    bool graph_failed = false;
    // chunked loop: kChunkBodies bodies in a plain graph, two chunks in flight
    cudaGraph_t chunk_graph = nullptr;
    cudaGraphExec_t chunk_exec = nullptr;
    int chunk_kernels = 0;
    int* h_running = nullptr;       // pinned host copies of the running count
    cudaEvent_t chunk_ev[2] = {nullptr, nullptr};
    ~SolveSet()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (chunk_exec) cudaGraphExecDestroy(chunk_exec);
        if (chunk_graph) cudaGraphDestroy(chunk_graph);
        if (h_running) cudaFreeHost(h_running);
        for (auto& e : chunk_ev) if (e) cudaEventDestroy(e);
        if (cap_stream) cudaStreamDestroy(cap_stream);
    }

    SetView view(bool in_graph, bool outer64) const
    {
        SetView v;
        v.tiles = tiles.p;
        v.n_tiles = n_tiles;
        v.n_sys = S;
        v.sys_tile_begin = stb.p;
        v.desc = outer64 ? desc64.p : desc.p;
        v.st = st.p;
        v.partials = partials.p;
        v.counters = counters.p;
        v.running = misc.p;
        v.err = misc.p + 1;
        v.cond = in_graph ? cond : 0;
        v.use_cond = in_graph ? 1 : 0;
        v.spin = ctx ? ctx->spin_limit : 0;
        return v;
    }
};

// After an expired device wait: the L sweeps' output (V_Z0) back to all
// sentinel, as the flat and grid sweeps expect before a sweep (the L sweep
// itself resets the U sweeps' outputs row by row).
inline int reset_set_sweep_buffers(SolveSet& ss)
{
    if (ss.path != PATH_SWEEP) return MTLG_OK;
    const size_t vb = ss.f32 ? 4 : 8;
    for (int s = 0; s < ss.S && s < int(ss.h_desc.size()); ++s)
        if (ss.h_desc[s].ws && ss.h_desc[s].ws_stride > 0)
            MTLG_TRY(fill_sentinel(ss.ctx,
                                   static_cast<unsigned char*>(ss.h_desc[s].ws) + size_t(V_Z0) * size_t(ss.h_desc[s].ws_stride) * vb,
                                   size_t(ss.h_desc[s].ws_stride) * vb));
    return MTLG_OK;
}

inline int plan_set_chunks(SolveSet& ss, const std::vector<const mtlg_pc*>& pcs);

inline size_t vsize(int f32) { return f32 ? 4 : 8; }

// Builds the set: tiling, descriptors, workspace, merged sweep schedules.
inline int build_set(mtlg_ctx* c, SolveSet& ss)
{
    MTLG_TRACE(9140, "set.build");
    ss.ctx = c;
    ss.S = int(ss.in.size());
    std::vector<Tile> tiles;
    std::vector<int> stb(ss.S + 1, 0);
    long long maxn = 1;
    bool all_identity = true, all_jacobi = true;
    for (int s = 0; s < ss.S; ++s) {
        const SysInput& si = ss.in[s];
        plan_tiles(si.A->h_rp.data(), int(si.A->n_rows), s, tiles);
        stb[s + 1] = int(tiles.size());
        maxn = std::max<long long>(maxn, si.A->n_rows);
        const int kind = si.P ? si.P->kind : MTLG_PC_IDENTITY;
        if (kind != MTLG_PC_IDENTITY) all_identity = false;
        if (kind != MTLG_PC_DIAGONAL) all_jacobi = false;
        if (si.P && (si.P->kind == MTLG_PC_DIAGONAL || si.P->has_factors())) ss.pc_f32 = si.P->storage == MTLG_F32;
    }
    ss.path = all_identity ? PATH_IDENTITY : (all_jacobi && ss.S == 1 && ss.pc_f32 == ss.f32 ? PATH_JACOBI : PATH_SWEEP);
    if (ss.path == PATH_SWEEP) {
        for (int s = 0; s < ss.S; ++s) {
            const mtlg_pc* P = ss.in[s].P;
            if (!P || P->kind == MTLG_PC_IDENTITY || (P->storage == MTLG_F32) != bool(ss.pc_f32)) {
                set_error("a batch with triangular/diagonal preconditioners needs one PC per system with one storage type");
                return MTLG_ERR_NOT_SUPPORTED;
            }
        }
    }
    if (ss.path == PATH_SWEEP) {
        // the chunked-sweep plan first: without one the set sweeps in flat
        // level order, which needs every preconditioner's flat entries before
        // its views go into the descriptors
        std::vector<const mtlg_pc*> pcs(ss.S);
        for (int s = 0; s < ss.S; ++s) pcs[s] = ss.in[s].P;
        MTLG_TRY(plan_set_chunks(ss, pcs));
        if (!ss.cplan.ok)
            for (int s = 0; s < ss.S; ++s) MTLG_TRY(ensure_flat(const_cast<mtlg_pc*>(ss.in[s].P)));
    }
    ss.n_tiles = int(tiles.size());
    MTLG_TRY(ss.tiles.upload(c, tiles.data(), std::max<size_t>(1, tiles.size())));
    MTLG_TRY(ss.stb.upload(c, stb.data(), stb.size()));
    MTLG_TRY(ss.partials.alloc(c, size_t(std::max(1, ss.n_tiles)) * kMaxDots));
    MTLG_TRY(ss.counters.alloc(c, ss.S));
    MTLG_CUDA(cudaMemsetAsync(ss.counters.p, 0, sizeof(unsigned) * ss.S, c->stream));
    MTLG_TRY(ss.misc.alloc(c, 4));
    MTLG_CUDA(cudaMemsetAsync(ss.misc.p, 0, 4 * sizeof(int), c->stream));
    MTLG_TRY(ss.tickets.alloc(c, 8));
    MTLG_CUDA(cudaMemsetAsync(ss.tickets.p, 0, 8 * sizeof(int), c->stream));
    MTLG_TRY(ss.st.alloc(c, ss.S));

    // workspace arena: system s owns kNumVec vectors of stride[s] elements
    std::vector<long long> off(ss.S + 1, 0);
    std::vector<long long> strides(ss.S);
    for (int s = 0; s < ss.S; ++s) {
        strides[s] = (long long)round_up(size_t(std::max<int64_t>(1, ss.in[s].A->n_rows)), 64);
        off[s + 1] = off[s] + strides[s] * kNumVec;
    }
    MTLG_TRY(ss.ws.alloc(c, size_t(off[ss.S]) * vsize(ss.f32)));
    if (ss.mixed) MTLG_TRY(ss.ws64.alloc(c, size_t(off[ss.S] / kNumVec) * 8));
    MTLG_CUDA(cudaMemsetAsync(ss.ws.p, 0, size_t(off[ss.S]) * vsize(ss.f32), c->stream));

    ss.h_desc.assign(ss.S, SysDesc{});
    ss.h_desc64.assign(ss.S, SysDesc{});
    for (int s = 0; s < ss.S; ++s) {
        const SysInput& si = ss.in[s];
        SysDesc& d = ss.h_desc[s];
        memset(&d, 0, sizeof d);
        d.n = int(si.A->n_rows);
        d.nnz = int(si.A->nnz);
        d.rp = si.A->rp.p;
        d.ci = si.A->ci.p;
        if (ss.f32) {
            MTLG_TRY(ensure_f32_values(si.A));
            d.val = si.A->v32.p;
        } else {
            d.val = si.A->v64.p;
        }
        d.val64 = si.A->v64.p;
        d.ws = ss.ws.p + size_t(off[s]) * vsize(ss.f32);
        d.ws_stride = strides[s];
        d.pc = si.P ? si.P->kind : MTLG_PC_IDENTITY;
        if (si.P && si.P->kind == MTLG_PC_DIAGONAL) d.inv_diag = si.P->inv_diag.p;
        if (si.P && (si.P->kind == MTLG_PC_DIAGONAL || si.P->has_factors())) {
            MTLG_TRY(pc_views(si.P, ss.f32, d.L, d.U));
        }
        if (ss.mixed) {
            // inner problem: x = d (slot V_W1), b = float(r / ||r||) (slot V_W0)
            d.x = static_cast<unsigned char*>(d.ws) + size_t(V_W1) * strides[s] * vsize(ss.f32);
            d.b = static_cast<unsigned char*>(d.ws) + size_t(V_W0) * strides[s] * vsize(ss.f32);
            d.x64 = static_cast<double*>(si.x);
            d.b64 = static_cast<const double*>(si.b);
            d.r64 = reinterpret_cast<double*>(ss.ws64.p) + off[s] / kNumVec;
            SysDesc& e = ss.h_desc64[s];
            e = d;
            e.val = si.A->v64.p;
            e.x = si.x;
            e.b = si.b;
            e.ws = d.r64;       // slot 0 of the FP64 view is r64
            e.ws_stride = 0;
        } else {
            d.x = si.x;
            d.b = si.b;
        }
    }
    MTLG_TRY(ss.desc.upload(c, ss.h_desc.data(), ss.S));
    if (ss.mixed) MTLG_TRY(ss.desc64.upload(c, ss.h_desc64.data(), ss.S));

    // sweep buffers start all-sentinel (V_Z0; V_Z / V_PHAT / V_SHAT are reset
    // row by row by the L sweep before the U sweep writes them)
    if (ss.path == PATH_SWEEP) {
        for (int s = 0; s < ss.S; ++s) {
            const size_t vb = vsize(ss.f32);
            MTLG_TRY(fill_sentinel(c, static_cast<unsigned char*>(ss.h_desc[s].ws) + size_t(V_Z0) * strides[s] * vb,
                                   size_t(strides[s]) * vb));
        }
        // merged level order across systems
        int maxlev = 0;
        for (int s = 0; s < ss.S; ++s) maxlev = std::max({maxlev, ss.in[s].P->L.nlev, ss.in[s].P->U.nlev});
        std::vector<SweepTask> tl, tu;
        for (int l = 0; l < maxlev; ++l) {
            for (int s = 0; s < ss.S; ++s) {
                const TriDev& L = ss.in[s].P->L;
                if (l < L.nlev)
                    for (int t = L.lev_task_begin[l]; t < L.lev_task_begin[l + 1]; ++t) tl.push_back({s, t * kSweepRows});
                const TriDev& U = ss.in[s].P->U;
                if (l < U.nlev)
                    for (int t = U.lev_task_begin[l]; t < U.lev_task_begin[l + 1]; ++t) tu.push_back({s, t * kSweepRows});
            }
        }
        ss.ntl = int(tl.size());
        ss.ntu = int(tu.size());
        MTLG_TRY(ss.tl.upload(c, tl.data(), std::max<size_t>(1, tl.size())));
        MTLG_TRY(ss.tu.upload(c, tu.data(), std::max<size_t>(1, tu.size())));
    }
    return MTLG_OK;
}

// Chunked-sweep plan of the systems with a preconditioner (pcs[s] ==
// nullptr: slot unused); the set runs chunked sweeps only if every one of
// them has the chunked layout.
inline int plan_set_chunks(SolveSet& ss, const std::vector<const mtlg_pc*>& pcs)
{
    std::vector<std::pair<const TriDev*, const TriDev*>> f(pcs.size(), {nullptr, nullptr});
    for (size_t s = 0; s < pcs.size(); ++s)
        if (pcs[s]) f[s] = {&pcs[s]->L, &pcs[s]->U};
    if (ss.f32) {
        if (ss.pc_f32) return plan_chunks<float, float>(ss.ctx, f, ss.cplan);
        return plan_chunks<float, double>(ss.ctx, f, ss.cplan);
    }
    if (ss.pc_f32) return plan_chunks<double, float>(ss.ctx, f, ss.cplan);
    return plan_chunks<double, double>(ss.ctx, f, ss.cplan);
}

template <typename T>
inline int launch_sweep(SolveSet& ss, cudaStream_t st, const SetView& sv, int which, int in, int out, int reset,
                        int skip, int ticket)
{
    if (ss.cplan.ok) {   // planned when the set was built (no plan under sweep_kernel 1)
        ChunkSweepOp op;
        memset(&op, 0, sizeof op);
        op.tasks = which == 0 ? ss.cplan.tl.p : ss.cplan.tu.p;
        op.ntasks = which == 0 ? ss.cplan.ntl : ss.cplan.ntu;
        op.ticket = ss.tickets.p + 4 + ticket;
        op.which = which;
        op.in = in;
        op.out = out;
        op.reset = reset;
        op.skip = skip;
        op.sleep_ns = ss.ctx->sweep_sleep_ns;
        if (ss.pc_f32) return launch_chunk_sweep<T, float>(ss.ctx, st, sv, op, ss.cplan);
        return launch_chunk_sweep<T, double>(ss.ctx, st, sv, op, ss.cplan);
    }
    SweepOp op;
    memset(&op, 0, sizeof op);
    op.tasks = which == 0 ? ss.tl.p : ss.tu.p;
    op.ntasks = which == 0 ? ss.ntl : ss.ntu;
    op.ticket = ss.tickets.p + ticket;
    op.which = which;
    op.in = in;
    op.out = out;
    op.reset = reset;
    op.skip = skip;
    op.fuse = SWF_NONE;
    op.sleep_ns = ss.ctx->sweep_sleep_ns;
    if (op.ntasks == 0) return MTLG_OK;
    const int grid = ss.ctx->sweep_blocks();
    if (ss.pc_f32) k_sweep<T, float><<<grid, kBlock, 0, st>>>(sv, op);
    else k_sweep<T, double><<<grid, kBlock, 0, st>>>(sv, op);
    ss.ctx->launches++;
    MTLG_CUDA(cudaGetLastError());
    return MTLG_OK;
}

inline void set_dot(SpmvOp& op, int j, int a, int b, int c = OPND_ONE)
{
    op.da[j] = a; op.db[j] = b; op.dc[j] = c;
    op.ndot = std::max(op.ndot, j + 1);
}
inline void set_dot(VecOp& op, int j, int a, int b, int c = OPND_ONE)
{
    op.da[j] = a; op.db[j] = b; op.dc[j] = c;
    op.ndot = std::max(op.ndot, j + 1);
}
// The reference expression a dot stands for, which fixes its summation order
// under "reduction_order" 1 (RK_DOT4 unless set): mtl::dot, two_norm, or the
// lazy_dot / lazy_unary_dot of a fused expression.
template <typename OpT>
inline void set_kinds(OpT& op, int k0, int k1 = RK_DOT4)
{
    op.rk[0] = k0;
    op.rk[1] = k1;
}

// ------------------------------------------------------------------ CG
// Reference body (itl/krylov/cg.hpp:76-111):
//   z = solve(L, r); rho = r.z; p = z + (rho/rho_1) p (first: p = z);
//   (q = A p) || (alpha_1 = p.q); alpha = rho/alpha_1; x += alpha p;
//   (r -= alpha q) || (rr = r.r);  loop while !finished(sqrt(|rr|)).
// Identity PC: cg.hpp:40-71 (z = r).
template <typename T>
inline int cg_init(SolveSet& ss, cudaStream_t st, const SetView& sv, bool inner_refine, int skip = -1)
{
    mtlg_ctx* c = ss.ctx;
    if (inner_refine) {
        VecOp op = vec_op_default(VOP_REF_CAST);
        op.a = V_W0; op.b = SLOT_X; op.c = V_R;
        set_dot(op, 0, V_R, V_R);
        if (ss.path == PATH_JACOBI) { set_dot(op, 1, V_R, V_R, OPND_D); op.fin = FIN_REF_CG_INIT_JAC; }
        else op.fin = FIN_REF_CG_INIT;
        op.skip = skip >= 0 ? skip : SKIP_OUTER;
        return launch_vec<T>(c, st, sv, op);
    }
    SpmvOp op = spmv_op_default();
    op.x = SLOT_X; op.w = SLOT_B; op.y = V_R;
    set_dot(op, 0, OPND_Y, OPND_Y);      // rr = dot(r, r)
    if (ss.path == PATH_JACOBI) { set_dot(op, 1, OPND_Y, OPND_Y, OPND_D); op.fin = FIN_CG_INIT_JAC; }   // dot(r, z)
    else op.fin = FIN_CG_INIT;
    set_kinds(op, RK_DOT4, RK_DOT4);
    if (skip >= 0) op.skip = skip;
    return launch_spmv<T>(c, st, sv, op, XF_PLAIN, ASG_WMINUS);
}

template <typename T>
inline int cg_half(SolveSet& ss, cudaStream_t st, const SetView& sv, int pin, int pout, bool count)
{
    mtlg_ctx* c = ss.ctx;
    int zslot = V_R;
    int xf = XF_CG_P;
    if (ss.path == PATH_SWEEP) {
        MTLG_TRY(launch_sweep<T>(ss, st, sv, 0, V_R, V_Z0, V_Z, SKIP_INNER, 0));
        MTLG_TRY(launch_sweep<T>(ss, st, sv, 1, V_Z0, V_Z, V_Z0, SKIP_INNER, 1));
        VecOp d = vec_op_default(VOP_DOT);
        set_dot(d, 0, V_R, V_Z);   // rho = dot(r, z)
        set_kinds(d, RK_DOT4);
        d.fin = FIN_CG_RHO;
        d.skip = SKIP_INNER;
        d.count_body = 0;
        MTLG_TRY(launch_vec<T>(c, st, sv, d));
        zslot = V_Z;
    } else if (ss.path == PATH_JACOBI) {
        xf = XF_CG_P_JAC;
    }
    SpmvOp op = spmv_op_default();
    op.z = zslot; op.p = pin; op.pnew = pout; op.y = V_Q;
    set_dot(op, 0, OPND_XP, OPND_Y);   // (q = A p) || (alpha_1 = lazy_dot(p, q))
    set_kinds(op, RK_LDOT4);
    op.fin = FIN_CG_ALPHA;
    op.skip = SKIP_INNER;
    op.count_body = count ? 1 : 0;
    MTLG_TRY(launch_spmv<T>(c, st, sv, op, xf, ASG_SET));
    VecOp u = vec_op_default(VOP_CG_UPDATE);
    u.a = SLOT_X; u.b = pout; u.c = V_R; u.e = V_Q;
    set_dot(u, 0, V_R, V_R);   // (r -= alpha q) || (rr = lazy_unary_dot(r))
    if (ss.path == PATH_JACOBI) { set_dot(u, 1, V_R, V_R, OPND_D); u.fin = FIN_CG_UPDATE_JAC; }   // dot(r, z)
    else if (ss.path == PATH_IDENTITY) u.fin = FIN_CG_UPDATE;
    else u.fin = FIN_CG_UPDATE_PC;
    set_kinds(u, RK_UDOT4, RK_DOT4);
    u.skip = SKIP_INNER;
    return launch_vec<T>(c, st, sv, u);
}

// ------------------------------------------------------------------ BiCGSTAB
// Reference body (itl/krylov/bicgstab.hpp:29-77), see k_vec VOP_BI_* and the
// FIN_BI_* finalize steps for the scalar updates and breakdown tests.
template <typename T>
inline int bicg_init(SolveSet& ss, cudaStream_t st, const SetView& sv, bool inner_refine, int skip = -1)
{
    mtlg_ctx* c = ss.ctx;
    if (inner_refine) {
        VecOp op = vec_op_default(VOP_REF_CAST);
        op.a = V_W0; op.b = SLOT_X; op.c = V_R; op.e = V_RT;
        set_dot(op, 0, V_RT, V_R);
        set_dot(op, 1, V_R, V_R);
        op.fin = FIN_REF_BI_INIT;
        op.skip = skip >= 0 ? skip : SKIP_OUTER;
        return launch_vec<T>(c, st, sv, op);
    }
    SpmvOp op = spmv_op_default();
    op.x = SLOT_X; op.w = SLOT_B; op.y = V_R; op.y2 = V_RT;   // r = b - A x; rtilde = r
    set_dot(op, 0, OPND_Y, OPND_Y);   // rho_1 = dot(rtilde, r)
    set_dot(op, 1, OPND_Y, OPND_Y);   // finished(r): two_norm(r)
    set_kinds(op, RK_DOT4, RK_NORM4);
    op.fin = FIN_BI_TOP;
    if (skip >= 0) op.skip = skip;
    return launch_spmv<T>(c, st, sv, op, XF_PLAIN, ASG_WMINUS);
}

template <typename T>
inline int bicg_body(SolveSet& ss, cudaStream_t st, const SetView& sv)
{
    mtlg_ctx* c = ss.ctx;
    // p = r + beta (p - omega v)
    VecOp pu = vec_op_default(VOP_BI_P);
    pu.a = V_P0; pu.b = V_R; pu.c = V_V;
    pu.skip = SKIP_INNER;
    pu.count_body = 1;
    MTLG_TRY(launch_vec<T>(c, st, sv, pu));
    // phat = solve(M, p); v = A phat; gamma = rtilde . v
    int xf = XF_PLAIN, xin = V_P0, pn = SLOT_NONE, phat = V_P0;
    if (ss.path == PATH_SWEEP) {
        MTLG_TRY(launch_sweep<T>(ss, st, sv, 0, V_P0, V_Z0, V_PHAT, SKIP_INNER, 0));
        MTLG_TRY(launch_sweep<T>(ss, st, sv, 1, V_Z0, V_PHAT, V_Z0, SKIP_INNER, 1));
        xin = V_PHAT; phat = V_PHAT;
    } else if (ss.path == PATH_JACOBI) {
        xf = XF_JAC; pn = V_PHAT; phat = V_PHAT;
    }
    SpmvOp v = spmv_op_default();
    v.x = xin; v.y = V_V; v.pnew = pn;
    set_dot(v, 0, V_RT, OPND_Y);   // gamma = dot(rtilde, v)
    set_kinds(v, RK_DOT4);
    v.fin = FIN_BI_GAMMA;
    v.skip = SKIP_INNER;
    MTLG_TRY(launch_spmv<T>(c, st, sv, v, xf, ASG_SET));
    // s = r - alpha v ; finished(s)?
    VecOp sop = vec_op_default(VOP_BI_S);
    sop.a = V_S; sop.b = V_R; sop.c = V_V;
    set_dot(sop, 0, V_S, V_S);   // finished(s): two_norm(s)
    set_kinds(sop, RK_NORM4);
    sop.fin = FIN_BI_S;
    sop.skip = SKIP_INNER;
    MTLG_TRY(launch_vec<T>(c, st, sv, sop));
    // shat = solve(M, s); t = A shat; omega = t.s / t.t
    int sin = V_S, sn = SLOT_NONE, shat = V_S;
    xf = XF_PLAIN;
    if (ss.path == PATH_SWEEP) {
        MTLG_TRY(launch_sweep<T>(ss, st, sv, 0, V_S, V_Z0, V_SHAT, SKIP_INNER, 2));
        MTLG_TRY(launch_sweep<T>(ss, st, sv, 1, V_Z0, V_SHAT, V_Z0, SKIP_INNER, 3));
        sin = V_SHAT; shat = V_SHAT;
    } else if (ss.path == PATH_JACOBI) {
        xf = XF_JAC; sn = V_SHAT; shat = V_SHAT;
    }
    SpmvOp t = spmv_op_default();
    t.x = sin; t.y = V_T; t.pnew = sn;
    set_dot(t, 0, OPND_Y, V_S);      // dot(t, s)
    set_dot(t, 1, OPND_Y, OPND_Y);   // dot(t, t)
    set_kinds(t, RK_DOT4, RK_DOT4);
    t.fin = FIN_BI_OMEGA;
    t.skip = SKIP_INNER;
    MTLG_TRY(launch_spmv<T>(c, st, sv, t, xf, ASG_SET));
    // x += omega shat + alpha phat ; r = s - omega t ; loop-top tests
    VecOp xr = vec_op_default(VOP_BI_XR);
    xr.a = SLOT_X; xr.b = phat; xr.c = shat; xr.e = V_S; xr.f = V_T; xr.g = V_R;
    set_dot(xr, 0, V_RT, V_R);   // rho_1 = dot(rtilde, r)
    set_dot(xr, 1, V_R, V_R);    // finished(r): two_norm(r)
    set_kinds(xr, RK_DOT4, RK_NORM4);
    xr.fin = FIN_BI_TOP;
    xr.skip = SKIP_RUNNING;
    return launch_vec<T>(c, st, sv, xr);
}

template <typename T>
inline int enqueue_body(SolveSet& ss, cudaStream_t st, const SetView& sv)
{
    if (ss.solver == MTLG_CG) {
        MTLG_TRY(cg_half<T>(ss, st, sv, V_P0, V_P1, true));
        return cg_half<T>(ss, st, sv, V_P1, V_P0, false);
    }
    return bicg_body<T>(ss, st, sv);
}

inline int iters_per_body(const SolveSet& ss) { return ss.solver == MTLG_CG ? 2 : 1; }

// Captures the loop body under a WHILE conditional node.
template <typename T>
inline int build_graph(SolveSet& ss)
{
    mtlg_ctx* c = ss.ctx;
    if (ss.exec || ss.graph_failed) return MTLG_OK;
    if (!ss.cap_stream) MTLG_CUDA(cudaStreamCreateWithFlags(&ss.cap_stream, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    MTLG_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    // cudaGraphNodeParams has no usable default constructor (union member)
    alignas(cudaGraphNodeParams) unsigned char cpbuf[sizeof(cudaGraphNodeParams)];
    memset(cpbuf, 0, sizeof cpbuf);
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cpbuf);
    cudaGraphNode_t node;
    if (e == cudaSuccess) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(g);
        ss.graph_failed = true;
        return MTLG_OK;
    }
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    ss.cond = (unsigned long long)h;
    const int64_t before = c->launches;
    MTLG_CUDA(cudaStreamBeginCaptureToGraph(ss.cap_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int s = enqueue_body<T>(ss, ss.cap_stream, ss.view(true, false));
    cudaGraph_t out = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(ss.cap_stream, &out);
    ss.body_kernels = int(c->launches - before);
    c->launches = before;
    if (s != MTLG_OK || e2 != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(g);
        ss.graph_failed = true;
        return s != MTLG_OK ? s : MTLG_OK;
    }
    e = cudaGraphInstantiate(&ss.exec, g, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(g);
        ss.exec = nullptr;
        ss.graph_failed = true;
        return MTLG_OK;
    }
    ss.graph = g;
    ss.iters_per_body = iters_per_body(ss);
    return MTLG_OK;
}

constexpr int kChunkBodies = 8;

// Chunked loop (default): kChunkBodies loop bodies captured in a plain CUDA
// graph; the host keeps two chunks in flight and reads the running count of
// the older one (pinned memory, event) before queueing the next, so the GPU
// never waits for the host.  Bodies queued after the last system stopped
// return at once.  Kernels of plain graphs can be profiled node by node.
template <typename T>
inline int run_loop_chunked(SolveSet& ss, int max_iter)
{
    mtlg_ctx* c = ss.ctx;
    if (!ss.chunk_exec) {
        MTLG_TRACE(9141, "set.capture");
        if (!ss.cap_stream) MTLG_CUDA(cudaStreamCreateWithFlags(&ss.cap_stream, cudaStreamNonBlocking));
        if (!ss.h_running) MTLG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&ss.h_running), 2 * sizeof(int), 0));
        for (auto& e : ss.chunk_ev)
            if (!e) MTLG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        const int64_t before = c->launches;
        MTLG_CUDA(cudaStreamBeginCapture(ss.cap_stream, cudaStreamCaptureModeThreadLocal));
        int s = MTLG_OK;
        const SetView sv = ss.view(false, false);
        for (int k = 0; k < kChunkBodies && s == MTLG_OK; ++k) s = enqueue_body<T>(ss, ss.cap_stream, sv);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(ss.cap_stream, &g);
        ss.chunk_kernels = int(c->launches - before);
        c->launches = before;
        MTLG_TRY(s);
        MTLG_CUDA(e);
        ss.chunk_graph = g;
        MTLG_CUDA(cudaGraphInstantiate(&ss.chunk_exec, g, 0));
    }
    const int ipb = iters_per_body(ss);
    const int max_chunks = max_iter / (ipb * kChunkBodies) + 2;
    int launched = 0;
    for (int k = 0; k < max_chunks; ++k) {
        MTLG_CUDA(cudaGraphLaunch(ss.chunk_exec, c->stream));
        c->launches += ss.chunk_kernels;
        MTLG_CUDA(cudaMemcpyAsync(ss.h_running + (k & 1), ss.misc.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        MTLG_CUDA(cudaEventRecord(ss.chunk_ev[k & 1], c->stream));
        ++launched;
        if (k >= 1) {
            MTLG_CUDA(cudaEventSynchronize(ss.chunk_ev[(k - 1) & 1]));
            if (ss.h_running[(k - 1) & 1] <= 0) break;
        }
    }
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    (void)launched;
    return MTLG_OK;
}

// Runs the loop until no system is running.  Default: chunked plain graphs
// (run_loop_chunked).  loop_mode 1: one graph with a WHILE conditional node,
// one launch per solve.  If a graph cannot be built, or under loop_mode 2
// (for profilers that do not see kernels inside graphs), the body is
// launched directly from the host, 8 at a time.
template <typename T>
inline int run_loop(SolveSet& ss, int max_iter)
{
    mtlg_ctx* c = ss.ctx;
    const int ipb = iters_per_body(ss);
    int hdr[3] = {0, 0, max_iter / ipb + 4};   // err flag, body runs, cap
    MTLG_CUDA(cudaMemcpyAsync(ss.misc.p + 1, hdr, sizeof hdr, cudaMemcpyHostToDevice, c->stream));
    if (c->loop_mode == 0) return run_loop_chunked<T>(ss, max_iter);
    if (c->loop_mode == 1) MTLG_TRY(build_graph<T>(ss));   // loop_mode 2: direct launches (profilers)
    if (c->loop_mode == 1 && ss.exec) {
        MTLG_CUDA(cudaGraphLaunch(ss.exec, c->stream));
        int runs = 0;
        MTLG_CUDA(cudaMemcpyAsync(&runs, ss.misc.p + 2, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        MTLG_CUDA(cudaStreamSynchronize(c->stream));
        c->launches += int64_t(runs) * ss.body_kernels;
        return MTLG_OK;
    }
    const SetView sv = ss.view(false, false);
    for (int it = 0; it <= max_iter / ipb + 1; it += 8) {
        for (int k = 0; k < 8; ++k) MTLG_TRY(enqueue_body<T>(ss, c->stream, sv));
        int running = 0;
        MTLG_CUDA(cudaMemcpyAsync(&running, ss.misc.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        MTLG_CUDA(cudaStreamSynchronize(c->stream));
        if (running <= 0) break;
    }
    return MTLG_OK;
}

inline SysState initial_state(const SysInput& si)
{
    SysState s;
    memset(&s, 0, sizeof s);
    s.max_iter = si.max_iter;
    s.rtol = si.rtol;
    s.atol = si.atol;
    s.norm_r0 = si.norm_r0;
    s.status = MTLG_ST_RUNNING;
    s.ostatus = MTLG_ST_RUNNING;
    s.log = si.log;
    s.log_cap = si.log_cap;
    s.log_n = 0;
    return s;
}

template <typename T>
inline int run_plain(SolveSet& ss)
{
    mtlg_ctx* c = ss.ctx;
    std::vector<SysState> h(ss.S);
    bool need_nb = false;
    int maxit = 0;
    for (int s = 0; s < ss.S; ++s) {
        h[s] = initial_state(ss.in[s]);
        need_nb |= ss.in[s].norm_r0 < 0;
        maxit = std::max(maxit, ss.in[s].max_iter);
    }
    MTLG_CUDA(cudaMemcpyAsync(ss.st.p, h.data(), sizeof(SysState) * ss.S, cudaMemcpyHostToDevice, c->stream));
    int running = ss.S;
    MTLG_CUDA(cudaMemcpyAsync(ss.misc.p, &running, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    const SetView sv = ss.view(false, false);
    if (need_nb) {
        VecOp nb = vec_op_default(VOP_DOT);
        set_dot(nb, 0, SLOT_B, SLOT_B);   // basic_iteration(b, ...): two_norm(b)
        set_kinds(nb, RK_NORM4);
        nb.fin = FIN_NORM_R0;
        MTLG_TRY(launch_vec<T>(c, c->stream, sv, nb));
    }
    if (ss.solver == MTLG_CG) MTLG_TRY(cg_init<T>(ss, c->stream, sv, false));
    else MTLG_TRY(bicg_init<T>(ss, c->stream, sv, false));
    MTLG_CUDA(cudaGetLastError());
    return run_loop<T>(ss, maxit);
}

// FP64 iterative refinement: the outer residual, its norm and the update run
// in FP64 on the FP64 values; the inner solve in FP32 on the FP32 values.
inline int run_refine(SolveSet& ss, const mtlg_refine_params& rp)
{
    mtlg_ctx* c = ss.ctx;
    std::vector<SysState> h(ss.S);
    for (int s = 0; s < ss.S; ++s) {
        SysInput si = ss.in[s];
        si.max_iter = rp.max_inner;
        si.rtol = rp.inner_rtol;
        si.atol = 0.0;
        h[s] = initial_state(si);
        h[s].outer_rtol = rp.rtol;
        h[s].max_outer = rp.max_outer;
        h[s].inner_rtol = rp.inner_rtol;
    }
    MTLG_CUDA(cudaMemcpyAsync(ss.st.p, h.data(), sizeof(SysState) * ss.S, cudaMemcpyHostToDevice, c->stream));
    const SetView v64 = ss.view(false, true), v32 = ss.view(false, false);
    VecOp nb = vec_op_default(VOP_DOT);
    set_dot(nb, 0, SLOT_B, SLOT_B);
    nb.fin = FIN_REF_NB;
    MTLG_TRY(launch_vec<double>(c, c->stream, v64, nb));
    for (int outer = 0; outer <= rp.max_outer; ++outer) {
        MTLG_CUDA(cudaMemsetAsync(ss.misc.p, 0, sizeof(int), c->stream));
        SpmvOp r = spmv_op_default();
        r.x = SLOT_X; r.w = SLOT_B; r.y = 0;
        set_dot(r, 0, OPND_Y, OPND_Y);
        r.fin = FIN_REF_OUTER;
        r.skip = SKIP_OUTER;
        MTLG_TRY(launch_spmv<double>(c, c->stream, v64, r, XF_PLAIN, ASG_WMINUS));
        int running = 0;
        MTLG_CUDA(cudaMemcpyAsync(&running, ss.misc.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        MTLG_CUDA(cudaStreamSynchronize(c->stream));
        if (running == 0) break;
        if (ss.solver == MTLG_CG) MTLG_TRY(cg_init<float>(ss, c->stream, v32, true));
        else MTLG_TRY(bicg_init<float>(ss, c->stream, v32, true));
        MTLG_TRY(run_loop<float>(ss, rp.max_inner));
        VecOp up = vec_op_default(VOP_REF_UPDATE);
        up.a = SLOT_X;
        up.skip = SKIP_OUTER;
        MTLG_TRY(launch_vec<float>(c, c->stream, v32, up));
    }
    MTLG_CUDA(cudaGetLastError());
    return MTLG_OK;
}

inline void fill_result(const SysState& s, bool mixed, mtlg_iter_result* r)
{
    r->iterations = mixed ? s.inner_total : s.iter;
    r->status = mixed ? s.ostatus : s.status;
    r->error_code = s.error;
    r->outer_iterations = mixed ? s.outer : 0;
    r->resid = s.resid;
    r->norm_r0 = mixed ? s.nb : s.norm_r0;
    r->relresid = r->norm_r0 != 0.0 ? s.resid / r->norm_r0 : s.resid;
    r->fp64_fallback = 0;
    r->reserved = 0;
}

}  // namespace mtlg
