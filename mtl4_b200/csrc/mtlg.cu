// mtl4_b200: C ABI of the sparse-solve hot path on one B200 (sm_100a).
// The declarations and the reference interface each entry point replaces are
// in include/mtl4_b200/mtlg.h.
#include "host_solve.cuh"
#include "host_krylov.cuh"

#include <map>
#include <cmath>
#include <type_traits>

using namespace mtlg;

namespace mtlg {

// Cache of single-system solve sets (reused across calls with the same
// operator and preconditioner so their loop graphs are built once).
struct SetKey {
    const mtlg_csr* A;
    const mtlg_pc* P;
    int solver, f32, mixed;
    int red_order;   // the loop graphs hold the reduction kernels of that mode
    bool operator<(const SetKey& o) const
    {
        return std::tie(A, P, solver, f32, mixed, red_order) < std::tie(o.A, o.P, o.solver, o.f32, o.mixed, o.red_order);
    }
};

struct CtxExtra {
    std::map<SetKey, std::unique_ptr<SolveSet>> sets;
    // vector-only tile sets, by length
    struct VecSet {
        DBuf<Tile> tiles;
        DBuf<int> stb;
        DBuf<double> partials;
        DBuf<unsigned> counters;
        DBuf<SysDesc> desc;
        DBuf<SysState> st;
        DBuf<int> misc;
        int n_tiles = 0;
    };
    std::map<int64_t, std::unique_ptr<VecSet>> vsets;
};

static std::mutex g_extra_mu;
static std::map<const mtlg_ctx*, std::unique_ptr<CtxExtra>> g_extra;

inline CtxExtra& extra(const mtlg_ctx* c)
{
    std::lock_guard<std::mutex> lk(g_extra_mu);
    auto& e = g_extra[c];
    if (!e) e.reset(new CtxExtra);
    return *e;
}

inline void purge_sets(const mtlg_ctx* c, const void* obj)
{
    MTLG_TRACE(9108, "sets.purge");
    CtxExtra& e = extra(c);
    for (auto it = e.sets.begin(); it != e.sets.end();) {
        if (it->first.A == obj || it->first.P == obj) it = e.sets.erase(it);
        else ++it;
    }
}

inline int vec_set(mtlg_ctx* c, int64_t n, SetView& sv)
{
    auto& vs = extra(c).vsets[n];
    if (!vs) {
        vs.reset(new CtxExtra::VecSet);
        std::vector<Tile> tiles;
        for (int64_t r = 0; r < n; r += kTileRows) tiles.push_back({0, int(r), int(std::min<int64_t>(n, r + kTileRows)), TILE_STREAM, 0, 0});
        vs->n_tiles = int(tiles.size());
        MTLG_TRY(vs->tiles.upload(c, tiles.data(), std::max<size_t>(1, tiles.size())));
        int stb[2] = {0, vs->n_tiles};
        MTLG_TRY(vs->stb.upload(c, stb, 2));
        MTLG_TRY(vs->partials.alloc(c, size_t(std::max(1, vs->n_tiles)) * kMaxDots));
        MTLG_TRY(vs->counters.alloc(c, 1));
        MTLG_CUDA(cudaMemsetAsync(vs->counters.p, 0, sizeof(unsigned), c->stream));
        MTLG_TRY(vs->desc.alloc(c, 1));
        MTLG_TRY(vs->st.alloc(c, 1));
        MTLG_TRY(vs->misc.alloc(c, 4));
        MTLG_CUDA(cudaMemsetAsync(vs->misc.p, 0, 4 * sizeof(int), c->stream));
    }
    sv = SetView{};
    sv.tiles = vs->tiles.p;
    sv.n_tiles = vs->n_tiles;
    sv.n_sys = 1;
    sv.sys_tile_begin = vs->stb.p;
    sv.desc = vs->desc.p;
    sv.st = vs->st.p;
    sv.partials = vs->partials.p;
    sv.counters = vs->counters.p;
    sv.running = vs->misc.p;
    sv.err = vs->misc.p + 1;
    return MTLG_OK;
}

inline int read_dots(mtlg_ctx* c, SysState* st, double* out, int nd)
{
    SysState h;
    MTLG_CUDA(cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    for (int j = 0; j < nd; ++j) out[j] = h.dots[j];
    return MTLG_OK;
}

inline bool ok_dtype(int d) { return d == MTLG_F64 || d == MTLG_F32; }

}  // namespace mtlg

namespace mtlg {
template <typename T, typename S>
int pc_sweeps(mtlg_pc* P, const mtlg_vec* x, mtlg_vec* y)
{
    mtlg_ctx* c = P->ctx;
    SetView sv = SetView{};
    sv.n_sys = 1;
    sv.desc = P->desc.p;
    sv.st = P->st.p;
    sv.running = P->misc.p;
    sv.err = P->misc.p + 1;
    sv.spin = c->spin_limit;
    SysDesc d;
    memset(&d, 0, sizeof d);
    d.n = P->n;
    d.x = x->p;
    d.b = y->p;
    d.ws = P->tmp.p;
    d.ws_stride = 0;
    ChunkPlan& pl = P->plan[sizeof(T) == 4 ? 1 : 0];
    int& made = P->plan_kernel[sizeof(T) == 4 ? 1 : 0];
    const int setting = plan_setting(c);
    if (made != setting) {
        std::vector<std::pair<const TriDev*, const TriDev*>> f(1, {&P->L, &P->U});
        MTLG_TRY((plan_chunks<T, S>(c, f, pl)));
        made = setting;
    }
    // flat sweeps (no chunked plan, or chosen by sweep_kernel) need the flat entries
    const bool chunked = pl.ok;
    if (!chunked) MTLG_TRY(ensure_flat(P));
    MTLG_TRY(pc_views(P, sizeof(T) == 4 ? 1 : 0, d.L, d.U));
    MTLG_CUDA(cudaMemcpyAsync(P->desc.p, &d, sizeof d, cudaMemcpyHostToDevice, c->stream));
    if (chunked) {
        ChunkSweepOp op;
        memset(&op, 0, sizeof op);
        op.skip = SKIP_NONE;
        op.sleep_ns = c->sweep_sleep_ns;
        // y0 = L^{-1} x  (temp, slot 0); clears y row by row
        op.tasks = pl.tl.p; op.ntasks = pl.ntl; op.ticket = P->tickets.p + 2; op.which = 0;
        op.in = SLOT_X; op.out = 0; op.reset = SLOT_B;
        MTLG_TRY((launch_chunk_sweep<T, S>(c, c->stream, sv, op, pl)));
        // y = U^{-1} y0; clears the temp again
        op.tasks = pl.tu.p; op.ntasks = pl.ntu; op.ticket = P->tickets.p + 3; op.which = 1;
        op.in = 0; op.out = SLOT_B; op.reset = 0;
        MTLG_TRY((launch_chunk_sweep<T, S>(c, c->stream, sv, op, pl)));
    } else {
        SweepOp op;
        memset(&op, 0, sizeof op);
        op.skip = SKIP_NONE;
        op.fuse = SWF_NONE;
        op.sleep_ns = c->sweep_sleep_ns;
        const int grid = c->sweep_blocks();
        op.tasks = P->L.tasks.p; op.ntasks = int(P->L.tasks.n); op.ticket = P->tickets.p + 0; op.which = 0;
        op.in = SLOT_X; op.out = 0; op.reset = SLOT_B;
        if (op.ntasks) { k_sweep<T, S><<<grid, kBlock, 0, c->stream>>>(sv, op); c->launches++; }
        op.tasks = P->U.tasks.p; op.ntasks = int(P->U.tasks.n); op.ticket = P->tickets.p + 1; op.which = 1;
        op.in = 0; op.out = SLOT_B; op.reset = 0;
        if (op.ntasks) { k_sweep<T, S><<<grid, kBlock, 0, c->stream>>>(sv, op); c->launches++; }
    }
    MTLG_CUDA(cudaGetLastError());
    // queued applies (pc_apply_sync = 0): an expired wait stays flagged on the
    // device and is reported by the next synchronous apply of this preconditioner
    if (!c->pc_apply_sync) return MTLG_OK;
    int err = 0;
    MTLG_CUDA(cudaMemcpyAsync(&err, P->misc.p + 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    if (err) {
        int z = 0;
        MTLG_CUDA(cudaMemcpy(P->misc.p + 1, &z, sizeof z, cudaMemcpyHostToDevice));
        MTLG_CUDA(cudaMemset(P->tickets.p, 0, 8 * sizeof(int)));
        MTLG_TRY(pc_reset_sweep_state(P));
        set_error("triangular sweep dependency wait expired");
        return MTLG_ERR_TIMEOUT;
    }
    return MTLG_OK;
}

// SpMV on raw device pointers of the CSR's size (GMRES workspace vectors);
// w (optional) is the W of y = W - A x.
int spmv_raw(mtlg_ctx* c, mtlg_csr* A, int dtype, const void* x, void* y, const void* w, int asg)
{
    const bool f32 = dtype == MTLG_F32;
    if (f32) MTLG_TRY(ensure_f32_values(A));
    SetView sv;
    MTLG_TRY(csr_op_set(A, sv));
    SysDesc d;
    memset(&d, 0, sizeof d);
    d.n = int(A->n_rows);
    d.nnz = int(A->nnz);
    d.rp = A->rp.p;
    d.ci = A->ci.p;
    d.val = f32 ? (const void*)A->v32.p : (const void*)A->v64.p;
    d.val64 = A->v64.p;
    d.x = const_cast<void*>(x);
    d.b = y;
    d.ws = const_cast<void*>(w);
    d.ws_stride = 0;
    MTLG_CUDA(cudaMemcpyAsync(sv.desc, &d, sizeof d, cudaMemcpyHostToDevice, c->stream));
    SpmvOp op = spmv_op_default();
    op.x = SLOT_X;
    op.y = SLOT_B;
    op.w = w ? 0 : SLOT_NONE;
    if (f32) return launch_spmv<float>(c, c->stream, sv, op, XF_PLAIN, asg);
    return launch_spmv<double>(c, c->stream, sv, op, XF_PLAIN, asg);
}

}  // namespace mtlg

namespace mtlg {
template <typename T>
int launch_spmv_rows(mtlg_ctx* c, mtlg_csr* A, const void* x, void* y, int asg)
{
    if (A->wtasks.empty()) return MTLG_OK;
    if (!A->d_wtasks.p) {
        MTLG_TRY(A->d_wtasks.upload(c, A->wtasks.data(), A->wtasks.size()));
        MTLG_TRY(A->wctr.alloc(c, 2));
        MTLG_CUDA(cudaMemsetAsync(A->wctr.p, 0, 2 * sizeof(int), c->stream));
    }
    const int ntasks = int(A->wtasks.size());
    // 3 CTAs per SM (measured faster than 4 on the 40M-entry power-law CSR)
    const int grid = std::min((ntasks + 7) / 8, c->sm_count * 3);
    const T* va = std::is_same<T, float>::value ? (const T*)A->v32.p : (const T*)A->v64.p;
#define MTLG_ROWS(ASG) k_spmv_rows<T, ASG><<<grid, kBlock, 0, c->stream>>>(A->d_wtasks.p, ntasks, A->wctr.p, A->rp.p, \
                                                                          A->ci.p, va, (const T*)x, (T*)y)
    switch (asg) {
    case ASG_SET: MTLG_ROWS(ASG_SET); break;
    case ASG_ADD: MTLG_ROWS(ASG_ADD); break;
    default: MTLG_ROWS(ASG_SUB); break;
    }
#undef MTLG_ROWS
    c->launches++;
    MTLG_CUDA(cudaGetLastError());
    return MTLG_OK;
}

}  // namespace mtlg

extern "C" int mtlg_pc_apply(mtlg_ctx* c, mtlg_pc* P, const mtlg_vec* x, mtlg_vec* y);

namespace mtlg {
int pc_adjoint_raw(mtlg_ctx* c, mtlg_pc* P, int64_t n, const double* x, double* y)
{
    if (!P || P->kind == MTLG_PC_IDENTITY) {
        if (x != y) MTLG_CUDA(cudaMemcpyAsync(y, x, size_t(n) * 8, cudaMemcpyDeviceToDevice, c->stream));
        return MTLG_OK;
    }
    mtlg_vec xv, yv;
    xv.ctx = yv.ctx = c;
    xv.n = yv.n = n;
    xv.dtype = yv.dtype = MTLG_F64;
    xv.p = const_cast<double*>(x);
    yv.p = y;
    return mtlg_pc_adjoint_apply(c, P, &xv, &yv);
}

int pc_apply_raw(mtlg_ctx* c, mtlg_pc* P, int dtype, int64_t n, const void* x, void* y)
{
    if (!P || P->kind == MTLG_PC_IDENTITY) {
        if (x != y) MTLG_CUDA(cudaMemcpyAsync(y, x, size_t(n) * (dtype == MTLG_F32 ? 4 : 8), cudaMemcpyDeviceToDevice, c->stream));
        return MTLG_OK;
    }
    mtlg_vec xv, yv;
    xv.ctx = yv.ctx = c;
    xv.n = yv.n = n;
    xv.dtype = yv.dtype = dtype;
    xv.p = const_cast<void*>(x);
    yv.p = y;
    return mtlg_pc_apply(c, P, &xv, &yv);
}
}  // namespace mtlg

extern "C" {

const char* mtlg_status_string(int s)
{
    switch (s) {
    case MTLG_OK: return "ok";
    case MTLG_ERR_INVALID_ARG: return "invalid argument";
    case MTLG_ERR_NOT_SQUARE: return "matrix not square";
    case MTLG_ERR_MISSING_DIAGONAL: return "missing diagonal";
    case MTLG_ERR_ZERO_PIVOT: return "zero pivot";
    case MTLG_ERR_BREAKDOWN: return "unexpected orthogonality (breakdown)";
    case MTLG_ERR_OOM: return "out of device memory";
    case MTLG_ERR_TIMEOUT: return "device wait timed out";
    case MTLG_ERR_CUDA: return "CUDA error";
    case MTLG_ERR_INCOMPATIBLE_SIZE: return "incompatible size";
    case MTLG_ERR_UNSORTED: return "CSR rows must be sorted and in range";
    case MTLG_ERR_TOO_LARGE: return "too large for 32-bit device indexing";
    case MTLG_ERR_NOT_SUPPORTED: return "not supported";
    case MTLG_ERR_ADMISSION: return "request exceeds the device budget";
    case MTLG_ERR_NOT_FOUND: return "unknown request";
    case MTLG_PENDING: return "pending";
    case MTLG_ERR_FILE_NOT_FOUND: return "file not found";
    case MTLG_ERR_FORMAT: return "malformed input";
    default: return "unknown status";
    }
}

const char* mtlg_last_error_message(void) { return last_error(); }

int mtlg_ctx_set_residual_log(mtlg_ctx* c, int capacity)
{
    MTLG_CHECK_ARG(c && capacity >= 0, "ctx/capacity");
    if (c->log_dev) {
        cudaStreamSynchronize(c->stream);
        cudaFree(c->log_dev);
        c->in_use -= size_t(c->log_cap) * 16;
        c->log_dev = nullptr;
    }
    c->log_cap = 0;
    c->log_n = 0;
    if (capacity > 0) {
        MTLG_CUDA(cudaSetDevice(c->device));
        if (cudaMalloc(&c->log_dev, size_t(capacity) * 16) != cudaSuccess) {
            cudaGetLastError();
            c->log_dev = nullptr;
            set_error("residual log of %d tests", capacity);
            return MTLG_ERR_OOM;
        }
        c->in_use += size_t(capacity) * 16;
        c->log_cap = capacity;
    }
    return MTLG_OK;
}

int mtlg_ctx_residual_log(mtlg_ctx* c, double* pairs, int capacity, int* count)
{
    MTLG_CHECK_ARG(c && count, "ctx/count");
    *count = c->log_n;
    const int k = std::min(std::min(c->log_n, c->log_cap), capacity);
    if (pairs && k > 0) MTLG_CUDA(cudaMemcpy(pairs, c->log_dev, size_t(k) * 16, cudaMemcpyDeviceToHost));
    return MTLG_OK;
}

int mtlg_trace_enable(int on)
{
    TraceState& t = trace_state();
    std::lock_guard<std::mutex> lk(t.mu);
    t.on = on ? 1 : 0;
    return MTLG_OK;
}

int mtlg_trace_reset(void)
{
    TraceState& t = trace_state();
    std::lock_guard<std::mutex> lk(t.mu);
    t.events.clear();
    return MTLG_OK;
}

int mtlg_trace_report(char* buf, size_t cap, size_t* needed)
{
    TraceState& t = trace_state();
    std::string out;
    {
        std::lock_guard<std::mutex> lk(t.mu);
        char line[160];
        for (const auto& kv : t.events) {
            snprintf(line, sizeof line, "%d %s %lld %.6f\n", kv.first, kv.second.name.c_str(), kv.second.calls,
                     kv.second.seconds * 1e3);
            out += line;
        }
    }
    if (needed) *needed = out.size() + 1;
    if (buf && cap) {
        const size_t k = std::min(cap - 1, out.size());
        memcpy(buf, out.data(), k);
        buf[k] = 0;
    }
    return MTLG_OK;
}

// ------------------------------------------------------------------ context
int mtlg_ctx_create(int device, size_t hbm_budget, mtlg_ctx** out)
{
    MTLG_CHECK_ARG(out, "out");
    *out = nullptr;
    int ndev = 0;
    MTLG_CUDA(cudaGetDeviceCount(&ndev));
    MTLG_CHECK_ARG(device >= 0 && device < ndev, "device index");
    MTLG_CUDA(cudaSetDevice(device));
    std::unique_ptr<mtlg_ctx> c(new mtlg_ctx);
    c->device = device;
    c->budget = hbm_budget;
    MTLG_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    MTLG_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
    MTLG_CUDA(cudaDeviceGetAttribute(&c->max_threads_per_sm, cudaDevAttrMaxThreadsPerMultiProcessor, device));
    MTLG_CUDA(cudaDeviceGetAttribute(&c->regs_per_sm, cudaDevAttrMaxRegistersPerMultiprocessor, device));
    MTLG_CUDA(cudaDeviceGetAttribute(&c->smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device));
    MTLG_CUDA(cudaDeviceGetAttribute(&c->smem_reserved_per_block, cudaDevAttrReservedSharedMemoryPerBlock, device));
    int nb = 1, nb2 = 1;
    MTLG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_sweep<double, double>, kBlock, 0));
    MTLG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, k_ilu0_factor, kBlock, 0));
    c->sweep_max_bpsm = std::max(1, std::min(nb, nb2));
    c->sweep_grid = c->sm_count * c->sweep_max_bpsm;
    MTLG_TRY(init_kernel_shapes());
    MTLG_TRY(init_chunk_shapes());
    MTLG_TRY(init_grid_shapes());
    {
        // stream-ordered pool of this context's device buffers, kept between
        // set-ups (release threshold: never); without one, cudaMalloc
        cudaMemPoolProps props;
        memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        if (cudaMemPoolCreate(&c->pool, &props) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        } else {
            cudaGetLastError();
            c->pool = nullptr;
        }
    }
    *out = c.release();
    return MTLG_OK;
}

int mtlg_ctx_destroy(mtlg_ctx* c)
{
    if (!c) return MTLG_OK;
    cudaStreamSynchronize(c->stream);
    {
        std::unique_ptr<CtxExtra> e;
        {
            std::lock_guard<std::mutex> lk(g_extra_mu);
            auto it = g_extra.find(c);
            if (it != g_extra.end()) {
                e = std::move(it->second);
                g_extra.erase(it);
            }
        }
    }
    if (c->log_dev) cudaFree(c->log_dev);
    cudaStreamSynchronize(c->stream);
    // the pool goes with the context once every buffer of it is back
    if (c->pool && c->in_use.load() == 0) cudaMemPoolDestroy(c->pool);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return MTLG_OK;
}

int mtlg_ctx_synchronize(mtlg_ctx* c)
{
    MTLG_CHECK_ARG(c, "ctx");
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    return MTLG_OK;
}

int mtlg_ctx_set_stream(mtlg_ctx* c, void* s)
{
    MTLG_CHECK_ARG(c, "ctx");
    // buffers are allocated and freed in the order of the context's stream:
    // the old stream's work ends before the new stream takes over
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    c->stream = s ? static_cast<cudaStream_t>(s) : c->own_stream;
    return MTLG_OK;
}

void* mtlg_ctx_stream(mtlg_ctx* c) { return c ? (void*)c->stream : nullptr; }

int mtlg_ctx_set_tuning(mtlg_ctx* c, const char* key, int64_t value)
{
    MTLG_CHECK_ARG(c && key, "ctx/key");
    const std::string k(key);
    if (k == "sweep_blocks_per_sm") c->sweep_bpsm = int(std::max<int64_t>(0, value));
    else if (k == "sweep_blocks") c->sweep_nblocks = int(std::max<int64_t>(0, std::min<int64_t>(value, 1 << 16)));
    else if (k == "loop_mode") c->loop_mode = int(std::max<int64_t>(0, std::min<int64_t>(value, 2)));
    else if (k == "spmv_kernel") c->spmv_kernel = int(std::max<int64_t>(0, std::min<int64_t>(value, 3)));
    else if (k == "sweep_sleep_ns") c->sweep_sleep_ns = int(std::max<int64_t>(0, std::min<int64_t>(value, 100000)));
    else if (k == "sweep_kernel") c->sweep_kernel = value ? 1 : 0;
    else if (k == "grid_sweep") c->grid_sweep = value ? 1 : 0;
    else if (k == "grid_warps") {
        if (value != 0 && value != 4 && value != 8) {
            set_error("grid_warps must be 0, 4 or 8");
            return MTLG_ERR_INVALID_ARG;
        }
        c->grid_warps = int(value);
    }
    else if (k == "pc_apply_sync") c->pc_apply_sync = value ? 1 : 0;
    else if (k == "reduction_order") c->red_order = value ? 1 : 0;
    else if (k == "spin_limit") c->spin_limit = std::max<int64_t>(0, value);
    else if (k == "admission_free_bytes") c->admission_free_bytes = std::max<int64_t>(0, value);
    else if (k == "admission_reserve_bytes") c->admission_reserve_bytes = std::max<int64_t>(-1, value);
    else if (k == "chunk_rows") c->chunk_rows = int(std::max<int64_t>(0, std::min<int64_t>(value, 1 << 15)));
    else if (k == "vec_ctas_per_sm") c->vec_ctas_per_sm = int(std::max<int64_t>(1, std::min<int64_t>(value, 16)));
    else if (k == "sweep_cluster") {
        if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8 && value != 16) {
            set_error("sweep_cluster must be 0, 1, 2, 4, 8 or 16");
            return MTLG_ERR_INVALID_ARG;
        }
        c->sweep_cluster = int(value);
    }
    else {
        set_error("unknown tuning key '%s'", key);
        return MTLG_ERR_INVALID_ARG;
    }
    return MTLG_OK;
}

int mtlg_ctx_get_tuning(mtlg_ctx* c, const char* key, int64_t* value)
{
    MTLG_CHECK_ARG(c && key && value, "ctx/key/value");
    const std::string k(key);
    if (k == "sweep_blocks_per_sm") *value = c->sweep_bpsm;
    else if (k == "sweep_blocks") *value = c->sweep_blocks();
    else if (k == "loop_mode") *value = c->loop_mode;
    else if (k == "spmv_kernel") *value = c->spmv_kernel;
    else if (k == "sweep_max_blocks_per_sm") *value = c->sweep_max_bpsm;
    else if (k == "sweep_sleep_ns") *value = c->sweep_sleep_ns;
    else if (k == "sm_count") *value = c->sm_count;
    else if (k == "sweep_kernel") *value = c->sweep_kernel;
    else if (k == "grid_sweep") *value = c->grid_sweep;
    else if (k == "grid_warps") *value = c->grid_warps;
    else if (k == "pc_apply_sync") *value = c->pc_apply_sync;
    else if (k == "reduction_order") *value = c->red_order;
    else if (k == "spin_limit") *value = c->spin_limit > 0 ? c->spin_limit : kSpinLimit;
    else if (k == "admission_free_bytes") *value = c->admission_free_bytes;
    else if (k == "admission_reserve_bytes") *value = c->admission_reserve_bytes;
    else if (k == "chunk_rows") *value = c->chunk_rows;
    else if (k == "sweep_cluster") *value = c->sweep_cluster;
    else if (k == "vec_ctas_per_sm") *value = c->vec_ctas_per_sm;
    else {
        set_error("unknown tuning key '%s'", key);
        return MTLG_ERR_INVALID_ARG;
    }
    return MTLG_OK;
}
int64_t mtlg_ctx_kernel_launches(mtlg_ctx* c) { return c ? c->launches : 0; }
size_t mtlg_ctx_bytes_in_use(mtlg_ctx* c) { return c ? c->in_use.load() : size_t(0); }

// ------------------------------------------------------------------ CSR
int mtlg_csr_create(mtlg_ctx* c, int64_t n_rows, int64_t n_cols, int64_t nnz, const int64_t* row_ptr,
                    const int32_t* col, const void* val, mtlg_dtype val_dtype, mtlg_csr** out)
{
    MTLG_TRACE(9001, "csr_create");
    MTLG_CHECK_ARG(c && out, "ctx/out");
    *out = nullptr;
    MTLG_CHECK_ARG(n_rows >= 0 && n_cols >= 0 && nnz >= 0, "negative size");
    MTLG_CHECK_ARG(row_ptr && (nnz == 0 || (col && val)), "null array");
    MTLG_CHECK_ARG(ok_dtype(val_dtype), "dtype");
    if (n_rows > INT32_MAX - 1 || n_cols > INT32_MAX || nnz > INT32_MAX - 1) {
        set_error("n or nnz beyond 32-bit device indexing");
        return MTLG_ERR_TOO_LARGE;
    }
    if (row_ptr[0] != 0 || row_ptr[n_rows] != nnz) {
        set_error("row_ptr must start at 0 and end at nnz");
        return MTLG_ERR_INVALID_ARG;
    }
    std::unique_ptr<mtlg_csr> A(new mtlg_csr);
    A->ctx = c;
    A->n_rows = n_rows;
    A->n_cols = n_cols;
    A->nnz = nnz;
    A->h_rp.assign(row_ptr, row_ptr + n_rows + 1);
    A->h_ci.assign(col, col + nnz);
    A->h_dpos.assign(size_t(n_rows), -1);
    std::vector<int> rp32(size_t(n_rows) + 1);
    for (int64_t i = 0; i < n_rows; ++i) {
        const int64_t a = row_ptr[i], e = row_ptr[i + 1];
        if (e < a) {
            set_error("row_ptr decreases at row %lld", (long long)i);
            return MTLG_ERR_INVALID_ARG;
        }
        A->max_row = std::max<int>(A->max_row, int(e - a));
        for (int64_t k = a; k < e; ++k) {
            if (col[k] < 0 || col[k] >= n_cols || (k > a && col[k] <= col[k - 1])) {
                set_error("row %lld: columns must be sorted, distinct and in range", (long long)i);
                return MTLG_ERR_UNSORTED;
            }
            if (col[k] == i) A->h_dpos[i] = int(k);
        }
        rp32[i] = int(a);
    }
    rp32[n_rows] = int(nnz);
    plan_tiles(A->h_rp.data(), int(n_rows), 0, A->tiles);
    for (const Tile& t : A->tiles) A->tiles_by_kind[t.kind]++;
    A->irregular = A->max_row > kShortRow;
    plan_warp_tasks(A->h_rp.data(), int(n_rows), A->wtasks);
    MTLG_TRY(A->rp.upload(c, rp32.data(), rp32.size()));
    MTLG_TRY(A->ci.upload(c, col, size_t(nnz)));
    MTLG_TRY(A->dpos.upload(c, A->h_dpos.data(), std::max<size_t>(1, A->h_dpos.size())));
    if (val_dtype == MTLG_F64) {
        MTLG_TRY(A->v64.upload(c, static_cast<const double*>(val), size_t(nnz)));
    } else {
        std::vector<double> w(static_cast<const float*>(val), static_cast<const float*>(val) + nnz);
        MTLG_TRY(A->v64.upload(c, w.data(), size_t(nnz)));
        MTLG_TRY(A->v32.upload(c, static_cast<const float*>(val), size_t(nnz)));
    }
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    *out = A.release();
    return MTLG_OK;
}

int mtlg_mm_read_host(const char* path, int64_t* n_rows, int64_t* n_cols, int64_t* nnz, int64_t* row_ptr,
                      int32_t* col, double* val)
{
    MTLG_TRACE(9003, "matrix_market_read");
    MTLG_CHECK_ARG(path && n_rows && n_cols && nnz, "path/sizes");
    MmCsr m;
    MTLG_TRY(mm_read_file(path, m));
    *n_rows = m.n_rows;
    *n_cols = m.n_cols;
    *nnz = int64_t(m.ci.size());
    if (row_ptr) std::copy(m.rp.begin(), m.rp.end(), row_ptr);
    if (col) std::copy(m.ci.begin(), m.ci.end(), col);
    if (val) std::copy(m.val.begin(), m.val.end(), val);
    return MTLG_OK;
}

int mtlg_mm_read(mtlg_ctx* c, const char* path, mtlg_csr** out)
{
    MTLG_TRACE(9003, "matrix_market_read");
    MTLG_CHECK_ARG(c && path && out, "ctx/path/out");
    MmCsr m;
    MTLG_TRY(mm_read_file(path, m));
    return mtlg_csr_create(c, m.n_rows, m.n_cols, int64_t(m.ci.size()), m.rp.data(), m.ci.data(), m.val.data(),
                           MTLG_F64, out);
}

int mtlg_csr_destroy(mtlg_csr* A)
{
    if (!A) return MTLG_OK;
    cudaStreamSynchronize(A->ctx->stream);
    if (A->AT) mtlg_csr_destroy(A->AT);
    purge_sets(A->ctx, A);
    delete A;
    return MTLG_OK;
}

int mtlg_csr_info(const mtlg_csr* A, int64_t* n_rows, int64_t* n_cols, int64_t* nnz)
{
    MTLG_CHECK_ARG(A, "csr");
    if (n_rows) *n_rows = A->n_rows;
    if (n_cols) *n_cols = A->n_cols;
    if (nnz) *nnz = A->nnz;
    return MTLG_OK;
}

int mtlg_csr_update_values(mtlg_csr* A, const void* val, mtlg_dtype dt)
{
    MTLG_CHECK_ARG(A && (val || A->nnz == 0) && ok_dtype(dt), "csr/val/dtype");
    mtlg_ctx* c = A->ctx;
    if (dt == MTLG_F64) {
        MTLG_CUDA(cudaMemcpyAsync(A->v64.p, val, size_t(A->nnz) * 8, cudaMemcpyHostToDevice, c->stream));
    } else {
        std::vector<double> w(static_cast<const float*>(val), static_cast<const float*>(val) + A->nnz);
        MTLG_CUDA(cudaMemcpyAsync(A->v64.p, w.data(), size_t(A->nnz) * 8, cudaMemcpyHostToDevice, c->stream));
    }
    if (A->v32.p) {
        A->v32.release();
        MTLG_TRY(ensure_f32_values(A));
    }
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    return MTLG_OK;
}

int mtlg_csr_plan_info(const mtlg_csr* A, int64_t* tiles_by_kind3, int* max_row_len)
{
    MTLG_CHECK_ARG(A, "csr");
    if (tiles_by_kind3) for (int k = 0; k < 3; ++k) tiles_by_kind3[k] = A->tiles_by_kind[k];
    if (max_row_len) *max_row_len = A->max_row;
    return MTLG_OK;
}

// ------------------------------------------------------------------ vectors
int mtlg_vec_create(mtlg_ctx* c, int64_t n, mtlg_dtype dt, mtlg_vec** out)
{
    MTLG_CHECK_ARG(c && out && n >= 0 && ok_dtype(dt), "ctx/out/n/dtype");
    *out = nullptr;
    std::unique_ptr<mtlg_vec> v(new mtlg_vec);
    v->ctx = c;
    v->n = n;
    v->dtype = dt;
    v->owned = true;
    MTLG_TRY(dalloc(c, &v->p, v->bytes()));
    MTLG_CUDA(cudaMemsetAsync(v->p, 0, v->bytes(), c->stream));
    *out = v.release();
    return MTLG_OK;
}

int mtlg_vec_wrap(mtlg_ctx* c, int64_t n, mtlg_dtype dt, void* p, mtlg_vec** out)
{
    MTLG_CHECK_ARG(c && out && n >= 0 && ok_dtype(dt) && (p || n == 0), "ctx/out/n/dtype/ptr");
    std::unique_ptr<mtlg_vec> v(new mtlg_vec);
    v->ctx = c;
    v->n = n;
    v->dtype = dt;
    v->p = p;
    v->owned = false;
    *out = v.release();
    return MTLG_OK;
}

int mtlg_vec_destroy(mtlg_vec* v)
{
    if (!v) return MTLG_OK;
    if (v->owned) {
        cudaStreamSynchronize(v->ctx->stream);
        dfree(v->ctx, v->p, v->bytes());
    }
    delete v;
    return MTLG_OK;
}

int mtlg_vec_upload(mtlg_vec* v, const void* h, int64_t n)
{
    MTLG_CHECK_ARG(v && (h || n == 0), "vec/host");
    if (n != v->n) {
        set_error("upload of %lld elements into a vector of %lld", (long long)n, (long long)v->n);
        return MTLG_ERR_INCOMPATIBLE_SIZE;
    }
    MTLG_CUDA(cudaMemcpyAsync(v->p, h, v->bytes(), cudaMemcpyHostToDevice, v->ctx->stream));
    return MTLG_OK;
}

int mtlg_vec_download(const mtlg_vec* v, void* h, int64_t n)
{
    MTLG_CHECK_ARG(v && (h || n == 0), "vec/host");
    if (n != v->n) {
        set_error("download of %lld elements from a vector of %lld", (long long)n, (long long)v->n);
        return MTLG_ERR_INCOMPATIBLE_SIZE;
    }
    MTLG_CUDA(cudaMemcpyAsync(h, v->p, v->bytes(), cudaMemcpyDeviceToHost, v->ctx->stream));
    MTLG_CUDA(cudaStreamSynchronize(v->ctx->stream));
    return MTLG_OK;
}

int mtlg_vec_fill(mtlg_vec* v, double value)
{
    MTLG_CHECK_ARG(v, "vec");
    mtlg_ctx* c = v->ctx;
    if (v->n == 0) return MTLG_OK;
    SetView sv;
    MTLG_TRY(vec_set(c, v->n, sv));
    SysDesc d;
    memset(&d, 0, sizeof d);
    d.n = int(v->n);
    d.x = v->p;
    MTLG_CUDA(cudaMemcpyAsync(sv.desc, &d, sizeof d, cudaMemcpyHostToDevice, c->stream));
    VecOp op = vec_op_default(VOP_FILL);
    op.a = SLOT_X;
    op.scalar = value;
    return v->dtype == MTLG_F64 ? launch_vec<double>(c, c->stream, sv, op) : launch_vec<float>(c, c->stream, sv, op);
}

void* mtlg_vec_device_ptr(const mtlg_vec* v) { return v ? v->p : nullptr; }
int64_t mtlg_vec_size(const mtlg_vec* v) { return v ? v->n : -1; }

// ------------------------------------------------------------------ SpMV / level 1
static int spmv_impl(mtlg_ctx* c, mtlg_csr* A, const mtlg_vec* x, mtlg_vec* y, int assign, double* pq)
{
    MTLG_CHECK_ARG(c && A && x && y, "null handle");
    MTLG_CHECK_ARG(x->dtype == y->dtype, "x and y dtypes differ");
    MTLG_CHECK_ARG(assign >= MTLG_ASSIGN && assign <= MTLG_MINUS, "assign");
    if (x->n != A->n_cols || y->n != A->n_rows) {
        set_error("SpMV sizes: A %lldx%lld, x %lld, y %lld", (long long)A->n_rows, (long long)A->n_cols,
                  (long long)x->n, (long long)y->n);
        return MTLG_ERR_INCOMPATIBLE_SIZE;
    }
    const bool f32 = x->dtype == MTLG_F32;
    if (f32) MTLG_TRY(ensure_f32_values(A));
    SetView sv;
    MTLG_TRY(csr_op_set(A, sv));
    SysDesc d;
    memset(&d, 0, sizeof d);
    d.n = int(A->n_rows);
    d.nnz = int(A->nnz);
    d.rp = A->rp.p;
    d.ci = A->ci.p;
    d.val = f32 ? (const void*)A->v32.p : (const void*)A->v64.p;
    d.val64 = A->v64.p;
    d.x = x->p;
    d.b = y->p;
    MTLG_CUDA(cudaMemcpyAsync(sv.desc, &d, sizeof d, cudaMemcpyHostToDevice, c->stream));
    SpmvOp op = spmv_op_default();
    op.x = SLOT_X;
    op.y = SLOT_B;
    if (pq) {
        set_dot(op, 0, OPND_XP, OPND_Y);   // (q = A p) || lazy_dot(p, q)
        set_kinds(op, RK_LDOT4);
        op.fin = FIN_STORE;
    }
    const int asg = assign == MTLG_ASSIGN ? ASG_SET : (assign == MTLG_PLUS ? ASG_ADD : ASG_SUB);
    // auto: thread per row for short regular rows, warp tasks for irregular
    // row lengths, stream tiles otherwise
    const int kern = c->spmv_kernel != 0 ? c->spmv_kernel
                     : A->irregular ? 2
                     : (A->n_rows > 0 && A->nnz <= int64_t(kScalarMeanRow) * A->n_rows) ? 3 : 1;
    if (!pq && kern == 3) {
        const int grid = int(std::min<int64_t>((A->n_rows + kBlock - 1) / kBlock, int64_t(c->sm_count) * 16));
        if (A->n_rows == 0) return MTLG_OK;
        const void* va = f32 ? (const void*)A->v32.p : (const void*)A->v64.p;
#define MTLG_SCALAR(T, ASG) k_spmv_scalar<T, ASG><<<grid, kBlock, 0, c->stream>>>(int(A->n_rows), A->rp.p, A->ci.p, (const T*)va, (const T*)x->p, (T*)y->p)
        if (f32) { if (asg == ASG_SET) MTLG_SCALAR(float, ASG_SET); else if (asg == ASG_ADD) MTLG_SCALAR(float, ASG_ADD); else MTLG_SCALAR(float, ASG_SUB); }
        else { if (asg == ASG_SET) MTLG_SCALAR(double, ASG_SET); else if (asg == ASG_ADD) MTLG_SCALAR(double, ASG_ADD); else MTLG_SCALAR(double, ASG_SUB); }
#undef MTLG_SCALAR
        c->launches++;
        MTLG_CUDA(cudaGetLastError());
        return MTLG_OK;
    }
    const bool warp = !pq && kern == 2;
    if (warp) {
        if (f32) return launch_spmv_rows<float>(c, A, x->p, y->p, asg);
        return launch_spmv_rows<double>(c, A, x->p, y->p, asg);
    }
    if (f32) MTLG_TRY(launch_spmv<float>(c, c->stream, sv, op, XF_PLAIN, asg));
    else MTLG_TRY(launch_spmv<double>(c, c->stream, sv, op, XF_PLAIN, asg));
    MTLG_CUDA(cudaGetLastError());
    if (pq) return read_dots(c, sv.st, pq, 1);
    return MTLG_OK;
}

int mtlg_spmv_gather_floor(mtlg_ctx* c, mtlg_csr* A, const mtlg_vec* x)
{
    MTLG_CHECK_ARG(c && A && x, "null handle");
    MTLG_CHECK_ARG(x->dtype == MTLG_F64 && x->n == A->n_cols, "x: FP64, n_cols entries");
    const int grid = c->sm_count * 8;
    if (!A->probe.p) MTLG_TRY(A->probe.alloc(c, size_t(grid) * kBlock));
    if (A->nnz == 0) return MTLG_OK;
    k_gather_floor<<<grid, kBlock, 0, c->stream>>>(A->nnz, A->ci.p, A->v64.p, static_cast<const double*>(x->p),
                                                   A->probe.p);
    c->launches++;
    MTLG_CUDA(cudaGetLastError());
    return MTLG_OK;
}

int mtlg_spmv(mtlg_ctx* c, mtlg_csr* A, const mtlg_vec* x, mtlg_vec* y, int assign)
{
    MTLG_TRACE(3049, "crs_cvec_mult");
    return spmv_impl(c, A, x, y, assign, nullptr);
}

int mtlg_spmv_dot(mtlg_ctx* c, mtlg_csr* A, const mtlg_vec* p, mtlg_vec* q, double* pq)
{
    MTLG_TRACE(9002, "crs_cvec_mult_dot");
    MTLG_CHECK_ARG(pq, "pq");
    return spmv_impl(c, A, p, q, MTLG_ASSIGN, pq);
}

static int vec_binary(mtlg_ctx* c, const mtlg_vec* x, const mtlg_vec* y, int kind, double scalar, double* out,
                      int rk = RK_DOT4)
{
    MTLG_CHECK_ARG(c && x && y, "null handle");
    MTLG_CHECK_ARG(x->dtype == y->dtype, "dtypes differ");
    if (x->n != y->n) {
        set_error("vector sizes %lld and %lld", (long long)x->n, (long long)y->n);
        return MTLG_ERR_INCOMPATIBLE_SIZE;
    }
    if (x->n == 0) {
        if (out) *out = 0.0;
        return MTLG_OK;
    }
    SetView sv;
    MTLG_TRY(vec_set(c, x->n, sv));
    SysDesc d;
    memset(&d, 0, sizeof d);
    d.n = int(x->n);
    d.x = x->p;
    d.b = y->p;
    MTLG_CUDA(cudaMemcpyAsync(sv.desc, &d, sizeof d, cudaMemcpyHostToDevice, c->stream));
    VecOp op = vec_op_default(kind);
    if (kind == VOP_DOT) {
        set_dot(op, 0, SLOT_X, SLOT_B);
        set_kinds(op, rk);
        op.fin = FIN_STORE;
    } else {  // VOP_AXPY: y += a x
        op.a = SLOT_B;
        op.b = SLOT_X;
        op.scalar = scalar;
    }
    if (x->dtype == MTLG_F64) MTLG_TRY(launch_vec<double>(c, c->stream, sv, op));
    else MTLG_TRY(launch_vec<float>(c, c->stream, sv, op));
    MTLG_CUDA(cudaGetLastError());
    if (out) return read_dots(c, sv.st, out, 1);
    return MTLG_OK;
}

extern "C++" {
namespace mtlg {
// dot of raw FP64 device vectors in the summation kind rk (used by the
// host-driven bodies)
int dot_raw(mtlg_ctx* c, int64_t n, const double* x, const double* y, int rk, double* out)
{
    mtlg_vec xv, yv;
    xv.ctx = yv.ctx = c;
    xv.n = yv.n = n;
    xv.dtype = yv.dtype = MTLG_F64;
    xv.p = const_cast<double*>(x);
    yv.p = const_cast<double*>(y);
    return vec_binary(c, &xv, &yv, VOP_DOT, 0.0, out, rk);
}
}  // namespace mtlg
}  // extern "C++"

int mtlg_dot(mtlg_ctx* c, const mtlg_vec* x, const mtlg_vec* y, double* out)
{
    MTLG_TRACE(2003, "dot");
    MTLG_CHECK_ARG(out, "out");
    return vec_binary(c, x, y, VOP_DOT, 0.0, out);
}

int mtlg_two_norm(mtlg_ctx* c, const mtlg_vec* x, double* out)
{
    MTLG_TRACE(2039, "two_norm");
    MTLG_CHECK_ARG(out, "out");
    MTLG_TRY(vec_binary(c, x, x, VOP_DOT, 0.0, out, RK_NORM4));
    *out = sqrt(fabs(*out));
    return MTLG_OK;
}

int mtlg_axpy(mtlg_ctx* c, double a, const mtlg_vec* x, mtlg_vec* y) { return vec_binary(c, x, y, VOP_AXPY, a, nullptr); }

// ------------------------------------------------------------------ preconditioners
int mtlg_pc_create(mtlg_ctx* c, mtlg_csr* A, int kind, mtlg_dtype storage, mtlg_pc** out)
{
    MTLG_TRACE(kind == MTLG_PC_ILU0 ? 5038 : kind == MTLG_PC_IC0 ? 5035 : kind == MTLG_PC_DIAGONAL ? 5050 : 9100,
               kind == MTLG_PC_ILU0 ? "ilu_0::factorize" : kind == MTLG_PC_IC0 ? "ic_0::factorize"
               : kind == MTLG_PC_DIAGONAL ? "diagonal::setup" : "identity::setup");
    MTLG_CHECK_ARG(c && A && out, "null handle");
    MTLG_CHECK_ARG(kind >= MTLG_PC_IDENTITY && kind <= MTLG_PC_IC0, "pc kind");
    MTLG_CHECK_ARG(ok_dtype(storage), "storage dtype");
    *out = nullptr;
    if (A->n_rows != A->n_cols) {
        set_error("preconditioner of a %lldx%lld matrix", (long long)A->n_rows, (long long)A->n_cols);
        return MTLG_ERR_NOT_SQUARE;
    }
    std::unique_ptr<mtlg_pc> P(new mtlg_pc);
    P->ctx = c;
    P->A = A;
    P->kind = kind;
    P->storage = storage;
    P->n = int(A->n_rows);
    MTLG_TRY(pc_build(P.get()));
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    *out = P.release();
    return MTLG_OK;
}

int mtlg_pc_destroy(mtlg_pc* P)
{
    if (!P) return MTLG_OK;
    MTLG_TRACE(9107, "pc.destroy");
    cudaStreamSynchronize(P->ctx->stream);
    if (P->fallback64) mtlg_pc_destroy(P->fallback64);
    if (P->adjoint) mtlg_pc_destroy(P->adjoint);
    purge_sets(P->ctx, P);
    delete P;
    return MTLG_OK;
}

int mtlg_pc_apply(mtlg_ctx* c, mtlg_pc* P, const mtlg_vec* x, mtlg_vec* y)
{
    MTLG_CHECK_ARG(c && P && x && y, "null handle");
    MTLG_TRACE(P->kind == MTLG_PC_ILU0 ? 5039 : P->kind == MTLG_PC_IC0 ? 5036 : P->kind == MTLG_PC_DIAGONAL ? 5051 : 9109,
               P->kind == MTLG_PC_ILU0 ? "ilu_0::solve" : P->kind == MTLG_PC_IC0 ? "ic_0::solve"
               : P->kind == MTLG_PC_DIAGONAL ? "diagonal::solve" : "identity::solve");
    MTLG_CHECK_ARG(x->dtype == y->dtype, "x and y dtypes differ");
    if (x->n != P->n || y->n != P->n) {
        set_error("preconditioner of size %d applied to %lld -> %lld", P->n, (long long)x->n, (long long)y->n);
        return MTLG_ERR_INCOMPATIBLE_SIZE;
    }
    if (P->n == 0) return MTLG_OK;
    if (P->kind == MTLG_PC_IDENTITY) {
        if (x->p != y->p) MTLG_CUDA(cudaMemcpyAsync(y->p, x->p, x->bytes(), cudaMemcpyDeviceToDevice, c->stream));
        return MTLG_OK;
    }
    const bool t32 = x->dtype == MTLG_F32, s32 = P->storage == MTLG_F32;
    if (t32 && !s32) return pc_sweeps<float, double>(P, x, y);
    if (t32 && s32) return pc_sweeps<float, float>(P, x, y);
    if (!t32 && s32) return pc_sweeps<double, float>(P, x, y);
    return pc_sweeps<double, double>(P, x, y);
}

int mtlg_pc_adjoint_apply(mtlg_ctx* c, mtlg_pc* P, const mtlg_vec* x, mtlg_vec* y)
{
    MTLG_CHECK_ARG(P, "pc");
    // identity, diagonal (real) and IC(0) are self-adjoint (ic_0.hpp:88-100)
    if (P->kind != MTLG_PC_ILU0) return mtlg_pc_apply(c, P, x, y);
    MTLG_TRACE(5040, "ilu_0::adjoint_solve");
    if (!P->adjoint) MTLG_TRY(pc_build_adjoint(P));
    return mtlg_pc_apply(c, P->adjoint, x, y);
}

int mtlg_pc_factor(const mtlg_pc* P, int which, int64_t* nnz, int64_t* row_ptr, int32_t* col, double* val)
{
    MTLG_CHECK_ARG(P && (which == 0 || which == 1), "pc/which");
    if (!P->has_factors()) {
        set_error("preconditioner has no triangular factors");
        return MTLG_ERR_NOT_SUPPORTED;
    }
    MTLG_TRY(ensure_flat(const_cast<mtlg_pc*>(P)));   // the download reads the flat layout
    const TriDev& T = which == 0 ? P->L : P->U;
    const bool has_diag = !(P->kind == MTLG_PC_ILU0 && which == 0);
    const bool diag_first = which == 1;  // U: diagonal first; IC's L: last
    const int64_t total = T.nnz + (has_diag ? P->n : 0);
    if (nnz) *nnz = total;
    if (!row_ptr && !col && !val) return MTLG_OK;
    mtlg_ctx* c = P->ctx;
    const size_t ss = P->ssize();
    std::vector<unsigned char> hv(size_t(std::max(T.nnz, 1)) * ss), hd(size_t(std::max(T.npad, 1)) * ss);
    MTLG_CUDA(cudaMemcpyAsync(hv.data(), T.val.p, size_t(T.nnz) * ss, cudaMemcpyDeviceToHost, c->stream));
    MTLG_CUDA(cudaMemcpyAsync(hd.data(), T.dia.p, size_t(T.npad) * ss, cudaMemcpyDeviceToHost, c->stream));
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    auto getv = [&](const std::vector<unsigned char>& b, size_t i) -> double {
        if (ss == 8) { double v; memcpy(&v, &b[i * 8], 8); return v; }
        float v; memcpy(&v, &b[i * 4], 4); return double(v);
    };
    std::vector<int> kof(P->n, -1);
    for (int k = 0; k < T.npad; ++k) if (T.h_row_of[k] >= 0) kof[T.h_row_of[k]] = k;
    int64_t o = 0;
    if (row_ptr) row_ptr[0] = 0;
    for (int i = 0; i < P->n; ++i) {
        const int k = kof[i];
        if (has_diag && diag_first) { if (col) col[o] = i; if (val) val[o] = getv(hd, k); ++o; }
        for (int e = T.h_rp[k]; e < T.h_rp[k + 1]; ++e, ++o) {
            if (col) col[o] = T.h_ci[e];
            if (val) val[o] = getv(hv, e);
        }
        if (has_diag && !diag_first) { if (col) col[o] = i; if (val) val[o] = getv(hd, k); ++o; }
        if (row_ptr) row_ptr[i + 1] = o;
    }
    return MTLG_OK;
}

int mtlg_pc_levels(const mtlg_pc* P, int* levels_L, int* levels_U)
{
    MTLG_CHECK_ARG(P, "pc");
    if (levels_L) *levels_L = P->L.nlev;
    if (levels_U) *levels_U = P->U.nlev;
    return MTLG_OK;
}

extern "C++" {
template <typename T, typename S>
static int sweep_plan_of(mtlg_ctx* c, mtlg_pc* P, int32_t* out)
{
    ChunkPlan& pl = P->plan[sizeof(T) == 4 ? 1 : 0];
    int& made = P->plan_kernel[sizeof(T) == 4 ? 1 : 0];
    const int setting = plan_setting(c);
    if (made != setting) {
        std::vector<std::pair<const TriDev*, const TriDev*>> f(1, {&P->L, &P->U});
        MTLG_TRY((plan_chunks<T, S>(c, f, pl)));
        made = setting;
    }
    for (int i = 0; i < 8; ++i) out[i] = 0;
    if (!pl.ok) return MTLG_OK;
    if (pl.grid) {
        out[2] = pl.gresident;
        out[3] = pl.gsmem;
        out[4] = 32 * pl.gnw;
        out[5] = P->L.gns;
        out[6] = pl.ntl;
        out[7] = pl.gsteps;
        return MTLG_OK;
    }
    const ChunkSide& sl = pl.side[0];
    out[0] = sl.rows;
    out[1] = P->L.nch;
    out[2] = sl.resident;
    out[3] = sl.smem;
    out[4] = sl.threads();
    out[5] = sl.entries();
    out[6] = sl.seg_rows;
    out[7] = sl.seg_ents;
    return MTLG_OK;
}
}

int mtlg_pc_sweep_plan(mtlg_ctx* c, mtlg_pc* P, int dtype, int32_t* out8)
{
    MTLG_CHECK_ARG(c && P && out8, "null handle");
    MTLG_CHECK_ARG(ok_dtype(dtype), "dtype");
    for (int i = 0; i < 8; ++i) out8[i] = 0;
    if (!P->has_factors() && P->kind != MTLG_PC_DIAGONAL) return MTLG_OK;
    const bool t32 = dtype == MTLG_F32, s32 = P->storage == MTLG_F32;
    if (t32 && !s32) return sweep_plan_of<float, double>(c, P, out8);
    if (t32 && s32) return sweep_plan_of<float, float>(c, P, out8);
    if (!t32 && s32) return sweep_plan_of<double, float>(c, P, out8);
    return sweep_plan_of<double, double>(c, P, out8);
}

int mtlg_grid_structure(int64_t n, const int64_t* row_ptr, const int32_t* col, int lower, int32_t* out8)
{
    MTLG_CHECK_ARG(out8 && n >= 0 && (n == 0 || (row_ptr && col)), "null array");
    for (int i = 0; i < 8; ++i) out8[i] = 0;
    MTLG_CHECK_ARG(n <= INT32_MAX && (n == 0 || row_ptr[n] <= INT32_MAX), "sizes beyond int32");
    // the strictly lower (upper) entries of each row, in storage order, as
    // the preconditioners' factor row lists hold them
    RowLists F;
    F.rp.assign(size_t(n) + 1, 0);
    for (int64_t r = 0; r < n; ++r) {
        for (int64_t e = row_ptr[r]; e < row_ptr[r + 1]; ++e)
            if (lower ? col[e] < r : col[e] > r) F.col.push_back(col[e]);
        F.rp[size_t(r) + 1] = int(F.col.size());
    }
    TriDev T;
    if (!detect_grid(F, int(n), lower != 0, T) || T.gnx == 0) return MTLG_OK;
    out8[0] = T.gnx;
    out8[1] = T.gny;
    out8[2] = T.gnz;
    out8[3] = T.gns;
    out8[4] = T.gns == 0 ? 0 : (T.gperm == (T.gns == 3 ? kGridFar3 : kGridFar2) ? 1 : 2);
    out8[5] = T.gskew;
    return MTLG_OK;
}

// ------------------------------------------------------------------ solves
static int check_solve_args(int solver, mtlg_csr* A, mtlg_vec* x, const mtlg_vec* b, const mtlg_pc* P)
{
    MTLG_CHECK_ARG(A && x && b, "null handle");
    MTLG_CHECK_ARG(solver >= MTLG_CG && solver <= MTLG_IDR_S, "solver");
    if (A->n_rows != A->n_cols) {
        set_error("solve with a %lldx%lld matrix", (long long)A->n_rows, (long long)A->n_cols);
        return MTLG_ERR_NOT_SQUARE;
    }
    if (x->n != A->n_rows || b->n != A->n_rows || (P && P->n != A->n_rows)) {
        set_error("solve sizes differ");
        return MTLG_ERR_INCOMPATIBLE_SIZE;
    }
    return MTLG_OK;
}

int mtlg_gmres_impl(mtlg_ctx* c, mtlg_csr* A, mtlg_pc* L, mtlg_pc* R, mtlg_vec* x, const mtlg_vec* b,
                    const mtlg_iter_params* p, mtlg_iter_result* r);

static int timed_result(mtlg_ctx* c, SolveSet& ss, cudaEvent_t e0, cudaEvent_t e1, mtlg_iter_result* res)
{
    MTLG_CUDA(cudaEventRecord(e1, c->stream));
    MTLG_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    MTLG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    SysState h;
    MTLG_CUDA(cudaMemcpy(&h, ss.st.p, sizeof h, cudaMemcpyDeviceToHost));
    int flags[1] = {0};
    MTLG_CUDA(cudaMemcpy(flags, ss.misc.p + 1, sizeof(int), cudaMemcpyDeviceToHost));
    if (res) {
        fill_result(h, ss.mixed != 0, res);
        res->seconds = ms * 1e-3;
    }
    if (c->log_cap) c->log_n = h.log_n;
    if (flags[0]) {
        int z = 0;
        MTLG_CUDA(cudaMemcpy(ss.misc.p + 1, &z, sizeof z, cudaMemcpyHostToDevice));
        MTLG_CUDA(cudaMemset(ss.tickets.p, 0, 8 * sizeof(int)));
        for (auto& si : ss.in) MTLG_TRY(pc_reset_sweep_state(si.P));
        MTLG_TRY(reset_set_sweep_buffers(ss));
        set_error("a device-side wait expired during the solve");
        return MTLG_ERR_TIMEOUT;
    }
    const int st = ss.mixed ? h.ostatus : h.status;
    if (st == MTLG_ST_BREAKDOWN && ss.solver == MTLG_BICGSTAB) {
        set_error("BiCGSTAB breakdown (zero rho, gamma or omega)");
        return MTLG_ERR_BREAKDOWN;
    }
    return MTLG_OK;
}

int mtlg_solve(mtlg_ctx* c, int solver, mtlg_csr* A, mtlg_pc* L, mtlg_pc* R, mtlg_vec* x, const mtlg_vec* b,
               const mtlg_iter_params* p, mtlg_iter_result* res)
{
    MTLG_TRACE(solver == MTLG_CG ? ((L && L->kind != MTLG_PC_IDENTITY) ? 7002 : 7001) : solver == MTLG_BICGSTAB ? 7004 : 9111,
               solver == MTLG_CG ? ((L && L->kind != MTLG_PC_IDENTITY) ? "cg" : "cg_without_pc")
               : solver == MTLG_BICGSTAB ? "bicgstab" : "gmres");
    MTLG_CHECK_ARG(c && p, "ctx/params");
    MTLG_TRY(check_solve_args(solver, A, x, b, L));
    MTLG_CHECK_ARG(x->dtype == b->dtype, "x and b dtypes differ");
    if (solver == MTLG_GMRES) {
        c->log_n = 0;   // GMRES runs its tests on the host: no residual log
        return mtlg_gmres_impl(c, A, L, R, x, b, p, res);
    }
    if (solver >= MTLG_BICG && solver <= MTLG_IDR_S) {
        c->log_n = 0;
        if (x->dtype != MTLG_F64) {
            set_error("the host-driven Krylov bodies take FP64 vectors");
            return MTLG_ERR_NOT_SUPPORTED;
        }
        KOp op;
        op.c = c;
        op.A = A;
        op.n = A->n_rows;
        return krylov_run(c, solver, op, L, R, static_cast<double*>(x->p), static_cast<const double*>(b->p), p, res);
    }
    const int f32 = x->dtype == MTLG_F32;
    if (L && L->kind == MTLG_PC_IDENTITY) L = nullptr;   // is_identity(P) short-cut (cg.hpp:80-81)
    SetKey key{A, L, solver, f32, 0, c->red_order};
    auto& slot = extra(c).sets[key];
    if (!slot) {
        std::unique_ptr<SolveSet> ss(new SolveSet);
        ss->solver = solver;
        ss->f32 = f32;
        SysInput si;
        si.A = A;
        si.P = L;
        ss->in.push_back(si);
        MTLG_TRY(build_set(c, *ss));
        slot = std::move(ss);
    }
    SolveSet& ss = *slot;
    SysInput& si = ss.in[0];
    si.x = x->p;
    si.b = b->p;
    si.max_iter = p->max_iter;
    si.rtol = p->rtol;
    si.atol = p->atol;
    si.norm_r0 = p->norm_r0;
    si.log = c->log_dev;
    si.log_cap = c->log_cap;
    c->log_n = 0;
    ss.h_desc[0].x = x->p;
    ss.h_desc[0].b = b->p;
    MTLG_CUDA(cudaMemcpyAsync(ss.desc.p, ss.h_desc.data(), sizeof(SysDesc), cudaMemcpyHostToDevice, c->stream));
    cudaEvent_t e0, e1;
    MTLG_CUDA(cudaEventCreate(&e0));
    MTLG_CUDA(cudaEventCreate(&e1));
    MTLG_CUDA(cudaEventRecord(e0, c->stream));
    int s = f32 ? run_plain<float>(ss) : run_plain<double>(ss);
    if (s == MTLG_OK) s = timed_result(c, ss, e0, e1, res);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return s;
}

// A refinement that stalled (the operator is too ill-conditioned for the
// FP32 inner solve) or broke down is finished by a plain FP64 solve of the
// same kind from its current iterate (from zero if that is not finite or
// its residual is not below ||b||), with
// the same stopping rule (relative to ||b||) and an iteration budget of
// max_iter; the result adds up both and sets fp64_fallback.  x and b are
// FP64 device vectors of A's size; P32 is the FP32 preconditioner (or null).
extern "C++" {
namespace mtlg {
int fp64_finish(mtlg_ctx* c, int solver, mtlg_csr* A, mtlg_pc* P32, double* x, const double* b, int max_iter,
                double rtol, mtlg_iter_result& r)
{
    mtlg_pc* P64 = nullptr;
    if (P32 && P32->kind != MTLG_PC_IDENTITY) {
        if (!P32->fallback64) MTLG_TRY(mtlg_pc_create(c, A, P32->kind, MTLG_F64, &P32->fallback64));
        P64 = P32->fallback64;
    }
    mtlg_vec xv, bv;
    xv.ctx = bv.ctx = c;
    xv.n = bv.n = A->n_rows;
    xv.dtype = bv.dtype = MTLG_F64;
    xv.p = x;
    bv.p = const_cast<double*>(b);
    // an iterate no better than zero (the FP32 solves may have driven it far
    // off before the stall showed) restarts from zero: from a huge start the
    // FP64 recursive residual would drift from the true one
    if (!std::isfinite(r.resid) || !(r.resid < r.norm_r0)) MTLG_CUDA(cudaMemsetAsync(x, 0, xv.bytes(), c->stream));
    mtlg_iter_params ip{};
    ip.max_iter = std::max(max_iter, 1);
    ip.rtol = rtol;
    ip.atol = 0.0;
    ip.norm_r0 = -1.0;
    mtlg_iter_result r2{};
    const int s = mtlg_solve(c, solver, A, P64, nullptr, &xv, &bv, &ip, &r2);
    r.iterations += r2.iterations;
    r.status = r2.status;
    r.error_code = r2.error_code;
    r.resid = r2.resid;
    r.relresid = r2.relresid;
    r.norm_r0 = r2.norm_r0;
    r.seconds += r2.seconds;
    r.fp64_fallback = 1;
    return s;
}

inline bool needs_fp64_finish(const mtlg_iter_result& r)
{
    return r.status == MTLG_ST_STALLED || r.status == MTLG_ST_BREAKDOWN;
}

// remaining refinement budget, at least one inner solve's worth
inline int fp64_budget(const mtlg_refine_params& rp, int used)
{
    const int64_t total = int64_t(std::max(rp.max_inner, 1)) * std::max(rp.max_outer, 1) - used;
    return int(std::max<int64_t>(std::max(rp.max_inner, 1), total));
}
}  // namespace mtlg
}

int mtlg_refine_solve(mtlg_ctx* c, int solver, mtlg_csr* A, mtlg_pc* P, mtlg_vec* x, const mtlg_vec* b,
                      const mtlg_refine_params* rp, mtlg_iter_result* res)
{
    MTLG_TRACE(9110, "refine");
    MTLG_CHECK_ARG(c && rp, "ctx/params");
    MTLG_TRY(check_solve_args(solver, A, x, b, P));
    MTLG_CHECK_ARG(x->dtype == MTLG_F64 && b->dtype == MTLG_F64, "refinement takes FP64 x and b");
    MTLG_CHECK_ARG(solver == MTLG_CG || solver == MTLG_BICGSTAB, "refinement runs CG or BiCGSTAB inside");
    if (P && P->kind == MTLG_PC_IDENTITY) P = nullptr;
    if (P && P->storage != MTLG_F32) {
        set_error("the inner FP32 solve needs a preconditioner stored in FP32");
        return MTLG_ERR_INVALID_ARG;
    }
    SetKey key{A, P, solver, 1, 1, c->red_order};
    auto& slot = extra(c).sets[key];
    if (!slot) {
        std::unique_ptr<SolveSet> ss(new SolveSet);
        ss->solver = solver;
        ss->f32 = 1;
        ss->mixed = 1;
        SysInput si;
        si.A = A;
        si.P = P;
        si.x = x->p;
        si.b = b->p;
        ss->in.push_back(si);
        MTLG_TRY(build_set(c, *ss));
        slot = std::move(ss);
    }
    SolveSet& ss = *slot;
    ss.in[0].x = x->p;
    ss.in[0].b = b->p;
    ss.h_desc[0].x64 = static_cast<double*>(x->p);
    ss.h_desc[0].b64 = static_cast<const double*>(b->p);
    ss.h_desc64[0].x = x->p;
    ss.h_desc64[0].b = b->p;
    MTLG_CUDA(cudaMemcpyAsync(ss.desc.p, ss.h_desc.data(), sizeof(SysDesc), cudaMemcpyHostToDevice, c->stream));
    MTLG_CUDA(cudaMemcpyAsync(ss.desc64.p, ss.h_desc64.data(), sizeof(SysDesc), cudaMemcpyHostToDevice, c->stream));
    cudaEvent_t e0, e1;
    MTLG_CUDA(cudaEventCreate(&e0));
    MTLG_CUDA(cudaEventCreate(&e1));
    MTLG_CUDA(cudaEventRecord(e0, c->stream));
    mtlg_iter_result r{};
    int s = run_refine(ss, *rp);
    if (s == MTLG_OK) s = timed_result(c, ss, e0, e1, &r);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if ((s == MTLG_OK || s == MTLG_ERR_BREAKDOWN) && needs_fp64_finish(r))
        s = fp64_finish(c, solver, A, P, static_cast<double*>(x->p), static_cast<const double*>(b->p),
                        fp64_budget(*rp, r.iterations), rp->rtol, r);
    if (res) *res = r;
    return s;
}

}  // extern "C"

#include "host_gmres.cuh"
#include "host_batch.cuh"
#include "formats.cuh"

extern "C" {

int mtlg_poisson2d_spmv(mtlg_ctx* c, int m, int n, const mtlg_vec* x, mtlg_vec* y, int assign)
{
    using namespace mtlg;
    MTLG_TRACE(3080, "poisson2D_dirichlet::mult");
    MTLG_CHECK_ARG(c && x && y && m >= 1 && n >= 1, "ctx/vectors/grid");
    MTLG_CHECK_ARG(x->dtype == MTLG_F64 && y->dtype == MTLG_F64, "poisson2D takes FP64 vectors");
    MTLG_CHECK_ARG(assign >= MTLG_ASSIGN && assign <= MTLG_MINUS, "assign");
    if (x->n != int64_t(m) * n || y->n != int64_t(m) * n) {
        set_error("poisson2D %dx%d needs vectors of %lld", m, n, (long long)m * n);
        return MTLG_ERR_INCOMPATIBLE_SIZE;
    }
    const int asg = assign == MTLG_ASSIGN ? ASG_SET : (assign == MTLG_PLUS ? ASG_ADD : ASG_SUB);
    return poisson2d_apply(c, m, n, static_cast<const double*>(x->p), static_cast<double*>(y->p), asg);
}

int mtlg_poisson2d_solve(mtlg_ctx* c, int solver, int m, int n, mtlg_vec* x, const mtlg_vec* b,
                         const mtlg_iter_params* p, mtlg_iter_result* res)
{
    using namespace mtlg;
    MTLG_TRACE(9112, "poisson2D_solve");
    MTLG_CHECK_ARG(c && x && b && p && m >= 1 && n >= 1, "ctx/vectors/params");
    MTLG_CHECK_ARG(x->dtype == MTLG_F64 && b->dtype == MTLG_F64, "FP64 vectors");
    MTLG_CHECK_ARG(solver != MTLG_GMRES && solver >= MTLG_CG && solver <= MTLG_IDR_S, "solver");
    if (x->n != int64_t(m) * n || b->n != int64_t(m) * n) {
        set_error("poisson2D %dx%d needs vectors of %lld", m, n, (long long)m * n);
        return MTLG_ERR_INCOMPATIBLE_SIZE;
    }
    KOp op;
    op.c = c;
    op.pm = m;
    op.pn = n;
    op.n = int64_t(m) * n;
    return krylov_run(c, solver, op, nullptr, nullptr, static_cast<double*>(x->p), static_cast<const double*>(b->p),
                      p, res);
}

}  // extern "C"
