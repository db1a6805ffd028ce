// Host side: context, device memory accounting, CSR / vector handles, tiling.
#pragma once
#include "sweep.cuh"
#include "gridsweep.cuh"
#include "refdot.cuh"
#include "trace.cuh"
#include "mmio.cuh"

#include <algorithm>
#include <atomic>
#include <thread>
#include <memory>
#include <mutex>

// Host-to-device copies of large host arrays through pinned staging blocks:
// a pageable cudaMemcpyAsync copies at a few GB/s and holds the calling
// thread; here the thread copies into a pinned block (a memcpy) and the DMA
// engine drains it while the thread fills the next one.  A block is reused
// once the copy recorded on its event has finished.
struct PinnedStage {
    static constexpr size_t kBlockBytes = size_t(8) << 20;
    static constexpr int kBlocks = 8;
    std::mutex init_mu;
    bool ready = false, failed = false;
    unsigned char* blk[kBlocks] = {};
    cudaEvent_t ev[kBlocks] = {};
    std::mutex mu[kBlocks];
    std::atomic<unsigned> next{0};
    bool init()
    {
        std::lock_guard<std::mutex> lk(init_mu);
        if (ready || failed) return ready;
        for (int i = 0; i < kBlocks; ++i) {
            if (cudaHostAlloc(reinterpret_cast<void**>(&blk[i]), kBlockBytes, cudaHostAllocDefault) != cudaSuccess ||
                cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                release();
                failed = true;
                return false;
            }
        }
        ready = true;
        return true;
    }
    void release()
    {
        for (int i = 0; i < kBlocks; ++i) {
            if (ev[i]) cudaEventSynchronize(ev[i]), cudaEventDestroy(ev[i]);
            if (blk[i]) cudaFreeHost(blk[i]);
            ev[i] = nullptr;
            blk[i] = nullptr;
        }
        ready = false;
    }
    ~PinnedStage() { release(); }
};

struct mtlg_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    size_t budget = 0;
    std::atomic<size_t> in_use{0};   // set-up may allocate from several host threads
    int64_t launches = 0;
    int sm_count = 148;
    int max_threads_per_sm = 2048, regs_per_sm = 65536;
    int smem_per_sm = 228 * 1024, smem_reserved_per_block = 1024;
    int sweep_grid = 148;       // persistent grid of the sweep / factor kernels
    int sweep_max_bpsm = 1;     // resident sweep CTAs per SM the device allows
    int sweep_bpsm = 0;         // tuning: sweep CTAs per SM (0: as many as fit)
    int sweep_sleep_ns = 0;     // tuning: back-off between polls of a dependency
    int sweep_nblocks = 0;      // tuning: absolute sweep grid (0: use sweep_bpsm)
    int loop_mode = 0;          // tuning: 0 chunked plain graphs, 1 WHILE conditional graph
    int spmv_kernel = 0;        // tuning: 0 auto (row-length statistics), 1 stream tiles, 2 warp tasks
    int chunk_rows = 0;         // tuning: rows per sweep chunk of new preconditioners (0: by size)
    int sweep_cluster = 0;      // tuning: CTAs per cluster of the chunked sweeps (0: automatic)
    int vec_ctas_per_sm = 2;    // tuning: CTAs per SM of the vector passes
    int sweep_kernel = 0;       // tuning: 0 chunked waves, 1 flat level order
    int grid_sweep = 1;         // tuning: 1 grid-stencil factors of new preconditioners get the grid layout and sweep
    int grid_warps = 0;         // tuning: compute warps per grid-sweep CTA (0: automatic, 4 or 8)
    int pc_apply_sync = 1;      // tuning: 1 each preconditioner apply checks its device waits (synchronizes), 0 queued
    int red_order = 0;          // tuning: FP64 dots and norms, 0 tile-parallel, 1 the reference's summation order
    int64_t admission_free_bytes = 0;     // tuning: stand-in for cudaMemGetInfo's free bytes (0: query)
    int64_t spin_limit = 0;               // tuning: polls before a device dependency wait gives up (0: kSpinLimit)
    double* log_dev = nullptr;            // residual log of single solves (2 * log_cap doubles)
    int log_cap = 0;
    int log_n = 0;                        // tests of the last logged solve (CG / BiCGSTAB)
    int64_t admission_reserve_bytes = -1; // tuning: bytes kept out of admission (-1: max(1 GiB, 2%))
    int* d_scratch_err = nullptr;
    PinnedStage stage;                    // staging blocks of large uploads
    cudaMemPool_t pool = nullptr;         // stream-ordered device memory (nullptr: cudaMalloc / cudaFree)
    int sweep_blocks() const
    {
        if (sweep_nblocks > 0) return std::min(sweep_nblocks, sm_count * sweep_max_bpsm);
        const int b = sweep_bpsm > 0 ? std::min(sweep_bpsm, sweep_max_bpsm) : 1;
        return sm_count * b;
    }
};

namespace mtlg {

static thread_local std::string g_err;
void set_error(const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}
const char* last_error() { return g_err.c_str(); }

inline size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Device allocation charged to the context (all buffers 256-byte aligned and
// padded by 16 bytes so vector loads of a tail never leave the allocation).
inline int dalloc(mtlg_ctx* c, void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    const size_t b = round_up(bytes + 16, 256);
    if (c->budget && c->in_use + b > c->budget) {
        set_error("device budget exceeded: %zu + %zu > %zu bytes", c->in_use.load(), b, c->budget);
        return MTLG_ERR_OOM;
    }
    // the context's pool: allocations and frees are ordered on its stream and
    // freed blocks stay in the pool for the next set-up (no device-wide
    // synchronization per buffer, as cudaMalloc / cudaFree have)
    cudaError_t e = c->pool ? cudaMallocFromPoolAsync(p, b, c->pool, c->stream) : cudaMalloc(p, b);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation of %zu bytes: %s", b, cudaGetErrorString(e));
        *p = nullptr;
        return MTLG_ERR_OOM;
    }
    c->in_use += b;
    return MTLG_OK;
}
inline void dfree(mtlg_ctx* c, void* p, size_t bytes)
{
    if (!p) return;
    if (bytes == 0) bytes = 16;
    if (c->pool) cudaFreeAsync(p, c->stream);
    else cudaFree(p);
    const size_t b = round_up(bytes + 16, 256);
    size_t cur = c->in_use.load();
    while (!c->in_use.compare_exchange_weak(cur, cur >= b ? cur - b : 0)) {
    }
}

// Runs f(i) for i in [0, n) on up to `threads` host threads (0: the
// hardware's), each taking the next index; f must be safe to run
// concurrently for different i.
template <typename F>
inline void parallel_for(int n, F&& f, int threads = 0)
{
    int t = threads > 0 ? threads : int(std::thread::hardware_concurrency());
    t = std::max(1, std::min(std::min(t, 32), n));
    if (t <= 1) {
        for (int i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    pool.reserve(size_t(t - 1));
    auto work = [&]() {
        for (int i = next++; i < n; i = next++) f(i);
    };
    for (int k = 1; k < t; ++k) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
}

// Host vectors whose elements are left uninitialized on resize (the large
// set-up arrays are written in full, in parallel, right after sizing: no
// single-threaded zeroing pass first).
template <typename T>
struct uninit_alloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = uninit_alloc<U>;
    };
    uninit_alloc() = default;
    template <typename U>
    uninit_alloc(const uninit_alloc<U>&) noexcept {}
    template <typename U>
    void construct(U* p) noexcept { ::new (static_cast<void*>(p)) U; }
    template <typename U, typename... A>
    void construct(U* p, A&&... a) { ::new (static_cast<void*>(p)) U(std::forward<A>(a)...); }
};
template <typename T>
using hvec = std::vector<T, uninit_alloc<T>>;

// out[0] = 0, out[i + 1] = out[i] + len(i) for i < n, in parallel blocks
// (block sums, their prefix, then each block's own prefix).
template <typename Len>
inline void parallel_prefix(int n, Len&& len, int* out)
{
    constexpr int kBlk = 1 << 16;
    const int nb = (n + kBlk - 1) / kBlk;
    std::vector<long long> bsum(size_t(nb) + 1, 0);
    parallel_for(nb, [&](int b) {
        long long t = 0;
        for (int i = b * kBlk; i < std::min(n, (b + 1) * kBlk); ++i) t += len(i);
        bsum[size_t(b) + 1] = t;
    });
    for (int b = 0; b < nb; ++b) bsum[size_t(b) + 1] += bsum[size_t(b)];
    out[0] = 0;
    parallel_for(nb, [&](int b) {
        long long t = bsum[size_t(b)];
        for (int i = b * kBlk; i < std::min(n, (b + 1) * kBlk); ++i) {
            t += len(i);
            out[i + 1] = int(t);
        }
    });
}

// Host -> device copy on the context's stream; arrays of 1 MiB and more go
// through the pinned staging blocks (not while the stream is capturing a
// graph: a captured copy would replay from a reused block).
inline int upload_bytes(mtlg_ctx* c, void* dst, const void* src, size_t bytes)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(c->stream, &cs);
    if (bytes < (size_t(1) << 20) || cs != cudaStreamCaptureStatusNone || !c->stage.init()) {
        MTLG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
        return MTLG_OK;
    }
    PinnedStage& S = c->stage;
    for (size_t off = 0; off < bytes; off += PinnedStage::kBlockBytes) {
        const size_t piece = std::min(PinnedStage::kBlockBytes, bytes - off);
        const int i = int(S.next++ % PinnedStage::kBlocks);
        std::lock_guard<std::mutex> lk(S.mu[i]);
        MTLG_CUDA(cudaEventSynchronize(S.ev[i]));
        memcpy(S.blk[i], static_cast<const unsigned char*>(src) + off, piece);
        MTLG_CUDA(cudaMemcpyAsync(static_cast<unsigned char*>(dst) + off, S.blk[i], piece, cudaMemcpyHostToDevice,
                                  c->stream));
        MTLG_CUDA(cudaEventRecord(S.ev[i], c->stream));
    }
    return MTLG_OK;
}

// Typed owning device buffer.
template <typename T>
struct DBuf {
    mtlg_ctx* ctx = nullptr;
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    int alloc(mtlg_ctx* c, size_t count)
    {
        release();
        ctx = c;
        n = count;
        void* q = nullptr;
        int s = dalloc(c, &q, count * sizeof(T));
        p = static_cast<T*>(q);
        return s;
    }
    int upload(mtlg_ctx* c, const T* h, size_t count)
    {
        MTLG_TRY(alloc(c, count));
        if (count) MTLG_TRY(upload_bytes(c, p, h, count * sizeof(T)));
        return MTLG_OK;
    }
    void release()
    {
        if (p && ctx) dfree(ctx, p, n * sizeof(T));
        p = nullptr;
        n = 0;
    }
};

template <typename T>
inline void tally(mtlg_ctx* c, int64_t k) { c->launches += k; }

// Tiling of one system's rows (see the Tile comment in common.cuh).
inline void plan_tiles(const int64_t* rp, int n, int sys, std::vector<Tile>& out)
{
    int r = 0;
    while (r < n) {
        int64_t len = rp[r + 1] - rp[r];
        if (len > kTileNnz) {
            out.push_back({sys, r, r + 1, TILE_LONG, int(rp[r]), int(rp[r + 1])});
            ++r;
            continue;
        }
        const int rb = r;
        int64_t nnz = 0;
        while (r < n && r - rb < kTileRows) {
            len = rp[r + 1] - rp[r];
            if (len > kTileNnz || nnz + len > kTileNnz) break;
            nnz += len;
            ++r;
        }
        out.push_back({sys, rb, r, TILE_STREAM, int(rp[rb]), int(rp[r])});
    }
}

inline void plan_warp_runs(const int64_t* rp, int n, std::vector<WarpTask>& out);

// Row-aligned warp tasks (see k_spmv_rows), listed in the order the warps
// take them: long-row tasks first (most entries first), then the runs.
inline void plan_warp_tasks(const int64_t* rp, int n, std::vector<WarpTask>& out)
{
    std::vector<WarpTask> runs;
    plan_warp_runs(rp, n, runs);
    out.clear();
    out.reserve(runs.size());
    for (const WarpTask& t : runs)
        if (t.row_end - t.row_begin == 1 && t.nnz_end - t.nnz_begin > kWarpNnz) out.push_back(t);
    std::stable_sort(out.begin(), out.end(), [](const WarpTask& a, const WarpTask& b) {
        return a.nnz_end - a.nnz_begin > b.nnz_end - b.nnz_begin;
    });
    for (const WarpTask& t : runs)
        if (!(t.row_end - t.row_begin == 1 && t.nnz_end - t.nnz_begin > kWarpNnz)) out.push_back(t);
}

// Tasks in row order: a run of consecutive rows with at most kWarpNnz
// entries (and rows), or one longer row.
inline void plan_warp_runs(const int64_t* rp, int n, std::vector<WarpTask>& out)
{
    int r = 0;
    while (r < n) {
        int64_t len = rp[r + 1] - rp[r];
        if (len > kWarpNnz) {
            out.push_back({r, r + 1, int(rp[r]), int(rp[r + 1])});
            ++r;
            continue;
        }
        const int rb = r;
        int64_t nnz = 0;
        while (r < n && r - rb < kWarpNnz) {
            len = rp[r + 1] - rp[r];
            if (len > kWarpNnz || nnz + len > kWarpNnz) break;
            nnz += len;
            ++r;
        }
        out.push_back({rb, r, int(rp[rb]), int(rp[r])});
    }
}

}  // namespace mtlg

using namespace mtlg;

struct mtlg_vec {
    mtlg_ctx* ctx = nullptr;
    int64_t n = 0;
    int dtype = MTLG_F64;
    void* p = nullptr;
    bool owned = false;
    size_t bytes() const { return size_t(n) * (dtype == MTLG_F64 ? 8 : 4); }
};

struct mtlg_csr {
    mtlg_ctx* ctx = nullptr;
    int64_t n_rows = 0, n_cols = 0, nnz = 0;
    DBuf<int> rp, ci;
    DBuf<double> v64;
    DBuf<float> v32;
    std::vector<int64_t> h_rp;
    std::vector<int> h_ci;
    std::vector<int> h_dpos;       // diagonal position per row (-1: none)
    DBuf<int> dpos;
    std::vector<Tile> tiles;
    int max_row = 0;
    int64_t tiles_by_kind[3] = {0, 0, 0};
    std::vector<WarpTask> wtasks;  // row-aligned warp tasks (irregular matrices)
    DBuf<WarpTask> d_wtasks;
    DBuf<int> wctr;                // k_spmv_rows task counter and exit count (self-resetting)
    DBuf<double> probe;            // k_gather_floor partial sums
    bool irregular = false;        // some row longer than kShortRow entries
    // single-system operation set (standalone SpMV / dot)
    DBuf<Tile> d_tiles;
    DBuf<int> d_stb;
    DBuf<double> partials;
    DBuf<unsigned> counters;
    DBuf<SysDesc> desc;
    DBuf<SysState> st;
    DBuf<int> misc;                // running, err[3]
    mtlg_csr* AT = nullptr;        // transpose (made for bicg / qmr on first need)
};

namespace mtlg {

inline int ensure_f32_values(mtlg_csr* A)
{
    if (A->v32.p) return MTLG_OK;
    MTLG_TRY(A->v32.alloc(A->ctx, size_t(A->nnz)));
    if (A->nnz) {
        const int grid = int(std::min<int64_t>((A->nnz + 255) / 256, 4096));
        k_cast_f64_f32<<<grid, 256, 0, A->ctx->stream>>>(A->nnz, A->v64.p, A->v32.p);
        A->ctx->launches++;
        MTLG_CUDA(cudaGetLastError());
    }
    return MTLG_OK;
}

// Single-system set over a CSR's own tiling (standalone operations).
inline int csr_op_set(mtlg_csr* A, SetView& sv)
{
    mtlg_ctx* c = A->ctx;
    if (!A->d_tiles.p) {
        MTLG_TRY(A->d_tiles.upload(c, A->tiles.data(), A->tiles.size()));
        int stb[2] = {0, int(A->tiles.size())};
        MTLG_TRY(A->d_stb.upload(c, stb, 2));
        MTLG_TRY(A->partials.alloc(c, std::max<size_t>(1, A->tiles.size()) * kMaxDots));
        MTLG_TRY(A->counters.alloc(c, 1));
        MTLG_CUDA(cudaMemsetAsync(A->counters.p, 0, sizeof(unsigned), c->stream));
        MTLG_TRY(A->desc.alloc(c, 1));
        MTLG_TRY(A->st.alloc(c, 1));
        MTLG_CUDA(cudaMemsetAsync(A->st.p, 0, sizeof(SysState), c->stream));
        MTLG_TRY(A->misc.alloc(c, 4));
        MTLG_CUDA(cudaMemsetAsync(A->misc.p, 0, 4 * sizeof(int), c->stream));
    }
    sv = SetView{};
    sv.tiles = A->d_tiles.p;
    sv.n_tiles = int(A->tiles.size());
    sv.n_sys = 1;
    sv.sys_tile_begin = A->d_stb.p;
    sv.desc = A->desc.p;
    sv.st = A->st.p;
    sv.partials = A->partials.p;
    sv.counters = A->counters.p;
    sv.running = A->misc.p;
    sv.err = A->misc.p + 1;
    sv.cond = 0;
    sv.use_cond = 0;
    return MTLG_OK;
}

inline SpmvOp spmv_op_default()
{
    SpmvOp op;
    memset(&op, 0, sizeof op);
    op.x = SLOT_X;
    op.y = SLOT_NONE;
    op.w = SLOT_NONE;
    op.y2 = SLOT_NONE;
    op.p = op.z = op.pnew = SLOT_NONE;
    op.ndot = 0;
    for (int j = 0; j < kMaxDots; ++j) op.da[j] = op.db[j] = op.dc[j] = OPND_ONE;
    op.fin = FIN_NONE;
    op.skip = SKIP_NONE;
    op.count_body = 0;
    return op;
}

inline VecOp vec_op_default(int kind)
{
    VecOp op;
    memset(&op, 0, sizeof op);
    op.op = kind;
    op.a = op.b = op.c = op.e = op.f = op.g = SLOT_NONE;
    for (int j = 0; j < kMaxDots; ++j) op.da[j] = op.db[j] = op.dc[j] = OPND_ONE;
    op.fin = FIN_NONE;
    op.skip = SKIP_NONE;
    return op;
}

// Kernel dispatchers ---------------------------------------------------------
// SpMV launch shape: persistent grid of (resident CTAs per SM) x SMs, two
// staging buffers of dynamic shared memory per CTA.
template <typename T, int XF, int ASG>
struct SpmvShape {
    static int occ;
    static int init()
    {
        const int smem = 2 * StageLayout<T>::BYTES;
        MTLG_CUDA(cudaFuncSetAttribute(k_spmv<T, XF, ASG>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int o = 1;
        MTLG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_spmv<T, XF, ASG>, kBlock, smem));
        occ = std::max(1, o);
        return MTLG_OK;
    }
};
template <typename T, int XF, int ASG> int SpmvShape<T, XF, ASG>::occ = 0;

#define MTLG_SPMV_VARIANTS(M)      \
    M(XF_PLAIN, ASG_SET)          \
    M(XF_PLAIN, ASG_ADD)          \
    M(XF_PLAIN, ASG_SUB)          \
    M(XF_PLAIN, ASG_WMINUS)       \
    M(XF_CG_P, ASG_SET)           \
    M(XF_CG_P_JAC, ASG_SET)       \
    M(XF_JAC, ASG_SET)

// Called once per context (kernel attributes may not change inside a stream
// capture).
inline int init_kernel_shapes()
{
#define MTLG_SPMV_INIT(XF, ASG)                              \
    MTLG_TRY((SpmvShape<double, XF, ASG>::init()));          \
    MTLG_TRY((SpmvShape<float, XF, ASG>::init()));
    MTLG_SPMV_VARIANTS(MTLG_SPMV_INIT)
#undef MTLG_SPMV_INIT
    MTLG_CUDA(cudaFuncSetAttribute(k_dot_ref, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDots * kRefWarpSmem));
    return MTLG_OK;
}

// Reference summation order (tuning "reduction_order" 1, FP64 only): a pass
// that reduces dots runs without them, and k_dot_ref then reduces the same
// vectors in the reference's order and finalizes.  Operand codes of the SpMV
// epilogue (its output y, its transformed input x') name the vectors that
// hold those values once the pass has run.
template <typename T>
inline bool ref_order_active(const mtlg_ctx* c, int ndot, int fin)
{
    return std::is_same<T, double>::value && c->red_order == 1 && ndot > 0 && fin != FIN_NONE;
}

inline int launch_dot_ref(mtlg_ctx* c, cudaStream_t st, const SetView& sv, const RefDotOp& r)
{
    if (sv.n_sys == 0) return MTLG_OK;
    k_dot_ref<<<sv.n_sys, 32 * r.ndot, r.ndot * kRefWarpSmem, st>>>(sv, r);
    c->launches++;
    return MTLG_OK;
}

template <typename OpT>
inline RefDotOp ref_dot_op(const OpT& op)
{
    RefDotOp r;
    memset(&r, 0, sizeof r);
    r.ndot = op.ndot;
    for (int j = 0; j < kMaxDots; ++j) {
        r.va[j] = op.da[j]; r.vb[j] = op.db[j]; r.vc[j] = op.dc[j];
        r.rk[j] = op.rk[j];
    }
    r.fin = op.fin;
    r.skip = op.skip;
    return r;
}

template <typename T>
inline int launch_spmv(mtlg_ctx* c, cudaStream_t st, const SetView& sv, const SpmvOp& op, int xf, int asg)
{
    if (sv.n_tiles == 0) return MTLG_OK;
    if (ref_order_active<T>(c, op.ndot, op.fin)) {
        RefDotOp r = ref_dot_op(op);
        auto resolve = [&](int code) {
            if (code == OPND_Y) return op.y;
            if (code == OPND_XP) return xf == XF_PLAIN ? op.x : op.pnew;
            return code;
        };
        for (int j = 0; j < op.ndot; ++j) {
            r.va[j] = resolve(op.da[j]); r.vb[j] = resolve(op.db[j]); r.vc[j] = resolve(op.dc[j]);
            if (r.va[j] == SLOT_NONE || r.vb[j] == SLOT_NONE || r.vc[j] == SLOT_NONE) {
                set_error("reference-order dot of an SpMV operand that is not stored");
                return MTLG_ERR_NOT_SUPPORTED;
            }
        }
        SpmvOp plain = op;
        plain.ndot = 0;
        plain.fin = FIN_NONE;
        MTLG_TRY(launch_spmv<T>(c, st, sv, plain, xf, asg));
        return launch_dot_ref(c, st, sv, r);
    }
    const int smem = 2 * StageLayout<T>::BYTES;
#define MTLG_SPMV_CASE(XF, ASG)                                                                    \
    if (xf == XF && asg == ASG) {                                                                 \
        const int grid = std::min(sv.n_tiles, c->sm_count * SpmvShape<T, XF, ASG>::occ);          \
        k_spmv<T, XF, ASG><<<grid, kBlock, smem, st>>>(sv, op);                                    \
        c->launches++;                                                                            \
        return MTLG_OK;                                                                           \
    }
    MTLG_SPMV_VARIANTS(MTLG_SPMV_CASE)
#undef MTLG_SPMV_CASE
    set_error("unsupported SpMV variant %d/%d", xf, asg);
    return MTLG_ERR_NOT_SUPPORTED;
}

template <typename T>
inline int launch_vec(mtlg_ctx* c, cudaStream_t st, const SetView& sv, const VecOp& op)
{
    if (sv.n_tiles == 0) return MTLG_OK;
    if (ref_order_active<T>(c, op.ndot, op.fin)) {
        // a finishing BiCGSTAB system still retires in the plain x/r pass
        VecOp plain = op;
        plain.ndot = 0;
        plain.fin = FIN_NONE;
        MTLG_TRY(launch_vec<T>(c, st, sv, plain));
        return launch_dot_ref(c, st, sv, ref_dot_op(op));
    }
    // one CTA per run of tiles, vec_ctas_per_sm per SM at most (each CTA
    // publishes its dot tally with one atomic on the system's counter)
    dim3 g(std::min(sv.n_tiles, c->vec_ctas_per_sm * c->sm_count)), b(kBlock);
    switch (op.op) {
#define MTLG_VEC_CASE(OP) \
    case OP: k_vec<T, OP><<<g, b, 0, st>>>(sv, op); break;
        MTLG_VEC_CASE(VOP_DOT)
        MTLG_VEC_CASE(VOP_AXPY)
        MTLG_VEC_CASE(VOP_CG_UPDATE)
        MTLG_VEC_CASE(VOP_BI_P)
        MTLG_VEC_CASE(VOP_BI_S)
        MTLG_VEC_CASE(VOP_BI_XR)
        MTLG_VEC_CASE(VOP_REF_CAST)
        MTLG_VEC_CASE(VOP_REF_UPDATE)
        MTLG_VEC_CASE(VOP_FILL)
        MTLG_VEC_CASE(VOP_COPY)
        MTLG_VEC_CASE(VOP_SCALE_COPY)
#undef MTLG_VEC_CASE
    default:
        set_error("unsupported vector op %d", op.op);
        return MTLG_ERR_NOT_SUPPORTED;
    }
    c->launches++;
    return MTLG_OK;
}

}  // namespace mtlg
