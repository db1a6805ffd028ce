// Level-scheduled sparse triangular solves and ILU(0)/IC(0) factorization.
//
// Rows are processed in dependency-level order (level = 1 + max level of the
// rows a row reads).  Work is handed out in tasks of kSweepRows rows through
// one atomic ticket, so a task is taken only by a running warp and every row
// it waits on belongs to an earlier task: the waits always end.  Each wait is
// still bounded (kSpinLimit polls); on expiry the kernel records a timeout
// in err[0] and finishes with a zero in place of the missing value.
//
// Readiness is carried by the value itself: the output vector is filled with
// an all-ones NaN pattern before the sweep and a finished row stores its
// result with one 4/8-byte relaxed store, which is single-copy atomic.  No
// separate flag, no fence.
//
// The per-row arithmetic is the reference's sequential row sweep
// (boost/numeric/mtl/operation/lower_trisolve.hpp:174-209,
//  upper_trisolve.hpp:161-176): rr = v[r]; rr -= a * w[c] for the row's
// off-diagonal entries in storage order; w[r] = rr * dia (dia = 1 for the
// unit diagonal of ILU's L, the stored inverse diagonal otherwise).
#pragma once
#include "kernels.cuh"

#include <type_traits>

namespace mtlg {

struct SweepOp {
    const SweepTask* tasks;
    int ntasks;
    int* ticket;        // zeroed before the launch
    int which;          // 0: L, 1: U
    int in, out;        // vector slots
    int reset;          // slot whose row is reset to the sentinel (SLOT_NONE: none)
    int skip;
    int fuse;           // SWF_* input transform of the L sweep
    int fuse_a, fuse_b, fuse_c;  // slots used by the transform
    int sleep_ns;       // back-off between polls
};

enum SweepFuse : int { SWF_NONE = 0, SWF_BI_P = 1 };

// Takes the next task index for the calling warp.  Every warp ends with
// exactly one grab past the last task; the final such grab (the
// (ntasks + warps)-th) returns the ticket to zero for the next launch.
__device__ __forceinline__ int grab_task(int* ticket, int ntasks)
{
    int t = 0;
    if ((threadIdx.x & 31) == 0) {
        t = atomicAdd(ticket, 1);
        const int W = int(gridDim.x) * int(blockDim.x >> 5);
        if (t == ntasks + W - 1) atomicExch(ticket, 0);
    }
    return __shfl_sync(0xffffffffu, t, 0);
}

// Polls p until it holds a value.  Gives up after kSpinLimit polls (sets
// err[0]) or as soon as another wait has given up, so a failed sweep drains
// in one bounded wait instead of one per row.
template <typename T>
__device__ __forceinline__ T wait_value(const T* p, int* err, int sleep_ns)
{
    T w = ld_volatile(p);
    if (!is_sentinel(w)) return w;
    long long spins = 0;
    do {
        if ((++spins & 255) == 0 && *(volatile int*)err) return T(0);
        if (spins > kSpinLimit) {
            atomicExch(err, 1);
            return T(0);
        }
        if (sleep_ns > 0) __nanosleep(sleep_ns);
        w = ld_volatile(p);
    } while (is_sentinel(w));
    return w;
}

// rr -= a * w as the reference evaluates it: fused for FP64 factors and
// vectors; with an FP32 factor or FP32 vector the product is rounded first.
template <typename T, typename S>
__device__ __forceinline__ T sweep_step(T rr, S a, T w);
template <> __device__ __forceinline__ double sweep_step<double, double>(double rr, double a, double w) { return fma(-a, w, rr); }
template <> __device__ __forceinline__ double sweep_step<double, float>(double rr, float a, double w) { return __dsub_rn(rr, __dmul_rn(double(a), w)); }
template <> __device__ __forceinline__ float sweep_step<float, float>(float rr, float a, float w) { return __fsub_rn(rr, __fmul_rn(a, w)); }
// FP32 vector, FP64 factor: the arithmetic is promoted to double, then stored
template <> __device__ __forceinline__ float sweep_step<float, double>(float rr, double a, float w) { return float(__dsub_rn(double(rr), __dmul_rn(a, double(w)))); }

// T: vector type, S: stored factor type (rr -= S * T is evaluated in T).
template <typename T, typename S>
__global__ void __launch_bounds__(kBlock) k_sweep(SetView sv, SweepOp op)
{
    const int lane = threadIdx.x & 31;
    for (;;) {
        const int t = grab_task(op.ticket, op.ntasks);
        if (t >= op.ntasks) break;
        const SweepTask task = op.tasks[t];
        const SysDesc& d = sv.desc[task.sys];
        if (skip_system(sv.st[task.sys], op.skip)) continue;
        if (*(volatile int*)sv.err) continue;   // a wait expired: drain
        const TriFactor& F = op.which == 0 ? d.L : d.U;
        const int k = task.first + lane;
        const int row = F.row_of[k];
        if (row < 0) continue;
        const int a = F.rp[k], e = F.rp[k + 1];
        const S* __restrict__ fv = static_cast<const S*>(F.val);
        const int* __restrict__ fc = F.ci;
        T* y = vptr<T>(d, op.out);
        const T* v = vptr<T>(d, op.in);
        T rr;
        if (op.fuse == SWF_BI_P) {
            // p = r + beta (p - omega v) for this row, then the sweep reads p
            // (bicgstab.hpp:48-55 with phat = solve(M, p))
            const SysState& s = sv.st[task.sys];
            T* P = vptr<T>(d, op.fuse_a);
            const T* R = vptr<T>(d, op.fuse_b);
            const T* V = vptr<T>(d, op.fuse_c);
            const T pr = (s.iter <= 1) ? R[row]
                                       : fma(T(s.beta), fma(-T(s.omega), V[row], P[row]), R[row]);
            P[row] = pr;
            rr = pr;
        } else {
            rr = v[row];
        }
        // Stage up to 8 entries in registers so their loads are in flight
        // before the first wait.
        int cc[8];
        S av[8];
        const int nr = min(e - a, 8);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (j < nr) { cc[j] = fc[a + j]; av[j] = fv[a + j]; }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (j < nr) rr = sweep_step<T, S>(rr, av[j], wait_value(y + cc[j], sv.err, op.sleep_ns));
        }
        for (int j = a + 8; j < e; ++j) rr = sweep_step<T, S>(rr, fv[j], wait_value(y + fc[j], sv.err, op.sleep_ns));
        const S dia = static_cast<const S*>(F.dia)[k];
        typedef typename std::conditional<(sizeof(S) > sizeof(T)), S, T>::type W;   // promoted type
        st_volatile(y + row, unsentinel(T(W(rr) * W(dia))));
        if (op.reset != SLOT_NONE) {
            // keeps the sentinel invariant of the sweep buffers: the L sweep
            // clears the U sweep's output row, the U sweep its consumed input
            T* R = vptr<T>(d, op.reset);
            R[row] = sentinel_value<T>();
        }
    }
}

// ------------------------------------------------------------ chunked sweep
// One CTA per chunk of contiguous rows (TriFactor's chunked layout), taken
// in processing order through one ticket.  The chunk's inputs are loaded
// into shared memory, then its waves run one after the other: a row reads
// the rows of its own chunk from shared memory (finished in earlier waves,
// made visible by the barrier between waves) and polls only rows of earlier
// chunks in global memory.  Every result is also published to global memory
// with a relaxed store for later chunks.  Chunks depend on earlier chunks
// only and waves on earlier waves, and a chunk is held by a running CTA, so
// the waits end; they are bounded all the same (wait_value).
//
// The chunk's structure (wave sizes, rows, multipliers, entries) streams
// through kStageBufs shared-memory buffers, one segment of waves per buffer,
// each segment brought in by one bulk copy per array (TMA, completion on an
// mbarrier) issued kStageBufs - 1 segments ahead of its use, so a wave's
// critical path is shared-memory reads, the arithmetic and the barrier.  The
// arithmetic per row is k_sweep's (same entry order, same roundings).
constexpr int kStageBufs = 3;

struct ChunkSweepOp {
    const GroupTask* tasks;
    int ntasks;
    int* ticket;        // zero before the launch; returned to zero by the last grab
    int which;          // 0: L, 1: U
    int in, out, reset; // vector slots (reset: SLOT_NONE or cleared to the sentinel)
    int skip;
    int sleep_ns;
    int vec_bytes;      // shared vector: rows of the largest chunk x sizeof(T), 16-byte multiple
    int rows_cap;       // staging buffer capacity in rows (multiple of 4)
    int ents_cap;       // ... and in entries (multiple of 4)
    int inbox;          // 1: a second shared vector receives the predecessor chunk's results
};

// Staging buffer layout: [wave sizes: rows_cap u32][rows: rows_cap int]
// [multipliers: rows_cap S][columns: ents_cap int][values: ents_cap S].
template <typename S>
__host__ __device__ __forceinline__ int stage_bytes(int rows_cap, int ents_cap)
{
    return rows_cap * (8 + int(sizeof(S))) + ents_cap * (4 + int(sizeof(S)));
}

__device__ __forceinline__ unsigned smem_u32(const void* p) { return unsigned(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for a staged segment: after kSpinLimit polls it records a
// timeout and keeps waiting up to the same bound again for the copy itself.
__device__ __forceinline__ void mbar_wait(unsigned long long* bar, unsigned parity, int* err)
{
    long long spins = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++spins == kSpinLimit) atomicExch(err, 1);
        if (spins > 2 * kSpinLimit) return;
    }
}

// Global -> shared bulk copy (16-byte aligned addresses, 16-byte multiple size).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ unsigned round16u(unsigned v) { return (v + 15u) & ~15u; }

// Issues the copies of segment `sg` into staging buffer `buf` (one thread).
template <typename S>
__device__ __forceinline__ void stage_segment(const TriFactor& F, const SegRec& sg, unsigned char* buf, int rows_cap,
                                              int ents_cap, unsigned long long* bar)
{
    const unsigned bw = round16u(unsigned(sg.nw) * 4u), br = round16u(unsigned(sg.np) * 4u);
    const unsigned bd = round16u(unsigned(sg.np) * unsigned(sizeof(S)));
    const unsigned bc = round16u(unsigned(sg.ne) * 4u), bv = round16u(unsigned(sg.ne) * unsigned(sizeof(S)));
    mbar_expect_tx(bar, bw + br + bd + bc + bv);
    unsigned char* o = buf;
    bulk_g2s(o, F.wv + sg.w0, bw, bar);
    o += rows_cap * 4;
    bulk_g2s(o, F.crow + sg.p0, br, bar);
    o += rows_cap * 4;
    bulk_g2s(o, static_cast<const S*>(F.cdia) + sg.p0, bd, bar);
    o += rows_cap * int(sizeof(S));
    if (bc) bulk_g2s(o, F.ccol + sg.e0, bc, bar);
    o += ents_cap * 4;
    if (bv) bulk_g2s(o, static_cast<const S*>(F.cval) + sg.e0, bv, bar);
}

// Relaxed accesses without a compiler memory clobber: the chunk kernel orders
// its shared-memory traffic with barriers, so these need not pin every other
// access in place (which would serialize a row's loads).
__device__ __forceinline__ float ld_relaxed_gpu(const float* p)
{
    float v;
    asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double ld_relaxed_gpu(const double* p)
{
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void st_relaxed_gpu(float* p, float v)
{
    asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v));
}
__device__ __forceinline__ void st_relaxed_gpu(double* p, double v)
{
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v));
}

// wait_value without the clobber (same bound and drain rule)
template <typename T>
__device__ __noinline__ T poll_value(const T* p, int* err, int sleep_ns)
{
    T w = ld_relaxed_gpu(p);
    long long spins = 0;
    while (is_sentinel(w)) {
        if ((++spins & 255) == 0 && *(volatile int*)err) return T(0);
        if (spins > kSpinLimit) {
            atomicExch(err, 1);
            return T(0);
        }
        if (sleep_ns > 0) __nanosleep(sleep_ns);
        w = ld_relaxed_gpu(p);
    }
    return w;
}

// One thread's row of a staged wave, in registers.
template <typename S, int KM>
struct WaveRow {
    int nw, K, row;
    S dia;
    int col[KM];
    S val[KM];
};

template <typename S, int KM>
__device__ __forceinline__ void wave_row(const unsigned* swv, const int* srow, const S* sdia, const int* scol,
                                         const S* sval, int w, int poff, int eoff, int tid, WaveRow<S, KM>& r)
{
    const unsigned m = swv[w];
    r.nw = int(m & 0xFFFFu);
    r.K = int(m >> 16);
    r.row = -1;
    if (tid < r.nw) {
        r.row = srow[poff + tid];
        r.dia = sdia[poff + tid];
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            r.col[k] = -1;
            if (k < r.K) {
                r.col[k] = scol[eoff + k * r.nw + tid];
                r.val[k] = sval[eoff + k * r.nw + tid];
            }
        }
    }
}

// ---- thread-block cluster helpers (distributed shared memory)
__device__ __forceinline__ unsigned cluster_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_size()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// shared::cluster address of `p` (own shared memory) in the CTA of rank `rank`
__device__ __forceinline__ unsigned map_rank(const void* p, unsigned rank)
{
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_cluster(unsigned addr, unsigned v)
{
    asm volatile("st.relaxed.cluster.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
__device__ __forceinline__ void st_cluster(unsigned addr, float v)
{
    asm volatile("st.relaxed.cluster.shared::cluster.f32 [%0], %1;" ::"r"(addr), "f"(v));
}
__device__ __forceinline__ void st_cluster(unsigned addr, double v)
{
    asm volatile("st.relaxed.cluster.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v));
}
__device__ __forceinline__ float ld_inbox(const float* p)
{
    float v;
    asm volatile("ld.relaxed.cluster.shared::cta.f32 %0, [%1];" : "=f"(v) : "r"(smem_u32(p)));
    return v;
}
__device__ __forceinline__ double ld_inbox(const double* p)
{
    double v;
    asm volatile("ld.relaxed.cluster.shared::cta.f64 %0, [%1];" : "=d"(v) : "r"(smem_u32(p)));
    return v;
}

// Polls an inbox entry (written by the previous CTA of the cluster); same
// bound and drain rule as poll_value.
template <typename T>
__device__ __noinline__ T poll_inbox(const T* p, int* err)
{
    T w = ld_inbox(p);
    long long spins = 0;
    while (is_sentinel(w)) {
        if ((++spins & 255) == 0 && *(volatile int*)err) return T(0);
        if (spins > kSpinLimit) {
            atomicExch(err, 1);
            return T(0);
        }
        w = ld_inbox(p);
    }
    return w;
}

// Launched in clusters of C CTAs (C = 1: plain launch).  A cluster takes a
// group of up to C consecutive chunks of one system; rank r works on chunk
// pos0 + r.  With op.inbox, rank r pushes each of its results into rank
// r + 1's inbox (a sentinel-filled shared vector indexed like the producer's
// rows), so the dependencies of a chunk on its predecessor are read from the
// CTA's own shared memory; all other dependencies on earlier chunks are
// polled in global memory.  Cluster barriers: after the group is handed out
// (all ranks see it), and after the inboxes are filled (no push lands before
// its inbox is reset); the next group's first barrier also ends this one, so
// no rank resets its inbox while the previous rank still pushes into it.
template <typename T, typename S, int NT, int KM>
__global__ void __launch_bounds__(NT) k_sweep_chunk(SetView sv, ChunkSweepOp op)
{
    extern __shared__ __align__(128) unsigned char chunk_smem[];
    __shared__ __align__(8) unsigned long long bars[kStageBufs];
    __shared__ unsigned s_task, s_go;
    __shared__ int s_nw[kStageBufs];
    typedef typename std::conditional<(sizeof(S) > sizeof(T)), S, T>::type W;   // promoted type
    T* yl = reinterpret_cast<T*>(chunk_smem);
    T* inbox = reinterpret_cast<T*>(chunk_smem + op.vec_bytes);
    unsigned char* stage = chunk_smem + op.vec_bytes * (op.inbox ? 2 : 1);
    const int sbytes = stage_bytes<S>(op.rows_cap, op.ents_cap);
    const int tid = threadIdx.x;
    const unsigned cr = cluster_rank(), C = cluster_size();
    const int nclusters = int(gridDim.x / C);
    if (tid == 0) {
        for (int b = 0; b < kStageBufs; ++b) mbar_init(&bars[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    unsigned consumed = 0;   // segments this CTA has consumed (uniform)
    for (;;) {
        if (cr == 0 && tid == 0) {
            const int t = atomicAdd(op.ticket, 1);
            if (t == op.ntasks + nclusters - 1) atomicExch(op.ticket, 0);
            unsigned go = 0;
            if (t < op.ntasks) {
                const GroupTask gt = op.tasks[t];
                go = !skip_system(sv.st[gt.sys], op.skip) && !*(volatile int*)sv.err;
            }
            for (unsigned q = 0; q < C; ++q) {
                st_cluster(map_rank(&s_task, q), unsigned(t));
                st_cluster(map_rank(&s_go, q), go);
            }
        }
        if (C > 1) cluster_sync(); else __syncthreads();
        const int t = int(s_task);
        const bool go = s_go != 0;
        GroupTask gt = {0, 0, 0, 0};
        if (t < op.ntasks && go) gt = op.tasks[t];
        const bool mine = int(cr) < gt.count;
        const SysDesc& d = sv.desc[gt.sys];
        const TriFactor& F = op.which == 0 ? d.L : d.U;
        const int pos = gt.pos0 + int(cr);
        const int B = F.chunk_rows;
        const int r0 = mine ? (op.which == 0 ? pos : F.nch - 1 - pos) * B : 0;
        const int nr = mine ? min(d.n - r0, B) : 0;
        const bool has_pred = op.inbox && mine && cr >= 1;
        const bool push = op.inbox && int(cr) + 1 < gt.count;
        const int r0p = op.which == 0 ? r0 - B : r0 + B;       // predecessor chunk's rows
        const int nrp = has_pred ? min(d.n - r0p, B) : 0;
        const int s0 = mine ? F.cseg[pos] : 0, nseg = mine ? F.cseg[pos + 1] - s0 : 0;
        SegRec ahead;   // thread 0: the next segment to stage
        if (tid == 0) {
            for (int i = 0; i < kStageBufs - 1 && i < nseg; ++i) {
                const SegRec sg = F.segs[s0 + i];
                const unsigned b = (consumed + i) % kStageBufs;
                s_nw[b] = sg.nw;
                stage_segment<S>(F, sg, stage + b * sbytes, op.rows_cap, op.ents_cap, &bars[b]);
            }
            if (kStageBufs - 1 < nseg) ahead = F.segs[s0 + kStageBufs - 1];
        }
        T* y = mine ? vptr<T>(d, op.out) : nullptr;
        T* R = mine && op.reset != SLOT_NONE ? vptr<T>(d, op.reset) : nullptr;
        if (mine) {
            const T* v = vptr<T>(d, op.in);
            for (int i = tid; i < nr; i += NT) yl[i] = v[r0 + i];
        }
        if (op.inbox)
            for (int i = tid; i < B; i += NT) inbox[i] = sentinel_value<T>();
        if (C > 1) cluster_sync(); else __syncthreads();
        if (t >= op.ntasks) break;
        if (!mine) continue;
        const unsigned rpush = push ? map_rank(inbox, cr + 1) : 0u;
        for (int i = 0; i < nseg; ++i) {
            const unsigned g = consumed + i, b = g % kStageBufs;
            if (tid == 0 && i + kStageBufs - 1 < nseg) {
                // buffer of segment i - 1, released by the barrier that ended it
                const unsigned bn = (g + kStageBufs - 1) % kStageBufs;
                s_nw[bn] = ahead.nw;
                stage_segment<S>(F, ahead, stage + bn * sbytes, op.rows_cap, op.ents_cap, &bars[bn]);
                if (i + kStageBufs < nseg) ahead = F.segs[s0 + i + kStageBufs];
            }
            mbar_wait(&bars[b], (g / kStageBufs) & 1u, sv.err);
            const unsigned char* buf = stage + b * sbytes;
            const unsigned* swv = reinterpret_cast<const unsigned*>(buf);
            const int* srow = reinterpret_cast<const int*>(buf + op.rows_cap * 4);
            const S* sdia = reinterpret_cast<const S*>(buf + op.rows_cap * 8);
            const int* scol = reinterpret_cast<const int*>(buf + op.rows_cap * (8 + int(sizeof(S))));
            const S* sval = reinterpret_cast<const S*>(buf + op.rows_cap * (8 + int(sizeof(S))) + op.ents_cap * 4);
            const int nwaves = s_nw[b];
            int poff = 0, eoff = 0;
            WaveRow<S, KM> cur, nxt;
            wave_row<S, KM>(swv, srow, sdia, scol, sval, 0, 0, 0, tid, cur);
            for (int w = 0; w < nwaves; ++w) {
                if (cur.row >= 0) {
                    // all in-chunk reads at once, then the waits on earlier chunks
                    T rr = yl[cur.row - r0];
                    T dv[KM];
                    bool ext = false;
#pragma unroll
                    for (int k = 0; k < KM; ++k) {
                        const unsigned lc = unsigned(cur.col[k] - r0);
                        dv[k] = T(0);
                        if (lc < unsigned(nr)) dv[k] = yl[lc];
                        else if (cur.col[k] >= 0) ext = true;
                    }
                    if (ext) {
#pragma unroll
                        for (int k = 0; k < KM; ++k) {
                            const int col = cur.col[k];
                            if (col >= 0 && unsigned(col - r0) >= unsigned(nr)) {
                                const unsigned lp = unsigned(col - r0p);
                                dv[k] = lp < unsigned(nrp) ? poll_inbox(inbox + lp, sv.err)
                                                           : poll_value(y + col, sv.err, op.sleep_ns);
                            }
                        }
                    }
#pragma unroll
                    for (int k = 0; k < KM; ++k)
                        if (cur.col[k] >= 0) rr = sweep_step<T, S>(rr, cur.val[k], dv[k]);
                    const T out = unsentinel(T(W(rr) * W(cur.dia)));
                    yl[cur.row - r0] = out;
                    if (push) st_cluster(rpush + unsigned(cur.row - r0) * unsigned(sizeof(T)), out);
                    st_relaxed_gpu(y + cur.row, out);
                    if (R) R[cur.row] = sentinel_value<T>();
                }
                poff += cur.nw;
                eoff += cur.K * cur.nw;
                if (w + 1 < nwaves) wave_row<S, KM>(swv, srow, sdia, scol, sval, w + 1, poff, eoff, tid, nxt);
                __syncthreads();
                cur = nxt;
            }
        }
        consumed += unsigned(nseg);
    }
}

// ---------------------------------------------------------------- factorization
// Device-side ILU(0) (boost/numeric/itl/pc/ilu_0.hpp:45-82, Saad's IKJ form
// without fill): row i, for each k < i in its pattern (ascending):
//   a_ik *= inv_dia[k];  a_ij -= a_ik * LU[k][j] for the later entries j of
//   row i that row k also holds;  then inv_dia[i] = 1 / LU[i][i].
// Rows wait for the rows k they read (levels of the L pattern).
struct FactorOp {
    const SweepTask* tasks;   // L schedule (row_of of the L factor)
    int ntasks;
    int* ticket;
    const int* row_of;        // level-ordered rows
    const int* rp;            // A's pattern
    const int* ci;
    double* lu;               // FP64 working values (A's order)
    double* inv_dia;          // [n] sentinel-filled
    const int* dpos;          // diagonal position per row
    // IC(0): transposed upper pattern: for row i the (k < i) entries a_ki
    const int* lt_rp;
    const int* lt_src;        // position of a_ki in A's values
    const int* lt_row;        // k
    const double* a;          // A's FP64 values (IC(0) reads, never writes)
    int* err;
};

__device__ __forceinline__ double wait_acquire(const double* p, int* err)
{
    double w;
    asm volatile("ld.acquire.gpu.global.f64 %0, [%1];" : "=d"(w) : "l"(p) : "memory");
    long long spins = 0;
    while (is_sentinel(w)) {
        if ((++spins & 255) == 0 && *(volatile int*)err) return 1.0;
        if (spins > kSpinLimit) {
            atomicExch(err, 1);
            return 1.0;
        }
        __nanosleep(32);
        asm volatile("ld.acquire.gpu.global.f64 %0, [%1];" : "=d"(w) : "l"(p) : "memory");
    }
    return w;
}

__device__ __forceinline__ void publish_release(double* p, double v)
{
    asm volatile("st.release.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(unsentinel(v)) : "memory");
}

__global__ void __launch_bounds__(kBlock) k_ilu0_factor(FactorOp op)
{
    const int lane = threadIdx.x & 31;
    for (;;) {
        const int t = grab_task(op.ticket, op.ntasks);
        if (t >= op.ntasks) break;
        const int i = op.row_of[op.tasks[t].first + lane];
        if (i < 0 || *(volatile int*)op.err) continue;
        const int a = op.rp[i], e = op.rp[i + 1];
        for (int kc = a; kc < e; ++kc) {
            const int k = op.ci[kc];
            if (k >= i) break;
            const double ik = wait_acquire(op.inv_dia + k, op.err);
            const double aik = __dmul_rn(op.lu[kc], ik);
            op.lu[kc] = aik;
            // merge-walk row k (sorted) against the rest of row i (sorted)
            int kp = op.rp[k];
            const int ke = op.rp[k + 1];
            for (int jc = kc + 1; jc < e; ++jc) {
                const int j = op.ci[jc];
                while (kp < ke && op.ci[kp] < j) ++kp;
                if (kp < ke && op.ci[kp] == j) op.lu[jc] = fma(-aik, __ldcg(op.lu + kp), op.lu[jc]);
            }
        }
        const double piv = op.lu[op.dpos[i]];
        __threadfence();
        publish_release(op.inv_dia + i, __ddiv_rn(1.0, piv));
    }
}

// Device-side IC(0) pivots (boost/numeric/itl/pc/ic_0.hpp:136-186).  The
// reference's elimination of row k touches, in row i of U, only entries with
// column in (k, i] -- the diagonal -- so each pivot is
//   u_ii = a_ii - sum_{k<i, a_ki != 0, ascending k} (a_ki / sqrt(u_kk))^2
// with the stored inverse 1/sqrt(u_ii).  Off-diagonals are a_ij / sqrt(u_ii),
// filled afterwards by k_fill_factor.
__global__ void __launch_bounds__(kBlock) k_ic0_factor(FactorOp op)
{
    const int lane = threadIdx.x & 31;
    for (;;) {
        const int t = grab_task(op.ticket, op.ntasks);
        if (t >= op.ntasks) break;
        const int i = op.row_of[op.tasks[t].first + lane];
        if (i < 0 || *(volatile int*)op.err) continue;
        double diag = op.a[op.dpos[i]];
        for (int q = op.lt_rp[i]; q < op.lt_rp[i + 1]; ++q) {
            const int k = op.lt_row[q];
            const double ik = wait_acquire(op.inv_dia + k, op.err);
            const double dk = __dmul_rn(op.a[op.lt_src[q]], ik);
            // u_ii -= d * d with the product rounded first, as the reference
            // evaluates it (no fused multiply-add)
            diag = __dsub_rn(diag, __dmul_rn(dk, dk));
        }
        publish_release(op.inv_dia + i, __ddiv_rn(1.0, __dsqrt_rn(diag)));
    }
}

// Level-ordered factor values: val[e] = S(src[idx[e]] * (mul[e] >= 0 ?
// inv_dia[mul[e]] : 1)); dia[k] = S(row_of[k] >= 0 && dia_mode ? inv_dia[row] : 1).
__global__ void k_fill_factor(int nent, const int* __restrict__ idx, const int* __restrict__ mul,
                              const double* __restrict__ src, const double* __restrict__ inv_dia, void* val,
                              int val_f32)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nent; e += gridDim.x * blockDim.x) {
        double v = src[idx[e]];
        if (mul[e] >= 0) v = v * inv_dia[mul[e]];
        if (val_f32) static_cast<float*>(val)[e] = float(v);
        else static_cast<double*>(val)[e] = v;
    }
}

__global__ void k_fill_dia(int nrows, const int* __restrict__ row_of, const double* __restrict__ inv_dia, int unit,
                           void* dia, int f32)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nrows; k += gridDim.x * blockDim.x) {
        const int r = row_of[k];
        double v = (unit || r < 0) ? 1.0 : inv_dia[r];
        if (f32) static_cast<float*>(dia)[k] = float(v);
        else static_cast<double*>(dia)[k] = v;
    }
}

// Jacobi: inv_diag[i] = 1 / a_ii in the storage precision
// (boost/numeric/itl/pc/diagonal.hpp:37-45, math::reciprocal).
__global__ void k_inv_diag(int n, const double* __restrict__ a, const int* __restrict__ dpos, void* out, int f32)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = dpos[i] >= 0 ? a[dpos[i]] : 0.0;
        if (f32) static_cast<float*>(out)[i] = 1.0f / float(v);
        else static_cast<double*>(out)[i] = 1.0 / v;
    }
}

__global__ void k_cast_f64_f32(long long n, const double* __restrict__ in, float* __restrict__ out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = float(in[i]);
}

// Sentinel fill of a vector before a sweep (all-ones bit pattern).
__global__ void k_fill_bits(long long nbytes4, unsigned* p)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nbytes4; i += (long long)gridDim.x * blockDim.x)
        p[i] = 0xFFFFFFFFu;
}

}  // namespace mtlg
