// Level-scheduled sparse triangular solves and ILU(0)/IC(0) factorization.
//
// Rows are processed in dependency-level order (level = 1 + max level of the
// rows a row reads).  Work is handed out in tasks of kSweepRows rows through
// one atomic ticket, so a task is taken only by a running warp and every row
// it waits on belongs to an earlier task: the waits always end.  Each wait is
// still bounded (the context's spin_limit polls, default kSpinLimit); on
// expiry the kernel records a timeout
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

// Polls p until it holds a value.  Gives up after lim polls (the context's
// "spin_limit"; sets
// err[0]) or as soon as another wait has given up, so a failed sweep drains
// in one bounded wait instead of one per row.
template <typename T>
__device__ __forceinline__ T wait_value(const T* p, int* err, int sleep_ns, long long lim)
{
    T w = ld_volatile(p);
    if (!is_sentinel(w)) return w;
    long long spins = 0;
    do {
        if ((++spins & 255) == 0 && *(volatile int*)err) return T(0);
        if (spins > (lim > 0 ? lim : kSpinLimit)) {
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
            if (j < nr) rr = sweep_step<T, S>(rr, av[j], wait_value(y + cc[j], sv.err, op.sleep_ns, sv.spin));
        }
        for (int j = a + 8; j < e; ++j) rr = sweep_step<T, S>(rr, fv[j], wait_value(y + fc[j], sv.err, op.sleep_ns, sv.spin));
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
// in processing order through one ticket.  Warp roles:
//  - CW compute warps (CT = 32 CW threads) run the chunk's waves one after
//    the other, RPT rows per thread (thread i holds rows i, i + CT, ... of a
//    wave of at most CT RPT rows; slots past the wave's rows repeat its last
//    row, so the rows need no branches), with a barrier among the compute
//    warps between waves: a row reads the rows of its own chunk from a
//    shared vector (finished in earlier waves), and its result is published
//    in position order (one coalesced store per warp, row group and wave)
//    for later chunks;
//  - kRecvWarps receiver warps fetch the results of earlier chunks this chunk
//    needs, in the order the waves consume them, many requests in flight,
//    into receive slots in shared memory, so a compute thread waits on the
//    value itself, never on an L2 round trip of its own;
//  - the producer warp streams the chunk's structure (wave sizes, rows,
//    multipliers, entries) through kStageBufs shared buffers, one segment of
//    waves per buffer, one bulk copy (TMA) per array, with full / empty
//    mbarrier pairs between it and the compute threads.
// The chunk's right-hand sides are loaded into the shared vector up front
// and the chunk's outputs written back at its end by all warps, coalesced.  Chunks
// depend on earlier chunks only and waves on earlier waves, and a chunk is
// held by a running CTA, so the waits end; they are bounded all the same
// (spin_limit polls, then a timeout flag and a drain).  The arithmetic per
// row is k_sweep's (same entry order, same roundings).
constexpr int kStageBufs = 3;
constexpr int kRecvDepth = 2;                       // receive quads in flight per receiver lane
constexpr int kRecvWarps = 3;                       // receiver warps
constexpr int kChunkExtraWarps = kRecvWarps + 1;    // receiver warps and the producer warp after the compute warps

struct ChunkSweepOp {
    const GroupTask* tasks;
    int ntasks;
    int* ticket;        // zero before the launch; returned to zero by the last grab
    int which;          // 0: L, 1: U
    int in, out, reset; // vector slots (reset: SLOT_NONE or cleared to the sentinel)
    int skip;
    int sleep_ns;
    int vec_bytes;      // shared cells (chunk rows, the +0 cell, receive slots) of the largest chunk, 16-byte multiple
    int rows_cap;       // staging buffer capacity in rows (multiple of 4)
    int ents_cap;       // ... and in entries (multiple of 4)
    int cl;             // cluster size the task table is built for (tasks: ntasks groups of cl entries)
    int pad;
};

// Staging buffer layout: [wave sizes: rows_cap u32][rows: rows_cap int]
// [push cells: rows_cap int][multipliers: rows_cap S][columns: ents_cap int]
// [values: ents_cap S].
template <typename S>
__host__ __device__ __forceinline__ int stage_bytes(int rows_cap, int ents_cap)
{
    return rows_cap * (12 + int(sizeof(S))) + ents_cap * (4 + int(sizeof(S)));
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

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
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

// Bounded mbarrier wait: after kSpinLimit polls it records a timeout and
// keeps waiting up to the same bound again (a staged copy always completes).
// The bound is fixed, not the context's spin_limit: it guards the copies of
// the chunk's own structure, which are in flight whatever the dependencies
// do, so a CTA never reads a buffer before its copy lands, never refills one
// the compute warps still read, and never ends with a copy in flight.
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

// A factor's chunked-layout arrays, copied into registers once per chunk
// (fields read through the system descriptor would be reloaded from global
// memory after every barrier).
struct ChunkArrays {
    const SegRec* segs;
    const unsigned* wv;
    const int* crow;
    const int* cpush;
    const void* cdia;
    const int* ccol;
    const void* cval;
};

// Issues the copies of segment `sg` into staging buffer `buf` (one thread).
template <typename S>
__device__ __forceinline__ void stage_segment(const ChunkArrays& F, const SegRec& sg, unsigned char* buf, int rows_cap,
                                              int ents_cap, unsigned long long* bar)
{
    const unsigned bw = round16u(unsigned(sg.nw) * 4u), br = round16u(unsigned(sg.np) * 4u);
    const unsigned bd = round16u(unsigned(sg.np) * unsigned(sizeof(S)));
    const unsigned bc = round16u(unsigned(sg.ne) * 4u), bv = round16u(unsigned(sg.ne) * unsigned(sizeof(S)));
    mbar_expect_tx(bar, bw + 2 * br + bd + bc + bv);
    unsigned char* o = buf;
    bulk_g2s(o, F.wv + sg.w0, bw, bar);
    o += rows_cap * 4;
    bulk_g2s(o, F.crow + sg.p0, br, bar);
    o += rows_cap * 4;
    bulk_g2s(o, F.cpush + sg.p0, br, bar);
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
// receive slots: written by the receiver warps, polled by the compute threads
__device__ __forceinline__ float ld_slot(const float* p)
{
    float v;
    asm volatile("ld.volatile.shared.f32 %0, [%1];" : "=f"(v) : "r"(smem_u32(p)));
    return v;
}
__device__ __forceinline__ double ld_slot(const double* p)
{
    double v;
    asm volatile("ld.volatile.shared.f64 %0, [%1];" : "=d"(v) : "r"(smem_u32(p)));
    return v;
}
__device__ __forceinline__ void st_slot(float* p, float v)
{
    asm volatile("st.volatile.shared.f32 [%0], %1;" ::"r"(smem_u32(p)), "f"(v));
}
__device__ __forceinline__ void st_slot(double* p, double v)
{
    asm volatile("st.volatile.shared.f64 [%0], %1;" ::"r"(smem_u32(p)), "d"(v));
}

// A result of an earlier chunk read directly (same bound and drain rule as wait_value).
template <typename T>
__device__ __noinline__ T poll_value(const T* p, int* err, int sleep_ns, long long lim)
{
    T w = ld_relaxed_gpu(p);
    long long spins = 0;
    while (is_sentinel(w)) {
        if ((++spins & 255) == 0 && *(volatile int*)err) return T(0);
        if (spins > (lim > 0 ? lim : kSpinLimit)) {
            atomicExch(err, 1);
            return T(0);
        }
        if (sleep_ns > 0) __nanosleep(sleep_ns);
        w = ld_relaxed_gpu(p);
    }
    return w;
}

// A receive slot not filled yet: wait for the receiver (same bound and drain rule).
template <typename T>
__device__ __noinline__ T poll_slot(const T* p, int* err, long long lim)
{
    T w = ld_slot(p);
    long long spins = 0;
    while (is_sentinel(w)) {
        if ((++spins & 255) == 0 && *(volatile int*)err) return T(0);
        if (spins > (lim > 0 ? lim : kSpinLimit)) {
            atomicExch(err, 1);
            return T(0);
        }
        w = ld_slot(p);
    }
    return w;
}

// 4 consecutive results (16-byte aligned for float, 32 for double), relaxed.
__device__ __forceinline__ void ld_relaxed_gpu4(const float* p, float* v)
{
    asm volatile("ld.relaxed.gpu.global.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3])
                 : "l"(p));
}
__device__ __forceinline__ void ld_relaxed_gpu4(const double* p, double* v)
{
    asm volatile("ld.relaxed.gpu.global.v2.f64 {%0, %1}, [%2];" : "=d"(v[0]), "=d"(v[1]) : "l"(p));
    asm volatile("ld.relaxed.gpu.global.v2.f64 {%0, %1}, [%2];" : "=d"(v[2]), "=d"(v[3]) : "l"(p + 2));
}
__device__ __forceinline__ void st_slot4(float* p, const float* v)
{
    asm volatile("st.volatile.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(smem_u32(p)), "f"(v[0]), "f"(v[1]), "f"(v[2]),
                 "f"(v[3]));
}
__device__ __forceinline__ void st_slot4(double* p, const double* v)
{
    asm volatile("st.volatile.shared.v2.f64 [%0], {%1, %2};" ::"r"(smem_u32(p)), "d"(v[0]), "d"(v[1]));
    asm volatile("st.volatile.shared.v2.f64 [%0], {%1, %2};" ::"r"(smem_u32(p + 2)), "d"(v[2]), "d"(v[3]));
}

// Receiver warps: fill slot[e] = ypos[cext[x0 + e]] for the chunk's nx slots
// (x0, nx multiples of 4), four slots (a quad) at a time, in slot order.
// Quads go in rows of 32 (lane l holds quad l of a row, so a row's loads
// coalesce); receiver warp rw of kRecvWarps takes rows rw, rw + kRecvWarps,
// ..., kRecvDepth of them at a time, and moves to its next batch when the
// batch is complete.  A quad whose used slots are 4 consecutive aligned
// positions moves with one vector load; the others slot by slot.  A value
// that is still the sentinel is requested again (the slot keeps the sentinel
// meanwhile); the wait is bounded like the others (on expiry the remaining
// slots get a zero so the compute threads drain).  With cqpull (the previous
// chunk runs in the previous CTA of the cluster and pushes its results into
// this chunk's slots; PULL) only the slots in cqpull's masks are fetched, one
// by one in quads that also hold pushed slots.
template <typename T, bool PULL>
__device__ __forceinline__ void receive_chunk(const int* __restrict__ cext, const int2* __restrict__ cquad,
                                              const int* __restrict__ cqpull, int x0, int nx, const T* ypos, T* slot,
                                              int rw, int lane, int* err, int sleep_ns, long long lim)
{
    const int q0 = x0 >> 2, nq = nx >> 2;
    for (int row0 = rw; 32 * row0 < nq; row0 += kRecvWarps * kRecvDepth) {
        int qd[kRecvDepth];
        int2 qi[kRecvDepth];
        unsigned pend[kRecvDepth];
#pragma unroll
        for (int j = 0; j < kRecvDepth; ++j) {
            qd[j] = 32 * (row0 + kRecvWarps * j) + lane;
            pend[j] = 0;
            if (qd[j] < nq) {
                qi[j] = __ldg(cquad + q0 + qd[j]);
                pend[j] = unsigned(qi[j].y);
                if constexpr (PULL) {
                    const unsigned pm = unsigned(__ldg(cqpull + q0 + qd[j]));
                    if (pm != pend[j]) qi[j].x = -1;   // pushed slots stay untouched
                    pend[j] = pm;
                }
            }
        }
        long long spins = 0;
        for (;;) {
            T v[kRecvDepth][4];
#pragma unroll
            for (int j = 0; j < kRecvDepth; ++j) {
                if (!pend[j]) continue;
                if (qi[j].x >= 0) {
                    ld_relaxed_gpu4(ypos + qi[j].x, v[j]);
                } else {
                    const int e = x0 + 4 * qd[j];
#pragma unroll
                    for (int l = 0; l < 4; ++l)
                        v[j][l] = (pend[j] >> l) & 1u ? ld_relaxed_gpu(ypos + __ldg(cext + e + l)) : sentinel_value<T>();
                }
            }
            unsigned left = 0;
#pragma unroll
            for (int j = 0; j < kRecvDepth; ++j) {
                if (!pend[j]) continue;
                T* dst = slot + 4 * qd[j];
                unsigned ready = 0;
#pragma unroll
                for (int l = 0; l < 4; ++l)
                    if (((pend[j] >> l) & 1u) && !is_sentinel(v[j][l])) ready |= 1u << l;
                if (qi[j].x >= 0) {
                    if (ready) st_slot4(dst, v[j]);   // not-ready lanes store the sentinel they hold
                } else {
#pragma unroll
                    for (int l = 0; l < 4; ++l)
                        if ((ready >> l) & 1u) st_slot(dst + l, v[j][l]);
                }
                pend[j] &= ~ready;
                left |= pend[j];
            }
            if (!left) break;
            if ((++spins & 255) == 0 && *(volatile int*)err) break;
            if (spins > (lim > 0 ? lim : kSpinLimit)) {
                atomicExch(err, 1);
                break;
            }
            if (sleep_ns > 0) __nanosleep(sleep_ns);
        }
#pragma unroll
        for (int j = 0; j < kRecvDepth; ++j)
#pragma unroll
            for (int l = 0; l < 4; ++l)
                if ((pend[j] >> l) & 1u) st_slot(slot + 4 * qd[j] + l, T(0));
    }
}

// Staging buffer views of segment buffer b.
template <typename S>
struct StageView {
    const unsigned* wv;
    const int* row;
    const int* push;
    const S* dia;
    const int* col;
    const S* val;
    __device__ __forceinline__ StageView(const unsigned char* buf, int rows_cap, int ents_cap)
        : wv(reinterpret_cast<const unsigned*>(buf)),
          row(reinterpret_cast<const int*>(buf + rows_cap * 4)),
          push(reinterpret_cast<const int*>(buf + rows_cap * 8)),
          dia(reinterpret_cast<const S*>(buf + rows_cap * 12)),
          col(reinterpret_cast<const int*>(buf + rows_cap * (12 + int(sizeof(S))))),
          val(reinterpret_cast<const S*>(buf + rows_cap * (12 + int(sizeof(S))) + ents_cap * 4))
    {
    }
};

// One compute thread's rows of a staged wave, in registers (RPT rows: i, i + CT, ...).
template <typename T, typename S, int RPT, int KM>
struct WaveRows {
    int row[RPT];     // chunk-local index
    int pos[RPT];     // position in the segment
    int push[RPT];    // receive slot of the next chunk this row's result fills, or -1
    T rhs[RPT];
    S dia[RPT];
    int col[RPT][KM];
    S val[RPT][KM];
};

// Loads compute thread i's rows of staged wave m (positions from poff,
// entries from eoff).  Row slots past the wave's rows repeat its last row (same reads,
// same result, same stores), and entries past the wave's K are the +0 cell
// with value 0, so the sweep needs no per-row branches; every index stays
// inside the staged segment.
template <typename T, typename S, int CT, int RPT, int KM>
__device__ __forceinline__ void wave_rows(unsigned m, const StageView<S>& V,
                                          const T* vec, int B, int r0, int poff, int eoff, int ents_cap, int lane,
                                          bool push, WaveRows<T, S, RPT, KM>& r)
{
    const int nw = int(m & 0x7FFFu), K = int(m >> 16);
    const int kl = max(K - 1, 0);
    const int elast = ents_cap - 1;   // a wave without entries (K = 0) may start at the end of the staged entries
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
        const int t = min(lane + CT * q, nw - 1);
        r.pos[q] = poff + t;
        r.row[q] = V.row[poff + t] - r0;
        r.push[q] = push && t == lane + CT * q ? V.push[poff + t] : -1;   // a repeated row pushes nothing
        r.dia[q] = V.dia[poff + t];
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            const int e = min(eoff + min(k, kl) * nw + t, elast);   // inside the wave's entries (K > 0)
            const int c = V.col[e];
            const S v = V.val[e];
            r.col[q][k] = k < K ? c : B;   // the +0 cell, value +0: neutral
            r.val[q][k] = k < K ? v : S(0);
        }
    }
#pragma unroll
    for (int q = 0; q < RPT; ++q) r.rhs[q] = vec[r.row[q]];
}

// Thread-block cluster helpers: rank and size, a barrier over all threads of
// the cluster (release / acquire: what a CTA wrote before it, in its own or a
// peer's shared memory, is visible after it), a peer's address of a shared
// variable, and stores into a peer CTA's shared memory.
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
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}
__device__ __forceinline__ unsigned peer_addr(const void* p, unsigned rank)
{
    unsigned a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
    return a;
}
__device__ __forceinline__ void st_peer(unsigned a, int v)
{
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void st_peer_relaxed(unsigned a, float v)
{
    asm volatile("st.relaxed.cluster.shared::cluster.f32 [%0], %1;" ::"r"(a), "f"(v));
}
__device__ __forceinline__ void st_peer_relaxed(unsigned a, double v)
{
    asm volatile("st.relaxed.cluster.shared::cluster.f64 [%0], %1;" ::"r"(a), "d"(v));
}

// Barrier among the CT compute threads (a warp barrier for one warp).
template <int CW>
__device__ __forceinline__ void compute_barrier()
{
    if constexpr (CW == 1)
        __syncwarp();
    else
        asm volatile("bar.sync 1, %0;" ::"n"(32 * CW) : "memory");
}

template <typename T, typename S, int CW, int RPT, int KM>
__global__ void __launch_bounds__(32 * (CW + kChunkExtraWarps)) k_sweep_chunk(SetView sv, ChunkSweepOp op)
{
    constexpr int CT = 32 * CW;
    constexpr int NTH = 32 * (CW + kChunkExtraWarps);
    if (blockDim.x != unsigned(NTH)) {   // launch shape mismatch: report, never wait
        if (threadIdx.x == 0) atomicExch(sv.err, 1);
        return;
    }
    extern __shared__ __align__(128) unsigned char chunk_smem[];
    __shared__ __align__(8) unsigned long long full[kStageBufs], empty[kStageBufs];
    __shared__ int s_task, s_go;
    __shared__ int s_nw[kStageBufs], s_p0[kStageBufs];
    typedef typename std::conditional<(sizeof(S) > sizeof(T)), S, T>::type W;   // promoted type
    T* vec = reinterpret_cast<T*>(chunk_smem);   // [chunk rows | +0 cell, kSlotBase - 1 unused | receive slots]
    unsigned char* stage = chunk_smem + op.vec_bytes;
    const int sbytes = stage_bytes<S>(op.rows_cap, op.ents_cap);
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int b = 0; b < kStageBufs; ++b) {
            mbar_init(&full[b], 1);
            mbar_init(&empty[b], 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const unsigned crank = cluster_rank(), csize = cluster_size();
    if (int(csize) != op.cl) {   // task table built for another cluster size: report (uniform over the cluster)
        if (tid == 0) atomicExch(sv.err, 1);
        return;
    }
    cluster_sync();      // every CTA of the cluster runs before any writes into a peer's shared memory
    unsigned gseg = 0;   // segments staged and consumed by this CTA so far (uniform)
    for (;;) {
        // the cluster's leader takes the next group of chunks for the cluster
        if (tid == 0 && crank == 0) {
            const int t = atomicAdd(op.ticket, 1);
            if (t == op.ntasks + int(gridDim.x / csize) - 1) atomicExch(op.ticket, 0);
            for (unsigned r = 0; r < csize; ++r) st_peer(peer_addr(&s_task, r), t);
        }
        cluster_sync();
        const int t = s_task;
        if (t >= op.ntasks) break;   // the same for the whole cluster
        const GroupTask gt = op.tasks[size_t(t) * csize + crank];
        if (tid == 0)
            s_go = (gt.count & kGroupActive) && !skip_system(sv.st[gt.sys], op.skip) && !*(volatile int*)sv.err;
        __syncthreads();
        const int go = s_go;
        const SysDesc& d = sv.desc[gt.sys];
        const TriFactor& TF = op.which == 0 ? d.L : d.U;
        const ChunkArrays F = {TF.segs, TF.wv, TF.crow, TF.cpush, TF.cdia, TF.ccol, TF.cval};
        const int pos = gt.pos0;
        const int B = TF.chunk_rows;
        const int r0 = (op.which == 0 ? pos : TF.nch - 1 - pos) * B;
        const int nr = min(d.n - r0, B);
        const int s0 = TF.cseg[pos], nseg = TF.cseg[pos + 1] - s0;
        const int x0 = TF.cxr[pos], nx = TF.cxr[pos + 1] - x0;
        const int* cext = TF.cext;
        T* ypos = static_cast<T*>(TF.ypos);
        // pushes: this chunk's results fill receive slots of the next chunk,
        // held by the next CTA of the cluster; the previous CTA fills ours
        const bool push_out = go && (gt.count & kGroupPushNext);
        const unsigned rvec = push_out ? peer_addr(vec, crank + 1) : 0u;
        const int* cqpull = (gt.count & kGroupPushedIn) ? TF.cqpull : nullptr;
        // chunk prologue (all threads): right-hand sides, empty receive slots,
        // this chunk's share of the other factor's result reset
        if (go) {
            const T* v = vptr<T>(d, op.in);
            for (int i = tid; i < nr; i += NTH) vec[i] = v[r0 + i];
            if (tid == 0) vec[B] = T(0);
            for (int i = tid; i < nx; i += NTH) vec[B + kSlotBase + i] = sentinel_value<T>();
            T* yr = static_cast<T*>(TF.ypos_reset);
            const long long a = (long long)TF.npos_reset * pos / TF.nch, e = (long long)TF.npos_reset * (pos + 1) / TF.nch;
            for (long long i = a + tid; i < e; i += NTH) yr[i] = sentinel_value<T>();
        }
        // every chunk of the group has empty receive slots before any push
        cluster_sync();
        if (!go) {
            // no chunk for this CTA in the group: the cluster's barriers only
        } else if (tid >= CT + 32 * kRecvWarps) {
            // producer warp: stage the chunk's segments (lane 0)
            if (tid == CT + 32 * kRecvWarps) {
                for (int i = 0; i < nseg; ++i) {
                    const unsigned g = gseg + i, b = g % kStageBufs;
                    const SegRec sg = F.segs[s0 + i];
                    if (g >= unsigned(kStageBufs)) mbar_wait(&empty[b], ((g / kStageBufs) + 1) & 1u, sv.err);
                    s_nw[b] = sg.nw;
                    s_p0[b] = sg.p0;
                    stage_segment<S>(F, sg, stage + b * sbytes, op.rows_cap, op.ents_cap, &full[b]);
                }
            }
        } else if (tid >= CT) {
            // receiver warps
            if (cqpull)
                receive_chunk<T, true>(cext, TF.cquad, cqpull, x0, nx, ypos, vec + B + kSlotBase, (tid - CT) >> 5,
                                       tid & 31, sv.err, op.sleep_ns, sv.spin);
            else
                receive_chunk<T, false>(cext, TF.cquad, nullptr, x0, nx, ypos, vec + B + kSlotBase, (tid - CT) >> 5,
                                        tid & 31, sv.err, op.sleep_ns, sv.spin);
        } else {
            // compute warps: all waves of the chunk, one cursor across
            // segments; the next wave's rows load while this one computes
            const int lane = tid;
            unsigned g = gseg, b = g % kStageBufs;
            mbar_wait(&full[b], (g / kStageBufs) & 1u, sv.err);
            StageView<S> V(stage + b * sbytes, op.rows_cap, op.ents_cap);
            int si = 0, nws = s_nw[b], p0 = s_p0[b];
            int w = 0, poff = 0, eoff = 0;
            unsigned m = V.wv[0];
            WaveRows<T, S, RPT, KM> cur, nxt;
            wave_rows<T, S, CT, RPT, KM>(m, V, vec, B, r0, 0, 0, op.ents_cap, lane, push_out, cur);
            for (;;) {
                // locate and load the next wave (possibly the next segment's first)
                const int nw = int(m & 0x7FFFu);
                const int poff_n = (poff + nw + 3) & ~3, eoff_n = eoff + int(m >> 16) * nw;   // waves start 4-aligned
                bool has_next = true, cross = false;
                unsigned mn = 0u;
                StageView<S> Vn = V;
                unsigned gn = g, bn = b;
                int pn = poff_n, en = eoff_n;
                if (w + 1 < nws) {
                    mn = V.wv[w + 1];
                } else if (si + 1 < nseg) {
                    cross = true;
                    gn = g + 1;
                    bn = gn % kStageBufs;
                    mbar_wait(&full[bn], (gn / kStageBufs) & 1u, sv.err);
                    Vn = StageView<S>(stage + bn * sbytes, op.rows_cap, op.ents_cap);
                    mn = Vn.wv[0];
                    pn = en = 0;
                } else {
                    has_next = false;
                }
                // all of the wave's reads at once (chunk rows, the +0 cell and
                // receive slots are cells of one shared vector; an entry coded
                // below zero is an earlier chunk's result read from global
                // memory); waits only for values not there yet
                T dv[RPT][KM];
                bool wait = false;
#pragma unroll
                for (int q = 0; q < RPT; ++q)
#pragma unroll
                    for (int k = 0; k < KM; ++k) {
                        const int c = cur.col[q][k];
                        const T x = vec[c >= 0 ? c : B];
                        dv[q][k] = c >= 0 ? x : sentinel_value<T>();
                        wait |= is_sentinel(dv[q][k]);
                    }
                if (has_next) wave_rows<T, S, CT, RPT, KM>(mn, Vn, vec, B, r0, pn, en, op.ents_cap, lane, push_out, nxt);
                if (wait) {
#pragma unroll
                    for (int q = 0; q < RPT; ++q)
#pragma unroll
                        for (int k = 0; k < KM; ++k) {
                            if (is_sentinel(dv[q][k])) {
                                const int c = cur.col[q][k];
                                dv[q][k] = c >= 0 ? poll_slot(vec + c, sv.err, sv.spin) : poll_value(ypos + (-c - 2), sv.err, op.sleep_ns, sv.spin);
                            }
                        }
                }
#pragma unroll
                for (int q = 0; q < RPT; ++q) {
                    T rr = cur.rhs[q];
#pragma unroll
                    for (int k = 0; k < KM; ++k) rr = sweep_step<T, S>(rr, cur.val[q][k], dv[q][k]);
                    const T out = unsentinel(T(W(rr) * W(cur.dia[q])));
                    vec[cur.row[q]] = out;
                    st_relaxed_gpu(ypos + p0 + cur.pos[q], out);
                    if (push_out) {
                        // rows the next chunk does not read go to an unused cell
                        const int ps = cur.push[q];
                        st_peer_relaxed(rvec + unsigned(ps >= 0 ? B + kSlotBase + ps : B + 1) * unsigned(sizeof(T)), out);
                    }
                }
                compute_barrier<CW>();
                if (!has_next) break;
                if (cross) {
                    // every compute thread has read its last rows of buffer b
                    if (lane == 0) mbar_arrive(&empty[b]);
                    g = gn;
                    b = bn;
                    V = Vn;
                    ++si;
                    nws = s_nw[b];
                    p0 = s_p0[b];
                    w = 0;
                    poff = eoff = 0;
                } else {
                    ++w;
                    poff = poff_n;
                    eoff = eoff_n;
                }
                m = mn;
                cur = nxt;
            }
            // last segment's buffer
            if (lane == 0) mbar_arrive(&empty[b]);
        }
        __syncthreads();
        // chunk epilogue (all warps): outputs and the reset of the buffer the
        // other sweep fills
        if (go) {
            gseg += unsigned(nseg);
            T* y = vptr<T>(d, op.out);
            T* R = op.reset != SLOT_NONE ? vptr<T>(d, op.reset) : nullptr;
            for (int i = tid; i < nr; i += NTH) {
                y[r0 + i] = vec[i];
                if (R) R[r0 + i] = sentinel_value<T>();
            }
        }
        // the group's pushes have landed and its CTAs are done with s_task
        cluster_sync();
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
    long long spin;           // polls before a dependency wait gives up
};

__device__ __forceinline__ double wait_acquire(const double* p, int* err, long long lim)
{
    double w;
    asm volatile("ld.acquire.gpu.global.f64 %0, [%1];" : "=d"(w) : "l"(p) : "memory");
    long long spins = 0;
    while (is_sentinel(w)) {
        if ((++spins & 255) == 0 && *(volatile int*)err) return 1.0;
        if (spins > (lim > 0 ? lim : kSpinLimit)) {
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
            const double ik = wait_acquire(op.inv_dia + k, op.err, op.spin);
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
            const double ik = wait_acquire(op.inv_dia + k, op.err, op.spin);
            const double dk = __dmul_rn(op.a[op.lt_src[q]], ik);
            // u_ii -= d * d with the product rounded first, as the reference
            // evaluates it (no fused multiply-add)
            diag = __dsub_rn(diag, __dmul_rn(dk, dk));
        }
        publish_release(op.inv_dia + i, __ddiv_rn(1.0, __dsqrt_rn(diag)));
    }
}

// Level-ordered factor values: val[e] = S(src[idx[e]] * (mul[e] >= 0 ?
// inv_dia[mul[e]] : 1)) (+0 where idx[e] < 0); dia[k] = S(row_of[k] >= 0 &&
// dia_mode ? inv_dia[row] : 1).
__global__ void k_fill_factor(int nent, const int* __restrict__ idx, const int* __restrict__ mul,
                              const double* __restrict__ src, const double* __restrict__ inv_dia, void* val,
                              int val_f32)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nent; e += gridDim.x * blockDim.x) {
        double v = idx[e] >= 0 ? src[idx[e]] : 0.0;   // idx < 0: padding, value +0
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
