// Shared definitions of the mtl4_b200 CUDA library (sm_100a).
//
// Execution model: every operation runs over a set of independent systems
// ("systems" = independent linear systems; a single solve is a set of one).
// Each system is described by a SysDesc (pointers into its own device
// buffers) and owns a SysState (its Krylov scalars and termination state,
// the device-side counterpart of itl::basic_iteration).  Work is cut into
// row tiles that never straddle two systems, so every per-system reduction
// sums the same partials in the same order whether the system runs alone or
// in a batch.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mtl4_b200/mtlg.h"

namespace mtlg {

// ----------------------------------------------------------------- errors
void set_error(const char* fmt, ...);
const char* last_error();

#define MTLG_CUDA(call)                                                                     \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            ::mtlg::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            return MTLG_ERR_CUDA;                                                           \
        }                                                                                   \
    } while (0)

#define MTLG_TRY(expr)                  \
    do {                                \
        int s_ = (expr);                \
        if (s_ != MTLG_OK) return s_;   \
    } while (0)

#define MTLG_CHECK_ARG(cond, msg)                       \
    do {                                                \
        if (!(cond)) {                                  \
            ::mtlg::set_error("invalid argument: %s", msg); \
            return MTLG_ERR_INVALID_ARG;                \
        }                                               \
    } while (0)

// ----------------------------------------------------------------- constants
constexpr int kTileRows = 256;        // rows per stream tile == threads per CTA
constexpr int kTileNnz = 2048;        // entries staged in shared memory per tile
constexpr int kShortRow = 32;         // rows up to this length: one thread, sequential sum
constexpr int kBlock = 256;
constexpr int kSweepRows = 32;        // rows per sweep task (one warp, one row per lane)
constexpr int kMaxDots = 4;           // dots a fused pass can reduce at once
constexpr int kNumVec = 16;           // workspace vectors per system
constexpr double kRefMinGain = 0.5;  // refinement: an outer step must at least halve the FP64 residual
constexpr int kScalarMeanRow = 12;   // SpMV auto choice: thread per row up to this mean row length
constexpr long long kSpinLimit = 1LL << 20;  // polls before a device wait gives up (~0.5 s); default spin_limit

// Tile kinds of the SpMV / vector tiling.
enum TileKind : int { TILE_STREAM = 0, TILE_LONG = 1 };

struct Tile {
    int sys;        // system index
    int row_begin;  // first row (system-local)
    int row_end;    // one past the last row
    int kind;       // TileKind
    int nnz_begin;  // row_ptr[row_begin]
    int nnz_end;    // row_ptr[row_end]
};

// One dependency-ordered sweep task: kSweepRows consecutive rows of a
// system's level-ordered triangular factor.
struct SweepTask {
    int sys;
    int first;      // first level-ordered row of the task
};

// One segment of a chunked triangular factor: waves [w0, w0 + nw), positions
// [p0, p0 + np), entries [e0, e0 + ne); the starts are multiples of 4.
struct __align__(16) SegRec {
    int w0, nw, p0, np, e0, ne, pad0, pad1;
};

constexpr unsigned kWaveOverflow = 0x8000u;   // wave reads rows of earlier chunks beyond the receive slots
constexpr int kSlotBase = 4;                  // receive slots start at shared cell chunk_rows + kSlotBase (16-byte aligned)
constexpr int kGridStepPad = 8;               // grid layout: steps per unit padded to a multiple of this

// Level-ordered triangular factor (device pointers).  Row k of the factor is
// original row `row_of[k]` (-1 marks padding that aligns levels to warps);
// its off-diagonal entries keep the reference's storage order and `dia[k]`
// is the multiplier applied last (inverse diagonal, 1 for a unit diagonal).
struct TriFactor {
    const int* rp;
    const int* ci;
    const void* val;   // T
    const void* dia;   // T
    const int* row_of;
    // Chunked layout (k_sweep_chunk).  Chunk q holds rows [q*chunk_rows,
    // (q+1)*chunk_rows); chunks are stored in processing order (ascending
    // rows for L, descending for U).  A chunk's rows are grouped in waves of
    // one dependency level (at most the launch's thread count rows each),
    // consecutive waves in segments that one bulk copy per array stages in
    // shared memory.  A wave's entries are column-major: entry k of its t-th
    // row sits at k * rows + t after the wave's first entry.  Columns are
    // coded as cells of the chunk's shared vector (B = chunk_rows): c < B a
    // row of the chunk, c == B a cell holding +0 (entries past a row's own,
    // with value +0: exactly neutral in the row's arithmetic), c >= B +
    // kSlotBase receive slot c - B - kSlotBase, filled by the receiver warps
    // with a row of an earlier chunk (cext lists those rows' positions per
    // chunk, in slot order, each chunk's list 4-aligned); c < 0 a row of an
    // earlier chunk at position -c - 2, read directly (its wave carries
    // kWaveOverflow).  Results cross chunks through ypos, in position order
    // (a wave's results are contiguous, starting 4-aligned).  Every segment
    // starts 16-byte aligned in every array.
    int chunk_rows;    // 0: no chunked layout
    int nch;
    int seg_rows;      // rows per segment, at most
    int pad1;
    const int* cseg;   // [nch + 1] segment range of each chunk
    const SegRec* segs;          // [segments]
    const unsigned* wv;// [waves] rows | kWaveOverflow | entries per row << 16
    const int* crow;   // row at each position
    const int* cxr;    // [nch + 1] receive-slot range of each chunk in cext
    const int* cext;   // positions of earlier chunks' rows, per chunk in slot order (-1: unused slot)
    const int2* cquad; // per 4 slots: {first of 4 consecutive positions or -1, mask of used slots}
    const int* cqpull; // per 4 slots: mask of the used slots the previous chunk does not push
    const int* cpush;  // per position: receive slot of the next chunk the row's result fills, or -1
    void* ypos;        // results by position (T), all sentinel before the sweep
    void* ypos_reset;  // the other factor's results by position: reset to the sentinel by this sweep
    int npos, npos_reset;
    const int* ccol;   // entries' columns
    const void* cval;  // entries' values (S)
    const void* cdia;  // multiplier per position (S)
    // Grid layout (k_sweep_grid): the factor's pattern is a 5- or 7-point
    // grid stencil.  Counting rows from the sweep's start (r' = r for L,
    // n - 1 - r for U), r' = i + gnx * (j + gny * k) and row r' reads rows
    // r' - 1 (x, when i > 0), r' - gnx (y, when j > 0) and r' - gnx*gny (z,
    // when k > 0) and nothing else.  A warp unit u = k * gnjb + jb holds the
    // x-lines j = 32 jb + lane of plane k; its step s is row i = s - lane of
    // each lane (i = s without skew).  gdata: [unit][step][slot][lane], slot
    // q < gns the entry of direction (gperm >> 2q) & 3 (0 x, 1 y, 2 z; +0
    // where the row has no such neighbour), slot gns the multiplier.
    int gnx, gny, gnz;  // gnx == 0: no grid layout
    int gns;            // entries per row (directions present): 0, 2 or 3
    int gperm;          // slot order of the directions (the reference's entry order)
    int gdirs;          // directions present (bit d)
    int gskew;          // 1: lane l runs row i at step i + l (rows depend on the lane below)
    int gnsteps;        // steps per unit
    int gnsp;           // steps per unit in the layout (a multiple of kGridStepPad)
    int gnjb;           // units along y
    const void* gdata;  // S
};

// One CTA's chunk in a group of chunks run by one thread-block cluster:
// chunk pos0 of system sys's factor; count holds the kGroup flags.
struct GroupTask {
    int sys;
    int pos0;
    int count;
    int pad;
};
constexpr int kGroupActive = 1;     // the CTA has a chunk in this group
constexpr int kGroupPushNext = 2;   // the next CTA of the cluster holds the next chunk: push results into it
constexpr int kGroupPushedIn = 4;   // the previous CTA holds the previous chunk and pushes into this one

// Workspace vector slots.
enum Vec : int {
    V_R = 0, V_P0, V_P1, V_Q, V_Z, V_Z0, V_RT, V_V, V_S, V_T, V_PHAT, V_SHAT, V_D, V_W0, V_W1, V_W2
};

struct SysDesc {
    int n;
    int nnz;
    const int* rp;
    const int* ci;
    const void* val;        // values in the solve precision T
    const double* val64;    // FP64 values (outer residual of refinement)
    void* x;                // solution (T)
    const void* b;          // right-hand side (T)
    void* ws;               // workspace: vector k at (T*)ws + k * ws_stride
    long long ws_stride;
    int pc;                 // mtlg_pc_kind
    int pad0;
    const void* inv_diag;   // T, Jacobi
    TriFactor L, U;
    double* x64;            // refinement: FP64 solution
    const double* b64;      // refinement: FP64 right-hand side
    double* r64;            // refinement: FP64 residual
};

// Device-side state of one system's solve (basic_iteration + Krylov scalars).
struct SysState {
    double rho, rho_1, alpha, beta, omega, gamma;
    double rr, resid, norm_r0, rtol, atol;
    double dots[kMaxDots];
    double scale;           // refinement: ||r|| of the current step
    double nb;              // refinement: ||b||
    int iter, max_iter, status, error;
    int ostatus;            // refinement (outer) status
    int phase;              // served solves: PH_* (ignored by the other engines)
    int first, flags;
    int outer, max_outer;
    int inner_total, inner_max;
    double inner_rtol, outer_rtol;
    double* log;            // residual log: (iteration, resid) of every termination test
    int log_cap, log_n;     // capacity in tests; tests made (log_n > log_cap: truncated)
};

// Per-launch view of the system set.
struct SetView {
    const Tile* tiles;
    int n_tiles;
    int n_sys;
    const int* sys_tile_begin;   // [n_sys + 1]
    SysDesc* desc;
    SysState* st;
    double* partials;            // [n_tiles * kMaxDots]
    unsigned* counters;          // [n_sys] last-block counters (self-resetting)
    int* running;                // systems still running
    int* err;                    // device error flags (timeouts)
    unsigned long long cond;     // cudaGraphConditionalHandle (0: not in a graph)
    int use_cond;
    long long spin;              // polls before a dependency wait gives up (context "spin_limit"; 0: kSpinLimit)
};

// ----------------------------------------------------------------- device helpers
template <typename T> struct Sentinel;
template <> struct Sentinel<double> {
    static constexpr unsigned long long bits = 0xFFFFFFFFFFFFFFFFull;
};
template <> struct Sentinel<float> {
    static constexpr unsigned bits = 0xFFFFFFFFu;
};

template <typename T> __device__ __forceinline__ T sentinel_value();
template <> __device__ __forceinline__ double sentinel_value<double>() { return __longlong_as_double(-1ll); }
template <> __device__ __forceinline__ float sentinel_value<float>() { return __uint_as_float(0xFFFFFFFFu); }

__device__ __forceinline__ double ld_volatile(const double* p)
{
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ float ld_volatile(const float* p)
{
    float v;
    asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_volatile(double* p, double v)
{
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_volatile(float* p, float v)
{
    asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ bool is_sentinel(double v)
{
    return (unsigned long long)__double_as_longlong(v) == Sentinel<double>::bits;
}
__device__ __forceinline__ bool is_sentinel(float v) { return (unsigned)__float_as_uint(v) == Sentinel<float>::bits; }
// A computed value must never look like "not ready": map the sentinel bit
// pattern (a NaN) to the canonical NaN.
__device__ __forceinline__ double unsentinel(double v) { return is_sentinel(v) ? __longlong_as_double(0x7FF8000000000000ll) : v; }
__device__ __forceinline__ float unsentinel(float v) { return is_sentinel(v) ? __uint_as_float(0x7FC00000u) : v; }

template <typename T>
__device__ __forceinline__ T* wsvec(const SysDesc& d, int k)
{
    return static_cast<T*>(d.ws) + (long long)k * d.ws_stride;
}

// Deterministic block reduction of kMaxDots doubles (fixed tree, fixed
// thread->element mapping).  Result valid in thread 0.
template <int ND>
__device__ __forceinline__ void block_reduce(double (&v)[ND], double* smem /* [ND * 32] */)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < ND; ++j) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], o);
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < ND; ++j) smem[j * 32 + warp] = v[j];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int j = 0; j < ND; ++j) {
            double t = lane < nw ? smem[j * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            v[j] = t;
        }
    }
}

// Writes tile `tile`'s partial dots (block_reduce results, valid in thread 0).
template <int ND>
__device__ __forceinline__ void store_partials(const SetView& sv, int tile, const double (&v)[ND])
{
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < ND; ++j) sv.partials[(long long)tile * kMaxDots + j] = v[j];
    }
}

// A CTA's count of finished tiles of one system (tiles whose partials it has
// stored), published with one atomic when the CTA moves on to another system
// or ends: one atomic per CTA and system instead of one per tile.
struct TileTally {
    int sys = -1;
    unsigned n = 0;
    unsigned need = 0;   // tiles that complete the system (0: all of its SpMV tiles)
};

// Publishes the tally (whole CTA, tally uniform) and reports whether it
// completed the system's tiles: the calling CTA then owns the system's
// finalize.  The counter resets itself for the next pass.
__device__ __forceinline__ bool publish_tally(const SetView& sv, TileTally& tt)
{
    __shared__ int s_last;
    if (tt.n == 0) return false;
    if (threadIdx.x == 0) {
        __threadfence();   // this CTA's partials before its count
        const unsigned ntiles =
            tt.need ? tt.need : unsigned(sv.sys_tile_begin[tt.sys + 1] - sv.sys_tile_begin[tt.sys]);
        const unsigned prev = atomicAdd(&sv.counters[tt.sys], tt.n);
        s_last = (prev + tt.n == ntiles);
        if (s_last) {
            sv.counters[tt.sys] = 0;
            __threadfence();
        }
    }
    __syncthreads();
    const bool last = s_last != 0;
    __syncthreads();
    tt.n = 0;
    return last;
}

// Sum of a system's tile partials (its first `count` tiles, or all of its
// SpMV tiles) in tile order (deterministic: thread i adds tiles i,
// i + blockDim, ... in turn, loads issued 8 tiles at a time); called by the
// whole last CTA, result valid in thread 0.
template <int ND>
__device__ __forceinline__ void gather_partials(const SetView& sv, int sys, double (&out)[ND], double* smem,
                                                int count = -1)
{
    const int t0 = sv.sys_tile_begin[sys], t1 = count >= 0 ? t0 + count : sv.sys_tile_begin[sys + 1];
    const int B = blockDim.x;
#pragma unroll
    for (int j = 0; j < ND; ++j) out[j] = 0.0;
    for (int t = t0 + threadIdx.x; t < t1; t += 8 * B) {
        double v[8][ND];
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int j = 0; j < ND; ++j)
                v[u][j] = t + u * B < t1 ? __ldcg(&sv.partials[(long long)(t + u * B) * kMaxDots + j]) : 0.0;
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int j = 0; j < ND; ++j)
                if (t + u * B < t1) out[j] += v[u][j];
    }
    block_reduce<ND>(out, smem);
}

// Phases of a served solve (continuous batching): each engine step runs the
// kernels of every phase, and each kernel acts only on the slots in its
// phase, so requests admitted at different times share the same launches.
enum Phase : int { PH_INIT = 0, PH_OUTER = 1, PH_CAST = 2, PH_INNER = 3, PH_UPDATE = 4, PH_DONE = 5 };

__device__ __forceinline__ void inner_done(SysState& s)
{
    // refinement solves go back for an FP64 update, plain ones are finished
    if (s.phase == PH_INNER) s.phase = (s.max_outer > 0) ? PH_UPDATE : PH_DONE;
}

__device__ __forceinline__ void set_cond(const SetView& sv, unsigned v)
{
    if (sv.use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)sv.cond, v);
}

// basic_iteration::finished(r) for a residual norm (basic_iteration.hpp:60-65,
// 85-93): converged if resid <= rtol*norm_r0 or resid <= atol (atol only when
// norm_r0 == 0); otherwise "too many iterations" once iter >= max_iter.
// Returns true when the system stops; retires it from the running count.
// One termination test into the system's residual log (when it has one):
// the (iteration, residual) pairs let the host replay the tests into an
// iteration object, e.g. a cyclic_iteration that prints every cycle.
__device__ __forceinline__ void log_check(SysState& s, double resid)
{
    if (s.log && s.log_n < s.log_cap) {
        s.log[2 * s.log_n] = double(s.iter);
        s.log[2 * s.log_n + 1] = resid;
    }
    s.log_n += 1;
}

__device__ __forceinline__ bool check_finished(const SetView& sv, SysState& s, double resid)
{
    log_check(s, resid);
    s.resid = resid;
    bool conv = (s.norm_r0 == 0.0) ? (resid <= s.atol) : (resid <= s.rtol * s.norm_r0 || resid <= s.atol);
    if (conv) {
        s.status = MTLG_ST_CONVERGED;
        s.error = 0;
    } else if (isnan(resid) || isinf(resid)) {
        s.status = MTLG_ST_BREAKDOWN;
        s.error = 1;
    } else if (s.iter >= s.max_iter) {
        s.status = MTLG_ST_MAXIT;
        s.error = 1;
    } else {
        return false;
    }
    inner_done(s);
    if (atomicSub(sv.running, 1) == 1) set_cond(sv, 0u);
    return true;
}

__device__ __forceinline__ void retire(const SetView& sv, SysState& s, int status, int error)
{
    s.status = status;
    s.error = error;
    inner_done(s);
    if (atomicSub(sv.running, 1) == 1) set_cond(sv, 0u);
}

}  // namespace mtlg
