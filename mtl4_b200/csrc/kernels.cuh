// CSR SpMV and fused vector passes with device-side Krylov scalar updates.
//
// SpMV follows the reference's row-major CSR product
// (boost/numeric/mtl/operation/mat_vec_mult.hpp:614-683): every row is an
// accumulator started at zero and updated entry by entry in storage order,
// tmp += A.data[j] * v[A.ref_minor()[j]], then assigned/added/subtracted
// into w (Assign::first_update).  The reference build (g++ -O3 with FMA
// available) evaluates that loop in groups of four entries whose products
// are rounded before the addition, and the row's last (L mod 4) entries as
// fused multiply-adds; in FP32 every product is rounded first.  row_step
// reproduces this, so rows of up to kShortRow entries, which keep the exact
// order (one thread per row), are bitwise the reference's in FP64 and FP32.
// Longer rows are split over a warp (or the whole CTA) and summed as a fixed
// tree.
#pragma once
#include "common.cuh"

namespace mtlg {

// ---------------------------------------------------------------- operands
// Vector operand codes: >= 0 workspace slot, negatives name descriptor
// vectors; OPND_* are per-row values available in epilogues.
enum Slot : int { SLOT_X = -1, SLOT_B = -2, SLOT_X64 = -3, SLOT_B64 = -4, SLOT_R64 = -5, SLOT_NONE = -100 };
enum Opnd : int { OPND_ONE = -1000, OPND_Y = -1001, OPND_XP = -1002, OPND_D = -1003 };

template <typename T>
__device__ __forceinline__ T* vptr(const SysDesc& d, int slot)
{
    if (slot >= 0) return wsvec<T>(d, slot);
    switch (slot) {
    case SLOT_X: return static_cast<T*>(d.x);
    case SLOT_B: return const_cast<T*>(static_cast<const T*>(d.b));
    default: return nullptr;
    }
}

// ---------------------------------------------------------------- finalize
enum Fin : int {
    FIN_NONE = 0,
    FIN_STORE,          // st.dots[j] = sum_j
    FIN_CG_INIT,        // rr -> finished?  (identity: rho = rr)
    FIN_CG_INIT_JAC,    // rr, r.Dr -> finished?  rho = r.z
    FIN_CG_ALPHA,       // p.q -> alpha = rho / p.q, ++iter
    FIN_CG_UPDATE,      // rr -> finished?  identity: beta = rr / rho
    FIN_CG_UPDATE_JAC,  // rr, r.z -> finished?  beta = r.z / rho
    FIN_CG_UPDATE_PC,   // rr -> finished?  (z follows from the sweeps)
    FIN_CG_RHO,         // r.z after the sweeps -> beta
    FIN_BI_TOP,         // rt.r, r.r at the loop top (init and after r update)
    FIN_BI_GAMMA,       // rt.v -> alpha
    FIN_BI_S,           // s.s -> finished(s)?
    FIN_BI_OMEGA,       // t.s, t.t -> omega
    FIN_REF_OUTER,      // FP64 r.r -> refinement stop test, scale
    FIN_NORM_R0,        // norm_r0 = sqrt(b.b)  (basic_iteration from b)
    FIN_REF_NB,         // refinement: nb = ||b||_FP64
    FIN_REF_CG_INIT,    // inner CG init on the scaled residual (norm_r0 = ||r||)
    FIN_REF_CG_INIT_JAC,
    FIN_REF_BI_INIT,    // inner BiCGSTAB init (norm_r0 = ||r||)
    FIN_PHASE_OUTER,    // served refinement: back to the outer residual
};

// Status flags
enum : int { FLAG_FINISHING = 1 };

__device__ __forceinline__ void bicg_top(const SetView& sv, SysState& s, double rtr, double rr, bool first_pass)
{
    if (!first_pass) s.rho_1 = s.rho;  // rho_2 = rho_1 (bicgstab.hpp:75)
    if (check_finished(sv, s, sqrt(fabs(rr)))) return;
    s.iter += 1;
    s.rho = rtr;  // rho_1 = dot(rtilde, r)
    if (s.rho == 0.0) { retire(sv, s, MTLG_ST_BREAKDOWN, 1); return; }
    if (s.iter > 1) {
        if (s.omega == 0.0) { retire(sv, s, MTLG_ST_BREAKDOWN, 1); return; }
        s.beta = (s.rho / s.rho_1) * (s.alpha / s.omega);
    }
}

__device__ void finalize(const SetView& sv, int fin, int sys, const double* dots)
{
    SysState& s = sv.st[sys];
    switch (fin) {
    case FIN_STORE:
        for (int j = 0; j < kMaxDots; ++j) s.dots[j] = dots[j];
        break;
    case FIN_NORM_R0:
        s.norm_r0 = sqrt(fabs(dots[0]));
        break;
    case FIN_REF_NB:
        s.nb = sqrt(fabs(dots[0]));
        break;
    case FIN_REF_CG_INIT:
        s.phase = PH_INNER;
        s.norm_r0 = sqrt(fabs(dots[0]));
        s.rr = dots[0];
        s.rho = dots[0];
        check_finished(sv, s, sqrt(fabs(dots[0])));
        break;
    case FIN_REF_CG_INIT_JAC:
        s.phase = PH_INNER;
        s.norm_r0 = sqrt(fabs(dots[0]));
        s.rr = dots[0];
        s.rho = dots[1];
        check_finished(sv, s, sqrt(fabs(dots[0])));
        break;
    case FIN_REF_BI_INIT:
        s.phase = PH_INNER;
        s.norm_r0 = sqrt(fabs(dots[1]));
        bicg_top(sv, s, dots[0], dots[1], true);
        break;
    case FIN_CG_INIT:
        s.phase = PH_INNER;
        s.rr = dots[0];
        s.rho = dots[0];
        s.iter = 0;
        check_finished(sv, s, sqrt(fabs(dots[0])));
        break;
    case FIN_CG_INIT_JAC:
        s.phase = PH_INNER;
        s.rr = dots[0];
        s.rho = dots[1];
        s.iter = 0;
        check_finished(sv, s, sqrt(fabs(dots[0])));
        break;
    case FIN_CG_ALPHA:
        s.dots[0] = dots[0];
        s.alpha = s.rho / dots[0];
        s.iter += 1;
        break;
    case FIN_CG_UPDATE:
        s.rr = dots[0];
        if (!check_finished(sv, s, sqrt(fabs(dots[0])))) {
            s.rho_1 = s.rho;
            s.rho = dots[0];
            s.beta = s.rho / s.rho_1;
        }
        break;
    case FIN_CG_UPDATE_JAC:
        s.rr = dots[0];
        if (!check_finished(sv, s, sqrt(fabs(dots[0])))) {
            s.rho_1 = s.rho;
            s.rho = dots[1];
            s.beta = s.rho / s.rho_1;
        }
        break;
    case FIN_CG_UPDATE_PC:
        s.rr = dots[0];
        check_finished(sv, s, sqrt(fabs(dots[0])));
        break;
    case FIN_CG_RHO:
        s.rho_1 = s.rho;
        s.rho = dots[0];
        s.beta = s.rho / s.rho_1;
        break;
    case FIN_BI_TOP:
        if (s.iter == 0) s.phase = PH_INNER;
        bicg_top(sv, s, dots[0], dots[1], s.iter == 0);
        break;
    case FIN_PHASE_OUTER:
        s.phase = PH_OUTER;
        break;
    case FIN_BI_GAMMA:
        s.gamma = dots[0];
        if (s.gamma == 0.0) { retire(sv, s, MTLG_ST_BREAKDOWN, 1); break; }
        s.alpha = s.rho / s.gamma;
        // a non-finite step would spoil the iterate: stop before the update
        if (!isfinite(s.alpha)) retire(sv, s, MTLG_ST_BREAKDOWN, 1);
        break;
    case FIN_BI_S: {
        // iter.finished(s) (bicgstab.hpp:64): on true, x += alpha*phat is
        // still due; the x/r pass does it and then retires the system.
        const double res = sqrt(fabs(dots[0]));
        log_check(s, res);
        s.resid = res;
        bool conv = (s.norm_r0 == 0.0) ? (res <= s.atol) : (res <= s.rtol * s.norm_r0 || res <= s.atol);
        if (conv) { s.flags |= FLAG_FINISHING; s.error = 0; s.dots[3] = MTLG_ST_CONVERGED; }
        else if (isnan(res) || isinf(res)) { retire(sv, s, MTLG_ST_BREAKDOWN, 1); }
        else if (s.iter >= s.max_iter) { s.flags |= FLAG_FINISHING; s.error = 1; s.dots[3] = MTLG_ST_MAXIT; }
        break;
    }
    case FIN_BI_OMEGA:
        s.omega = dots[0] / dots[1];
        // t.t == 0 or an overflow: stop before x and r take a non-finite step
        if (!isfinite(s.omega)) retire(sv, s, MTLG_ST_BREAKDOWN, 1);
        break;
    case FIN_REF_OUTER: {
        // Refinement stop test on the FP64 residual: ||b - A x|| <= rtol*||b||.
        const double rn = sqrt(fabs(dots[0]));
        const double prev = s.scale;   // the previous outer residual (outer >= 1)
        s.inner_total += s.iter;
        s.iter = 0;
        s.scale = rn;
        s.resid = rn;
        s.flags = 0;
        if (rn <= s.outer_rtol * s.nb) {
            s.ostatus = MTLG_ST_CONVERGED; s.status = MTLG_ST_CONVERGED; s.error = 0; s.phase = PH_DONE;
        } else if (isnan(rn) || isinf(rn)) {
            s.ostatus = MTLG_ST_BREAKDOWN; s.status = MTLG_ST_BREAKDOWN; s.error = 1; s.phase = PH_DONE;
        } else if (s.outer >= 1 && !(rn <= kRefMinGain * prev)) {
            // the FP32 inner solves no longer reduce the FP64 residual (the
            // operator is too ill-conditioned for FP32): stop; the host
            // finishes the system in FP64
            s.ostatus = MTLG_ST_STALLED; s.status = MTLG_ST_STALLED; s.error = 1; s.phase = PH_DONE;
        } else if (s.outer >= s.max_outer) {
            s.ostatus = MTLG_ST_MAXIT; s.status = MTLG_ST_MAXIT; s.error = 1; s.phase = PH_DONE;
        } else {
            s.outer += 1;
            s.status = MTLG_ST_RUNNING;
            s.phase = PH_CAST;
            atomicAdd(sv.running, 1);
        }
        break;
    }
    default:
        break;
    }
}

// ---------------------------------------------------------------- SpMV
enum XForm : int { XF_PLAIN = 0, XF_CG_P = 1, XF_CG_P_JAC = 2, XF_JAC = 3 };
enum Assign : int { ASG_SET = 0, ASG_ADD = 1, ASG_SUB = 2, ASG_WMINUS = 3 };
enum Skip : int { SKIP_NONE = 0, SKIP_INNER = 1, SKIP_OUTER = 2, SKIP_RUNNING = 3, SKIP_PH_BASE = 16 };
// SKIP_PH_BASE + p: act only on systems in phase p (served solves)

struct SpmvOp {
    int x, y, w;        // input slot, output slot, W for y = W - A x
    int y2;             // optional second output (copy of y)
    int p, z, pnew;     // XF_CG_*: old p, z (or r), new p
    int ndot;
    int da[kMaxDots], db[kMaxDots], dc[kMaxDots];
    int rk[kMaxDots];   // reference summation order of each dot (RK_*, refdot.cuh)
    int fin;
    int skip;
    int count_body;     // increments the body counter (first kernel of a loop body)
};

__device__ __forceinline__ bool skip_system(const SysState& s, int mode)
{
    if (mode == SKIP_INNER) return s.status != MTLG_ST_RUNNING || (s.flags & FLAG_FINISHING);
    if (mode == SKIP_OUTER) return s.ostatus != MTLG_ST_RUNNING;
    if (mode == SKIP_RUNNING) return s.status != MTLG_ST_RUNNING;
    if (mode >= SKIP_PH_BASE) return s.phase != mode - SKIP_PH_BASE;
    return false;
}

// acc + a*x with the product rounded first (no contraction)
__device__ __forceinline__ double mac(double acc, double a, double x) { return __dadd_rn(acc, __dmul_rn(a, x)); }
__device__ __forceinline__ float mac(float acc, float a, float x) { return __fadd_rn(acc, __fmul_rn(a, x)); }
// One step of a sequential row sum: entries before the row's last (L mod 4)
// add the rounded product, the last ones are fused (FP64 only), as in the
// reference build's row loop.  `fused` = the entry lies in that tail.
__device__ __forceinline__ double row_step(double acc, double a, double x, bool fused)
{
    return fused ? __fma_rn(a, x, acc) : mac(acc, a, x);
}
__device__ __forceinline__ float row_step(float acc, float a, float x, bool) { return mac(acc, a, x); }
// first entry of a row's fused tail: a + 4 * floor((e - a) / 4)
__device__ __forceinline__ int fused_tail(int a, int e) { return a + ((e - a) & ~3); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

template <typename T, int XF>
struct XIn {
    const T* x;
    const T* p;
    const T* z;
    const T* dinv;
    T beta;
    bool first;
    __device__ __forceinline__ T operator()(int j) const
    {
        if (XF == XF_PLAIN) return x[j];
        if (XF == XF_JAC) return dinv[j] * x[j];
        T zj = (XF == XF_CG_P_JAC) ? dinv[j] * z[j] : z[j];
        return first ? zj : fma(beta, p[j], zj);
    }
};

// Slot codes that name a vector (workspace slot or descriptor vector).
__device__ __forceinline__ bool names_vector(int code) { return code >= SLOT_B; }

template <typename T, int ASG>
__device__ __forceinline__ T assign_out(T old_or_w, T acc)
{
    if (ASG == ASG_SET) return acc;
    if (ASG == ASG_ADD) return old_or_w + acc;
    return old_or_w - acc;  // ASG_SUB and ASG_WMINUS
}

// Per-row epilogue operand (a dot factor): a vector, or y / x' / D of the row.
template <typename T>
struct Opnd1 {
    int code;
    const T* v;
    __device__ __forceinline__ T get(int i, T y, T xp, const T* dinv) const
    {
        switch (code) {
        case OPND_ONE: return T(1);
        case OPND_Y: return y;
        case OPND_XP: return xp;
        case OPND_D: return dinv[i];
        default: return v[i];
        }
    }
};

template <typename T, int ASG, int XF>
struct RowEpilogue {
    T* y;
    T* y2;
    const T* w;
    T* pnew;
    int ndot;
    Opnd1<T> a0, b0, c0, a1, b1, c1;
    __device__ __forceinline__ void operator()(int i, T acc, T xp, const T* dinv, double& d0, double& d1) const
    {
        const T base = (ASG == ASG_SET) ? T(0) : ((ASG == ASG_WMINUS) ? w[i] : y[i]);
        const T out = assign_out<T, ASG>(base, acc);
        y[i] = out;
        if (y2) y2[i] = out;
        if (XF != XF_PLAIN) pnew[i] = xp;
        if (ndot > 0) d0 += double(a0.get(i, out, xp, dinv) * b0.get(i, out, xp, dinv) * c0.get(i, out, xp, dinv));
        if (ndot > 1) d1 += double(a1.get(i, out, xp, dinv) * b1.get(i, out, xp, dinv) * c1.get(i, out, xp, dinv));
    }
};

// ---- shared-memory staging of a stream tile (16-byte cp.async copies)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Buffer layout: values (kTileNnz + one chunk), columns (kTileNnz + one
// chunk), row pointers (kTileRows + 1 + one chunk).  Every copy is widened to
// 16-byte boundaries; the device arrays carry 16 bytes of tail padding, so
// the widened range stays inside the allocation.
template <typename T>
struct StageLayout {
    static constexpr int VE = 16 / sizeof(T);
    static constexpr int VBYTES = (kTileNnz + 2 * VE) * sizeof(T);
    static constexpr int CBYTES = (kTileNnz + 8) * 4;
    static constexpr int RBYTES = ((kTileRows + 1 + 8) * 4 + 15) / 16 * 16;
    static constexpr int BYTES = VBYTES + CBYTES + RBYTES;
    static_assert(VBYTES % 16 == 0 && CBYTES % 16 == 0 && BYTES % 16 == 0, "16-byte aligned sections");
};

template <typename T>
__device__ __forceinline__ void stage_tile(const Tile& t, const int* rp, const int* ci, const T* va, unsigned char* buf)
{
    typedef StageLayout<T> SL;
    const int ka = t.nnz_begin & ~(SL::VE - 1);
    const int kb = (t.nnz_end + SL::VE - 1) & ~(SL::VE - 1);
    for (int c = threadIdx.x; c < (kb - ka) / SL::VE; c += blockDim.x)
        cp_async16(buf + c * 16, va + ka + c * SL::VE);
    const int ca = t.nnz_begin & ~3, cb = (t.nnz_end + 3) & ~3;
    for (int c = threadIdx.x; c < (cb - ca) / 4; c += blockDim.x)
        cp_async16(buf + SL::VBYTES + c * 16, ci + ca + c * 4);
    const int ra = t.row_begin & ~3, rb = (t.row_end + 1 + 3) & ~3;
    for (int c = threadIdx.x; c < (rb - ra) / 4; c += blockDim.x)
        cp_async16(buf + SL::VBYTES + SL::CBYTES + c * 16, rp + ra + c * 4);
}

// Persistent CTAs walk the tiles with a stride of the grid.  A stream tile's
// values, columns and row pointers are copied into one of two shared-memory
// buffers while the previous tile is summed from the other.  Every thread
// then sums one row sequentially; rows longer than kShortRow are summed by a
// warp from shared memory.  A long tile (one row with more than kTileNnz
// entries) is summed by the whole CTA straight from global memory.
// Publishes a CTA's tally of a system's finished SpMV tiles; the CTA that
// completes the system gathers its partials and finalizes.
template <typename OpT>
__device__ __forceinline__ void spmv_publish(const SetView& sv, const OpT& op, TileTally& tally, double* s_red)
{
    if (publish_tally(sv, tally)) {
        double tot[kMaxDots];
        gather_partials<kMaxDots>(sv, tally.sys, tot, s_red);
        if (threadIdx.x == 0) finalize(sv, op.fin, tally.sys, tot);
    }
}

template <typename T, int XF, int ASG>
__global__ void __launch_bounds__(kBlock, 3) k_spmv(SetView sv, SpmvOp op)
{
    typedef StageLayout<T> SL;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_med[kTileRows];
    __shared__ int s_nmed;
    __shared__ double s_red[kMaxDots * 32];
    __shared__ T s_acc[32];

    if (op.count_body && blockIdx.x == 0 && threadIdx.x == 0) {
        // loop-body counter: bounds a graph while-loop independently of the
        // solver's own termination test
        int runs = atomicAdd(&sv.err[1], 1) + 1;
        if (runs > sv.err[2] || *(volatile int*)sv.running <= 0) set_cond(sv, 0u);
    }
    const int G = gridDim.x;
    int t = blockIdx.x;
    if (t >= sv.n_tiles) return;
    TileTally tally;   // finished tiles of the current system, published per system run

    Tile cur = sv.tiles[t];
    {
        const SysDesc& d0 = sv.desc[cur.sys];
        if (cur.kind == TILE_STREAM && !skip_system(sv.st[cur.sys], op.skip))
            stage_tile<T>(cur, d0.rp, d0.ci, static_cast<const T*>(d0.val), smem_raw);
        cp_async_commit();
    }
    Tile nxt = (t + G < sv.n_tiles) ? sv.tiles[t + G] : cur;

    for (int it = 0; t < sv.n_tiles; t += G, ++it) {
        const int tn = t + G;
        Tile nn = (tn + G < sv.n_tiles) ? sv.tiles[tn + G] : nxt;   // metadata one tile ahead
        unsigned char* buf = smem_raw + (it & 1) * SL::BYTES;
        if (tn < sv.n_tiles) {
            const SysDesc& dn = sv.desc[nxt.sys];
            if (nxt.kind == TILE_STREAM && !skip_system(sv.st[nxt.sys], op.skip))
                stage_tile<T>(nxt, dn.rp, dn.ci, static_cast<const T*>(dn.val), smem_raw + ((it + 1) & 1) * SL::BYTES);
        }
        cp_async_commit();
        cp_async_wait_1();
        __syncthreads();

        const Tile tile = cur;
        const int sys = tile.sys;
        if (op.fin != FIN_NONE && sys != tally.sys) {
            spmv_publish(sv, op, tally, s_red);
            tally.sys = sys;
        }
        const SysDesc& d = sv.desc[sys];
        const SysState& s = sv.st[sys];
        if (!skip_system(s, op.skip)) {
            XIn<T, XF> xin;
            xin.x = vptr<T>(d, op.x);
            xin.p = op.p != SLOT_NONE ? vptr<T>(d, op.p) : nullptr;
            xin.z = op.z != SLOT_NONE ? vptr<T>(d, op.z) : nullptr;
            xin.dinv = static_cast<const T*>(d.inv_diag);
            xin.beta = T(s.beta);
            xin.first = (s.iter == 0);
            const T* dinv = xin.dinv;

            RowEpilogue<T, ASG, XF> epi;
            epi.y = vptr<T>(d, op.y);
            epi.y2 = op.y2 != SLOT_NONE ? vptr<T>(d, op.y2) : nullptr;
            epi.w = op.w != SLOT_NONE ? vptr<T>(d, op.w) : nullptr;
            epi.pnew = op.pnew != SLOT_NONE ? vptr<T>(d, op.pnew) : nullptr;
            epi.ndot = op.ndot;
            epi.a0 = {op.da[0], names_vector(op.da[0]) ? vptr<T>(d, op.da[0]) : nullptr};
            epi.b0 = {op.db[0], names_vector(op.db[0]) ? vptr<T>(d, op.db[0]) : nullptr};
            epi.c0 = {op.dc[0], names_vector(op.dc[0]) ? vptr<T>(d, op.dc[0]) : nullptr};
            epi.a1 = {op.da[1], names_vector(op.da[1]) ? vptr<T>(d, op.da[1]) : nullptr};
            epi.b1 = {op.db[1], names_vector(op.db[1]) ? vptr<T>(d, op.db[1]) : nullptr};
            epi.c1 = {op.dc[1], names_vector(op.dc[1]) ? vptr<T>(d, op.dc[1]) : nullptr};
            double d0 = 0.0, d1 = 0.0;

            if (tile.kind == TILE_STREAM) {
                const T* s_val = reinterpret_cast<const T*>(buf);
                const int* s_col = reinterpret_cast<const int*>(buf + SL::VBYTES);
                const int* s_rp = reinterpret_cast<const int*>(buf + SL::VBYTES + SL::CBYTES);
                const int ka = tile.nnz_begin & ~(SL::VE - 1), ca = tile.nnz_begin & ~3, ra = tile.row_begin & ~3;
                if (threadIdx.x == 0) s_nmed = 0;
                __syncthreads();
                const int i = tile.row_begin + threadIdx.x;
                if (i < tile.row_end) {
                    const int a = s_rp[i - ra], e = s_rp[i + 1 - ra];
                    if (e - a <= kShortRow) {
                        // gathers issued 8 at a time, summed in storage order
                        T acc = T(0);
                        const int q = fused_tail(a, e);
                        int k = a;
                        for (; k + 8 <= e; k += 8) {
                            T xv[8];
#pragma unroll
                            for (int u = 0; u < 8; ++u) xv[u] = xin(s_col[k + u - ca]);
#pragma unroll
                            for (int u = 0; u < 8; ++u) acc = row_step(acc, s_val[k + u - ka], xv[u], k + u >= q);
                        }
                        T xv[8];
#pragma unroll
                        for (int u = 0; u < 8; ++u) if (k + u < e) xv[u] = xin(s_col[k + u - ca]);
#pragma unroll
                        for (int u = 0; u < 8; ++u)
                            if (k + u < e) acc = row_step(acc, s_val[k + u - ka], xv[u], k + u >= q);
                        epi(i, acc, xin(i), dinv, d0, d1);
                    } else {
                        s_med[atomicAdd(&s_nmed, 1)] = i;
                    }
                }
                __syncthreads();
                const int nmed = s_nmed;
                const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
                for (int m = warp; m < nmed; m += nw) {
                    const int r = s_med[m];
                    const int a = s_rp[r - ra], e = s_rp[r + 1 - ra];
                    T acc = T(0);
                    int k = a + lane;
                    for (; k + 3 * 32 < e; k += 4 * 32) {
                        const T x0 = xin(s_col[k - ca]), x1 = xin(s_col[k + 32 - ca]);
                        const T x2 = xin(s_col[k + 64 - ca]), x3 = xin(s_col[k + 96 - ca]);
                        acc = mac(acc, s_val[k - ka], x0);
                        acc = mac(acc, s_val[k + 32 - ka], x1);
                        acc = mac(acc, s_val[k + 64 - ka], x2);
                        acc = mac(acc, s_val[k + 96 - ka], x3);
                    }
                    for (; k < e; k += 32) acc = mac(acc, s_val[k - ka], xin(s_col[k - ca]));
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
                    if (lane == 0) epi(r, acc, xin(r), dinv, d0, d1);
                }
            } else {
                const int r = tile.row_begin;
                const int* __restrict__ ci = d.ci;
                const T* __restrict__ va = static_cast<const T*>(d.val);
                T acc = T(0);
                int k = tile.nnz_begin + threadIdx.x;
                const int B = blockDim.x;
                for (; k + 3 * B < tile.nnz_end; k += 4 * B) {
                    const int c0 = ci[k], c1 = ci[k + B], c2 = ci[k + 2 * B], c3 = ci[k + 3 * B];
                    const T v0 = va[k], v1 = va[k + B], v2 = va[k + 2 * B], v3 = va[k + 3 * B];
                    const T x0 = xin(c0), x1 = xin(c1), x2 = xin(c2), x3 = xin(c3);
                    acc = mac(acc, v0, x0);
                    acc = mac(acc, v1, x1);
                    acc = mac(acc, v2, x2);
                    acc = mac(acc, v3, x3);
                }
                for (; k < tile.nnz_end; k += B) acc = mac(acc, va[k], xin(ci[k]));
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
                const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
                if (lane == 0) s_acc[warp] = acc;
                __syncthreads();
                if (warp == 0) {
                    acc = lane < (int)(blockDim.x >> 5) ? s_acc[lane] : T(0);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
                    if (lane == 0) epi(r, acc, xin(r), dinv, d0, d1);
                }
            }
            if (op.fin != FIN_NONE) {
                double dd[kMaxDots] = {d0, d1, 0.0, 0.0};
                block_reduce<kMaxDots>(dd, s_red);
                store_partials<kMaxDots>(sv, t, dd);
                ++tally.n;
            }
        }
        __syncthreads();   // the buffer is refilled two tiles later
        cur = nxt;
        nxt = nn;
    }
    cp_async_wait_0();
    if (op.fin != FIN_NONE) spmv_publish(sv, op, tally, s_red);
}

// ---------------------------------------------------------------- SpMV, warp tasks
// Row-aligned warp tasks for matrices with irregular row lengths.  A task is
// either a run of consecutive rows with at most kWarpNnz entries in total
// (and at most kWarpNnz rows), or one row with more entries.
constexpr int kWarpNnz = 256;
constexpr int kSeqRow = 32;   // rows of a run task summed by one lane in storage order

struct WarpTask {
    int row_begin, row_end, nnz_begin, nnz_end;
};

// Element copies global -> shared without register staging (cp.async of 4
// or 8 bytes, cached in L1 as the only size-generic form allows).
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(s), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_drain_warp()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
    __syncwarp();
}

// Run tasks: each lane loads 8 column indices (coalesced) and issues, without
// register staging, the copies of the matching values and the 8 gathers of x
// into the warp's shared buffers (cp.async), plus the task's row pointers;
// every lane then sums whole rows of up to kSeqRow entries from there,
// sequentially in storage order with row_step (so such a row's result is
// bitwise the reference's row sum); longer rows are summed by the whole warp.
// Long-row tasks: the warp strides over the row 256 entries at a time
// through the same buffers and reduces with a fixed tree.
// Scheduling: warps take tasks from a counter (one atomic per task) in the
// order of the task list -- long-row tasks first, most entries first, then
// the runs in row order -- so no warp is left holding several long rows at
// the end; the next task's descriptor is loaded while the current one runs.
// The last warp to finish resets the counter for the next launch.  No CTA
// barrier: warps proceed independently.
template <typename T, int ASG>
__global__ void __launch_bounds__(kBlock, 3)
k_spmv_rows(const WarpTask* __restrict__ tasks, int ntasks, int* __restrict__ ctr, const int* __restrict__ rp,
            const int* __restrict__ ci, const T* __restrict__ va, const T* __restrict__ x, T* __restrict__ y)
{
    __shared__ T s_a[kBlock / 32][kWarpNnz];
    __shared__ T s_x[kBlock / 32][kWarpNnz];
    __shared__ int s_rp[kBlock / 32][kWarpNnz + 1];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    T* sa = s_a[wib];
    T* sx = s_x[wib];
    int* srp = s_rp[wib];
    auto grab = [&]() {
        int v = 0;
        if (lane == 0) v = atomicAdd(ctr, 1);
        return __shfl_sync(0xffffffffu, v, 0);
    };
    int t = grab();
    WarpTask nxt;
    if (t < ntasks) nxt = tasks[t];
    while (t < ntasks) {
        const WarpTask task = nxt;
        t = grab();
        if (t < ntasks) nxt = tasks[t];
        const int k0 = task.nnz_begin, k1 = task.nnz_end;
        if (task.row_end - task.row_begin == 1 && k1 - k0 > kWarpNnz) {
            T acc = T(0);
            for (int kb = k0; kb < k1; kb += 32 * 8) {
                int cc[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int k = kb + lane + 32 * u;
                    if (k < k1) {
                        cc[u] = __ldg(ci + k);
                        cp_async_elem<sizeof(T)>(sa + lane + 32 * u, va + k);
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (kb + lane + 32 * u < k1) cp_async_elem<sizeof(T)>(sx + lane + 32 * u, x + cc[u]);
                cp_async_drain_warp();
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (kb + lane + 32 * u < k1) acc = mac(acc, sa[lane + 32 * u], sx[lane + 32 * u]);
                __syncwarp();   // the buffers are refilled by the next 256 entries
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
            if (lane == 0) {
                const int r = task.row_begin;
                const T base = (ASG == ASG_SET) ? T(0) : y[r];
                y[r] = assign_out<T, ASG>(base, acc);
            }
            continue;
        }
        const int nr = task.row_end - task.row_begin;
        int cc[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int k = k0 + lane + 32 * u;
            if (k < k1) {
                cc[u] = __ldg(ci + k);
                cp_async_elem<sizeof(T)>(sa + lane + 32 * u, va + k);
            }
        }
#pragma unroll
        for (int u = 0; u < 9; ++u) {
            const int r = lane + 32 * u;
            if (r <= nr) cp_async_elem<4>(srp + r, rp + task.row_begin + r);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (k0 + lane + 32 * u < k1) cp_async_elem<sizeof(T)>(sx + lane + 32 * u, x + cc[u]);
        cp_async_drain_warp();
        // rows of up to kSeqRow entries: one lane each, summed sequentially
        // (bitwise the sequential row sum); longer rows: the whole warp,
        // lane-strided partial sums and a fixed shuffle tree, so no lane
        // walks a long row alone while the others wait
        for (int base = 0; base < nr; base += 32) {
            const int r = base + lane;
            int a = 0, e = 0;
            if (r < nr) {
                a = srp[r] - k0;
                e = srp[r + 1] - k0;
            }
            const bool seq = r < nr && e - a <= kSeqRow;
            if (seq) {
                T acc = T(0);
                const int q = fused_tail(a, e);
                for (int j = a; j < e; ++j) acc = row_step(acc, sa[j], sx[j], j >= q);
                const int row = task.row_begin + r;
                const T yb = (ASG == ASG_SET) ? T(0) : y[row];
                y[row] = assign_out<T, ASG>(yb, acc);
            }
            unsigned lng = __ballot_sync(0xffffffffu, r < nr && !seq);
            while (lng) {
                const int rr = base + __ffs(lng) - 1;
                lng &= lng - 1;
                T acc = T(0);
                const int ra = srp[rr] - k0, re = srp[rr + 1] - k0;
                for (int j = ra + lane; j < re; j += 32) acc = mac(acc, sa[j], sx[j]);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
                if (lane == 0) {
                    const int row = task.row_begin + rr;
                    const T yb = (ASG == ASG_SET) ? T(0) : y[row];
                    y[row] = assign_out<T, ASG>(yb, acc);
                }
            }
        }
        __syncwarp();
    }
    // self-reset: the last warp out zeroes the task counter and itself
    if (lane == 0) {
        const int nw = gridDim.x * (blockDim.x >> 5);
        if (atomicAdd(ctr + 1, 1) == nw - 1) {
            ctr[0] = 0;
            ctr[1] = 0;
            __threadfence();
        }
    }
}

// Gather floor of y = A x (a measurement kernel): every entry's value and
// column are streamed and x[col] gathered, 8 entries in flight per thread,
// with no row structure; one partial sum per thread.
__global__ void __launch_bounds__(kBlock) k_gather_floor(long long nnz, const int* __restrict__ ci,
                                                         const double* __restrict__ va, const double* __restrict__ x,
                                                         double* __restrict__ out)
{
    double acc = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; k0 < nnz; k0 += 8 * stride) {
        int c[8];
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const long long k = k0 + u * stride;
            c[u] = k < nnz ? __ldg(ci + k) : 0;
            v[u] = k < nnz ? __ldg(va + k) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) acc = fma(v[u], __ldg(x + c[u]), acc);
    }
    out[blockIdx.x * (long long)blockDim.x + threadIdx.x] = acc;
}

// Thread per row straight from global memory (rows of consecutive threads are
// adjacent, so a warp's value and column loads stay in the sectors L1 just
// fetched); gathers issued 8 at a time, summed in storage order.
template <typename T, int ASG>
__global__ void __launch_bounds__(kBlock)
k_spmv_scalar(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ va,
              const T* __restrict__ x, T* __restrict__ y)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int a = rp[i], e = rp[i + 1], q = fused_tail(a, e);
        T acc = T(0);
        int k = a;
        for (; k + 8 <= e; k += 8) {
            T xv[8], av[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) { av[u] = va[k + u]; xv[u] = x[ci[k + u]]; }
#pragma unroll
            for (int u = 0; u < 8; ++u) acc = row_step(acc, av[u], xv[u], k + u >= q);
        }
        T xv[8], av[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) if (k + u < e) { av[u] = va[k + u]; xv[u] = x[ci[k + u]]; }
#pragma unroll
        for (int u = 0; u < 8; ++u) if (k + u < e) acc = row_step(acc, av[u], xv[u], k + u >= q);
        const T base = (ASG == ASG_SET) ? T(0) : y[i];
        y[i] = assign_out<T, ASG>(base, acc);
    }
}

// ---------------------------------------------------------------- vector passes
enum VOp : int {
    VOP_DOT = 0,        // dots only
    VOP_AXPY,           // y += a x             (a = op.scalar)
    VOP_CG_UPDATE,      // x += alpha p ; r -= alpha q
    VOP_BI_P,           // p = r + beta (p - omega v)   (first: p = r)
    VOP_BI_S,           // s = r - alpha v
    VOP_BI_XR,          // x += omega shat + alpha phat ; r = s - omega t  (finishing: x += alpha phat)
    VOP_REF_CAST,       // r32 = float(r64 / scale); d = 0; z/r inner init
    VOP_REF_UPDATE,     // x64 += scale * double(d)
    VOP_FILL,           // v = scalar
    VOP_COPY,           // y = x
    VOP_SCALE_COPY,     // y = a x
};

struct VecOp {
    int op;
    int a, b, c, e, f, g;   // slots (meaning per op)
    int ndot;
    int da[kMaxDots], db[kMaxDots], dc[kMaxDots];
    int rk[kMaxDots];   // reference summation order of each dot (RK_*, refdot.cuh)
    int fin;
    int skip;
    int count_body;
    double scalar;
};

template <typename T>
__device__ __forceinline__ T vpick(const T* const* v, int j, int code, int i, const T* dinv)
{
    if (code == OPND_ONE) return T(1);
    if (code == OPND_D) return dinv[i];
    return v[j][i];
}

// Publishes a CTA's tally of a system's finished vector-pass tiles; the CTA
// that completes the system gathers its partials and finalizes (or retires a
// finishing BiCGSTAB system).
template <int OP>
__device__ __forceinline__ void vec_publish(const SetView& sv, const VecOp& op, TileTally& tally, double* s_red)
{
    const int count = int(tally.need);
    if (publish_tally(sv, tally)) {
        double tot[kMaxDots];
        gather_partials<kMaxDots>(sv, tally.sys, tot, s_red, count);
        if (threadIdx.x == 0) {
            SysState& s = sv.st[tally.sys];
            if (OP == VOP_BI_XR && (s.flags & FLAG_FINISHING)) {
                s.flags &= ~FLAG_FINISHING;
                retire(sv, s, (int)s.dots[3], s.error);
            } else {
                finalize(sv, op.fin, tally.sys, tot);
            }
        }
    }
}

constexpr int kVecGroup = 4;   // tiles a vector-pass CTA works on at once (one row of each per thread)

// A vector pass splits each system into row tiles of kTileRows (tile v:
// rows v kTileRows .. + kTileRows), as many as fit in the system's share of
// the SpMV tile indices (at least that many: SpMV tiles hold at most
// kTileRows rows), whose partial slots it uses.  One CTA per run of
// consecutive tile indices (the launch sizes the grid to the SMs),
// kVecGroup tiles of one system at a time (thread k takes row k of each, so
// its loads of the group's rows are in flight together, with no tile
// metadata to read); the system's vectors and scalars are read once per run.
// Each tile's partial dots are block reduced on their own in a fixed order,
// so the sums do not depend on the grid, the grouping or the batch.
template <typename T, int OP>
__global__ void __launch_bounds__(kBlock) k_vec(SetView sv, VecOp op)
{
    static_assert(kBlock == kTileRows, "a vector-pass thread takes one row of each tile");
    constexpr int NR = kVecGroup * kMaxDots;
    __shared__ double s_red[NR * 32];
    if (op.count_body && blockIdx.x == 0 && threadIdx.x == 0) {
        int runs = atomicAdd(&sv.err[1], 1) + 1;
        if (runs > sv.err[2] || *(volatile int*)sv.running <= 0) set_cond(sv, 0u);
    }
    const int t_begin = int((long long)sv.n_tiles * blockIdx.x / gridDim.x);
    const int t_end = int((long long)sv.n_tiles * (blockIdx.x + 1) / gridDim.x);
    TileTally tally;
    int t = t_begin;
    while (t < t_end) {
        const int sys = sv.tiles[t].sys;
        const int tb = sv.sys_tile_begin[sys];
        const int te = min(t_end, sv.sys_tile_begin[sys + 1]);   // this system's tile indices in the CTA's range
        const SysDesc& d = sv.desc[sys];
        const int n = sv.tiles[sv.sys_tile_begin[sys + 1] - 1].row_end;   // its rows (the last tile's end)
        const int nvt = (n + kTileRows - 1) / kTileRows;                   // its row tiles
        if (sys != tally.sys) {
            vec_publish<OP>(sv, op, tally, s_red);
            tally.sys = sys;
            tally.need = unsigned(nvt);
        }
        SysState& s = sv.st[sys];
        if (skip_system(s, op.skip)) {
            t = te;
            continue;
        }
        const T* dinv = static_cast<const T*>(d.inv_diag);
        const T* dv[3 * kMaxDots];
#pragma unroll
        for (int j = 0; j < kMaxDots; ++j) {
            dv[3 * j + 0] = (j < op.ndot && names_vector(op.da[j])) ? vptr<T>(d, op.da[j]) : nullptr;
            dv[3 * j + 1] = (j < op.ndot && names_vector(op.db[j])) ? vptr<T>(d, op.db[j]) : nullptr;
            dv[3 * j + 2] = (j < op.ndot && names_vector(op.dc[j])) ? vptr<T>(d, op.dc[j]) : nullptr;
        }
        T* A = op.a != SLOT_NONE ? vptr<T>(d, op.a) : nullptr;
        T* B = op.b != SLOT_NONE ? vptr<T>(d, op.b) : nullptr;
        T* C = op.c != SLOT_NONE ? vptr<T>(d, op.c) : nullptr;
        T* E = op.e != SLOT_NONE ? vptr<T>(d, op.e) : nullptr;
        T* F = op.f != SLOT_NONE ? vptr<T>(d, op.f) : nullptr;
        T* G = op.g != SLOT_NONE ? vptr<T>(d, op.g) : nullptr;
        const bool finishing = (s.flags & FLAG_FINISHING) != 0;
        const T alpha = T(s.alpha), beta = T(s.beta), omega = T(s.omega);
        const bool first = (s.iter <= 1);
        const double scale = s.scale;
        const bool reduce = op.fin != FIN_NONE || (OP == VOP_BI_XR && finishing);
        // one row: the pass and its dot terms
        auto row = [&](int i, double* dot) {
            if (OP == VOP_AXPY) {
                A[i] = fma(T(op.scalar), B[i], A[i]);                       // A += s B
            } else if (OP == VOP_CG_UPDATE) {
                A[i] = fma(alpha, B[i], A[i]);                              // x += alpha p
                C[i] = fma(-alpha, E[i], C[i]);                             // r -= alpha q
            } else if (OP == VOP_BI_P) {
                // p = r + beta * (p - omega * v)     (bicgstab.hpp:49-53)
                A[i] = first ? B[i] : fma(beta, fma(-omega, C[i], A[i]), B[i]);
            } else if (OP == VOP_BI_S) {
                A[i] = fma(-alpha, C[i], B[i]);                             // s = r - alpha v
            } else if (OP == VOP_BI_XR) {
                // A x, B phat, C shat, E s, F t, G r
                if (finishing) {
                    A[i] = fma(alpha, B[i], A[i]);                          // x += alpha phat
                } else {
                    // x += omega shat + alpha phat, evaluated as the reference
                    // build does: x + fma(alpha, phat, omega shat)
                    A[i] = A[i] + fma(alpha, B[i], omega * C[i]);
                    G[i] = fma(-omega, F[i], E[i]);                         // r = s - omega t
                }
            } else if (OP == VOP_REF_CAST) {
                // inner right-hand side float(r64 / ||r64||); inner x = 0, r = b
                const T bi = T(d.r64[i] / scale);
                A[i] = bi;
                if (B) B[i] = T(0);
                if (C) C[i] = bi;
                if (E) E[i] = bi;
            } else if (OP == VOP_REF_UPDATE) {
                d.x64[i] = fma(scale, double(A[i]), d.x64[i]);            // x += ||r|| * d
            } else if (OP == VOP_FILL) {
                A[i] = T(op.scalar);
            } else if (OP == VOP_COPY) {
                A[i] = B[i];
            } else if (OP == VOP_SCALE_COPY) {
                A[i] = T(op.scalar) * B[i];
            }
#pragma unroll
            for (int j = 0; j < kMaxDots; ++j)
                if (j < op.ndot)
                    dot[j] += double(vpick<T>(dv, 3 * j + 0, op.da[j], i, dinv) * vpick<T>(dv, 3 * j + 1, op.db[j], i, dinv) *
                                     vpick<T>(dv, 3 * j + 2, op.dc[j], i, dinv));
        };
        for (; t < te; t += kVecGroup) {
            const int v0 = t - tb;
            const int ng = max(0, min(min(kVecGroup, te - t), nvt - v0));   // row tiles among these indices
            double dot[NR];
#pragma unroll
            for (int k = 0; k < NR; ++k) dot[k] = 0.0;
#pragma unroll
            for (int q = 0; q < kVecGroup; ++q) {
                const int i = (v0 + q) * kTileRows + int(threadIdx.x);
                if (q < ng && i < n) row(i, dot + q * kMaxDots);
            }
            if (!reduce || ng == 0) continue;
            block_reduce<NR>(dot, s_red);
            if (threadIdx.x == 0) {
#pragma unroll
                for (int q = 0; q < kVecGroup; ++q)
                    if (q < ng)
#pragma unroll
                        for (int j = 0; j < kMaxDots; ++j) sv.partials[(long long)(t + q) * kMaxDots + j] = dot[q * kMaxDots + j];
            }
            tally.n += unsigned(ng);
        }
        t = te;
    }
    vec_publish<OP>(sv, op, tally, s_red);
}

}  // namespace mtlg
