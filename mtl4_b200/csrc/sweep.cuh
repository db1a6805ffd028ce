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
