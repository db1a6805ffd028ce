// Dots and norms in the reference build's summation order (FP64), for the
// context's "reduction_order" 1 (reference order) mode.
//
// MTL4 reduces a vector with four partial sums t[k] over the entries
// i = k (mod 4) of the first 4*floor(n/4) entries, each partial added in
// index order, the remaining entries into t[0], and then combines the four.
// The four kinds below differ in whether the products are rounded or fused
// and in the order of the final combination (determined against the
// reference build, g++ -O3 -march=x86-64-v3 -ffp-contract=fast):
//   RK_DOT4   mtl::dot (operation/dot.hpp:99-145, Unroll 4): rounded
//             products throughout; (t0 + t1) + (t2 + t3)
//   RK_NORM4  two_norm squared (operation/two_norm.hpp:35-56,
//             vector/reduction.hpp:85-175): rounded products, fused tail;
//             t0 + (t1 + (t2 + t3))
//   RK_LDOT4  lazy_dot inside a fused expression (vector/dot_index_evaluator
//             .hpp:20-45, operation/fused_expr.hpp:60-75): rounded products;
//             ((t0 + t1) + t2) + t3
//   RK_UDOT4  lazy_unary_dot inside a fused expression
//             (vector/reduction_index_evaluator.hpp:31-34): fused products;
//             (t0 + t1) + (t2 + t3)
// A partial sum is a chain of n/4 dependent additions, which no parallel
// scheme reproduces bitwise: one warp per dot stages blocks of the operands
// in shared memory (16-byte cp.async, double-buffered) and four lanes run
// the four chains.  This costs about a microsecond per thousand entries; the
// default mode's tile-parallel reductions do not follow this order.
#pragma once
#include "kernels.cuh"

namespace mtlg {

enum RedKind : int { RK_DOT4 = 0, RK_NORM4 = 1, RK_LDOT4 = 2, RK_UDOT4 = 3 };

constexpr int kRefBlk = 1024;                 // entries staged per block and operand
constexpr int kRefOps = 3;                    // operands per product: a * (b * c)
constexpr int kRefWarpSmem = 2 * kRefOps * kRefBlk * 8;   // two buffers per warp

struct RefDotOp {
    int ndot;
    int va[kMaxDots], vb[kMaxDots], vc[kMaxDots];   // vector codes (slots), OPND_D or OPND_ONE
    int rk[kMaxDots];
    int fin;
    int skip;
};

__device__ __forceinline__ const double* ref_operand(const SysDesc& d, int code)
{
    if (code == OPND_ONE) return nullptr;
    if (code == OPND_D) return static_cast<const double*>(d.inv_diag);
    return vptr<double>(d, code);
}

// One system per CTA, one warp per dot (blockDim.x = 32 * ndot).
__global__ void __launch_bounds__(32 * kMaxDots) k_dot_ref(SetView sv, RefDotOp op)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double s_res[kMaxDots];
    const int sys = blockIdx.x;
    SysState& s = sv.st[sys];
    // (a finishing BiCGSTAB system was retired by its x/r pass, which still
    // reduces in that case, so it is skipped here like any finished system)
    if (skip_system(s, op.skip)) return;
    const SysDesc& d = sv.desc[sys];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = d.n, nb = n / 4 * 4;
    const double* src[kRefOps] = {ref_operand(d, op.va[w]), ref_operand(d, op.vb[w]), ref_operand(d, op.vc[w])};
    const int kind = op.rk[w];
    double* buf = reinterpret_cast<double*>(smem_raw + w * kRefWarpSmem);   // [2][kRefOps][kRefBlk]
    auto stage = [&](int blk, int which) {
        const int base = blk * kRefBlk, cnt = min(kRefBlk, nb - base);   // a multiple of 4: 32-byte chunks
        for (int o = 0; o < kRefOps; ++o) {
            if (!src[o]) continue;
            double* dst = buf + (which * kRefOps + o) * kRefBlk;
            if ((reinterpret_cast<uintptr_t>(src[o]) & 15) == 0) {
                for (int c = lane; c < cnt / 2; c += 32) cp_async16(dst + 2 * c, src[o] + base + 2 * c);
            } else {   // a borrowed vector that is not 16-byte aligned: plain loads
                for (int c = lane; c < cnt; c += 32) dst[c] = src[o][base + c];
            }
        }
        cp_async_commit();
    };
    const int nblk = (nb + kRefBlk - 1) / kRefBlk;
    double t = 0.0;   // lane k < 4: partial sum k
    if (nblk > 0) stage(0, 0);
    for (int blk = 0; blk < nblk; ++blk) {
        if (blk + 1 < nblk) stage(blk + 1, (blk + 1) & 1);
        else cp_async_commit();
        cp_async_wait_1();
        __syncwarp();
        if (lane < 4) {
            const double* a = buf + ((blk & 1) * kRefOps + 0) * kRefBlk;
            const double* b = buf + ((blk & 1) * kRefOps + 1) * kRefBlk;
            const double* c = buf + ((blk & 1) * kRefOps + 2) * kRefBlk;
            const int cnt = min(kRefBlk, nb - blk * kRefBlk);
            const bool hb = src[1] != nullptr, hc = src[2] != nullptr;
            for (int e = lane; e < cnt; e += 4) {
                const double bc = hc ? (hb ? __dmul_rn(b[e], c[e]) : c[e]) : (hb ? b[e] : 1.0);
                t = kind == RK_UDOT4 ? __fma_rn(a[e], bc, t) : __dadd_rn(t, __dmul_rn(a[e], bc));
            }
        }
        __syncwarp();   // the buffer is refilled by the next iteration's stage
    }
    cp_async_wait_0();
    // gather the four partials in lane 0, add the tail to t[0], combine
    const double t1 = __shfl_sync(0xffffffffu, t, 1), t2 = __shfl_sync(0xffffffffu, t, 2),
                 t3 = __shfl_sync(0xffffffffu, t, 3);
    if (lane == 0) {
        double t0 = t;
        for (int i = nb; i < n; ++i) {
            const double av = src[0][i];
            const double bv = src[1] ? src[1][i] : 1.0;
            const double bc = src[2] ? __dmul_rn(bv, src[2][i]) : bv;
            const bool fused = kind == RK_UDOT4 || kind == RK_NORM4;
            t0 = fused ? __fma_rn(av, bc, t0) : __dadd_rn(t0, __dmul_rn(av, bc));
        }
        double r;
        if (kind == RK_NORM4) r = __dadd_rn(t0, __dadd_rn(t1, __dadd_rn(t2, t3)));
        else if (kind == RK_LDOT4) r = __dadd_rn(__dadd_rn(__dadd_rn(t0, t1), t2), t3);
        else r = __dadd_rn(__dadd_rn(t0, t1), __dadd_rn(t2, t3));
        s_res[w] = r;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double dots[kMaxDots] = {0.0, 0.0, 0.0, 0.0};
        for (int j = 0; j < op.ndot; ++j) dots[j] = s_res[j];
        finalize(sv, op.fin, sys, dots);
    }
}

}  // namespace mtlg
