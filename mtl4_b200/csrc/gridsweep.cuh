// Structured-grid triangular sweeps (k_sweep_grid).
//
// Used when a factor's pattern is exactly a 5- or 7-point grid stencil in
// natural order (TriFactor's grid layout, detected at preconditioner
// set-up); other factors keep the chunked and flat sweeps.  The arithmetic
// of a row is k_sweep's, entry for entry: rr = v[r]; rr -= a * w for the
// row's off-diagonal entries in the reference's storage order; w[r] = rr *
// dia (boost/numeric/mtl/operation/lower_trisolve.hpp:174-209,
// upper_trisolve.hpp:161-176).  Only the schedule differs:
//  - lane l of a warp owns the x-line j = 32 jb + l of plane k and runs its
//    rows in x order, row i at step i + l: the x neighbour is the lane's own
//    previous result (a register) and the y neighbour the lower lane's
//    result of the previous step (a warp shuffle), so consecutive levels of
//    a warp need no barrier;
//  - the lane below lane 0 (the previous y-block) and the plane below run in
//    other warps.  A CTA runs the NW warps of one tile (NW consecutive planes
//    of one y-block, or NW consecutive y-blocks of a 2D grid) and hands
//    results between them through shared-memory rings whose cells carry
//    readiness in the value (the sentinel pattern marks an empty cell; the
//    consumer empties a cell after reading it);
//  - results of earlier tiles (other CTAs) are read from the output vector,
//    which is all-sentinel before a sweep (each sweep resets the vector the
//    next one writes), by two receiver warps that poll many steps at once
//    and fill the same rings;
//  - each warp's factor values, laid out step by step 32 lanes wide, stream
//    into shared memory with bulk copies (TMA) several steps ahead, its
//    right-hand sides with per-lane cp.async.
// Tiles are taken through one ticket in an order in which every tile a tile
// reads comes earlier, and a tile runs to its end on a running CTA, so the
// waits end; every wait is still bounded (the context's spin_limit polls),
// after which the kernel records a timeout and drains with zeros.
// The same kernel computes the FP64 pivots of an ILU(0) or IC(0)
// factorization of a grid-stencil pattern (OPK kGridILU0 / kGridIC0): a
// row's pivot needs its earlier neighbours' pivots exactly as an L sweep's
// row needs their results (boost/numeric/itl/pc/ilu_0.hpp:45-82,
// ic_0.hpp:124-186, with k_ilu0_factor's and k_ic0_factor's roundings).
#pragma once
#include "sweep.cuh"

namespace mtlg {

constexpr int kGridNB = 3;                  // staged factor blocks per compute warp
constexpr int kGridG = 8;                   // steps per block (staged factor values, right-hand sides)
constexpr int kGridRing = 32;               // steps per z / y ring (power of two)
constexpr int kGridRhs = 32;                // right-hand-side ring (power of two, four blocks)
constexpr int kGridRecvWarps = 2;           // receiver warps after the compute warps
constexpr int kGridBatch = 16;              // steps per receiver batch
static_assert(kGridRecvWarps * kGridBatch <= kGridRing, "receiver batches in flight must fit a ring");
static_assert(kGridStepPad % kGridG == 0, "layout padding must hold whole staged blocks");
static_assert(kGridRhs >= 3 * kGridG, "the right-hand-side ring holds the current block and two ahead");

// Row operations of the grid kernel: a triangular sweep, or the FP64 pivots
// of an ILU(0) or IC(0) factorization (the same dependencies: a row's pivot
// needs its three earlier neighbours' pivots).
constexpr int kGridSweep = 0, kGridILU0 = 1, kGridIC0 = 2;
// Slots per step (capacity): a sweep's entries and multiplier fit four; an
// ILU(0) pivot reads its L entries, the neighbours' entries in its column and
// its diagonal (up to seven).
__host__ __device__ constexpr int grid_cap(int opk) { return opk == kGridILU0 ? 8 : 4; }

// Staged S elements per compute warp (kGridNB blocks of up to grid_cap slots).
template <typename S, int OPK = kGridSweep>
__host__ __device__ constexpr int grid_stage_elems()
{
    return kGridNB * kGridG * grid_cap(OPK) * 32;
}

// Dynamic shared memory of a k_sweep_grid CTA of nw compute warps.
template <typename T, typename S, int OPK = kGridSweep>
__host__ __device__ inline int grid_smem_bytes(int nw)
{
    return nw * (grid_stage_elems<S, OPK>() * int(sizeof(S)) + (kGridRhs + kGridRing) * 32 * int(sizeof(T)) +
                 kGridRing * int(sizeof(T)));
}

// Slot orders the kernel runs (TriFactor::gperm): the farthest neighbour's
// entry first (z, y, x / y, x: rows stored by ascending column from below),
// or the nearest first (x, y, z / x, y).
constexpr int kGridFar3 = 2 | (1 << 2) | (0 << 4);
constexpr int kGridNear3 = 0 | (1 << 2) | (2 << 4);
constexpr int kGridFar2 = 1 | (0 << 2);
constexpr int kGridNear2 = 0 | (1 << 2);

__device__ __forceinline__ long long grid_row(long long rp, int n, int rev) { return rev ? (long long)n - 1 - rp : rp; }

// Predicated stores (one instruction, no branch around it).
__device__ __forceinline__ void st_slot_if(float* p, float v, bool c)
{
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.volatile.shared.f32 [%0], %1;\n\t}" ::"r"(smem_u32(p)),
                 "f"(v), "r"(int(c)));
}
__device__ __forceinline__ void st_slot_if(double* p, double v, bool c)
{
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.volatile.shared.f64 [%0], %1;\n\t}" ::"r"(smem_u32(p)),
                 "d"(v), "r"(int(c)));
}
__device__ __forceinline__ void st_relaxed_gpu_if(float* p, float v, bool c)
{
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.relaxed.gpu.global.f32 [%0], %1;\n\t}" ::"l"(p), "f"(v),
                 "r"(int(c)));
}
__device__ __forceinline__ void st_relaxed_gpu_if(double* p, double v, bool c)
{
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.relaxed.gpu.global.f64 [%0], %1;\n\t}" ::"l"(p), "d"(v),
                 "r"(int(c)));
}

// Ring handoffs of a compute warp, warp-uniform: every lane takes part, a
// lane without a cell to serve (act false) reads the CTA's dummy cell, which
// always holds +0; the warp waits (bounded, then +0 and a timeout flag) until
// every acting lane sees its value, then the acting lanes empty their cells.
template <typename T>
__device__ __noinline__ T grid_wait_take(T* p, T v, int* err, long long lim)
{
    long long spins = 0;
    while (__any_sync(0xffffffffu, is_sentinel(v))) {
        if ((++spins & 255) == 0 && *(volatile int*)err) break;
        if (spins > (lim > 0 ? lim : kSpinLimit)) {
            atomicExch(err, 1);
            break;
        }
        if (spins > 32) __nanosleep(32);   // a long wait leaves the issue slots to the producers
        if (is_sentinel(v)) v = ld_slot(p);
    }
    return is_sentinel(v) ? T(0) : v;
}
template <typename T>
__device__ __forceinline__ T grid_take(T* cell, bool act, T* dummy, int* err, long long lim)
{
    T* p = act ? cell : dummy;
    T v = ld_slot(p);
    if (__any_sync(0xffffffffu, is_sentinel(v))) v = grid_wait_take(p, v, err, lim);
    st_slot_if(cell, sentinel_value<T>(), act);
    return v;
}
// Fills ring cells once their previous values have been taken (same rules).
template <typename T>
__device__ __noinline__ void grid_wait_free(T* p, bool act, int* err, long long lim)
{
    long long spins = 0;
    while (__any_sync(0xffffffffu, act && !is_sentinel(ld_slot(p)))) {
        if ((++spins & 255) == 0 && *(volatile int*)err) return;
        if (spins > (lim > 0 ? lim : kSpinLimit)) {
            atomicExch(err, 1);
            return;
        }
        if (spins > 32) __nanosleep(32);
    }
}
template <typename T>
__device__ __forceinline__ void grid_put(T* cell, bool act, T v, T* dummy, int* err, long long lim)
{
    T* p = act ? cell : dummy;
    if (__any_sync(0xffffffffu, act && !is_sentinel(ld_slot(p)))) grid_wait_free(p, act, err, lim);
    st_slot_if(cell, v, act);
}

// A compute warp's unit of one tile (pointers already offset by the lane
// where the cell is per lane).
template <typename T, typename S>
struct GridWarp {
    const S* src;              // the unit's layout
    S* stg;                    // its staged blocks (kGridNB)
    unsigned long long* fb;    // their barriers
    const T* vin;
    T* vout;
    T* vres;                   // nullptr: no reset vector
    T* rr;                     // right-hand-side ring, this lane's column
    T* zin;                    // incoming z ring, this lane's column
    T* yin;                    // incoming y ring (lane 0)
    T* zo;                     // outgoing z ring (the next plane's warp), this lane's column
    T* yo;                     // outgoing y ring (the next y-block's warp; lane 31)
    T* dummy;                  // the CTA's cell that always holds +0
    long long rbase;           // r' of this lane's row i = 0
    int n, nx, nsteps, lane;
    bool lane_on, has_z, has_y, z_out, y_out;
    int* err;
    long long spin;
};

// The steps of one compute warp's unit: blocks of kGridG steps, each block's
// factor values staged by a bulk copy kGridNB blocks ahead and its
// right-hand sides by cp.async two blocks ahead; blocks where every lane has
// a row at every step run without per-step validity tests.  NS entries per
// row, FAR: the farthest neighbour's entry first (z, y, x; else x, y, z),
// REV: rows counted from the end (U sweeps).
template <typename T, typename S, int NS, bool FAR, bool REV, int OPK = kGridSweep>
__device__ __forceinline__ void grid_warp_run(const GridWarp<T, S>& g, unsigned& phase)
{
    typedef typename std::conditional<(sizeof(S) > sizeof(T)), S, T>::type W;   // promoted type
    constexpr int G = kGridG;
    constexpr int SES = (OPK == kGridILU0 ? 2 * NS + 1 : NS + 1) * 32;   // S elements per step
    constexpr int BE = G * grid_cap(OPK) * 32;                          // S elements per staged block (capacity)
    constexpr bool SKEW = NS > 0;        // rows depend on the lane below: lane l runs row i at step i + l
    const int lane = g.lane;
    const int nblk = (g.nsteps + G - 1) / G;
    const unsigned bbytes = unsigned(G * SES * int(sizeof(S)));
    if (lane == 0)
        for (int b = 0; b < kGridNB && b < nblk; ++b) {
            mbar_expect_tx(&g.fb[b], bbytes);
            bulk_g2s(g.stg + b * BE, g.src + size_t(b) * G * SES, bbytes, &g.fb[b]);
        }
    // right-hand sides of block m into their ring cells (one cp.async group)
    auto fetch = [&](int m) {
        if (OPK == kGridSweep && m < nblk) {
            const int i0 = SKEW ? m * G - lane : m * G;
            const long long r0 = g.rbase + i0;
            const T* p = g.vin + (REV ? (long long)g.n - 1 - r0 : r0);
            T* cell = g.rr + (((m * G) & (kGridRhs - 1)) << 5);
#pragma unroll
            for (int u = 0; u < G; ++u)
                if (g.lane_on && i0 + u >= 0 && i0 + u < g.nx && r0 + u < g.n)
                    cp_async_elem<sizeof(T)>(cell + (u << 5), REV ? p - u : p + u);
        }
        cp_async_commit();
    };
    fetch(0);
    fetch(1);
    T wx = T(0), wy = T(0);
    for (int m = 0; m < nblk; ++m) {
        const int s0 = m * G, b = m % kGridNB;
        mbar_wait(&g.fb[b], (phase >> b) & 1u, g.err);
        phase ^= 1u << b;
        fetch(m + 2);
        asm volatile("cp.async.wait_group 2;" ::: "memory");
        const S* bk = g.stg + b * BE + lane;
        const int c0 = s0 & (kGridRing - 1);   // ring cells of the block's steps: c0 + u (no wrap)
        const T* rc = g.rr + (c0 << 5);
        T* zi = g.zin + (c0 << 5);
        T* zo = g.zo + (c0 << 5);
        T* yi = g.yin + c0;
        const int i0 = SKEW ? s0 - lane : s0;
        const long long r0 = g.rbase + i0;
        T* po = g.vout + (REV ? (long long)g.n - 1 - r0 : r0);
        T* pr = g.vres ? g.vres + (REV ? (long long)g.n - 1 - r0 : r0) : nullptr;
        auto steps = [&](auto edge) {
            constexpr bool EDGE = decltype(edge)::value;
#pragma unroll
            for (int u = 0; u < G; ++u) {
                const int i = i0 + u;
                bool valid = true;
                if (EDGE) valid = g.lane_on && i >= 0 && i < g.nx && r0 + u < g.n;
                T wz = T(0), wl = wy;
                if (NS == 3 && g.has_z) wz = grid_take(zi + (u << 5), valid, g.dummy, g.err, g.spin);
                if (NS >= 2 && g.has_y) {
                    const T yv = grid_take(yi + u, valid && lane == 0, g.dummy, g.err, g.spin);
                    wl = lane == 0 ? yv : wy;
                } else if (NS >= 2) {
                    wl = lane == 0 ? T(0) : wy;
                }
                const S* e = bk + u * SES;
                T acc = OPK == kGridSweep ? rc[u << 5] : T(e[(SES / 32 - 1) * 32]);   // a pivot starts from a_ii
                if constexpr (OPK == kGridILU0) {
                    // k_ilu0_factor on a grid stencil: per earlier neighbour k
                    // (ascending column) l = a_ik / u_kk (rounded), u_ii -= l a_ki
                    // (fused); L's entries and the other U entries do not change
                    if (NS == 3) {
                        acc = __fma_rn(-__dmul_rn(e[0], wz), e[96], acc);
                        acc = __fma_rn(-__dmul_rn(e[32], wl), e[128], acc);
                        acc = __fma_rn(-__dmul_rn(e[64], wx), e[160], acc);
                    } else if (NS == 2) {
                        acc = __fma_rn(-__dmul_rn(e[0], wl), e[64], acc);
                        acc = __fma_rn(-__dmul_rn(e[32], wx), e[96], acc);
                    }
                } else if constexpr (OPK == kGridIC0) {
                    // k_ic0_factor: d = a_ki / sqrt(u_kk) (rounded), u_ii -= d d
                    // (rounded product), per earlier neighbour k ascending
                    if (NS == 3) {
                        T d = __dmul_rn(e[0], wz);
                        acc = __dsub_rn(acc, __dmul_rn(d, d));
                        d = __dmul_rn(e[32], wl);
                        acc = __dsub_rn(acc, __dmul_rn(d, d));
                        d = __dmul_rn(e[64], wx);
                        acc = __dsub_rn(acc, __dmul_rn(d, d));
                    } else if (NS == 2) {
                        T d = __dmul_rn(e[0], wl);
                        acc = __dsub_rn(acc, __dmul_rn(d, d));
                        d = __dmul_rn(e[32], wx);
                        acc = __dsub_rn(acc, __dmul_rn(d, d));
                    }
                } else if constexpr (NS == 3) {
                    if (FAR) {
                        acc = sweep_step<T, S>(acc, e[0], wz);
                        acc = sweep_step<T, S>(acc, e[32], wl);
                        acc = sweep_step<T, S>(acc, e[64], wx);
                    } else {
                        acc = sweep_step<T, S>(acc, e[0], wx);
                        acc = sweep_step<T, S>(acc, e[32], wl);
                        acc = sweep_step<T, S>(acc, e[64], wz);
                    }
                } else if (NS == 2) {
                    if (FAR) {
                        acc = sweep_step<T, S>(acc, e[0], wl);
                        acc = sweep_step<T, S>(acc, e[32], wx);
                    } else {
                        acc = sweep_step<T, S>(acc, e[0], wx);
                        acc = sweep_step<T, S>(acc, e[32], wl);
                    }
                }
                T out;
                if constexpr (OPK == kGridILU0) out = unsentinel(T(__ddiv_rn(1.0, double(acc))));
                else if constexpr (OPK == kGridIC0) out = unsentinel(T(__ddiv_rn(1.0, __dsqrt_rn(double(acc)))));
                else out = unsentinel(T(W(acc) * W(e[NS * 32])));
                if (EDGE) out = valid ? out : T(0);   // +0 outside the lane's line: an absent neighbour
                st_relaxed_gpu_if(REV ? po - u : po + u, out, valid);
                if (pr && valid) *(REV ? pr - u : pr + u) = sentinel_value<T>();
                if (NS == 3 && g.z_out) grid_put(zo + (u << 5), valid, out, g.dummy, g.err, g.spin);
                if (NS >= 2 && g.y_out)
                    grid_put(g.yo + ((i) & (kGridRing - 1)), valid && lane == 31, out, g.dummy, g.err, g.spin);
                if (SKEW) {
                    wx = out;   // +0 before a lane's first row: its x neighbour is absent
                    wy = __shfl_up_sync(0xffffffffu, out, 1);
                }
            }
        };
        const bool inner = g.lane_on && i0 >= 0 && i0 + G <= g.nx && r0 + G <= g.n;
        if (__all_sync(0xffffffffu, inner)) steps(std::integral_constant<bool, false>());
        else steps(std::integral_constant<bool, true>());
        // every lane is done with block m: refill its buffer with block m + kGridNB
        __syncwarp();
        if (lane == 0 && m + kGridNB < nblk) {
            mbar_expect_tx(&g.fb[b], bbytes);
            bulk_g2s(g.stg + b * BE, g.src + size_t(m + kGridNB) * G * SES, bbytes, &g.fb[b]);
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// One sweep over the grid tiles of a set of systems.  op.tasks: GroupTask
// {sys, first unit along y, first plane, units along y per tile (jw)}; a
// tile's warp q runs unit (first + q % jw, plane + q / jw).  Systems with z
// neighbours are tiled with jw = 1 (the warps are consecutive planes).
template <typename T, typename S, int NW, bool REV, int OPK = kGridSweep>
__global__ void __launch_bounds__(32 * (NW + kGridRecvWarps)) k_sweep_grid(SetView sv, ChunkSweepOp op)
{
    constexpr int NTH = 32 * (NW + kGridRecvWarps);
    constexpr int SE = grid_stage_elems<S, OPK>();
    if (blockDim.x != unsigned(NTH) || op.which != int(REV)) {   // launch shape mismatch: report, never wait
        if (threadIdx.x == 0) atomicExch(sv.err, 1);
        return;
    }
    extern __shared__ __align__(128) unsigned char grid_smem[];
    __shared__ __align__(8) unsigned long long full[NW * kGridNB];
    __shared__ int s_task, s_go;
    __shared__ __align__(8) T grid_dummy;   // read by lanes without a ring cell to serve: always +0
    S* stage = reinterpret_cast<S*>(grid_smem);
    T* rhs_ring = reinterpret_cast<T*>(grid_smem + size_t(NW) * SE * sizeof(S));
    T* zring = rhs_ring + NW * kGridRhs * 32;   // [warp][step % ring][lane]
    T* yring = zring + NW * kGridRing * 32;     // [warp][row % ring]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        grid_dummy = T(0);
        for (int b = 0; b < NW * kGridNB; ++b) mbar_init(&full[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    unsigned phase = 0;   // compute warps: parity of the next wait on each of their staged blocks (bit b)
    for (;;) {
        if (tid == 0) {
            const int t = atomicAdd(op.ticket, 1);
            if (t == op.ntasks + int(gridDim.x) - 1) atomicExch(op.ticket, 0);
            s_task = t;
            s_go = t < op.ntasks && !skip_system(sv.st[op.tasks[t].sys], op.skip) && !*(volatile int*)sv.err;
        }
        for (int e = tid; e < NW * kGridRing * 33; e += NTH) zring[e] = sentinel_value<T>();   // z and y rings empty
        __syncthreads();
        const int t = s_task;
        if (t >= op.ntasks) break;
        if (s_go) {
            const GroupTask gt = op.tasks[t];
            const SysDesc& d = sv.desc[gt.sys];
            const TriFactor& F = op.which == 0 ? d.L : d.U;
            const int rev = int(REV);   // U: rows counted from the end
            const int n = d.n, nx = F.gnx, ny = F.gny, nz = F.gnz, ns = F.gns, perm = F.gperm, dirs = F.gdirs;
            const int nsteps = F.gnsteps, njb = F.gnjb;
            const int jw = gt.pad, kw = NW / jw, ju0 = gt.pos0, k0 = gt.count;
            T* vout = vptr<T>(d, op.out);
            if (warp < NW) {
                // ------------------------------------------------ compute warp
                const int q = warp, qj = q % jw, qk = q / jw;
                const int ju = ju0 + qj, k = k0 + qk;
                if (ju < njb && k < nz) {
                    const int j = 32 * ju + lane;
                    GridWarp<T, S> g;
                    const int slots = OPK == kGridILU0 ? 2 * ns + 1 : ns + 1;
                    g.src = static_cast<const S*>(F.gdata) + (size_t(k) * njb + ju) * size_t(F.gnsp) * size_t(slots) * 32;
                    g.stg = stage + size_t(q) * SE;
                    g.fb = full + q * kGridNB;
                    g.vin = vptr<T>(d, op.in);
                    g.vout = vout;
                    g.vres = op.reset != SLOT_NONE ? vptr<T>(d, op.reset) : nullptr;
                    g.rr = rhs_ring + q * kGridRhs * 32 + lane;
                    g.zin = zring + q * kGridRing * 32 + lane;
                    g.yin = yring + q * kGridRing;
                    g.zo = zring + (q + jw) * kGridRing * 32 + lane;   // used only when z_out
                    g.yo = yring + (q + 1) * kGridRing;                // used only when y_out
                    g.dummy = &grid_dummy;
                    g.rbase = (long long)nx * ((long long)j + (long long)ny * k);
                    g.n = n;
                    g.nx = nx;
                    g.nsteps = nsteps;
                    g.lane = lane;
                    g.lane_on = j < ny;
                    g.has_z = (dirs & 4) && k > 0;
                    g.has_y = (dirs & 2) && ju > 0;
                    g.z_out = (dirs & 4) && qk + 1 < kw && k + 1 < nz;
                    g.y_out = (dirs & 2) && qj + 1 < jw && ju + 1 < njb;
                    g.err = sv.err;
                    g.spin = sv.spin;
                    if constexpr (OPK != kGridSweep) {
                        // pivots: L's geometry, farthest neighbour first
                        if (ns == 3) grid_warp_run<T, S, 3, true, false, OPK>(g, phase);
                        else grid_warp_run<T, S, 2, true, false, OPK>(g, phase);
                    } else if (ns == 3) {
                        if (perm == kGridFar3) grid_warp_run<T, S, 3, true, REV>(g, phase);
                        else grid_warp_run<T, S, 3, false, REV>(g, phase);
                    } else if (ns == 2) {
                        if (perm == kGridFar2) grid_warp_run<T, S, 2, true, REV>(g, phase);
                        else grid_warp_run<T, S, 2, false, REV>(g, phase);
                    } else {
                        grid_warp_run<T, S, 0, false, REV>(g, phase);
                    }
                }
            } else {
                // ------------------------------------------------ receiver warps
                // Receiver 0: the plane below the tile (jw == 1; lane l for
                // lane l of the first plane's warp).  Receiver 1: the row
                // below each warp's lane 0 (jw == 1: lane q for warp q;
                // otherwise lane 0 for warp 0).  Each lane walks its own
                // steps with a cursor: kGridBatch loads in flight, the ready
                // prefix whose ring cells are free goes in, the rest waits
                // for the next round, so no lane ever blocks another.
                const int rw = warp - NW;
                bool on;
                long long base;     // r' of the lane's step 0 (Z: row i = s - lane; Y: row i = s)
                T* cells;
                int stride, c, end;
                if (rw == 0) {
                    on = jw == 1 && (dirs & 4) && k0 > 0 && 32 * ju0 + lane < ny;
                    base = (long long)nx * ((long long)(32 * ju0 + lane) + (long long)ny * (k0 - 1)) - lane;
                    cells = zring + lane;
                    stride = 32;
                    c = lane;
                    end = min(nsteps, lane + nx);
                } else {
                    const int yk = jw == 1 ? k0 + lane : k0;
                    on = rw == 1 && (dirs & 2) && ju0 > 0 && (jw == 1 ? (lane < kw && yk < nz) : lane == 0);
                    base = (long long)nx * ((long long)(32 * ju0 - 1) + (long long)ny * yk);
                    cells = yring + (jw == 1 ? lane : 0) * kGridRing;
                    stride = 1;
                    c = 0;
                    end = nx;
                }
                if (!on) end = c;
                const long long lim = sv.spin > 0 ? sv.spin : kSpinLimit;
                long long spins = 0;
                while (__any_sync(0xffffffffu, c < end)) {
                    T v[kGridBatch];
#pragma unroll
                    for (int u = 0; u < kGridBatch; ++u)
                        v[u] = c + u < end ? ld_relaxed_gpu(vout + grid_row(base + c + u, n, rev)) : sentinel_value<T>();
                    int adv = 0;
                    bool go = true;
#pragma unroll
                    for (int u = 0; u < kGridBatch; ++u) {
                        T* cell = cells + ((c + u) & (kGridRing - 1)) * stride;
                        go = go && c + u < end && !is_sentinel(v[u]) && is_sentinel(ld_slot(cell));
                        st_slot_if(cell, v[u], go);
                        adv += go ? 1 : 0;
                    }
                    c += adv;
                    if (__any_sync(0xffffffffu, adv > 0)) continue;
                    if ((++spins & 255) == 0 && *(volatile int*)sv.err) break;
                    if (spins > lim) {
                        atomicExch(sv.err, 1);
                        break;
                    }
                    __nanosleep(op.sleep_ns > 0 ? op.sleep_ns : 64);
                }
                // after an expired wait: +0 into the cells still owed, so the compute warps drain
                for (; c < end; ++c) {
                    T* cell = cells + (c & (kGridRing - 1)) * stride;
                    st_slot_if(cell, T(0), is_sentinel(ld_slot(cell)));
                }
            }
        }
        __syncthreads();
    }
}

// Grid layout values straight from the matrix's CSR (no per-element index
// arrays): element (unit, step, slot, lane) is row r's entry of the slot's
// direction, found in A's row, with the sources and pivot rows of the
// preconditioner's factor row lists -- ILU(0): the entry (r, c) of the
// factorized values, no pivot; IC(0): L's (r, c) is a_cr times the inverse
// pivot of c, U's (r, c) is a_rc times the inverse pivot of r -- and the
// multiplier slot the inverse pivot of r (1 for a unit diagonal); padding +0.
// The same values and roundings as k_fill_grid and the chunked layout's fill.
// lmul: ILU(0) factorized on the grid (A's values in `src`): L's entries are
// a_rc times the inverse pivot of c, as k_ilu0_factor forms them.
struct GridFillGeom {
    int n, nx, ny, nz, ns, perm, skew, nsteps, nsp, njb;
};
constexpr int kGridFillILU = 0, kGridFillIC = 1;
__global__ void k_fill_grid_csr(long long nent, GridFillGeom g, int lower, int kind, int unit, int lmul,
                                const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ src,
                                const double* __restrict__ inv_dia, void* val, int f32)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nent;
         e += (long long)gridDim.x * blockDim.x) {
        const int lane = int(e & 31);
        long long rest = e >> 5;
        const int q = int(rest % (g.ns + 1));
        rest /= (g.ns + 1);
        const int s = int(rest % g.nsp);
        const long long u = rest / g.nsp;
        const int ju = int(u % g.njb), k = int(u / g.njb);
        const int i = g.skew ? s - lane : s, j = 32 * ju + lane;
        const long long rpr = i + (long long)g.nx * (j + (long long)g.ny * k);
        double v = 0.0;
        if (s < g.nsteps && i >= 0 && i < g.nx && j < g.ny && rpr < g.n) {
            const int r = lower ? int(rpr) : int(g.n - 1 - rpr);
            if (q == g.ns) {
                v = unit ? 1.0 : inv_dia[r];
            } else {
                const int d = (g.perm >> (2 * q)) & 3;
                const bool present = d == 0 ? i > 0 : d == 1 ? j > 0 : k > 0;
                if (present) {
                    const long long off = d == 0 ? 1 : d == 1 ? g.nx : (long long)g.nx * g.ny;
                    const int c = int(lower ? r - off : r + off);
                    const bool tr = kind == kGridFillIC && lower;   // IC(0)'s L holds the transposed upper entries
                    const int row = tr ? c : r, col = tr ? r : c;
                    int pos = -1;
                    for (int f = rp[row]; f < rp[row + 1]; ++f)
                        if (ci[f] == col) pos = f;
                    if (pos >= 0) {
                        v = src[pos];
                        if (kind == kGridFillIC) v = v * inv_dia[lower ? c : r];
                        else if (lmul && lower) v = v * inv_dia[c];   // ILU(0)'s l_rc = a_rc / u_cc, as the factorization rounds it
                    }
                }
            }
        }
        if (f32) static_cast<float*>(val)[e] = float(v);
        else static_cast<double*>(val)[e] = v;
    }
}

// Layout of a grid factorization (L's geometry, farthest neighbour first):
// per step and lane the row's entries toward its earlier neighbours a_ik
// (ILU(0) only), those neighbours' entries in the row's column a_ki, then
// a_ii; +0 where the row has no such neighbour.  FP64 values of A.
__global__ void k_fill_grid_factor(long long nent, GridFillGeom g, int kind, const int* __restrict__ rp,
                                   const int* __restrict__ ci, const double* __restrict__ a, double* __restrict__ out)
{
    const int slots = kind == kGridILU0 ? 2 * g.ns + 1 : g.ns + 1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nent;
         e += (long long)gridDim.x * blockDim.x) {
        const int lane = int(e & 31);
        long long rest = e >> 5;
        const int q = int(rest % slots);
        rest /= slots;
        const int s = int(rest % g.nsp);
        const long long u = rest / g.nsp;
        const int ju = int(u % g.njb), k = int(u / g.njb);
        const int i = g.skew ? s - lane : s, j = 32 * ju + lane;
        const long long r = i + (long long)g.nx * (j + (long long)g.ny * k);
        double v = 0.0;
        if (s < g.nsteps && i >= 0 && i < g.nx && j < g.ny && r < g.n) {
            int row = int(r), col = int(r);   // q == slots - 1: the diagonal
            bool present = true;
            if (q < slots - 1) {
                const int qd = q < g.ns ? q : q - g.ns;
                const int d = (g.perm >> (2 * qd)) & 3;
                present = d == 0 ? i > 0 : d == 1 ? j > 0 : k > 0;
                const long long off = d == 0 ? 1 : d == 1 ? g.nx : (long long)g.nx * g.ny;
                const int nb = int(r - off);
                const bool toward = kind == kGridILU0 && q < g.ns;   // a_ik (row r, column nb); else a_ki
                row = toward ? int(r) : nb;
                col = toward ? nb : int(r);
            }
            if (present)
                for (int f = rp[row]; f < rp[row + 1]; ++f)
                    if (ci[f] == col) v = a[f];
        }
        out[e] = v;
    }
}

// Flat-layout values copied from the grid layout (a factor built with the
// grid layout only, when a flat sweep, a factor download or the ILU(0)
// adjoint needs its flat layout): flat position p is row row_of[p], its
// entry k (column ci[k]) the grid element of that row and direction.
__global__ void k_flat_from_grid(int npos, const int* __restrict__ row_of, const int* __restrict__ rp,
                                 const int* __restrict__ ci, GridFillGeom g, int lower,
                                 const unsigned char* __restrict__ gval, unsigned char* __restrict__ val, int ssz)
{
    int rank[3] = {-1, -1, -1};
    for (int q = 0; q < g.ns; ++q) rank[(g.perm >> (2 * q)) & 3] = q;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npos; p += gridDim.x * blockDim.x) {
        const int r = row_of[p];
        if (r < 0) continue;
        const long long rpr = lower ? r : (long long)g.n - 1 - r;
        const int i = int(rpr % g.nx), j = int((rpr / g.nx) % g.ny), k = int(rpr / ((long long)g.nx * g.ny));
        const long long u = (long long)k * g.njb + j / 32;
        const int lane = j & 31, s = g.skew ? i + lane : i;
        for (int e = rp[p]; e < rp[p + 1]; ++e) {
            const long long off = lower ? (long long)r - ci[e] : (long long)ci[e] - r;
            const int d = off == 1 ? 0 : off == g.nx ? 1 : 2;
            const long long src = ((u * g.nsp + s) * (g.ns + 1) + rank[d]) * 32 + lane;
            if (ssz == 8) reinterpret_cast<double*>(val)[e] = reinterpret_cast<const double*>(gval)[src];
            else reinterpret_cast<float*>(val)[e] = reinterpret_cast<const float*>(gval)[src];
        }
    }
}

// Grid layout values: per element a value source (>= 0, times the inverse
// pivot named by gmul when >= 0), -2 for a row's multiplier (the inverse
// pivot of row gmul, 1 for a unit diagonal), -1 for padding (+0).
__global__ void k_fill_grid(long long nent, const int* __restrict__ gsrc, const int* __restrict__ gmul,
                            const double* __restrict__ src, const double* __restrict__ inv_dia, int unit, void* val,
                            int f32)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nent;
         e += (long long)gridDim.x * blockDim.x) {
        const int c = gsrc[e], m = gmul[e];
        double v = 0.0;
        if (c >= 0) {
            v = src[c];
            if (m >= 0) v = v * inv_dia[m];
        } else if (c == -2) {
            v = (unit || m < 0) ? 1.0 : inv_dia[m];
        }
        if (f32) static_cast<float*>(val)[e] = float(v);
        else static_cast<double*>(val)[e] = v;
    }
}

}  // namespace mtlg
