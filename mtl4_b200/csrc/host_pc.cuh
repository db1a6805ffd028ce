// Host side: preconditioner structure (factor patterns, dependency levels,
// level-ordered layout) and the device factorization launches.
#pragma once
#include "host_core.cuh"

namespace mtlg {

// Off-diagonal entries of a triangular factor in natural row order, each with
// the source of its value (index into a value array) and the row whose
// inverse pivot multiplies it (-1: none).
struct RowLists {
    std::vector<int> rp;   // n + 1
    std::vector<int> col, src, mul;
};

// Level-ordered, warp-padded triangular factor.
struct TriDev {
    int n = 0, npad = 0, nnz = 0, nlev = 0;
    bool lower = true;
    hvec<int> h_row_of;                // npad
    hvec<int> h_rp;                    // npad + 1
    hvec<int> h_ci, h_src, h_mul;
    std::vector<int> lev_task_begin;   // nlev + 1, in units of tasks
    DBuf<int> row_of, rp, ci, src, mul;
    DBuf<unsigned char> val, dia;      // storage type S
    DBuf<SweepTask> tasks;             // single-system task list (sys = 0)
    // chunked layout (k_sweep_chunk); nch == 0: not built (flat sweeps only)
    int chunk_rows = 0, nch = 0, nseg = 0, nwaves = 0, cnpos = 0, cnent = 0;
    int kmax = 0;       // entries per row, at most
    int threads = 0;    // rows per wave, at most (the launch's CTA size)
    int seg_rows = 0;   // rows per segment, at most
    int seg_ents = 0;   // entries per segment, at most
    int max_slots = 0;  // receive slots of a chunk, at most
    DBuf<int> cseg, cxr, cext, crow, ccol, csrc, cmul;
    DBuf<int2> cquad;
    DBuf<int> cqpull, cpush;
    DBuf<SegRec> segs;
    DBuf<unsigned> wv;
    DBuf<unsigned char> cval, cdia;    // storage type S
    DBuf<unsigned char> ypos[2];       // results by position for FP64 [0] / FP32 [1] vectors (all sentinel between sweeps)
    // flat layout entries (h_rp, h_ci, h_src, h_mul; rp, ci, src, mul, val,
    // dia on the device): built at set-up only when the factor has no
    // chunked layout, else on first need (ensure_flat) from the kept row lists
    bool flat_entries = false;
    RowLists F;
    // grid layout (k_sweep_grid; gnx == 0: the pattern is not a grid
    // stencil): geometry as in TriFactor, per element the value source and
    // pivot row (kept until the values are filled), the values (type S)
    int gnx = 0, gny = 0, gnz = 0, gns = 0, gperm = 0, gdirs = 0, gskew = 0, gnsteps = 0, gnsp = 0, gnjb = 0;
    long long gnent = 0;
    bool grid_indices = true;   // false: values filled straight from the matrix's CSR (no gsrc / gmul)
    DBuf<int> gsrc, gmul;
    DBuf<unsigned char> gval;
};

constexpr int kChunkMaxEntries = 16;   // longer factor rows: flat sweeps only

inline int round4(int v) { return (v + 3) & ~3; }
inline int entries_bucket(int k) { return k <= 2 ? 2 : k <= 3 ? 3 : k <= 4 ? 4 : k <= 8 ? 8 : 16; }

// Wave cap (rows) of a factor whose rows hold up to kb entries (bucket),
// stored in ssz-byte values: the largest shape built for it.
inline int chunk_wave_cap(int kb, int ssz)
{
    return ssz == 8 && kb > 8 ? 128 : 256;
}

// Chunked layout of a triangular factor: chunks of B contiguous rows in
// processing order; inside a chunk the rows are grouped by dependency level
// (waves, split to at most `threads` rows), a wave's rows in the order of
// the flat layout; consecutive waves form segments of at most seg_rows rows
// and seg_ents entries; entries wave-major as described at TriFactor.  The
// columns are coded as cells of the chunk's shared vector: a row of the
// chunk as its index in the chunk, B (a cell holding +0, with value 0) past a
// row's entries, B + kSlotBase + slot for entries whose row lies in an
// earlier chunk, up to B slots per chunk (in wave order; that row's position
// listed in cext, where the chunk's receiver warps fetch it from the
// position-ordered results); any further ones as -(position + 2), polled
// directly, their wave flagged with kWaveOverflow.  Waves start 4-aligned in
// positions, and in slots when they read several earlier-chunk rows.
inline int build_chunks(mtlg_ctx* c, const RowLists& F, const std::vector<int>& lev, int n, bool lower, int B,
                        int ssz, TriDev& T)
{
    T.nch = 0;
    T.max_slots = 0;
    int kmax = 0;
    for (int i = 0; i < n; ++i) kmax = std::max(kmax, F.rp[i + 1] - F.rp[i]);
    if (n == 0 || B <= 0 || kmax > kChunkMaxEntries) return MTLG_OK;
    B = std::max(32, (B + 31) / 32 * 32);
    const int nch = (n + B - 1) / B;
    // rows of each chunk in (level, flat order): a counting sort by level per
    // chunk (rows visited ascending for L, descending for U, so rows of one
    // level keep the flat layout's order), and the largest wave
    TracePhases ph;
    ph.next(9153, "pc.chunk_order");
    std::vector<int> order(size_t(n), 0);
    std::vector<int> cbeg(nch + 1, 0);
    for (int p = 0; p < nch; ++p) {
        const int ch = lower ? p : nch - 1 - p;
        cbeg[p + 1] = cbeg[p] + (std::min(n, ch * B + B) - ch * B);
    }
    std::vector<int> maxw_p(nch, 0);
    parallel_for(nch, [&](int p) {
        const int ch = lower ? p : nch - 1 - p;
        const int r0 = ch * B, r1 = std::min(n, r0 + B);
        int lo = lev[r0], hi = lev[r0];
        for (int r = r0; r < r1; ++r) {
            lo = std::min(lo, lev[r]);
            hi = std::max(hi, lev[r]);
        }
        std::vector<int> cnt(size_t(hi - lo + 2), 0);
        for (int r = r0; r < r1; ++r) cnt[size_t(lev[r] - lo + 1)]++;
        int mw = 0;
        for (size_t k = 1; k < cnt.size(); ++k) {
            mw = std::max(mw, cnt[k]);
            cnt[k] += cnt[k - 1];
        }
        int* out = order.data() + cbeg[p];
        if (lower)
            for (int r = r0; r < r1; ++r) out[cnt[size_t(lev[r] - lo)]++] = r;
        else
            for (int r = r1 - 1; r >= r0; --r) out[cnt[size_t(lev[r] - lo)]++] = r;
        maxw_p[p] = mw;
    });
    int maxw = 0;
    for (int p = 0; p < nch; ++p) maxw = std::max(maxw, maxw_p[p]);
    const int KB = entries_bucket(kmax);
    const int NT = std::min(chunk_wave_cap(KB, ssz), std::max(32, (maxw + 31) / 32 * 32));
    // segment capacity: a multiple of 32 rows, so every staged array (and
    // every staging buffer) starts 16-byte aligned in shared memory
    const int SR = std::max(NT, (1024 / KB + 31) / 32 * 32);
    const int SE = SR * KB;

    // Each chunk's layout is built on its own (host threads), positions and
    // entries counted from the chunk's start; rows of earlier chunks are
    // kept as row ids (cext) or -(row + 2) (overflow codes) until every
    // chunk's position is known.  A chunk's arrays start 4-aligned in the
    // concatenation (its first segment opens 4-aligned).
    ph.next(9154, "pc.chunk_waves");
    struct ChunkLocal {
        std::vector<unsigned> wv;
        std::vector<int> crow, ccol, csrc, cmul, cext;
        std::vector<SegRec> segs;
        int nslot = 0;
    };
    std::vector<ChunkLocal> loc(static_cast<size_t>(nch));
    std::vector<int> lpos(size_t(n), -1);   // position of each row inside its chunk
    parallel_for(nch, [&](int p) {
        ChunkLocal& L = loc[size_t(p)];
        std::vector<unsigned>& wv = L.wv;
        std::vector<int>&crow = L.crow, &ccol = L.ccol, &csrc = L.csrc, &cmul = L.cmul, &cext = L.cext;
        std::vector<SegRec>& segs = L.segs;
        SegRec cur{};
        bool open = false;
        auto close_seg = [&]() {
            if (!open) return;
            cur.np = int(crow.size()) - cur.p0;
            cur.ne = int(ccol.size()) - cur.e0;
            cur.nw = int(wv.size()) - cur.w0;
            segs.push_back(cur);
            open = false;
        };
        auto open_seg = [&]() {
            wv.resize(round4(int(wv.size())), 0u);
            crow.resize(round4(int(crow.size())), -1);
            const int e = round4(int(ccol.size()));
            ccol.resize(e, -1);
            csrc.resize(e, 0);
            cmul.resize(e, -1);
            cur = SegRec{int(wv.size()), 0, int(crow.size()), 0, int(ccol.size()), 0, 0, 0};
            open = true;
        };
        const int ch = lower ? p : nch - 1 - p;
        const int r0 = ch * B, r1 = std::min(n, r0 + B);
        int nslot = 0;
        for (int q = cbeg[p]; q < cbeg[p + 1];) {
            int qe = q + 1;
            while (qe < cbeg[p + 1] && qe - q < NT && lev[order[qe]] == lev[order[q]]) ++qe;
            const int nw = qe - q;
            int K = 0;
            for (int j = q; j < qe; ++j) K = std::max(K, F.rp[order[j] + 1] - F.rp[order[j]]);
            // a wave's positions start 4-aligned
            if (open && (round4(int(crow.size())) - cur.p0 + nw > SR || int(ccol.size()) - cur.e0 + K * nw > SE))
                close_seg();
            if (!open) open_seg();
            crow.resize(round4(int(crow.size())), -1);
            // a wave with several earlier-chunk reads starts its receive slots
            // 4-aligned too, so runs of consecutive positions move 4 at a time
            int next = 0;
            for (int j = q; j < qe; ++j)
                for (int e = F.rp[order[j]]; e < F.rp[order[j] + 1]; ++e) next += (F.col[e] < r0 || F.col[e] >= r1);
            if (next >= 4 && round4(nslot) < B)
                while (nslot % 4) {
                    cext.push_back(-1);
                    ++nslot;
                }
            const size_t wvi = wv.size();
            wv.push_back(unsigned(nw) | (unsigned(K) << 16));
            bool ovf = false;
            const size_t ent = ccol.size();
            for (int j = q; j < qe; ++j) {
                lpos[order[j]] = int(crow.size());
                crow.push_back(order[j]);
            }
            ccol.resize(ent + size_t(K) * nw, B);     // padding: the zero cell, value 0
            csrc.resize(ent + size_t(K) * nw, -1);
            cmul.resize(ent + size_t(K) * nw, -1);
            for (int t = 0; t < nw; ++t) {
                const int r = order[q + t];
                for (int k = 0; k < F.rp[r + 1] - F.rp[r]; ++k) {
                    const size_t e = ent + size_t(k) * nw + t;
                    const int col = F.col[F.rp[r] + k];
                    int code;
                    if (col >= r0 && col < r1) {
                        code = col - r0;                 // row of this chunk
                    } else if (nslot < B) {
                        cext.push_back(col);             // earlier chunk: receive slot (row id for now)
                        code = B + kSlotBase + nslot;
                        ++nslot;
                    } else {
                        code = -(col + 2);               // earlier chunk beyond the slots (row id for now)
                        ovf = true;
                    }
                    ccol[e] = code;
                    csrc[e] = F.src[F.rp[r] + k];
                    cmul[e] = F.mul[F.rp[r] + k];
                }
            }
            if (ovf) wv[wvi] |= kWaveOverflow;
            q = qe;
        }
        close_seg();
        while (cext.size() % 4) cext.push_back(-1);
        L.nslot = round4(nslot);
    });
    // concatenation: chunk bases, then the arrays with row ids turned into
    // positions (every earlier chunk's position is known now)
    ph.next(9157, "pc.chunk_concat");
    std::vector<size_t> bw(nch), bp(nch), be(nch), bx(nch), bs(nch);
    size_t sw = 0, sp = 0, se = 0, sx = 0, ss = 0;
    std::vector<int> cpbeg(size_t(nch) + 1, 0);   // first position of each chunk (and the end)
    for (int p = 0; p < nch; ++p) {
        const ChunkLocal& L = loc[size_t(p)];
        sw = size_t(round4(int(sw)));
        sp = size_t(round4(int(sp)));
        se = size_t(round4(int(se)));
        bw[p] = sw; bp[p] = sp; be[p] = se; bx[p] = sx; bs[p] = ss;
        cpbeg[p] = int(sp);
        sw += L.wv.size(); sp += L.crow.size(); se += L.ccol.size(); sx += L.cext.size(); ss += L.segs.size();
        T.max_slots = std::max(T.max_slots, L.nslot);
    }
    cpbeg[nch] = int(sp);
    std::vector<int> cseg(size_t(nch) + 1, 0), cxr(size_t(nch) + 1, 0);
    for (int p = 0; p < nch; ++p) {
        cseg[p + 1] = int(bs[p] + loc[size_t(p)].segs.size());
        cxr[p + 1] = int(bx[p] + loc[size_t(p)].cext.size());
    }
    // capacities include the 16-byte tails added at the end (no
    // reallocation); every element is written by the parallel copy below
    // (chunk data, then the alignment gap up to the next chunk's base)
    const size_t tw = size_t(round4(int(sw))) + 4, tp = size_t(round4(int(sp))) + 4;
    const size_t te = size_t(round4(int(se))) + 4, tx = sx + 4;
    hvec<unsigned> wv;
    hvec<int> crow, ccol, csrc, cmul, cext;
    wv.reserve(tw);
    wv.resize(sw);
    crow.reserve(tp);
    crow.resize(sp);
    for (hvec<int>* v : {&ccol, &csrc, &cmul}) {
        v->reserve(te);
        v->resize(se);
    }
    cext.reserve(tx);
    cext.resize(sx);
    std::vector<SegRec> segs(ss);
    auto pos_of = [&](int row) {
        const int ch = row / B;
        const int p = lower ? ch : nch - 1 - ch;
        return int(bp[p]) + lpos[row];
    };
    parallel_for(nch, [&](int p) {
        const ChunkLocal& L = loc[size_t(p)];
        const bool last = p + 1 == nch;
        std::copy(L.wv.begin(), L.wv.end(), wv.begin() + bw[p]);
        std::fill(wv.begin() + bw[p] + L.wv.size(), last ? wv.end() : wv.begin() + bw[p + 1], 0u);
        std::copy(L.crow.begin(), L.crow.end(), crow.begin() + bp[p]);
        std::fill(crow.begin() + bp[p] + L.crow.size(), last ? crow.end() : crow.begin() + bp[p + 1], -1);
        for (size_t k = 0; k < L.ccol.size(); ++k) {
            const int v = L.ccol[k];
            ccol[be[p] + k] = v <= -2 ? -(pos_of(-v - 2) + 2) : v;
        }
        std::copy(L.csrc.begin(), L.csrc.end(), csrc.begin() + be[p]);
        std::copy(L.cmul.begin(), L.cmul.end(), cmul.begin() + be[p]);
        const size_t ge = last ? ccol.size() : be[p + 1];
        std::fill(ccol.begin() + be[p] + L.ccol.size(), ccol.begin() + ge, -1);
        std::fill(csrc.begin() + be[p] + L.ccol.size(), csrc.begin() + ge, 0);
        std::fill(cmul.begin() + be[p] + L.ccol.size(), cmul.begin() + ge, -1);
        for (size_t k = 0; k < L.cext.size(); ++k) cext[bx[p] + k] = L.cext[k] >= 0 ? pos_of(L.cext[k]) : -1;
        for (size_t k = 0; k < L.segs.size(); ++k) {
            SegRec g = L.segs[k];
            g.w0 += int(bw[p]);
            g.p0 += int(bp[p]);
            g.e0 += int(be[p]);
            segs[bs[p] + k] = g;
        }
    });
    loc.clear();
    ph.next(9155, "pc.chunk_pushes");
    // pushes: a row of chunk p - 1 fills the first slot of chunk p that reads
    // it (when the two chunks run in neighbouring CTAs of a cluster); the
    // receivers fetch the other slots
    // (chunk p writes only positions of chunk p - 1: chunks run in parallel)
    std::vector<int> cpush;
    cpush.reserve(tp);
    cpush.assign(crow.size(), -1);
    std::vector<char> pushed(cext.size(), 0);
    parallel_for(nch - 1, [&](int pm) {
        const int p = pm + 1;
        for (int e = cxr[p]; e < cxr[p + 1]; ++e) {
            const int x = cext[e];
            if (x < cpbeg[p - 1] || x >= cpbeg[p] || cpush[x] >= 0) continue;
            cpush[x] = e - cxr[p];
            pushed[e] = 1;
        }
    });
    const int nq = int(cext.size() / 4);
    constexpr int kQuadBlock = 65536;
    std::vector<int> cqpull(size_t(nq) + 1, 0);
    // receive quads (slots 4q .. 4q+3): {first position, mask of used slots};
    // first position -1 where the used slots are not four consecutive
    // positions starting 4-aligned (fetched one by one)
    std::vector<int2> cquad(size_t(nq) + 1, make_int2(-1, 0));
    parallel_for((nq + kQuadBlock - 1) / kQuadBlock, [&](int blk) {
    for (int q = blk * kQuadBlock; q < std::min(nq, (blk + 1) * kQuadBlock); ++q) {
        for (int j = 0; j < 4; ++j)
            if (cext[4 * q + j] >= 0 && !pushed[4 * q + j]) cqpull[q] |= 1 << j;
        int mask = 0, p = -2;
        bool vec = true;
        for (int j = 0; j < 4; ++j) {
            const int x = cext[4 * q + j];
            if (x < 0) continue;
            mask |= 1 << j;
            if (p == -2) p = x - j;
            if (x != p + j) vec = false;
        }
        if (p < 0 || p % 4) vec = false;
        cquad[q] = make_int2(vec && mask ? p : -1, mask);
    }
    });
    ph.next(9158, "pc.chunk_tails");
    // tails: a staged copy rounds each array's segment up to 16 bytes
    wv.resize(round4(int(wv.size())) + 4, 0u);
    crow.resize(round4(int(crow.size())) + 4, -1);
    cpush.resize(crow.size(), -1);
    cext.resize(cext.size() + 4, 0);
    const int e = round4(int(ccol.size())) + 4;
    ccol.resize(e, -1);
    csrc.resize(e, 0);
    cmul.resize(e, -1);
    T.chunk_rows = B;
    T.nch = nch;
    T.nseg = int(segs.size());
    T.nwaves = int(wv.size());
    T.cnpos = int(crow.size());
    T.cnent = int(ccol.size());
    T.kmax = kmax;
    T.threads = NT;
    T.seg_rows = SR;
    T.seg_ents = SE;
    ph.next(9156, "pc.chunk_upload");
    MTLG_TRY(T.cseg.upload(c, cseg.data(), cseg.size()));
    MTLG_TRY(T.cxr.upload(c, cxr.data(), cxr.size()));
    MTLG_TRY(T.cext.upload(c, cext.data(), cext.size()));
    MTLG_TRY(T.cquad.upload(c, cquad.data(), cquad.size()));
    MTLG_TRY(T.cqpull.upload(c, cqpull.data(), cqpull.size()));
    MTLG_TRY(T.cpush.upload(c, cpush.data(), cpush.size()));
    MTLG_TRY(T.segs.upload(c, segs.data(), segs.size()));
    MTLG_TRY(T.wv.upload(c, wv.data(), wv.size()));
    MTLG_TRY(T.crow.upload(c, crow.data(), crow.size()));
    MTLG_TRY(T.ccol.upload(c, ccol.data(), ccol.size()));
    MTLG_TRY(T.csrc.upload(c, csrc.data(), csrc.size()));
    MTLG_TRY(T.cmul.upload(c, cmul.data(), cmul.size()));
    return MTLG_OK;
}

// ------------------------------------------------------------ chunked sweeps
constexpr int kChunkSmemMax = 225 * 1024;   // dynamic shared memory of one chunk CTA, at most

// Launch shape of the chunked sweeps of one side (the L or the U factors)
// of a set of systems.
struct ChunkSide {
    int nt = 0, km = 0;          // wave cap (rows), entries per row
    int rows = 0;                // rows of the largest chunk
    int slots = 0;               // receive slots of the largest chunk
    int seg_rows = 0, seg_ents = 0;
    int smem = 0;                // dynamic shared memory per CTA
    int resident = 1;            // CTAs resident at once (whole clusters)
    int cl = 1;                  // CTAs per cluster
    int vec_bytes = 0;
    int cells = 0;               // shared cells of the largest chunk (rows, +0 cell, slots)
    void add(const TriDev& T)
    {
        nt = std::max(nt, T.threads);
        km = std::max(km, T.kmax);
        rows = std::max(rows, T.chunk_rows);
        slots = std::max(slots, T.max_slots);
        cells = std::max(cells, T.chunk_rows + kSlotBase + T.max_slots);
        seg_rows = std::max(seg_rows, T.seg_rows);
        seg_ents = std::max(seg_ents, T.seg_ents);
    }
    int threads() const { return nt <= 32 ? 32 : nt <= 64 ? 64 : nt <= 128 ? 128 : 256; }
    int entries() const { return entries_bucket(km); }
};

// Launch plan of the chunked sweeps of a set of factors (computed outside
// any stream capture: it queries the occupancy): a shape per side and the
// task lists (ntl / ntu groups of cl GroupTask entries, one per CTA of a
// cluster).
struct ChunkPlan {
    bool ok = false;
    ChunkSide side[2];           // L [0], U [1]
    DBuf<GroupTask> tl, tu;      // grid sweeps: tiles {sys, first unit along y, first plane, jw}
    int ntl = 0, ntu = 0;
    bool grid = false;           // k_sweep_grid: every factor of the set has a grid layout
    int gnw = 0, gsmem = 0, gresident = 0;   // compute warps, dynamic shared memory, CTAs resident at once
    int gsteps = 0;              // steps per unit (the largest factor's)
};

// Context settings a sweep plan depends on (a plan is remade when they change).
inline int plan_setting(const mtlg_ctx* c)
{
    return c->sweep_kernel | (c->sweep_cluster << 4) | (c->grid_sweep << 9) | (c->grid_warps << 10);
}

// Kernel shape of a wave cap of NT rows and KM entries per row: up to four
// compute warps, two rows per thread beyond 128 rows.
template <typename T, typename S, int NT, int KM>
struct ChunkShape {
    static constexpr int CW = NT >= 128 ? 4 : NT / 32;
    static constexpr int RPT = NT / (32 * CW);
    static constexpr int THREADS = 32 * (CW + kChunkExtraWarps);
    static int init()
    {
        MTLG_CUDA(cudaFuncSetAttribute(k_sweep_chunk<T, S, CW, RPT, KM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kChunkSmemMax));
        // clusters of 16 CTAs (beyond the portable 8) where the device has them
        if (cudaFuncSetAttribute(k_sweep_chunk<T, S, CW, RPT, KM>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess)
            cudaGetLastError();
        return MTLG_OK;
    }
    // CTAs resident at once, in whole clusters of cl CTAs (0: does not fit)
    static int resident(mtlg_ctx* c, int smem, int cl)
    {
        if (cl == 1) {
            int n = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sweep_chunk<T, S, CW, RPT, KM>, THREADS,
                                                              size_t(smem)) != cudaSuccess) {
                cudaGetLastError();
                return 0;
            }
            return n * c->sm_count;
        }
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = unsigned(cl);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(unsigned(cl * c->sm_count));
        cfg.blockDim = dim3(THREADS);
        cfg.dynamicSmemBytes = size_t(smem);
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, (const void*)k_sweep_chunk<T, S, CW, RPT, KM>, &cfg) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        return n * cl;
    }
    static int launch(mtlg_ctx* c, cudaStream_t st, const SetView& sv, const ChunkSweepOp& op, const ChunkSide& pl)
    {
        const int grid = std::max(1, std::min(op.ntasks, pl.resident / pl.cl)) * pl.cl;
        if (pl.cl == 1) {
            k_sweep_chunk<T, S, CW, RPT, KM><<<grid, THREADS, pl.smem, st>>>(sv, op);
            c->launches++;
            MTLG_CUDA(cudaGetLastError());
            return MTLG_OK;
        }
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = unsigned(pl.cl);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(unsigned(grid));
        cfg.blockDim = dim3(THREADS);
        cfg.dynamicSmemBytes = size_t(pl.smem);
        cfg.stream = st;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        MTLG_CUDA(cudaLaunchKernelEx(&cfg, k_sweep_chunk<T, S, CW, RPT, KM>, sv, op));
        c->launches++;
        return MTLG_OK;
    }
};

// The shapes built, by stored type: with FP64 values, rows of 16 entries
// stay at one row per thread (the rows of a wave, the next wave's and their
// reads stay in registers).
#define MTLG_CHUNK_SHAPES_F32(M, T, S) \
    M(T, S, 32, 2) M(T, S, 32, 3) M(T, S, 32, 4) M(T, S, 32, 8) M(T, S, 32, 16) \
    M(T, S, 64, 2) M(T, S, 64, 3) M(T, S, 64, 4) M(T, S, 64, 8) M(T, S, 64, 16) \
    M(T, S, 128, 2) M(T, S, 128, 3) M(T, S, 128, 4) M(T, S, 128, 8) M(T, S, 128, 16) \
    M(T, S, 256, 2) M(T, S, 256, 3) M(T, S, 256, 4) M(T, S, 256, 8) M(T, S, 256, 16)
#define MTLG_CHUNK_SHAPES_F64(M, T, S) \
    M(T, S, 32, 2) M(T, S, 32, 3) M(T, S, 32, 4) M(T, S, 32, 8) M(T, S, 32, 16) \
    M(T, S, 64, 2) M(T, S, 64, 3) M(T, S, 64, 4) M(T, S, 64, 8) M(T, S, 64, 16) \
    M(T, S, 128, 2) M(T, S, 128, 3) M(T, S, 128, 4) M(T, S, 128, 8) M(T, S, 128, 16) \
    M(T, S, 256, 2) M(T, S, 256, 3) M(T, S, 256, 4) M(T, S, 256, 8)

inline int init_chunk_shapes()
{
#define MTLG_CHUNK_INIT(T, S, NT, KM) MTLG_TRY((ChunkShape<T, S, NT, KM>::init()));
    MTLG_CHUNK_SHAPES_F64(MTLG_CHUNK_INIT, double, double)
    MTLG_CHUNK_SHAPES_F32(MTLG_CHUNK_INIT, double, float)
    MTLG_CHUNK_SHAPES_F32(MTLG_CHUNK_INIT, float, float)
    MTLG_CHUNK_SHAPES_F64(MTLG_CHUNK_INIT, float, double)
#undef MTLG_CHUNK_INIT
    return MTLG_OK;
}

// Calls fn(ChunkShape<T, S, NT, KM>()) for the built shape of (nt, km);
// false if none is built.
template <typename T, typename S, typename Fn>
inline bool with_chunk_shape(int nt, int km, Fn&& fn)
{
    bool found = false;
#define MTLG_CHUNK_WITH(TT, SS, NT, KM) \
    if (!found && nt == NT && km == KM) { fn(ChunkShape<TT, SS, NT, KM>()); found = true; }
    if constexpr (sizeof(S) == 4) {
        MTLG_CHUNK_SHAPES_F32(MTLG_CHUNK_WITH, T, S)
    } else {
        MTLG_CHUNK_SHAPES_F64(MTLG_CHUNK_WITH, T, S)
    }
#undef MTLG_CHUNK_WITH
    return found;
}

// Groups of chunks, one per cluster of cl CTAs (cl GroupTask entries each):
// each factor's chunks (nch[s] of system s, in processing order) in runs of
// cl consecutive chunks, run by run (all systems' first runs, then their
// second runs, ...), runs packed into groups while they fit; the chunks of a
// run sit in neighbouring CTAs and push to each other.  Returns the number
// of groups.
inline int chunk_groups(const std::vector<int>& nch, int cl, std::vector<GroupTask>& g)
{
    g.clear();
    int ng = 0, used = cl, maxch = 0;
    for (int n : nch) maxch = std::max(maxch, n);
    for (int a = 0; a < maxch; a += cl)
        for (size_t s = 0; s < nch.size(); ++s) {
            const int len = std::min(cl, nch[s] - a);
            if (len <= 0) continue;
            if (used + len > cl) {
                // CTAs without a chunk in the group read the descriptors of
                // the group's first chunk (a live system) and do nothing else
                g.resize(g.size() + size_t(cl), GroupTask{int(s), a, 0, 0});
                ++ng;
                used = 0;
            }
            GroupTask* t = g.data() + size_t(ng - 1) * size_t(cl) + used;
            for (int i = 0; i < len; ++i)
                t[i] = GroupTask{int(s), a + i,
                                 kGroupActive | (i + 1 < len ? kGroupPushNext : 0) | (i > 0 ? kGroupPushedIn : 0), 0};
            used += len;
        }
    return ng;
}

// Shape and task lists of a set of systems' factors (f[s]: the system's L
// and U, or nulls for an unused slot), in groups (chunk_groups) of the
// side's cluster size.  Not ok (flat sweeps) when a side's shape is not built
// or its shared memory does not fit.
// Grid-sweep launch shapes: NW compute warps (4 or 8) and two receiver warps.
template <typename T, typename S, int NW>
struct GridShape {
    static constexpr int THREADS = 32 * (NW + kGridRecvWarps);
    static int init()
    {
        if (grid_smem_bytes<T, S>(NW) > kChunkSmemMax) return MTLG_OK;   // not built for this type pair
        MTLG_CUDA(cudaFuncSetAttribute(k_sweep_grid<T, S, NW, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       grid_smem_bytes<T, S>(NW)));
        MTLG_CUDA(cudaFuncSetAttribute(k_sweep_grid<T, S, NW, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       grid_smem_bytes<T, S>(NW)));
        return MTLG_OK;
    }
    static int resident(mtlg_ctx* c)
    {
        int n = 0, m = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sweep_grid<T, S, NW, false>, THREADS,
                                                          size_t(grid_smem_bytes<T, S>(NW))) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k_sweep_grid<T, S, NW, true>, THREADS,
                                                          size_t(grid_smem_bytes<T, S>(NW))) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        return std::min(n, m) * c->sm_count;
    }
    static int launch(mtlg_ctx* c, cudaStream_t st, const SetView& sv, const ChunkSweepOp& op, int resident)
    {
        const int grid = std::max(1, std::min(op.ntasks, resident));
        if (op.which) k_sweep_grid<T, S, NW, true><<<grid, THREADS, grid_smem_bytes<T, S>(NW), st>>>(sv, op);
        else k_sweep_grid<T, S, NW, false><<<grid, THREADS, grid_smem_bytes<T, S>(NW), st>>>(sv, op);
        c->launches++;
        MTLG_CUDA(cudaGetLastError());
        return MTLG_OK;
    }
};

// Grid factorizations: FP64, ILU(0) pivots with two compute warps (its
// steps carry seven values), IC(0) pivots with four.
constexpr int kGridFactorWarpsILU = 2, kGridFactorWarpsIC = 4;
template <int OPK, int NW>
struct GridFactorShape {
    static constexpr int THREADS = 32 * (NW + kGridRecvWarps);
    static int smem() { return grid_smem_bytes<double, double, OPK>(NW); }
    static int init()
    {
        MTLG_CUDA(cudaFuncSetAttribute(k_sweep_grid<double, double, NW, false, OPK>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem()));
        return MTLG_OK;
    }
    static int resident(mtlg_ctx* c)
    {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sweep_grid<double, double, NW, false, OPK>, THREADS,
                                                          size_t(smem())) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        return n * c->sm_count;
    }
};

inline int init_grid_shapes()
{
    MTLG_TRY((GridFactorShape<kGridILU0, kGridFactorWarpsILU>::init()));
    MTLG_TRY((GridFactorShape<kGridIC0, kGridFactorWarpsIC>::init()));
    MTLG_TRY((GridShape<double, double, 4>::init()));
    MTLG_TRY((GridShape<double, double, 8>::init()));
    MTLG_TRY((GridShape<double, float, 4>::init()));
    MTLG_TRY((GridShape<double, float, 8>::init()));
    MTLG_TRY((GridShape<float, float, 4>::init()));
    MTLG_TRY((GridShape<float, float, 8>::init()));
    MTLG_TRY((GridShape<float, double, 4>::init()));
    MTLG_TRY((GridShape<float, double, 8>::init()));
    return MTLG_OK;
}

template <typename T, typename S, typename Fn>
inline void with_grid_shape(int nw, Fn&& fn)
{
    if (nw == 8) fn(GridShape<T, S, 8>());
    else fn(GridShape<T, S, 4>());
}

// Grid-sweep plan of a set whose factors all have grid layouts: compute
// warps (the context's grid_warps, else 8 where the shared memory fits,
// else 4), and per side the tiles of every system, taken round-robin over
// the systems (a system's tiles plane block by plane block, y-blocks
// ascending inside: every tile a tile reads comes earlier).  Systems with z
// neighbours tile NW planes of one y-block (jw = 1), the others NW y-blocks.
template <typename T, typename S>
inline int plan_grid(mtlg_ctx* c, const std::vector<std::pair<const TriDev*, const TriDev*>>& f, ChunkPlan& pl)
{
    int nw = c->grid_warps > 0 ? c->grid_warps : 8;
    if (grid_smem_bytes<T, S>(nw) > kChunkSmemMax) nw = 4;
    if (grid_smem_bytes<T, S>(nw) > kChunkSmemMax) return MTLG_OK;
    int res = 0;
    with_grid_shape<T, S>(nw, [&](auto shape) { res = decltype(shape)::resident(c); });
    if (res < 1) return MTLG_OK;
    int steps = 0;
    for (int w = 0; w < 2; ++w) {
        std::vector<std::vector<GroupTask>> per(f.size());
        size_t most = 0;
        for (size_t s = 0; s < f.size(); ++s) {
            if (!f[s].first) continue;
            const TriDev& F = w == 0 ? *f[s].first : *f[s].second;
            steps = std::max(steps, F.gnsteps);
            const int jw = (F.gdirs & 4) ? 1 : nw, kw = nw / jw;
            for (int k0 = 0; k0 < F.gnz; k0 += kw)
                for (int j0 = 0; j0 < F.gnjb; j0 += jw) per[s].push_back(GroupTask{int(s), j0, k0, jw});
            most = std::max(most, per[s].size());
        }
        std::vector<GroupTask> g;
        for (size_t a = 0; a < most; ++a)
            for (size_t s = 0; s < f.size(); ++s)
                if (a < per[s].size()) g.push_back(per[s][a]);
        if (w == 0) {
            pl.ntl = int(g.size());
            MTLG_TRY(pl.tl.upload(c, g.data(), std::max<size_t>(1, g.size())));
        } else {
            pl.ntu = int(g.size());
            MTLG_TRY(pl.tu.upload(c, g.data(), std::max<size_t>(1, g.size())));
        }
    }
    pl.grid = true;
    pl.gnw = nw;
    pl.gsmem = grid_smem_bytes<T, S>(nw);
    pl.gresident = res;
    pl.gsteps = steps;
    pl.ok = true;
    return MTLG_OK;
}

template <typename T, typename S>
inline int plan_chunks(mtlg_ctx* c, const std::vector<std::pair<const TriDev*, const TriDev*>>& f, ChunkPlan& pl)
{
    pl.ok = false;
    pl.grid = false;
    pl.side[0] = pl.side[1] = ChunkSide();
    pl.ntl = pl.ntu = 0;
    if (c->grid_sweep && c->sweep_kernel == 0) {
        bool all = false;
        for (const auto& lu : f) {
            if (!lu.first) continue;
            const bool g = lu.first->gnx > 0 && lu.first->gval.p && lu.second->gnx > 0 && lu.second->gval.p;
            if (!g) {
                all = false;
                break;
            }
            all = true;
        }
        if (all) {
            MTLG_TRY((plan_grid<T, S>(c, f, pl)));
            if (pl.ok) return MTLG_OK;
        }
    }
    bool any = false;
    for (const auto& lu : f) {
        if (!lu.first) continue;
        any = true;
        if (lu.first->nch == 0 || lu.second->nch == 0 || !lu.first->cval.p || !lu.second->cval.p) return MTLG_OK;
        pl.side[0].add(*lu.first);
        pl.side[1].add(*lu.second);
    }
    if (!any || c->sweep_kernel != 0) return MTLG_OK;
    for (ChunkSide& sd : pl.side) {
        if (sd.seg_rows % 4 || sd.seg_ents % 4) {
            set_error("chunked sweep: staging capacity %d/%d is not a multiple of 4", sd.seg_rows, sd.seg_ents);
            return MTLG_ERR_NOT_SUPPORTED;
        }
        sd.vec_bytes = int((size_t(sd.cells) * sizeof(T) + 15) / 16 * 16);
        sd.smem = sd.vec_bytes + kStageBufs * stage_bytes<S>(sd.seg_rows, sd.seg_ents);
        if (sd.smem > kChunkSmemMax) return MTLG_OK;
    }
    for (int w = 0; w < 2; ++w) {
        ChunkSide& sd = pl.side[w];
        std::vector<int> nch(f.size(), 0);
        int maxch = 0;
        for (size_t s = 0; s < f.size(); ++s)
            if (f[s].first) {
                nch[s] = w == 0 ? f[s].first->nch : f[s].second->nch;
                maxch = std::max(maxch, nch[s]);
            }
        // clusters when some factor has several chunks: the context's size,
        // else the largest of 16, 8, 4 CTAs whose groups run at once (a
        // cluster takes its next group only when all of its CTAs are done, so
        // queued groups leave CTAs idle), else 2; one CTA per chunk (taken in
        // order as CTAs free up) when clusters do not fit
        int res = 0, ng = 0;
        std::vector<GroupTask> g;
        const int smem = sd.smem;
        const bool forced = c->sweep_cluster > 0;
        const int cands[5] = {forced ? c->sweep_cluster : 16, forced ? 1 : 8, forced ? 1 : 4, forced ? 1 : 2, 1};
        for (int cl : cands) {
            if (cl > 1 && maxch < 2) continue;
            if (!with_chunk_shape<T, S>(sd.threads(), sd.entries(),
                                        [&](auto shape) { res = decltype(shape)::resident(c, smem, cl); }))
                return MTLG_OK;
            sd.cl = cl;
            ng = chunk_groups(nch, cl, g);
            const int rc = res / cl;   // clusters resident at once
            // 16 and 8 only when every group is resident at once, 4 when
            // about all are, 2 always
            const bool fits = cl >= 8 ? ng <= rc : cl == 4 ? 4 * ng <= 5 * rc : true;
            if (cl == 1 || (rc >= 1 && (forced || fits))) break;
        }
        if (res < 1) return MTLG_OK;
        sd.resident = res;
        if (w == 0) {
            pl.ntl = ng;
            MTLG_TRY(pl.tl.upload(c, g.data(), std::max<size_t>(1, g.size())));
        } else {
            pl.ntu = ng;
            MTLG_TRY(pl.tu.upload(c, g.data(), std::max<size_t>(1, g.size())));
        }
    }
    pl.ok = true;
    return MTLG_OK;
}

template <typename T, typename S>
inline int launch_chunk_sweep(mtlg_ctx* c, cudaStream_t st, const SetView& sv, ChunkSweepOp op, const ChunkPlan& plan)
{
    if (op.ntasks == 0) return MTLG_OK;
    if (plan.grid) {
        int rc = MTLG_OK;
        with_grid_shape<T, S>(plan.gnw, [&](auto shape) { rc = decltype(shape)::launch(c, st, sv, op, plan.gresident); });
        return rc;
    }
    const ChunkSide& pl = plan.side[op.which];
    op.vec_bytes = pl.vec_bytes;
    op.rows_cap = pl.seg_rows;
    op.ents_cap = pl.seg_ents;
    op.cl = pl.cl;
    int rc = MTLG_OK;
    if (!with_chunk_shape<T, S>(pl.threads(), pl.entries(),
                                [&](auto shape) { rc = decltype(shape)::launch(c, st, sv, op, pl); })) {
        set_error("chunk sweep shape %d/%d", pl.threads(), pl.entries());
        return MTLG_ERR_NOT_SUPPORTED;
    }
    return rc;
}

// Device view of a factor (both layouts).
inline TriFactor tri_view(const TriDev& T)
{
    TriFactor f;
    memset(&f, 0, sizeof f);
    f.rp = T.rp.p;
    f.ci = T.ci.p;
    f.val = T.val.p;
    f.dia = T.dia.p;
    f.row_of = T.row_of.p;
    if (T.nch > 0 && T.cval.p && T.cdia.p) {
        f.chunk_rows = T.chunk_rows;
        f.nch = T.nch;
        f.seg_rows = T.seg_rows;
        f.cseg = T.cseg.p;
        f.segs = T.segs.p;
        f.wv = T.wv.p;
        f.crow = T.crow.p;
        f.cxr = T.cxr.p;
        f.cext = T.cext.p;
        f.cquad = T.cquad.p;
        f.cqpull = T.cqpull.p;
        f.cpush = T.cpush.p;
        f.ccol = T.ccol.p;
        f.cval = T.cval.p;
        f.cdia = T.cdia.p;
    }
    if (T.gnx > 0 && T.gval.p) {
        f.gnx = T.gnx;
        f.gny = T.gny;
        f.gnz = T.gnz;
        f.gns = T.gns;
        f.gperm = T.gperm;
        f.gdirs = T.gdirs;
        f.gskew = T.gskew;
        f.gnsteps = T.gnsteps;
        f.gnsp = T.gnsp;
        f.gnjb = T.gnjb;
        f.gdata = T.gval.p;
    }
    return f;
}

inline void compute_levels(const RowLists& F, int n, bool lower, std::vector<int>& lev, int& nlev)
{
    lev.assign(n, 0);
    int mx = -1;
    if (lower) {
        for (int i = 0; i < n; ++i) {
            int l = 0;
            for (int e = F.rp[i]; e < F.rp[i + 1]; ++e) l = std::max(l, lev[F.col[e]] + 1);
            lev[i] = l;
            mx = std::max(mx, l);
        }
    } else {
        for (int i = n - 1; i >= 0; --i) {
            int l = 0;
            for (int e = F.rp[i]; e < F.rp[i + 1]; ++e) l = std::max(l, lev[F.col[e]] + 1);
            lev[i] = l;
            mx = std::max(mx, l);
        }
    }
    nlev = mx + 1;
}

// Rows per sweep chunk: 64 KB of vector values per CTA (8192 FP64 or 16384
// FP32 rows), or the context's setting.
inline int default_chunk_rows(const mtlg_ctx* c, int storage)
{
    if (c->chunk_rows > 0) return c->chunk_rows;
    return storage == MTLG_F32 ? 16384 : 8192;
}

// Flat layout entries of a factor whose flat row order is built: per
// position its row's entries (columns, value sources, multipliers), on the
// host and the device.
inline int build_flat_entries(mtlg_ctx* c, const RowLists& F, TriDev& T)
{
    MTLG_TRACE(9159, "pc.flat_entries");
    T.h_rp.resize(size_t(T.npad) + 1);
    parallel_prefix(T.npad, [&](int k) {
        const int r = T.h_row_of[k];
        return r >= 0 ? F.rp[r + 1] - F.rp[r] : 0;
    }, T.h_rp.data());
    T.nnz = T.h_rp[T.npad];
    T.h_ci.resize(T.nnz);
    T.h_src.resize(T.nnz);
    T.h_mul.resize(T.nnz);
    constexpr int kRowsPerBlock = 16384;
    parallel_for((T.npad + kRowsPerBlock - 1) / kRowsPerBlock, [&](int blk) {
        const int k1 = std::min(T.npad, (blk + 1) * kRowsPerBlock);
        for (int k = blk * kRowsPerBlock; k < k1; ++k) {
            const int r = T.h_row_of[k];
            if (r < 0) continue;
            int o = T.h_rp[k];
            for (int e = F.rp[r]; e < F.rp[r + 1]; ++e, ++o) {
                T.h_ci[o] = F.col[e];
                T.h_src[o] = F.src[e];
                T.h_mul[o] = F.mul[e];
            }
        }
    });
    MTLG_TRY(T.rp.upload(c, T.h_rp.data(), T.h_rp.size()));
    MTLG_TRY(T.ci.upload(c, T.h_ci.data(), T.h_ci.size()));
    MTLG_TRY(T.src.upload(c, T.h_src.data(), T.h_src.size()));
    MTLG_TRY(T.mul.upload(c, T.h_mul.data(), T.h_mul.size()));
    T.flat_entries = true;
    return MTLG_OK;
}

// Grid geometry of a triangular factor's pattern (natural row order): the
// distinct offsets between a row and the rows it reads must be {1, nx} (2D)
// or {1, nx, nx*ny} (3D) with n = nx*ny(*nz), every row must read exactly
// its in-grid neighbours (x when i > 0, y when j > 0, z when k > 0; rows
// counted from the sweep's start: r' = r for L, n - 1 - r for U), and the
// rows' entries must follow one order of the directions (the slot order of
// the layout).  A factor without entries (Jacobi's trivial factors) is a
// grid of independent rows, run unskewed in lines of 256.
inline bool detect_grid(const RowLists& F, int n, bool lower, TriDev& T)
{
    T.gnx = 0;
    if (n < 1) return false;
    constexpr int kBlk = 1 << 16;
    const int nb = (n + kBlk - 1) / kBlk;
    std::vector<long long> bo(size_t(nb) * 4, 0);
    std::vector<int> bn(nb, 0);
    parallel_for(nb, [&](int b) {
        long long* o = bo.data() + size_t(b) * 4;
        int cnt = 0;
        const int r1 = std::min(n, (b + 1) * kBlk);
        for (int r = b * kBlk; r < r1 && cnt <= 3; ++r)
            for (int e = F.rp[r]; e < F.rp[r + 1]; ++e) {
                const long long off = lower ? (long long)r - F.col[e] : (long long)F.col[e] - r;
                bool seen = false;
                for (int x = 0; x < cnt; ++x) seen |= o[x] == off;
                if (seen) continue;
                if (cnt == 3) {
                    cnt = 4;   // more than three offsets: not a grid stencil
                    break;
                }
                o[cnt++] = off;
            }
        bn[b] = cnt;
    });
    std::vector<long long> offs;
    for (int b = 0; b < nb; ++b) {
        if (bn[b] > 3) return false;
        for (int x = 0; x < bn[b]; ++x)
            if (std::find(offs.begin(), offs.end(), bo[size_t(b) * 4 + x]) == offs.end())
                offs.push_back(bo[size_t(b) * 4 + x]);
    }
    if (offs.size() > 3) return false;
    std::sort(offs.begin(), offs.end());
    int nx, ny, nz;
    if (offs.empty()) {
        T.gnx = std::min(n, 256);
        T.gny = (n + T.gnx - 1) / T.gnx;
        T.gnz = 1;
        T.gns = T.gperm = T.gdirs = T.gskew = 0;
        return true;
    }
    if (offs.size() == 1 || offs[0] != 1 || offs[1] < 2 || offs[1] > n) return false;
    nx = int(offs[1]);
    if (offs.size() == 2) {
        if (n % nx) return false;
        ny = n / nx;
        nz = 1;
    } else {
        if (offs[2] % offs[1] || offs[2] / offs[1] < 2 || n % offs[2]) return false;
        ny = int(offs[2] / offs[1]);
        nz = int(n / offs[2]);
    }
    if (ny < 2 || (offs.size() == 3 && nz < 2)) return false;
    const int ns = int(offs.size());
    auto dir_of = [&](long long off) { return off == 1 ? 0 : off == nx ? 1 : 2; };
    // slot order: the directions of an interior row's entries
    const long long rint = 1 + (long long)nx * (1 + (long long)ny * (ns == 3 ? 1 : 0));
    if (rint >= n) return false;
    const int ri = lower ? int(rint) : int(n - 1 - rint);
    if (F.rp[ri + 1] - F.rp[ri] != ns) return false;
    int perm = 0, rank[3] = {-1, -1, -1};
    for (int q = 0; q < ns; ++q) {
        const int e = F.rp[ri] + q;
        const int d = dir_of(lower ? (long long)ri - F.col[e] : (long long)F.col[e] - ri);
        if (rank[d] >= 0) return false;
        rank[d] = q;
        perm |= d << (2 * q);
    }
    // the kernel runs the farthest-first and nearest-first orders
    if (ns == 3 ? (perm != kGridFar3 && perm != kGridNear3) : (perm != kGridFar2 && perm != kGridNear2)) return false;
    // every row reads exactly its in-grid neighbours, in slot order
    std::vector<char> bad(nb, 0);
    parallel_for(nb, [&](int b) {
        const int r1 = std::min(n, (b + 1) * kBlk);
        for (int r = b * kBlk; r < r1; ++r) {
            const long long rp = lower ? r : (long long)n - 1 - r;
            const long long i = rp % nx, j = (rp / nx) % ny, k = rp / ((long long)nx * ny);
            const int want = (i > 0) + (j > 0) + (k > 0);
            if (F.rp[r + 1] - F.rp[r] != want) {
                bad[b] = 1;
                return;
            }
            int last = -1;
            for (int e = F.rp[r]; e < F.rp[r + 1]; ++e) {
                const long long off = lower ? (long long)r - F.col[e] : (long long)F.col[e] - r;
                if (off != 1 && off != nx && off != (long long)nx * ny) {
                    bad[b] = 1;
                    return;
                }
                const int d = dir_of(off);
                const bool inside = d == 0 ? i > 0 : d == 1 ? j > 0 : k > 0;
                if (!inside || rank[d] < 0 || rank[d] <= last) {
                    bad[b] = 1;
                    return;
                }
                last = rank[d];
            }
        }
    });
    for (char x : bad)
        if (x) return false;
    T.gnx = nx;
    T.gny = ny;
    T.gnz = nz;
    T.gns = ns;
    T.gperm = perm;
    T.gdirs = ns == 3 ? 7 : 3;
    T.gskew = 1;
    return true;
}

// Grid layout of a factor whose pattern detect_grid accepted: per unit,
// step, slot and lane the value source and pivot row of the element
// (k_fill_grid fills the values after the factorization).
inline int build_grid(mtlg_ctx* c, const RowLists& F, int n, bool lower, TriDev& T)
{
    T.gnx = 0;
    T.gnent = 0;
    if (!c->grid_sweep) return MTLG_OK;
    {
        MTLG_TRACE(9160, "pc.grid_detect");
        if (!detect_grid(F, n, lower, T)) {
            T.gnx = 0;
            return MTLG_OK;
        }
    }
    MTLG_TRACE(9161, "pc.grid_layout");
    T.gnjb = (T.gny + 31) / 32;
    T.gnsteps = T.gskew ? T.gnx + std::min(T.gny, 32) - 1 : T.gnx;
    T.gnsp = (T.gnsteps + kGridStepPad - 1) / kGridStepPad * kGridStepPad;
    const int se = (T.gns + 1) * 32;
    const long long units = (long long)T.gnjb * T.gnz;
    const long long nent = units * T.gnsp * se;
    if (nent > (long long)INT32_MAX) {
        T.gnx = 0;
        return MTLG_OK;
    }
    T.gnent = nent;
    if (!T.grid_indices) return MTLG_OK;
    hvec<int> gsrc(static_cast<size_t>(nent)), gmul(static_cast<size_t>(nent));
    const int nx = T.gnx, ny = T.gny, ns = T.gns, perm = T.gperm, skew = T.gskew, nsteps = T.gnsteps;
    const long long nxy = (long long)nx * ny;
    parallel_for(int(units), [&](int u) {
        const int ju = u % T.gnjb, k = u / T.gnjb;
        long long e = (long long)u * T.gnsp * se;
        for (int s = 0; s < T.gnsp; ++s)
            for (int q = 0; q <= ns; ++q)
                for (int l = 0; l < 32; ++l, ++e) {
                    const int i = skew ? s - l : s, j = 32 * ju + l;
                    const long long rp = i + (long long)nx * (j + (long long)ny * k);
                    if (s >= nsteps || i < 0 || i >= nx || j >= ny || rp >= n) {
                        gsrc[e] = -1;
                        gmul[e] = -1;
                        continue;
                    }
                    const int r = lower ? int(rp) : int(n - 1 - rp);
                    if (q == ns) {
                        gsrc[e] = -2;
                        gmul[e] = r;
                        continue;
                    }
                    const int d = (perm >> (2 * q)) & 3;
                    const long long off = d == 0 ? 1 : d == 1 ? nx : nxy;
                    const long long col = lower ? r - off : r + off;
                    gsrc[e] = -1;
                    gmul[e] = -1;
                    for (int f = F.rp[r]; f < F.rp[r + 1]; ++f)
                        if (F.col[f] == col) {
                            gsrc[e] = F.src[f];
                            gmul[e] = F.mul[f];
                        }
                }
    });
    MTLG_TRY(T.gsrc.upload(c, gsrc.data(), gsrc.size()));
    MTLG_TRY(T.gmul.upload(c, gmul.data(), gmul.size()));
    return MTLG_OK;
}

inline int build_tri(mtlg_ctx* c, RowLists&& F, int n, bool lower, TriDev& T, int chunk_rows, int ssz, bool defer_flat)
{
    MTLG_TRY(build_grid(c, F, n, lower, T));
    // a factor swept on its grid layout (values filled from the CSR) needs no
    // chunked layout; its flat entries come on first need (ensure_flat)
    const bool grid_only = T.gnx > 0 && !T.grid_indices;
    if (grid_only) chunk_rows = 0;
    T.n = n;
    T.lower = lower;
    std::vector<int> lev;
    {
        MTLG_TRACE(9150, "pc.levels");
        compute_levels(F, n, lower, lev, T.nlev);
    }
    TracePhases ph;
    ph.next(9151, "pc.flat_layout");
    std::vector<int> cnt(T.nlev + 1, 0);
    for (int i = 0; i < n; ++i) cnt[lev[i]]++;
    // padded level starts
    std::vector<int> start(T.nlev + 1, 0);
    T.lev_task_begin.assign(T.nlev + 1, 0);
    for (int l = 0; l < T.nlev; ++l) {
        const int padded = (cnt[l] + kSweepRows - 1) / kSweepRows * kSweepRows;
        start[l + 1] = start[l] + padded;
        T.lev_task_begin[l + 1] = T.lev_task_begin[l] + padded / kSweepRows;
    }
    T.npad = start[T.nlev];
    T.h_row_of.resize(T.npad);
    // rows ascending within a level (lower) / descending (upper): a counting
    // sort by level; with few levels, blocks of rows scatter in parallel
    // (per-block offsets per level keep the sequential order)
    constexpr int kSortBlk = 1 << 16;
    const int nsb = (n + kSortBlk - 1) / kSortBlk;
    parallel_for(T.nlev, [&](int l) {
        for (int k = start[l] + cnt[l]; k < start[l + 1]; ++k) T.h_row_of[k] = -1;   // level padding
    });
    if (nsb > 1 && size_t(nsb) * size_t(T.nlev) <= (size_t(1) << 22)) {
        std::vector<int> bc(size_t(nsb) * T.nlev, 0);
        // block b of the visiting order (ascending rows for L, descending for U)
        auto row_at = [&](int v) { return lower ? v : n - 1 - v; };
        parallel_for(nsb, [&](int b) {
            int* c0 = bc.data() + size_t(b) * T.nlev;
            for (int v = b * kSortBlk; v < std::min(n, (b + 1) * kSortBlk); ++v) c0[lev[row_at(v)]]++;
        });
        parallel_for(T.nlev, [&](int l) {
            int o = start[l];
            for (int b = 0; b < nsb; ++b) {
                const int t = bc[size_t(b) * T.nlev + l];
                bc[size_t(b) * T.nlev + l] = o;
                o += t;
            }
        });
        parallel_for(nsb, [&](int b) {
            int* c0 = bc.data() + size_t(b) * T.nlev;
            for (int v = b * kSortBlk; v < std::min(n, (b + 1) * kSortBlk); ++v) {
                const int r = row_at(v);
                T.h_row_of[c0[lev[r]]++] = r;
            }
        });
    } else {
        std::vector<int> fill(start.begin(), start.end() - 1);
        if (lower) {
            for (int i = 0; i < n; ++i) T.h_row_of[fill[lev[i]]++] = i;
        } else {
            for (int i = n - 1; i >= 0; --i) T.h_row_of[fill[lev[i]]++] = i;
        }
    }
    std::vector<SweepTask> tasks(T.npad / kSweepRows);
    for (size_t t = 0; t < tasks.size(); ++t) tasks[t] = {0, int(t) * kSweepRows};
    ph.next(9152, "pc.flat_upload");
    MTLG_TRY(T.row_of.upload(c, T.h_row_of.data(), T.h_row_of.size()));
    MTLG_TRY(T.tasks.upload(c, tasks.data(), tasks.size()));
    T.nnz = F.rp[n];
    ph.end();
    MTLG_TRY(build_chunks(c, F, lev, n, lower, chunk_rows, ssz, T));
    if ((T.nch == 0 && !grid_only) || !defer_flat) return build_flat_entries(c, F, T);
    T.F = std::move(F);
    return MTLG_OK;
}

}  // namespace mtlg

struct mtlg_pc {
    mtlg_ctx* ctx = nullptr;
    mtlg_csr* A = nullptr;
    int kind = MTLG_PC_IDENTITY;
    int storage = MTLG_F64;
    int n = 0;
    DBuf<unsigned char> inv_diag;   // Jacobi, storage type
    TriDev L, U;
    DBuf<double> inv_dia;           // FP64 pivots (ILU: 1/u_ii, IC: 1/sqrt(u_ii))
    DBuf<unsigned char> tmp;        // sentinel-filled temporary (n x 8 bytes)
    DBuf<int> tickets;              // self-resetting work tickets
    DBuf<SysDesc> desc;
    DBuf<SysState> st;
    DBuf<int> misc;
    mtlg_pc* fallback64 = nullptr;  // FP32 storage: the FP64 preconditioner of the same kind a stalled
                                    // refinement finishes with (made on first need)
    ChunkPlan plan[2];              // chunked sweeps with FP64 [0] / FP32 [1] vectors
    int plan_kernel[2] = {-1, -1};  // context's sweep_kernel / cluster setting the plan was made for
    mtlg_pc* adjoint = nullptr;     // ILU(0): factors of (LU)^H, made on the first adjoint apply
    bool grid_factored = false;     // pivots computed by the grid kernel (ILU(0): A's values, no factorized copy)
    RowLists lt;                    // IC(0): transposed upper pattern (natural order)
    DBuf<int> lt_rp, lt_row, lt_src;
    bool has_factors() const { return kind == MTLG_PC_ILU0 || kind == MTLG_PC_IC0; }
    size_t ssize() const { return storage == MTLG_F64 ? 8 : 4; }
};

namespace mtlg {

inline int fill_sentinel(mtlg_ctx* c, void* p, size_t bytes)
{
    if (!bytes) return MTLG_OK;
    MTLG_CUDA(cudaMemsetAsync(p, 0xFF, bytes, c->stream));
    return MTLG_OK;
}

inline int sweep_grid(mtlg_ctx* c) { return c->sweep_grid; }

// Position-ordered results of a chunked factor for vectors of one type,
// allocated on first use and filled with the sentinel.
inline int ensure_ypos(mtlg_ctx* c, TriDev& T, int f32)
{
    if (T.nch == 0 || T.ypos[f32].p) return MTLG_OK;
    const size_t bytes = size_t(std::max(T.cnpos, 4)) * (f32 ? 4 : 8);
    MTLG_TRY(T.ypos[f32].alloc(c, bytes));
    return fill_sentinel(c, T.ypos[f32].p, bytes);
}

// Device views of a preconditioner's factors for vectors of one type: each
// sweep publishes into its own position-ordered results and resets the
// other factor's (the next sweep of the other kind reads them sentinel).
inline int pc_views(mtlg_pc* P, int f32, TriFactor& L, TriFactor& U)
{
    L = tri_view(P->L);
    U = tri_view(P->U);
    if (L.chunk_rows > 0 && U.chunk_rows > 0) {
        MTLG_TRY(ensure_ypos(P->ctx, P->L, f32));
        MTLG_TRY(ensure_ypos(P->ctx, P->U, f32));
        L.ypos = P->L.ypos[f32].p;
        L.npos = P->L.cnpos;
        L.ypos_reset = P->U.ypos[f32].p;
        L.npos_reset = P->U.cnpos;
        U.ypos = P->U.ypos[f32].p;
        U.npos = P->U.cnpos;
        U.ypos_reset = P->L.ypos[f32].p;
        U.npos_reset = P->L.cnpos;
    }
    return MTLG_OK;
}

// After an expired device wait: back to all-sentinel sweep buffers.
inline int pc_reset_sweep_state(mtlg_pc* P)
{
    if (!P) return MTLG_OK;
    for (TriDev* T : {&P->L, &P->U})
        for (int k = 0; k < 2; ++k)
            if (T->ypos[k].p) MTLG_TRY(fill_sentinel(P->ctx, T->ypos[k].p, T->ypos[k].n));
    if (P->tmp.p) MTLG_TRY(fill_sentinel(P->ctx, P->tmp.p, size_t(P->n) * 8));
    return MTLG_OK;
}

inline int pc_setup_single_set(mtlg_pc* P)
{
    mtlg_ctx* c = P->ctx;
    MTLG_TRY(P->desc.alloc(c, 1));
    MTLG_TRY(P->st.alloc(c, 1));
    MTLG_CUDA(cudaMemsetAsync(P->st.p, 0, sizeof(SysState), c->stream));
    MTLG_TRY(P->misc.alloc(c, 4));
    MTLG_CUDA(cudaMemsetAsync(P->misc.p, 0, 4 * sizeof(int), c->stream));
    MTLG_TRY(P->tickets.alloc(c, 8));
    MTLG_CUDA(cudaMemsetAsync(P->tickets.p, 0, 8 * sizeof(int), c->stream));
    MTLG_TRY(P->tmp.alloc(c, size_t(std::max(P->n, 1)) * 8));
    MTLG_TRY(fill_sentinel(c, P->tmp.p, size_t(P->n) * 8));
    return MTLG_OK;
}

inline int launch_grid(int64_t n, int maxg = 8192) { return int(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, maxg))); }

// Values of the chunked layout: entries from `srcvals` (times the inverse
// pivot named by cmul), multipliers from inv_dia (1 for a unit diagonal).
inline int fill_chunk_values(mtlg_pc* P, TriDev& T, const double* srcvals, const double* inv_dia, int unit)
{
    mtlg_ctx* c = P->ctx;
    if (T.nch == 0) return MTLG_OK;
    const int f32 = P->storage == MTLG_F32;
    MTLG_TRY(T.cval.alloc(c, size_t(std::max(T.cnent, 4)) * P->ssize()));
    MTLG_TRY(T.cdia.alloc(c, size_t(std::max(T.cnpos, 4)) * P->ssize()));
    if (T.cnent) {
        k_fill_factor<<<launch_grid(T.cnent), 256, 0, c->stream>>>(T.cnent, T.csrc.p, T.cmul.p, srcvals, inv_dia,
                                                                   T.cval.p, f32);
        c->launches++;
    }
    if (T.cnpos) {
        k_fill_dia<<<launch_grid(T.cnpos), 256, 0, c->stream>>>(T.cnpos, T.crow.p, inv_dia, unit, T.cdia.p, f32);
        c->launches++;
    }
    MTLG_CUDA(cudaGetLastError());
    return MTLG_OK;
}

// Values of the grid layout (same sources and roundings as the chunked
// layout's); the per-element sources are released afterwards.
inline int fill_grid_values(mtlg_pc* P, TriDev& T, const double* srcvals, const double* inv_dia, int unit)
{
    mtlg_ctx* c = P->ctx;
    if (T.gnx == 0 || T.gnent == 0) return MTLG_OK;
    const int f32 = P->storage == MTLG_F32;
    MTLG_TRY(T.gval.alloc(c, size_t(T.gnent) * P->ssize()));
    if (!T.grid_indices) {
        const GridFillGeom g = {T.n, T.gnx, T.gny, T.gnz, T.gns, T.gperm, T.gskew, T.gnsteps, T.gnsp, T.gnjb};
        const int kind = P->kind == MTLG_PC_IC0 ? kGridFillIC : kGridFillILU;
        k_fill_grid_csr<<<launch_grid(T.gnent), 256, 0, c->stream>>>(T.gnent, g, T.lower ? 1 : 0, kind, unit,
                                                                   P->grid_factored ? 1 : 0, P->A->rp.p, P->A->ci.p,
                                                                   srcvals, inv_dia, T.gval.p, f32);
        c->launches++;
        MTLG_CUDA(cudaGetLastError());
        return MTLG_OK;
    }
    k_fill_grid<<<launch_grid(T.gnent), 256, 0, c->stream>>>(T.gnent, T.gsrc.p, T.gmul.p, srcvals, inv_dia, unit,
                                                           T.gval.p, f32);
    c->launches++;
    MTLG_CUDA(cudaGetLastError());
    MTLG_CUDA(cudaStreamSynchronize(c->stream));   // the sources are released next
    T.gsrc.release();
    T.gmul.release();
    return MTLG_OK;
}

// Values of the flat layout: entries from `srcvals` (times the inverse
// pivot named by mul), multipliers from the FP64 pivots (1 for a unit
// diagonal).
inline int fill_flat_values(mtlg_pc* P, TriDev& T, const double* srcvals, int unit)
{
    mtlg_ctx* c = P->ctx;
    const int f32 = P->storage == MTLG_F32;
    MTLG_TRY(T.val.alloc(c, size_t(std::max(T.nnz, 1)) * P->ssize()));
    MTLG_TRY(T.dia.alloc(c, size_t(std::max(T.npad, 1)) * P->ssize()));
    if (T.nnz) {
        k_fill_factor<<<launch_grid(T.nnz), 256, 0, c->stream>>>(T.nnz, T.src.p, T.mul.p, srcvals, P->inv_dia.p,
                                                                 T.val.p, f32);
        c->launches++;
    }
    if (T.npad) {
        k_fill_dia<<<launch_grid(T.npad), 256, 0, c->stream>>>(T.npad, T.row_of.p, P->inv_dia.p, unit, T.dia.p, f32);
        c->launches++;
    }
    MTLG_CUDA(cudaGetLastError());
    return MTLG_OK;
}

// inv[csrc[e]] = e for the chunk entries with a value source (padding: src
// < 0; alignment gaps: column code -1).
__global__ void k_chunk_inverse(int nent, const int* __restrict__ csrc, const int* __restrict__ ccol,
                                int* __restrict__ inv)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nent; e += gridDim.x * blockDim.x)
        if (csrc[e] >= 0 && ccol[e] != -1) inv[csrc[e]] = e;
}
// val[k] = cval[inv[src[k]]]: a flat entry's value, copied from the chunked
// layout's entry of the same source (the same value, already in S).
__global__ void k_flat_from_chunk(int nnz, const int* __restrict__ src, const int* __restrict__ inv,
                                  const unsigned char* __restrict__ cval, unsigned char* __restrict__ val, int ssz)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x) {
        const int e = src[k] >= 0 ? inv[src[k]] : -1;   // every entry has its chunk twin; -1 stays 0
        if (ssz == 8) reinterpret_cast<double*>(val)[k] = e >= 0 ? reinterpret_cast<const double*>(cval)[e] : 0.0;
        else reinterpret_cast<float*>(val)[k] = e >= 0 ? reinterpret_cast<const float*>(cval)[e] : 0.0f;
    }
}

// The flat layout of a preconditioner whose factors were built with the
// chunked layout only: entries from the kept row lists, values copied from
// the chunked layout, multipliers from the pivots.  Needed by flat sweeps,
// factor downloads and the ILU(0) adjoint.
inline int ensure_flat(mtlg_pc* P)
{
    if (!P || !P->has_factors()) return MTLG_OK;
    mtlg_ctx* c = P->ctx;
    for (TriDev* T : {&P->L, &P->U}) {
        if (T->flat_entries) continue;
        MTLG_TRY(build_flat_entries(c, T->F, *T));
        T->F = RowLists();
        const int unit = (P->kind == MTLG_PC_ILU0 && T == &P->L);
        MTLG_TRY(T->val.alloc(c, size_t(std::max(T->nnz, 1)) * P->ssize()));
        MTLG_TRY(T->dia.alloc(c, size_t(std::max(T->npad, 1)) * P->ssize()));
        if (T->nnz && T->nch == 0 && T->gnx > 0 && T->gval.p) {
            // values from the grid layout
            const GridFillGeom g = {T->n, T->gnx, T->gny, T->gnz, T->gns, T->gperm, T->gskew, T->gnsteps, T->gnsp, T->gnjb};
            k_flat_from_grid<<<launch_grid(T->npad), 256, 0, c->stream>>>(T->npad, T->row_of.p, T->rp.p, T->ci.p, g,
                                                                          T->lower ? 1 : 0, T->gval.p, T->val.p,
                                                                          int(P->ssize()));
            c->launches++;
            MTLG_CUDA(cudaGetLastError());
        } else if (T->nnz) {
            DBuf<int> inv;
            const int64_t asz = std::max<int64_t>(1, P->A->nnz);
            MTLG_TRY(inv.alloc(c, size_t(asz)));
            MTLG_CUDA(cudaMemsetAsync(inv.p, 0xFF, size_t(asz) * sizeof(int), c->stream));
            k_chunk_inverse<<<launch_grid(T->cnent), 256, 0, c->stream>>>(T->cnent, T->csrc.p, T->ccol.p, inv.p);
            k_flat_from_chunk<<<launch_grid(T->nnz), 256, 0, c->stream>>>(T->nnz, T->src.p, inv.p, T->cval.p,
                                                                          T->val.p, int(P->ssize()));
            c->launches += 2;
            MTLG_CUDA(cudaGetLastError());
            MTLG_CUDA(cudaStreamSynchronize(c->stream));   // inv is freed at scope end
        }
        if (T->npad) {
            k_fill_dia<<<launch_grid(T->npad), 256, 0, c->stream>>>(T->npad, T->row_of.p, P->inv_dia.p, unit, T->dia.p,
                                                                     P->storage == MTLG_F32);
            c->launches++;
            MTLG_CUDA(cudaGetLastError());
        }
    }
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    return MTLG_OK;
}

// FP64 pivots of an ILU(0) / IC(0) preconditioner whose L factor has the
// grid layout (farthest neighbour first), on the grid kernel: the factor
// layout (A's values per row and neighbour) is filled on the device, the
// pivots land in P->inv_dia (all sentinel before).  ILU(0) grids with a
// side of 2 stay on the level-scheduled kernel (the rule holds there as
// well, but this kernel is exercised on sides of 3 and more).  Sets `done`
// when it ran.
inline int grid_factorize(mtlg_pc* P, bool& done)
{
    done = false;
    mtlg_ctx* c = P->ctx;
    const TriDev& L = P->L;
    if (L.gnx == 0 || L.gns < 2 || !L.gskew) return MTLG_OK;
    if (L.gperm != (L.gns == 3 ? kGridFar3 : kGridFar2)) return MTLG_OK;
    const int kind = P->kind == MTLG_PC_IC0 ? kGridIC0 : kGridILU0;
    if (kind == kGridILU0 && (L.gnx < 3 || (L.gns == 3 && L.gny < 3) || (L.gns == 2 && L.gny < 2))) return MTLG_OK;
    const int nw = kind == kGridILU0 ? kGridFactorWarpsILU : kGridFactorWarpsIC;
    const int res = kind == kGridILU0 ? GridFactorShape<kGridILU0, kGridFactorWarpsILU>::resident(c)
                                      : GridFactorShape<kGridIC0, kGridFactorWarpsIC>::resident(c);
    if (res < 1) return MTLG_OK;
    MTLG_TRACE(9162, "pc.grid_factor");
    const int slots = kind == kGridILU0 ? 2 * L.gns + 1 : L.gns + 1;
    const long long nent = (long long)L.gnjb * L.gnz * L.gnsp * slots * 32;
    DBuf<double> lay;
    MTLG_TRY(lay.alloc(c, size_t(nent)));
    const GridFillGeom gg = {L.n, L.gnx, L.gny, L.gnz, L.gns, L.gperm, L.gskew, L.gnsteps, L.gnsp, L.gnjb};
    k_fill_grid_factor<<<launch_grid(nent), 256, 0, c->stream>>>(nent, gg, kind, P->A->rp.p, P->A->ci.p, P->A->v64.p,
                                                                 lay.p);
    c->launches++;
    // one system: inv_dia is the output vector, L's view carries the factor layout
    SysDesc d;
    memset(&d, 0, sizeof d);
    d.n = P->n;
    d.x = P->inv_dia.p;
    d.L = tri_view(L);
    d.L.gnx = L.gnx;
    d.L.gny = L.gny;
    d.L.gnz = L.gnz;
    d.L.gns = L.gns;
    d.L.gperm = L.gperm;
    d.L.gdirs = L.gdirs;
    d.L.gskew = L.gskew;
    d.L.gnsteps = L.gnsteps;
    d.L.gnsp = L.gnsp;
    d.L.gnjb = L.gnjb;
    d.L.gdata = lay.p;
    MTLG_CUDA(cudaMemcpyAsync(P->desc.p, &d, sizeof d, cudaMemcpyHostToDevice, c->stream));
    std::vector<GroupTask> tiles;
    const int jw = L.gns == 3 ? 1 : nw, kw = nw / jw;
    for (int k0 = 0; k0 < L.gnz; k0 += kw)
        for (int j0 = 0; j0 < L.gnjb; j0 += jw) tiles.push_back(GroupTask{0, j0, k0, jw});
    DBuf<GroupTask> tl;
    MTLG_TRY(tl.upload(c, tiles.data(), tiles.size()));
    SetView sv;
    memset(&sv, 0, sizeof sv);
    sv.n_sys = 1;
    sv.desc = P->desc.p;
    sv.st = P->st.p;
    sv.running = P->misc.p;
    sv.err = P->misc.p + 1;
    sv.spin = c->spin_limit;
    ChunkSweepOp op;
    memset(&op, 0, sizeof op);
    op.tasks = tl.p;
    op.ntasks = int(tiles.size());
    op.ticket = P->tickets.p + 6;
    op.which = 0;
    op.in = SLOT_NONE;
    op.out = SLOT_X;
    op.reset = SLOT_NONE;
    op.skip = SKIP_NONE;
    op.sleep_ns = c->sweep_sleep_ns;
    const int grid = std::max(1, std::min(op.ntasks, res));
    if (kind == kGridILU0) {
        using Sh = GridFactorShape<kGridILU0, kGridFactorWarpsILU>;
        k_sweep_grid<double, double, kGridFactorWarpsILU, false, kGridILU0><<<grid, Sh::THREADS, Sh::smem(), c->stream>>>(sv, op);
    } else {
        using Sh = GridFactorShape<kGridIC0, kGridFactorWarpsIC>;
        k_sweep_grid<double, double, kGridFactorWarpsIC, false, kGridIC0><<<grid, Sh::THREADS, Sh::smem(), c->stream>>>(sv, op);
    }
    c->launches++;
    MTLG_CUDA(cudaGetLastError());
    MTLG_CUDA(cudaStreamSynchronize(c->stream));   // the layout and task list are released next
    done = true;
    return MTLG_OK;
}

// Structure + device factorization.
inline int pc_build(mtlg_pc* P)
{
    mtlg_csr* A = P->A;
    mtlg_ctx* c = P->ctx;
    const int n = P->n;
    const int64_t* rp = A->h_rp.data();
    const int* ci = A->h_ci.data();
    if (P->kind == MTLG_PC_DIAGONAL) {
        MTLG_TRY(P->inv_diag.alloc(c, size_t(n) * P->ssize()));
        if (n) {
            k_inv_diag<<<launch_grid(n), 256, 0, c->stream>>>(n, A->v64.p, A->dpos.p, P->inv_diag.p, P->storage == MTLG_F32);
            c->launches++;
            MTLG_CUDA(cudaGetLastError());
        }
        // trivial factors so the batched sweep path can apply Jacobi too:
        // L: no entries, dia = 1/a_ii; U: no entries, dia = 1.
        RowLists E;
        E.rp.assign(n + 1, 0);
        const int B = c->sweep_kernel == 0 ? default_chunk_rows(c, P->storage) : 0;
        P->L.grid_indices = P->U.grid_indices = false;
        MTLG_TRY(build_tri(c, RowLists(E), n, true, P->L, B, int(P->ssize()), false));
        MTLG_TRY(build_tri(c, RowLists(E), n, false, P->U, B, int(P->ssize()), false));
        MTLG_TRY(P->L.val.alloc(c, 16));
        MTLG_TRY(P->U.val.alloc(c, 16));
        MTLG_TRY(P->L.dia.alloc(c, size_t(P->L.npad) * P->ssize()));
        MTLG_TRY(P->U.dia.alloc(c, size_t(P->U.npad) * P->ssize()));
        MTLG_TRY(P->inv_dia.alloc(c, std::max(n, 1)));
        if (n) {
            // inv_dia (FP64) = 1 / a_ii for the trivial L's diagonal multiplier
            k_inv_diag<<<launch_grid(n), 256, 0, c->stream>>>(n, A->v64.p, A->dpos.p, P->inv_dia.p, 0);
            k_fill_dia<<<launch_grid(P->L.npad), 256, 0, c->stream>>>(P->L.npad, P->L.row_of.p, P->inv_dia.p, 0,
                                                                       P->L.dia.p, P->storage == MTLG_F32);
            k_fill_dia<<<launch_grid(P->U.npad), 256, 0, c->stream>>>(P->U.npad, P->U.row_of.p, P->inv_dia.p, 1,
                                                                       P->U.dia.p, P->storage == MTLG_F32);
            c->launches += 3;
            MTLG_CUDA(cudaGetLastError());
        }
        for (TriDev* T : {&P->L, &P->U}) {
            MTLG_TRY(fill_chunk_values(P, *T, P->inv_dia.p, P->inv_dia.p, T == &P->U));
            MTLG_TRY(fill_grid_values(P, *T, P->inv_dia.p, P->inv_dia.p, T == &P->U));
        }
        return pc_setup_single_set(P);
    }
    if (!P->has_factors()) return pc_setup_single_set(P);

    for (int i = 0; i < n; ++i) {
        if (A->h_dpos[i] < 0) {
            set_error("row %d has no diagonal entry", i);
            return MTLG_ERR_MISSING_DIAGONAL;
        }
    }
    RowLists Lr, Ur;
    Lr.rp.assign(n + 1, 0);
    Ur.rp.assign(n + 1, 0);
    {
    MTLG_TRACE(9101, "pc.structure");
    if (P->kind == MTLG_PC_ILU0) {
        // L = strict_lower(LU) (unit diagonal), U = upper(LU) with the
        // inverted diagonal first (ilu_0.hpp:79-81, ilu.hpp:84-91)
        // row counts, offsets, then the entries (rows in parallel)
        parallel_prefix(n, [&](int i) {
            int nl = 0;
            for (int64_t e = rp[i]; e < rp[i + 1] && ci[e] < i; ++e) ++nl;
            return nl;
        }, Lr.rp.data());
        parallel_prefix(n, [&](int i) {
            int nu = 0;
            for (int64_t e = rp[i + 1] - 1; e >= rp[i] && ci[e] > i; --e) ++nu;
            return nu;
        }, Ur.rp.data());
        for (RowLists* R : {&Lr, &Ur}) {
            R->col.resize(size_t(R->rp[n]));
            R->src.resize(size_t(R->rp[n]));
            R->mul.assign(size_t(R->rp[n]), -1);
        }
        constexpr int kRowBlock = 16384;
        parallel_for((n + kRowBlock - 1) / kRowBlock, [&](int blk) {
            for (int i = blk * kRowBlock; i < std::min(n, (blk + 1) * kRowBlock); ++i) {
                int ol = Lr.rp[i], ou = Ur.rp[i];
                for (int64_t e = rp[i]; e < rp[i + 1]; ++e) {
                    if (ci[e] < i) { Lr.col[ol] = ci[e]; Lr.src[ol++] = int(e); }
                    else if (ci[e] > i) { Ur.col[ou] = ci[e]; Ur.src[ou++] = int(e); }
                }
            }
        });
    } else {
        // U = upper(A) scaled by its row's inverse pivot; L = trans(U) with
        // the diagonal last (ic_0.hpp:47-57, 80-87)
        std::vector<int> cntT(n + 1, 0);
        for (int i = 0; i < n; ++i)
            for (int64_t e = rp[i]; e < rp[i + 1]; ++e)
                if (ci[e] > i) cntT[ci[e] + 1]++;
        for (int i = 0; i < n; ++i) cntT[i + 1] += cntT[i];
        Lr.rp = cntT;
        Lr.col.resize(cntT[n]);
        Lr.src.resize(cntT[n]);
        Lr.mul.resize(cntT[n]);
        std::vector<int> pos(cntT.begin(), cntT.end() - 1);
        for (int i = 0; i < n; ++i) {
            for (int64_t e = rp[i]; e < rp[i + 1]; ++e) {
                if (ci[e] > i) {
                    const int j = ci[e], o = pos[j]++;
                    Lr.col[o] = i; Lr.src[o] = int(e); Lr.mul[o] = i;
                    Ur.col.push_back(j); Ur.src.push_back(int(e)); Ur.mul.push_back(i);
                }
            }
            Ur.rp[i + 1] = int(Ur.col.size());
        }
        MTLG_TRY(P->lt_rp.upload(c, Lr.rp.data(), Lr.rp.size()));
        MTLG_TRY(P->lt_row.upload(c, Lr.col.data(), std::max<size_t>(1, Lr.col.size())));
        MTLG_TRY(P->lt_src.upload(c, Lr.src.data(), std::max<size_t>(1, Lr.src.size())));
    }
    }
    const int B = c->sweep_kernel == 0 ? default_chunk_rows(c, P->storage) : 0;
    P->L.grid_indices = P->U.grid_indices = false;   // grid values straight from the CSR
    {
        // the two factors' schedules are independent: U on a second host thread
        MTLG_TRACE(9102, "pc.schedule");
        int su = MTLG_OK;
        std::string eu;
        std::thread tu([&]() {
            cudaSetDevice(c->device);   // the thread's uploads go to the context's device
            MTLG_TRACE(9103, "pc.schedule_U");
            su = build_tri(c, std::move(Ur), n, false, P->U, B, int(P->ssize()), true);
            if (su != MTLG_OK) eu = last_error();
        });
        int sl = MTLG_OK;
        {
            MTLG_TRACE(9105, "pc.schedule_L");
            sl = build_tri(c, std::move(Lr), n, true, P->L, B, int(P->ssize()), true);
        }
        tu.join();
        if (sl != MTLG_OK) return sl;
        if (su != MTLG_OK) {
            set_error("%s", eu.c_str());
            return su;
        }
    }
    MTLG_TRY(pc_setup_single_set(P));
    MTLG_TRACE(9104, "pc.factor_and_fill");

    // ---- numeric factorization on the device (FP64)
    MTLG_TRY(P->inv_dia.alloc(c, std::max(n, 1)));
    MTLG_TRY(fill_sentinel(c, P->inv_dia.p, size_t(n) * 8));
    DBuf<double> lu;
    const double* srcvals = A->v64.p;
    FactorOp op;
    memset(&op, 0, sizeof op);
    op.tasks = P->L.tasks.p;
    op.ntasks = int(P->L.tasks.n);
    op.ticket = P->tickets.p + 7;
    op.row_of = P->L.row_of.p;
    op.rp = A->rp.p;
    op.ci = A->ci.p;
    op.inv_dia = P->inv_dia.p;
    op.dpos = A->dpos.p;
    op.err = P->misc.p + 1;
    op.spin = c->spin_limit;
    bool gdone = false;
    if (c->grid_sweep) MTLG_TRY(grid_factorize(P, gdone));
    P->grid_factored = gdone;
    if (gdone) {
        // pivots done on the grid kernel; factor values come from A's values
    } else if (P->kind == MTLG_PC_ILU0) {
        MTLG_TRY(lu.alloc(c, size_t(std::max<int64_t>(1, A->nnz))));
        MTLG_CUDA(cudaMemcpyAsync(lu.p, A->v64.p, size_t(A->nnz) * 8, cudaMemcpyDeviceToDevice, c->stream));
        op.lu = lu.p;
        if (op.ntasks) {
            k_ilu0_factor<<<sweep_grid(c), kBlock, 0, c->stream>>>(op);
            c->launches++;
        }
        srcvals = lu.p;
    } else {
        op.lt_rp = P->lt_rp.p;
        op.lt_row = P->lt_row.p;
        op.lt_src = P->lt_src.p;
        op.a = A->v64.p;
        if (op.ntasks) {
            k_ic0_factor<<<sweep_grid(c), kBlock, 0, c->stream>>>(op);
            c->launches++;
        }
    }
    MTLG_CUDA(cudaGetLastError());
    for (TriDev* T : {&P->L, &P->U}) {
        const int unit = (P->kind == MTLG_PC_ILU0 && T == &P->L);
        if (T->flat_entries) MTLG_TRY(fill_flat_values(P, *T, srcvals, unit));
        MTLG_TRY(fill_chunk_values(P, *T, srcvals, P->inv_dia.p, unit));
        MTLG_TRY(fill_grid_values(P, *T, srcvals, P->inv_dia.p, unit));
    }
    int err = 0;
    MTLG_CUDA(cudaMemcpyAsync(&err, P->misc.p + 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    if (err) {
        set_error("factorization dependency wait expired");
        return MTLG_ERR_TIMEOUT;
    }
    return MTLG_OK;
}

// FP64 copies of factor values stored as S (exact for FP32).
__global__ void k_widen(int n, const void* __restrict__ v, int f32, double* __restrict__ out)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        out[k] = f32 ? double(static_cast<const float*>(v)[k]) : static_cast<const double*>(v)[k];
}

// Row lists of the transpose of a factor (from its flat layout): row j of
// the result holds the entries (i, j) of T, each with src = src_off + its
// flat index, columns ascending or descending.
inline void transpose_rows(const TriDev& T, int n, int src_off, bool descending, RowLists& R)
{
    R.rp.assign(size_t(n) + 1, 0);
    for (int k = 0; k < T.nnz; ++k) R.rp[size_t(T.h_ci[k]) + 1]++;
    for (int i = 0; i < n; ++i) R.rp[size_t(i) + 1] += R.rp[size_t(i)];
    R.col.assign(size_t(T.nnz), 0);
    R.src.assign(size_t(T.nnz), 0);
    R.mul.assign(size_t(T.nnz), -1);
    std::vector<int> pos(R.rp.begin(), R.rp.end() - 1);
    for (int p = 0; p < T.npad; ++p) {
        const int i = T.h_row_of[p];
        if (i < 0) continue;
        for (int k = T.h_rp[p]; k < T.h_rp[p + 1]; ++k) {
            const int o = pos[size_t(T.h_ci[k])]++;
            R.col[size_t(o)] = i;
            R.src[size_t(o)] = src_off + k;
        }
    }
    parallel_for(n, [&](int j) {
        const int a = R.rp[size_t(j)], e = R.rp[size_t(j) + 1];
        if (e - a < 2) return;
        std::vector<std::pair<int, int>> v;
        v.reserve(size_t(e - a));
        for (int o = a; o < e; ++o) v.push_back({R.col[size_t(o)], R.src[size_t(o)]});
        if (descending) std::sort(v.begin(), v.end(), [](auto x, auto y) { return x.first > y.first; });
        else std::sort(v.begin(), v.end());
        for (int o = a; o < e; ++o) {
            R.col[size_t(o)] = v[size_t(o - a)].first;
            R.src[size_t(o)] = v[size_t(o - a)].second;
        }
    });
}

// ILU(0) adjoint apply, (LU)^H y = x: first U^H y0 = x (lower, the inverse
// pivots as multipliers), then L^H y = y0 (upper, unit diagonal) -- the
// reference's adjoint_lower_solver / adjoint_upper_solver on the transposed
// views (itl/pc/ilu.hpp:104-115).  Those run column-oriented
// (lower_trisolve.hpp:155-170, upper_trisolve.hpp:129-149): a row of U^H
// takes its contributions in ascending column order, a row of L^H in
// descending order (columns are processed from the last one down); the row
// lists keep those orders, so the row-oriented sweeps add in the same
// sequence.
inline int pc_build_adjoint(mtlg_pc* P)
{
    MTLG_TRY(ensure_flat(P));
    mtlg_ctx* c = P->ctx;
    const int n = P->n;
    const TriDev& L = P->L;
    const TriDev& U = P->U;
    const int f32 = P->storage == MTLG_F32;
    std::unique_ptr<mtlg_pc> Q(new mtlg_pc);
    Q->ctx = c;
    Q->A = P->A;
    Q->kind = MTLG_PC_ILU0;
    Q->storage = P->storage;
    Q->n = n;
    DBuf<double> v64;
    MTLG_TRY(v64.alloc(c, size_t(std::max(1, L.nnz + U.nnz))));
    if (L.nnz) k_widen<<<launch_grid(L.nnz), 256, 0, c->stream>>>(L.nnz, L.val.p, f32, v64.p);
    if (U.nnz) k_widen<<<launch_grid(U.nnz), 256, 0, c->stream>>>(U.nnz, U.val.p, f32, v64.p + L.nnz);
    c->launches += (L.nnz > 0) + (U.nnz > 0);
    MTLG_CUDA(cudaGetLastError());
    RowLists Lh, Uh;   // U^H (lower), L^H (upper)
    transpose_rows(U, n, L.nnz, false, Lh);
    transpose_rows(L, n, 0, true, Uh);
    const int B = c->sweep_kernel == 0 ? default_chunk_rows(c, P->storage) : 0;
    MTLG_TRY(build_tri(c, std::move(Lh), n, true, Q->L, B, int(P->ssize()), false));
    MTLG_TRY(build_tri(c, std::move(Uh), n, false, Q->U, B, int(P->ssize()), false));
    MTLG_TRY(pc_setup_single_set(Q.get()));
    MTLG_TRY(Q->inv_dia.alloc(c, size_t(std::max(n, 1))));
    if (n) MTLG_CUDA(cudaMemcpyAsync(Q->inv_dia.p, P->inv_dia.p, size_t(n) * 8, cudaMemcpyDeviceToDevice, c->stream));
    for (TriDev* T : {&Q->L, &Q->U}) {
        const int unit = T == &Q->U;
        MTLG_TRY(T->val.alloc(c, size_t(std::max(T->nnz, 1)) * Q->ssize()));
        MTLG_TRY(T->dia.alloc(c, size_t(std::max(T->npad, 1)) * Q->ssize()));
        if (T->nnz) {
            k_fill_factor<<<launch_grid(T->nnz), 256, 0, c->stream>>>(T->nnz, T->src.p, T->mul.p, v64.p, Q->inv_dia.p,
                                                                      T->val.p, f32);
            c->launches++;
        }
        if (T->npad) {
            k_fill_dia<<<launch_grid(T->npad), 256, 0, c->stream>>>(T->npad, T->row_of.p, Q->inv_dia.p, unit, T->dia.p, f32);
            c->launches++;
        }
        MTLG_CUDA(cudaGetLastError());
        MTLG_TRY(fill_chunk_values(Q.get(), *T, v64.p, Q->inv_dia.p, unit));
        MTLG_TRY(fill_grid_values(Q.get(), *T, v64.p, Q->inv_dia.p, unit));
    }
    MTLG_CUDA(cudaStreamSynchronize(c->stream));
    P->adjoint = Q.release();
    return MTLG_OK;
}

}  // namespace mtlg
