// numeric_flat.cu - step 3 (values) of the tiled SpGEMM without a copy
// pipeline: one CTA per C tile row, each warp owns RPW scalar rows and runs
// Gustavson over its own A entries with no CTA-wide synchronisation inside
// the product phase.
//
//   C(i, :) = sum over k in A(i, :) of a_ik * B(k, :)        (rows i of tile row I)
//
// (Reference: spgemm_cpu step 4, src/spgemm-cpu.h:284-367, row-organised as in
// the Super16 path, src/super16_symbolic.cuh:973-1073.)
//
// Every B row is used about once per tile row (a tile row's A entries hit
// distinct k almost always), so staging B in shared memory buys no reuse; what
// matters is the instruction count per product and the number of warps with
// loads in flight.  Per warp:
//   1. lanes take 32 A tiles of the tile row at a time and read the row ranges
//      of the warp's rows; a warp scan numbers the entries;
//   2. lanes take 32 of those entries at a time: each lane finds its tile with
//      a 5-step shuffle search, reads a_ik and B's row range [fs, fe) for
//      k - all 32 lanes' loads in flight together - and writes the entry to
//      the warp's list in shared memory;
//   3. the warp walks the list GROUP entries at a time: it loads the GROUP B
//      rows' heads (lane l: entry fs + l), then adds a_ik * b_kj into the
//      row's accumulator slot, entry by entry in list order.
// The accumulator is the C tile row in CSR order in shared memory, one FP64
// per structural entry; (tile s, row r, col c) sits at
// base[r][s] + popc(mask[r][s] >> (16 - c)).  The [row][slot] table has an odd
// row stride, so the lanes of one B row (same C row, different slots) read
// distinct banks.  A warp's rows are its own and lanes of one B row hit
// distinct columns, so the adds need no atomics and every output is summed in
// the fixed order (K, k) ascending - bitwise reproducible.  (With repeated
// columns in a B row the SAFE instantiation adds with shared atomics.)
//
// Windows of C tiles (<= F_SLOT_CAP tiles, <= ACC entries) bound shared
// memory; products whose C tile is outside the window are skipped and the A
// list is walked again for the next window.  Each product also stores its
// column beside its accumulator slot, so the CSR write-out of a row is two
// contiguous copies.  Shared memory (~43 KB) and
// registers (<= 48) are sized so that five CTAs share an SM: the kernel is
// latency-bound and lives on the number of warps in flight.
#include "rtt_internal.cuh"

namespace rtt
{
namespace
{

constexpr int FW = 8;                       // warps per CTA
constexpr int RPW = TD / FW;                // rows per warp
constexpr int F_THREADS = FW * 32;
// 2048 accumulator slots at five CTAs per SM.  (A second shape with 4608
// slots at three CTAs per SM, one window for tile rows up to 4608 entries,
// measured slower on banded batches than this one with row windows: the
// kernel lives on warps in flight.)
constexpr int ACC_SMALL = FLAT_ACC, CTAS_SMALL = 5;
constexpr int F_SLOT_CAP = FLAT_SLOT_CAP;   // C tiles per window
constexpr int F_CM_STRIDE = F_SLOT_CAP + 1; // row stride of cm: rows land in distinct banks
constexpr int F_SPAN_CAP = 4096;            // tile-column span of the slot table
#ifndef FLAT_GROUP
#define FLAT_GROUP 2
#endif
constexpr int GROUP = FLAT_GROUP;           // B rows loaded together
static_assert(RPW == 1 || RPW == 2, "one or two rows per warp");

template <int ACC>
struct FlatSmem
{
    double acc[ACC];
    int ccol[ACC];                    // column of each accumulator slot (written by the products)
    uint32_t cm[TD * F_CM_STRIDE];    // [row][slot]: (acc base << 16) | row mask
    int cJ[F_SLOT_CAP];
    uint8_t slot8[F_SPAN_CAP];        // tile column - Jlo -> slot (255 = none)
    int4 ent[FW][32];                 // per warp: B row start, length, cm row offset, -
    double enta[FW][32];              // per warp: a_ik
    int rowtot[TD];
    int rowacc0[TD + 1];
    int rowcsr0[TD];
    int rowrun[TD];
    int paircnt[FW]; // entries of each warp's rows (row windows)
    int rowwin, win_begin, win_end;
    int task;        // window task taken from the queue (split tile rows)
};

struct Window
{
    int Jlo, Jspan, nW;
    bool table;
};

template <class Smem>
__device__ __forceinline__ int flat_slot(const Smem &S, const Window &W, int J)
{
    const int d = J - W.Jlo;
    if ((unsigned)d > (unsigned)W.Jspan)
        return -1;
    if (W.table)
    {
        const int s = S.slot8[d];
        return s == 255 ? -1 : s;
    }
    const int s = lower_bound(S.cJ, 0, W.nW, J);
    return (s < W.nW && S.cJ[s] == J) ? s : -1;
}

// One product into the accumulator.  CHECK = false is the single-window case
// with a slot table: every product's C tile is in the window by construction
// (the symbolic step saw the same A tiles and B rows), so the lookup runs
// without branches; the two clamps only keep inconsistent operands inside
// this CTA's shared memory.
template <bool SAFE, bool CHECK, int ACC>
__device__ __forceinline__ void flat_add(FlatSmem<ACC> &S, const Window &W, const uint32_t *cmr,
                                         int col, double a, double b)
{
    int slot;
    if (CHECK)
    {
        slot = flat_slot(S, W, col >> 4);
        if (slot < 0)
            return;
    }
    else
    {
        slot = S.slot8[min((unsigned)((col >> 4) - W.Jlo), (unsigned)(F_SPAN_CAP - 1))];
    }
    const uint32_t w = cmr[slot];
    int pos = (int)(w >> 16) + __popc((w & 0xFFFFu) >> (16 - (col & 15)));
    if (!CHECK)
        pos = min(pos, ACC - 1);
    if (SAFE)
        atomicAdd(&S.acc[pos], a * b);
    else
        S.acc[pos] = fma(a, b, S.acc[pos]);
    S.ccol[pos] = col; // every structural entry receives at least one product
}

// The warp's products for one window: every A entry (r, k) of its rows r0, r1
// times B's row k.  Returns the number of products when count is set.
// first index in [lo, hi) with a[i] >= key, probing lo, lo + 1, lo + 3,
// lo + 7, ... before a binary search: cheap when the answer is near lo
__device__ __forceinline__ int gallop_lower_bound(const int *a, int lo, int hi, int key)
{
    int p = lo, d = 1;
    while (p < hi && __ldg(a + p) < key)
    {
        lo = p + 1;
        p += d;
        d <<= 1;
    }
    return lower_bound(a, lo, min(p, hi), key);
}

// Cursors of a persistent worker CTA (cur != nullptr): for the first
// cursor_cap(A) A entries of its task's tile row, where each B row's part in
// the current window ended.  The task's windows follow each other in column
// order, so the next window's part starts there: one galloping search over
// that part instead of two binary searches over the whole row.  A tile row
// holds at most A.nnz entries, so a CTA's cursor array needs no more.
constexpr int CUR_CAP = 32768;
__host__ __device__ __forceinline__ int cursor_cap(const DevTiles &A)
{
    return A.nnz < CUR_CAP ? (A.nnz > 1 ? A.nnz : 1) : CUR_CAP;
}

// The warp's A entries, in batches of 32 (lane l: entry l of the batch):
// calls fn(valid, k, a_ik, row, place) for each batch, place being the
// entry's index inside its tile row (the same in every window).  ACSR: the
// warp's rows are contiguous in A's CSR (the device path), entries in column
// order; otherwise they come from A's tiles, tile by tile (the tile
// drop-in), which is the same (K, k) order for sorted rows.
template <bool ACSR, class F>
__device__ __forceinline__ void warp_entries(const DevTiles &A, int a0, int a1, int r0, int r1,
                                             int e_a, int e_m, int e_e, int ebase, F &&fn)
{
    const int lane = lane_id();
    if (ACSR)
    {
        for (int q0 = e_a; q0 < e_e; q0 += 32)
        {
            const int e = q0 + lane;
            const bool ok = e < e_e;
            const int k = ok ? __ldg(A.csr_col + e) : 0;
            const double a = ok ? __ldg(A.csr_val + e) : 0.0;
            fn(ok, k, a, e < e_m ? r0 : r1, e - ebase, min(32, e_e - q0));
        }
        return;
    }
    for (int t0 = a0; t0 < a1; t0 += 32)
    {
        const int t = t0 + lane;
        int eb = 0, em = 0, n = 0, tn0 = 0, K = 0;
        if (t < a1)
        {
            tn0 = __ldg(A.tile_nnz + t);
            const int tcnt = __ldg(A.tile_nnz + t + 1) - tn0;
            const uint8_t *pp = A.ptr + (size_t)t * TD;
            eb = pp[r0];
            const int ee = r1 + 1 < TD ? (int)pp[r1 + 1] : tcnt;
            em = RPW == 2 ? (int)pp[r1] : ee; // first entry of row r1
            n = max(ee - eb, 0);
            K = __ldg(A.tile_col + t);
        }
        const int incl = warp_incl_scan(n);
        const int total = __shfl_sync(FULL, incl, 31);
        for (int q0 = 0; q0 < total; q0 += 32)
        {
            // lane's entry q of the batch: owner tile by shuffle search
            const int q = q0 + lane;
            int own = 0;
#pragma unroll
            for (int b = 16; b > 0; b >>= 1)
                if (__shfl_sync(FULL, incl, own + b - 1) <= q)
                    own += b;
            own = min(own, 31);
            const int o_incl = __shfl_sync(FULL, incl, own);
            const int o_n = __shfl_sync(FULL, n, own);
            const int o_eb = __shfl_sync(FULL, eb, own);
            const int o_em = __shfl_sync(FULL, em, own);
            const int o_tn0 = __shfl_sync(FULL, tn0, own);
            const int o_K = __shfl_sync(FULL, K, own);
            const bool ok = q < total;
            int k = 0, rq = r0, place = 0;
            double a = 0.0;
            if (ok)
            {
                const int e = o_eb + (q - (o_incl - o_n));
                rq = e < o_em ? r0 : r1;
                k = o_K * TD + (A.col[o_tn0 + e] & 15);
                a = __ldg(A.val + o_tn0 + e);
                place = o_tn0 + e - ebase;
            }
            fn(ok, k, a, rq, place, min(32, total - q0));
        }
    }
}

template <bool SAFE, bool CHECK, int ACC, bool NARROW, bool ACSR>
__device__ __forceinline__ long long warp_products(FlatSmem<ACC> &S, const Window &W, const DevTiles &A,
                                                   const DevTiles &B, int a0, int a1, int r0,
                                                   int r1, int e_a, int e_m, int e_e, bool count,
                                                   int4 *ent, double *enta, int *cur, int ebase,
                                                   bool first)
{
    const int lane = lane_id();
    long long n_fma = 0;
    warp_entries<ACSR>(A, a0, a1, r0, r1, e_a, e_m, e_e, ebase, [&](bool ok, int k, double a,
                                                                    int rq, int place, int nbatch) {
            int fs = 0, len = 0;
            if (ok)
            {
                if (k < B.m)
                {
                    fs = min(max(__ldg(B.csr_rowptr + k), 0), B.nnz);
                    len = min(max(__ldg(B.csr_rowptr + k + 1), fs), B.nnz) - fs;
                }
                if (count) // each pair once, in the first window
                    n_fma += len;
                // one window of several: a long sorted B row contributes only
                // its columns inside the window's tile-column range
                if (NARROW && CHECK && !SAFE && len > NARROW_MIN)
                {
                    const int lo = W.Jlo * TD, hi = (W.Jlo + W.Jspan + 1) * TD;
                    const int fe = fs + len;
                    const int ci = place; // the entry's place in its tile row
                    const bool keep = cur != nullptr && (unsigned)ci < (unsigned)cursor_cap(A);
                    int sb;
                    if (keep && !first)
                    {
                        sb = min(max(cur[ci], fs), fe);
                        if (sb < fe && __ldg(B.csr_col + sb) < lo)
                            sb = lower_bound(B.csr_col, sb, fe, lo);
                    }
                    else
                        sb = lower_bound(B.csr_col, fs, fe, lo);
                    const int se = gallop_lower_bound(B.csr_col, sb, fe, hi);
                    if (keep)
                        cur[ci] = se;
                    len = se - sb;
                    fs = sb;
                }
            }
            // items of at most 32 B entries: an entry whose B row is longer
            // than a warp becomes one item per 32 entries of the row, so the
            // loads of every item are issued ahead like any other
            auto run_items = [&](int nb) {
                for (int j = 0; j < nb; j += GROUP)
                {
                    int4 ge[GROUP];
                    int gcol[GROUP];
                    double gb[GROUP];
#pragma unroll
                    for (int u = 0; u < GROUP; ++u)
                    {
                        ge[u] = ent[(j + u) & 31];
                        if (j + u >= nb)
                            ge[u].y = 0;
                    }
#pragma unroll
                    for (int u = 0; u < GROUP; ++u)
                    {
                        gcol[u] = 0;
                        gb[u] = 0.0;
                        if (lane < ge[u].y)
                        {
                            gcol[u] = __ldg(B.csr_col + ge[u].x + lane);
                            gb[u] = __ldg(B.csr_val + ge[u].x + lane);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < GROUP; ++u)
                        if (lane < ge[u].y)
                            flat_add<SAFE, CHECK, ACC>(S, W, S.cm + ge[u].z, gcol[u],
                                                       enta[(j + u) & 31], gb[u]);
                }
            };
            if (!__any_sync(FULL, len > 32))
            {
                if (NARROW && CHECK)
                {
                    // entries whose B row has nothing in this window (narrowed
                    // to zero) are left out of the list, which keeps its order
                    const unsigned live = __ballot_sync(FULL, len > 0);
                    if (len > 0)
                    {
                        const int at = __popc(live & ((1u << lane) - 1u));
                        ent[at] = make_int4(fs, len, rq * F_CM_STRIDE, 0);
                        enta[at] = a;
                    }
                    __syncwarp();
                    run_items(__popc(live));
                }
                else
                {
                    ent[lane] = make_int4(fs, len, rq * F_CM_STRIDE, 0);
                    enta[lane] = a;
                    __syncwarp();
                    run_items(nbatch);
                }
            }
            else
            {
                const int nch = (len + 31) >> 5;
                const int cincl = warp_incl_scan(nch);
                const int ctotal = __shfl_sync(FULL, cincl, 31);
                for (int i0 = 0; i0 < ctotal; i0 += 32)
                {
                    const int qi = i0 + lane;
                    int ow = 0;
#pragma unroll
                    for (int b = 16; b > 0; b >>= 1)
                        if (__shfl_sync(FULL, cincl, ow + b - 1) <= qi)
                            ow += b;
                    ow = min(ow, 31);
                    const int k = qi - (__shfl_sync(FULL, cincl, ow) - __shfl_sync(FULL, nch, ow));
                    const int ofs = __shfl_sync(FULL, fs, ow), olen = __shfl_sync(FULL, len, ow);
                    const int orq = __shfl_sync(FULL, rq, ow);
                    const double oa = __shfl_sync(FULL, a, ow);
                    __syncwarp(); // the previous items are consumed
                    ent[lane] = qi < ctotal ? make_int4(ofs + 32 * k, min(32, olen - 32 * k),
                                                        orq * F_CM_STRIDE, 0)
                                            : make_int4(0, 0, 0, 0);
                    enta[lane] = oa;
                    __syncwarp();
                    run_items(min(32, ctotal - i0));
                }
            }
            __syncwarp(); // the next batch overwrites this warp's list
        });
    return n_fma;
}

// The warp's products from B's row segments (one window, B rows of at most
// SEGW_MAX segments, no repeated columns): half-warp h walks the A entries of
// its row (r0 or r1) one by one, in column order, and its lanes take the
// segments of that entry's B row - lane l the segments l, l + 16, ..., each
// with its tile column J and 16-bit mask.  A lane finds the segment's C tile slot and the row's
// (base, mask) word once, then adds the segment's entries (the mask's set
// bits, in column order; their values are consecutive in B's row, from the
// offset a half-warp scan of the masks' popcounts gives) into the row's
// accumulator.  The lanes of one half hit distinct columns of one row, the
// halves distinct rows; every output entry is still summed in the order of
// its row's A entries, as in warp_products.
constexpr int SEGW_MAX = 32; // segments of a B row the segment walk takes (two rounds)

template <int ACC>
__device__ __forceinline__ long long warp_products_seg(FlatSmem<ACC> &S, const Window &W,
                                                       const DevTiles &A, const DevTiles &B,
                                                       int r0, int r1, int e_a, int e_m,
                                                       int e_e, bool count)
{
    const int lane = lane_id(), h = lane >> 4, hl = lane & 15;
    const int rh = h ? r1 : r0;
    const uint32_t *cmr = S.cm + rh * F_CM_STRIDE;
    int e = h ? e_m : e_a;
    const int eend = h ? e_e : e_m;
    const int steps = max(e_m - e_a, e_e - e_m);
    long long n_fma = 0;
    for (int st = 0; st < steps; ++st, ++e)
    {
        int k = -1, s0 = 0, ns = 0, fs = 0;
        double a = 0.0;
        if (e < eend)
        {
            k = __ldg(A.csr_col + e);
            a = __ldg(A.csr_val + e);
            if (k < B.m)
            {
                s0 = __ldg(B.seg_ptr + k);
                ns = min(__ldg(B.seg_ptr + k + 1) - s0, SEGW_MAX);
                fs = __ldg(B.csr_rowptr + k);
            }
        }
        // up to SEGW_MAX segments: lane hl takes segments hl, hl + 16, ...
        const int rounds = (int)(__reduce_max_sync(FULL, (unsigned)ns) + 15) >> 4;
        int before = 0; // entries of the B row in the earlier rounds' segments
        for (int rd = 0; rd < rounds; ++rd)
        {
            const int sl = rd * 16 + hl;
            unsigned long long sg = 0ull;
            if (sl < ns)
                sg = __ldg(B.seg + s0 + sl);
            const int pc = __popc((unsigned)sg & 0xFFFFu);
            const int incl = half_incl_scan(pc);
            const int round_total = __shfl_sync(FULL, incl, (lane & 16) | 15);
            if (count)
                n_fma += pc;
            if (sl < ns)
            {
                const int J = (int)(sg >> 16);
                const int slot = S.slot8[min((unsigned)(J - W.Jlo), (unsigned)(F_SPAN_CAP - 1))];
                const uint32_t w = cmr[slot];
                const int base = (int)(w >> 16);
                const uint32_t cmask = w & 0xFFFFu;
                int eo = min(max(fs + before + incl - pc, 0), B.nnz - 1);
                uint32_t bm = (uint32_t)sg & 0xFFFFu;
                while (bm)
                {
                    const int c = __clz(bm) - 16; // column in the tile, left to right
                    bm &= ~(0x8000u >> c);
                    const double b = __ldg(B.csr_val + eo);
                    eo = min(eo + 1, B.nnz - 1);
                    const int pos = min(base + __popc(cmask >> (16 - c)), ACC - 1);
                    S.acc[pos] = fma(a, b, S.acc[pos]);
                    S.ccol[pos] = J * TD + c;
                }
            }
            before += round_total;
        }
    }
    return n_fma;
}

// ---------------------------------------------------------------------------
// Split execution of heavy tile rows (the early split of the reference's
// numeric step, src/dmma_tile_early_split.h:152-229, applied to C tile rows).
//
// A tile row is heavy when its C tiles need more than one window (more than
// F_SLOT_CAP tiles, or more than ACC entries that row windows cannot divide).
// One CTA would walk its A entries once per window, one window after another,
// and become the tail of the launch (an R-MAT hub row has hundreds of
// windows).  Instead k_win_plan cuts every heavy tile row into windows up
// front and queues them as tasks; the first CTAs of the numeric launch are
// persistent workers that take tasks from the queue, and the CTA of a heavy
// tile row itself exits.  Each task knows, for each of its rows, how many
// entries the row has in the tiles before the window, so it writes its part
// of C's CSR without waiting for the other windows.  Every output entry is
// still summed by one warp in the fixed (K, k) order: bitwise the same result.
struct WinTask
{
    int I, w0, w1, pad; // tile row, C tiles [w0, w1)
    int run[TD];        // per row: entries in the tile row's tiles before w0
};
static_assert(sizeof(WinTask) == 80, "task record layout");

struct WinQueue
{
    int count;    // tasks written by the plan
    int head;     // next task to take
    int overflow; // some heavy tile row found no room and kept its own CTA
    int next;     // next tile row for the persistent tile-row CTAs
};

constexpr int PLAN_WARPS = 8;
// Products walked by one window task (about a millisecond of one CTA): tile
// rows whose windows together walk fewer are not split.
constexpr long long SPLIT_TARGET = 1ll << 20;

// Window starts of a heavy tile row, chosen so that the tiles can be cut
// independently: tile t starts a window when t is the row's first tile, when
// t - cs0 is a multiple of F_SLOT_CAP, or when the entries before t cross a
// multiple of H = ACC - 256.  A window then holds <= F_SLOT_CAP tiles and
// fewer than H entries before its last tile, which adds at most 256.
template <int ACC>
__device__ __forceinline__ bool win_cut(const int *c_tile_nnz, int cs0, int cs1, int P0, int t)
{
    constexpr int H = ACC - 256;
    if (t >= cs1)
        return false;
    if (t == cs0 || (t - cs0) % F_SLOT_CAP == 0)
        return true;
    return (__ldg(c_tile_nnz + t) - P0) / H != (__ldg(c_tile_nnz + t - 1) - P0) / H;
}

// Global accumulation of heavy tile rows (NumericConfig::global_rows): a task
// is a run of consecutive C tiles of a heavy row holding about GLOB_H
// entries (at most GLOB_H + 255), with no cap on its tiles: its products
// accumulate in C's own value array, so no shared-memory window bounds it.
constexpr int GLOB_H = 8192;
constexpr int GLOB_RELCAP = GLOB_H + 256; // C tiles of one task, at most
// The atomic form keeps a task's tile table (an open-addressing hash of its
// tile columns: a task's tiles may lie anywhere in the row) and (row offset,
// mask) words in shared memory: a task holds at most GNT C tiles.
constexpr int GNT = 256, GHASH = 2 * GNT;
// rows of fewer shared-memory windows than this stay with the windows
constexpr int GLOB_MIN_WINDOWS = 4;
__device__ __forceinline__ bool glob2_cut(const int *c_tile_col, int cs0, int cs1, int t)
{
    (void)c_tile_col;
    return t < cs1 && (t == cs0 || (t - cs0) % GNT == 0);
}
__device__ __forceinline__ int glob2_hash(int J)
{
    return (int)(((unsigned)J * 0x9E3779B1u) >> 23) & (GHASH - 1); // 9 bits
}
__device__ __forceinline__ bool glob_cut(const int *c_tile_nnz, int cs0, int cs1, int P0, int t)
{
    if (t >= cs1)
        return false;
    if (t == cs0)
        return true;
    return (__ldg(c_tile_nnz + t) - P0) / GLOB_H != (__ldg(c_tile_nnz + t - 1) - P0) / GLOB_H;
}

// One warp per C tile row: decide heavy or not, and queue the windows of a
// heavy one.  heavy[I] = 1 tells the numeric kernel's CTA for I to exit.
template <int ACC, int GMODE = 0>
__global__ void __launch_bounds__(PLAN_WARPS * 32)
    k_win_plan(int tilem, int m, DevTiles A, DevTiles B,
               const int *__restrict__ c_tile_ptr, const int *__restrict__ c_tile_col,
               const int *__restrict__ c_tile_nnz,
               const uint16_t *__restrict__ c_mask, const int *__restrict__ csr_rowptr,
               uint8_t *__restrict__ heavy, WinTask *__restrict__ tasks, int cap,
               long long target, WinQueue *q, long long *counters)
{
    const int lane = lane_id();
    const int I = blockIdx.x * PLAN_WARPS + (threadIdx.x >> 5);
    if (I >= tilem)
        return;
    const int cs0 = __ldg(c_tile_ptr + I), cs1 = __ldg(c_tile_ptr + I + 1);
    const int a0 = __ldg(A.tile_ptr + I), a1 = __ldg(A.tile_ptr + I + 1);
    bool multi = false;
    if (cs1 > cs0 && a0 < a1)
    {
        const int E = __ldg(c_tile_nnz + cs1) - __ldg(c_tile_nnz + cs0);
        multi = cs1 - cs0 > F_SLOT_CAP || E > ACC;
        if (multi && cs1 - cs0 <= F_SLOT_CAP && csr_rowptr != nullptr)
        {
            // the numeric kernel's row windows: every warp's rows fit
            const int nrows = min(TD, m - I * TD);
            int pc = 0;
            if (lane < FW)
            {
                const int ra = min(lane * RPW, nrows), rb = min(lane * RPW + RPW, nrows);
                pc = __ldg(csr_rowptr + I * TD + rb) - __ldg(csr_rowptr + I * TD + ra);
            }
            multi = __any_sync(FULL, pc > ACC);
        }
    }
    if (!multi)
    {
        if (lane == 0)
            heavy[I] = 0;
        return;
    }
    const int P0 = __ldg(c_tile_nnz + cs0);
    constexpr bool GLOB = GMODE != 0;
    auto cuts = [&](int t) {
        return GMODE == 2   ? glob2_cut(c_tile_col, cs0, cs1, t)
               : GMODE == 1 ? glob_cut(c_tile_nnz, cs0, cs1, P0, t)
                            : win_cut<ACC>(c_tile_nnz, cs0, cs1, P0, t);
    };
    int nwin = 0;
    for (int t0 = cs0; t0 < cs1; t0 += 32)
        nwin += __popc(__ballot_sync(FULL, cuts(t0 + lane)));
    if (GMODE == 2)
    {
        // only rows that the shared-memory kernel would walk in many windows
        // go to device memory: a row of a few windows keeps its CTA (the
        // atomic adds cost more than its re-walks)
        int nstd = 0;
        for (int t0 = cs0; t0 < cs1; t0 += 32)
            nstd += __popc(__ballot_sync(FULL, win_cut<ACC>(c_tile_nnz, cs0, cs1, P0, t0 + lane)));
        if (nstd < GLOB_MIN_WINDOWS)
        {
            if (lane == 0)
                heavy[I] = 0;
            return;
        }
    }
    // Cost of one window: the tile row's products, since every window walks
    // all of them (the cost model of the reference's tail queue, products
    // standing in for its scan/match terms).  A task takes g consecutive
    // windows, about SPLIT_TARGET products of walking; a row whose windows all
    // fit one task keeps its own CTA and the L1 reuse of its B rows.
    long long P = 0;
    if (GLOB)
        ; // one task per run of GLOB_H entries: no grouping of windows
    else if (A.csr_rowptr != nullptr && A.csr_col != nullptr)
    {
        // the tile row's entries straight from A's CSR rows
        const int e0 = __ldg(A.csr_rowptr + I * TD), e1 = __ldg(A.csr_rowptr + min(A.m, I * TD + TD));
        for (int e = e0 + lane; e < e1; e += 32)
        {
            const int k = __ldg(A.csr_col + e);
            if (k < B.m)
                P += __ldg(B.csr_rowptr + k + 1) - __ldg(B.csr_rowptr + k);
        }
    }
    else
        for (int t = a0 + lane; t < a1; t += 32)
        {
            const int e0 = __ldg(A.tile_nnz + t), e1 = __ldg(A.tile_nnz + t + 1);
            const int K = __ldg(A.tile_col + t);
            for (int e = e0; e < e1; ++e)
            {
                const int k = K * TD + (A.col[e] & 15);
                if (k < B.m)
                    P += __ldg(B.csr_rowptr + k + 1) - __ldg(B.csr_rowptr + k);
            }
        }
    P = warp_sum(P);
    const int g = GLOB ? 1 : (int)max(1ll, min((long long)nwin, target / max(P, 1ll)));
    const int ntask = (nwin + g - 1) / g;
    int base = -1;
    // globally accumulated rows are queued even as a single task: their CTA
    // would walk the entries once per shared-memory window
    if ((GLOB ? ntask >= 1 : ntask >= 2) && lane == 0)
    {
        // room for all the tasks, or none at all (then the row keeps its own CTA)
        int old = *(volatile int *)&q->count;
        for (int it = 0; it < (1 << 20); ++it)
        {
            if (old + ntask > cap)
                break;
            const int seen = atomicCAS(&q->count, old, old + ntask);
            if (seen == old)
            {
                base = old;
                break;
            }
            old = seen;
        }
        if (base < 0)
            q->overflow = 1;
        else if (counters != nullptr)
        {
            atomicAdd((unsigned long long *)&counters[2], (unsigned long long)ntask);
            // tasks of two or more windows (the last task holds the remainder)
            const int last = nwin - (ntask - 1) * g;
            const int multi_tasks = g >= 2 ? ntask - (last < 2 ? 1 : 0) : 0;
            if (multi_tasks > 0)
                atomicAdd((unsigned long long *)&counters[3], (unsigned long long)multi_tasks);
        }
    }
    base = __shfl_sync(FULL, base, 0);
    if (lane == 0)
        heavy[I] = base >= 0;
    if (base < 0)
        return;
    // the tasks: window bounds and the rows' entries before each window
    int run[TD];
#pragma unroll
    for (int r = 0; r < TD; ++r)
        run[r] = 0;
    int widx = base, nw = 0; // tasks written, windows seen
    for (int t0 = cs0; t0 < cs1; t0 += 32)
    {
        const int t = t0 + lane;
        const bool cut = cuts(t);
        const unsigned wbal = __ballot_sync(FULL, cut);
        // a task starts at every g-th window
        const bool start = cut && (nw + __popc(wbal & ((1u << lane) - 1u))) % g == 0;
        nw += __popc(wbal);
        uint32_t w[TD / 2];
        if (t < cs1)
        {
            const uint4 *mp = reinterpret_cast<const uint4 *>(c_mask + (size_t)t * TD);
            const uint4 u0 = __ldg(mp), u1 = __ldg(mp + 1);
            w[0] = u0.x, w[1] = u0.y, w[2] = u0.z, w[3] = u0.w;
            w[4] = u1.x, w[5] = u1.y, w[6] = u1.z, w[7] = u1.w;
        }
        else
        {
#pragma unroll
            for (int p = 0; p < TD / 2; ++p)
                w[p] = 0u;
        }
        // per row pair: two 16-bit counts in one word (a chunk adds <= 512)
        int excl[TD / 2], tot[TD / 2];
#pragma unroll
        for (int p = 0; p < TD / 2; ++p)
        {
            const int pc = __popc(w[p] & 0xFFFFu) | (__popc(w[p] >> 16) << 16);
            const int incl = warp_incl_scan(pc);
            excl[p] = incl - pc;
            tot[p] = __shfl_sync(FULL, incl, 31);
        }
        const unsigned bal = __ballot_sync(FULL, start);
        if (start)
        {
            WinTask *tk = tasks + widx + __popc(bal & ((1u << lane) - 1u));
            tk->I = I;
            tk->w0 = t;
            tk->pad = 0;
            const unsigned later = lane == 31 ? 0u : bal & (0xFFFFFFFFu << (lane + 1));
            if (later) // the task ends at the next start in this chunk
                tk->w1 = t0 + __ffs(later) - 1;
#pragma unroll
            for (int p = 0; p < TD / 2; ++p)
            {
                tk->run[2 * p] = run[2 * p] + (excl[p] & 0xFFFF);
                tk->run[2 * p + 1] = run[2 * p + 1] + (excl[p] >> 16);
            }
        }
        // the last task of the chunks before ends at this chunk's first start
        if (bal != 0u && widx > base && lane == __ffs(bal) - 1)
            tasks[widx - 1].w1 = t;
        widx += __popc(bal);
#pragma unroll
        for (int p = 0; p < TD / 2; ++p)
        {
            run[2 * p] += tot[p] & 0xFFFF;
            run[2 * p + 1] += tot[p] >> 16;
        }
    }
    if (lane == 0)
        tasks[widx - 1].w1 = cs1;
}

// WORKER: the persistent CTAs that take window tasks from the queue (launched
// on a second stream, ahead of the tile-row CTAs); otherwise one CTA per C
// tile row, which exits if its row was split.  NARROW: some tile row has
// several windows, so long sorted B rows are cut to each window's columns
// (compiled out when every tile row fits one window: the registers are the
// kernel's limit).
template <bool SAFE, int ACC, int MIN_CTAS, bool WORKER, bool NARROW, bool ACSR, bool SEGW = false,
          bool PERSIST = false>
__global__ void __launch_bounds__(F_THREADS, MIN_CTAS)
    k_numeric_flat(DevTiles A, DevTiles B, int tilem, long long nnzC,
                   const int *__restrict__ c_tile_ptr, const int *__restrict__ c_tile_col,
                   const uint16_t *__restrict__ c_mask, const int *__restrict__ c_tile_nnz,
                   uint8_t *__restrict__ c_ptr, uint8_t *__restrict__ c_colb,
                   double *__restrict__ c_val, const int *__restrict__ csr_rowptr,
                   int *__restrict__ csr_col, double *__restrict__ csr_val, long long *counters,
                   int *err, const uint8_t *__restrict__ heavy, const WinTask *__restrict__ tasks,
                   WinQueue *q, int *__restrict__ cursors)
{
    extern __shared__ __align__(128) unsigned char dyn[];
    FlatSmem<ACC> &S = *reinterpret_cast<FlatSmem<ACC> *>(dyn);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = warp * RPW, r1 = r0 + RPW - 1;
    long long n_fma = 0;
    int4 *ent = S.ent[warp];
    double *enta = S.enta[warp];
    constexpr bool worker = WORKER;
    for (;;)
    {
        int I, wbeg = 0, wend = 0;
        if (worker)
        {
            __syncthreads(); // the previous task is done with shared memory
            if (tid == 0)
                S.task = atomicAdd(&q->head, 1);
            __syncthreads();
            const int tk = S.task;
            if (tk >= __ldg(&q->count))
                break;
            I = __ldg(&tasks[tk].I);
            wbeg = __ldg(&tasks[tk].w0);
            wend = __ldg(&tasks[tk].w1);
            if (tid < TD)
                S.rowrun[tid] = __ldg(&tasks[tk].run[tid]);
            if (I < 0 || I >= tilem)
                break; // not a task of this product (uniform)
        }
        else if (PERSIST)
        {
            // persistent tile-row CTAs: the next tile row from the queue
            // (every instance of a batch: its block diagonal's tile rows)
            __syncthreads(); // the previous tile row is done with shared memory
            if (tid == 0)
                S.task = atomicAdd(&q->next, 1);
            __syncthreads();
            I = S.task;
            if (I >= tilem)
                break;
            if (heavy != nullptr && heavy[I])
                continue; // a split row: the workers take its windows
        }
        else
        {
            I = blockIdx.x;
            if (I >= tilem || (heavy != nullptr && heavy[I]))
                break;
        }
        const int a0 = __ldg(A.tile_ptr + I), a1 = __ldg(A.tile_ptr + I + 1);
        const int cs0 = __ldg(c_tile_ptr + I), cs1 = __ldg(c_tile_ptr + I + 1);
        if (cs0 == cs1 || a0 == a1)
        {
            if (PERSIST)
                continue;
            break; // no C tiles in this tile row (uniform)
        }
        if (!worker)
        {
            wbeg = cs0;
            wend = cs1;
            if (tid < TD)
                S.rowrun[tid] = 0;
        }
        else if (wbeg < cs0 || wend > cs1)
            break;
        const int nrows = min(TD, A.m - I * TD);

        // Row windows: a tile row with more entries than the accumulator holds,
        // but few enough C tiles for one slot table, is processed in groups of
        // warps (row pairs) whose entries fit - every product is computed once,
        // warps outside the group wait, and the SM's other CTAs use the issue
        // slots.  Otherwise (or for the tile output) windows of C tiles are used
        // and the warps walk their A entries once per window.
        // (window state lives in shared memory: registers are the kernel's limit)
        if (tid == 0)
        {
            S.rowwin = 0;
            S.win_begin = 0;
            S.win_end = FW;
        }
        if (!worker && c_val == nullptr && csr_rowptr != nullptr && cs1 - cs0 <= F_SLOT_CAP &&
            __ldg(c_tile_nnz + cs1) - __ldg(c_tile_nnz + cs0) > ACC)
        {
            if (tid < FW)
            {
                const int ra = min(tid * RPW, nrows), rb = min(tid * RPW + RPW, nrows);
                S.paircnt[tid] = __ldg(csr_rowptr + I * TD + rb) - __ldg(csr_rowptr + I * TD + ra);
            }
            const int ok = __syncthreads_and(tid >= FW || S.paircnt[tid] <= ACC);
            if (tid == 0)
                S.rowwin = ok;
        }
        __syncthreads();

        for (int w0 = wbeg; w0 < wend;)
        {
            int nW;
            if (S.rowwin)
            {
                // ---- row window: warps [win_begin, win_end), all C tiles of the tile row
                if (tid == 0)
                {
                    const int wa = S.win_begin;
                    int e = wa + 1, sum = S.paircnt[wa];
                    while (e < FW && sum + S.paircnt[e] <= ACC)
                        sum += S.paircnt[e++];
                    S.win_end = e;
                }
                __syncthreads();
                nW = cs1 - cs0;
            }
            else
            {
                // ---- window [w0, w1): longest run of <= F_SLOT_CAP tiles, <= ACC entries
                const int base_nnz = __ldg(c_tile_nnz + w0);
                bool ok = false;
                if (tid < F_SLOT_CAP && w0 + tid < wend)
                    ok = __ldg(c_tile_nnz + w0 + tid + 1) - base_nnz <= ACC;
                nW = __syncthreads_count(ok);
                if (nW == 0)
                {
                    if (tid == 0)
                        set_error(err, DERR_NUM_BOUNDS); // a C tile holds at most 256 entries
                    return;
                }
            }
            const int w1 = w0 + nW;
            {
                // two rows' masks per 32-bit word (c_mask rows are 32-byte aligned per tile)
                const uint32_t *src = reinterpret_cast<const uint32_t *>(c_mask + (size_t)w0 * TD);
                for (int i = tid; i < nW * (TD / 2); i += F_THREADS)
                {
                    const int s = i >> 3, r = (i & 7) * 2;
                    // rows outside the row window count as empty
                    const bool in = r / RPW >= S.win_begin && r / RPW < S.win_end;
                    const uint32_t v = in ? __ldg(src + i) : 0u;
                    S.cm[r * F_CM_STRIDE + s] = v & 0xFFFFu;
                    S.cm[(r + 1) * F_CM_STRIDE + s] = v >> 16;
                }
            }
            for (int i = tid; i < nW; i += F_THREADS)
                S.cJ[i] = __ldg(c_tile_col + w0 + i);
            {
                // the slot table covers the window's tile-column span only
                const int span = __ldg(c_tile_col + w1 - 1) - __ldg(c_tile_col + w0) + 1;
                for (int i = tid; i < min((span + 3) / 4, F_SPAN_CAP / 4); i += F_THREADS)
                    reinterpret_cast<uint32_t *>(S.slot8)[i] = 0xFFFFFFFFu;
            }
            __syncthreads();
            Window W;
            W.Jlo = S.cJ[0];
            W.Jspan = S.cJ[nW - 1] - W.Jlo;
            W.nW = nW;
            W.table = W.Jspan < F_SPAN_CAP;
            if (W.table)
                for (int i = tid; i < nW; i += F_THREADS)
                    S.slot8[S.cJ[i] - W.Jlo] = (uint8_t)i;
            // accumulator bases: (row r, slot s) starts at the entries of rows < r
            // plus those of row r in slots < s.  Thread (r = tid / 16, part =
            // tid % 16) owns a run of slots: sum, half-warp scan, write.
            {
                static_assert(F_THREADS == TD * 16, "one half-warp per row");
                const int r = tid >> 4, part = tid & 15;
                const int per = (nW + 15) >> 4;
                const int s0 = min(part * per, nW), s1 = min(s0 + per, nW);
                uint32_t *cmr = S.cm + r * F_CM_STRIDE;
                int sum = 0;
                for (int s = s0; s < s1; ++s)
                    sum += __popc(cmr[s]);
                const int incl = half_incl_scan(sum);
                if (part == 15)
                    S.rowtot[r] = incl;
                __syncthreads();
                int racc = 0; // entries of rows < r
                for (int q = 0; q < r; ++q)
                    racc += S.rowtot[q];
                if (tid == 0)
                {
                    int t = 0;
                    for (int q = 0; q < TD; ++q)
                    {
                        S.rowacc0[q] = t;
                        t += S.rowtot[q];
                    }
                    S.rowacc0[TD] = t;
                }
                int run = racc + incl - sum;
                for (int s = s0; s < s1; ++s)
                {
                    const uint32_t m = cmr[s];
                    cmr[s] = ((uint32_t)run << 16) | m;
                    run += __popc(m);
                }
            }
            if (tid < nrows && csr_rowptr != nullptr)
                S.rowcsr0[tid] = __ldg(csr_rowptr + I * TD + tid) + S.rowrun[tid];
            __syncthreads(); // rowacc0 complete
            for (int i = tid; i < S.rowacc0[TD]; i += F_THREADS)
                S.acc[i] = 0.0;
            __syncthreads();

            // ---- products: warp-private, no CTA barrier
            if (r0 < nrows && warp >= S.win_begin && warp < S.win_end)
            {
                // each pair counted once: in the first tile window, in its row window
                const bool count = S.rowwin || w0 == cs0;
                int *cur = nullptr;
                // the warp's entries in A's CSR (ACSR) and the tile row's first
                int e_a = 0, e_m = 0, e_e = 0, ebase = 0;
                if (ACSR)
                {
                    const int *rp = A.csr_rowptr + (size_t)I * TD;
                    ebase = __ldg(rp);
                    e_a = __ldg(rp + min(r0, nrows));
                    e_m = __ldg(rp + min(r1, nrows));
                    e_e = __ldg(rp + min(r1 + 1, nrows));
                }
                if (WORKER && cursors != nullptr)
                {
                    cur = cursors + (size_t)blockIdx.x * cursor_cap(A);
                    if (!ACSR)
                        ebase = __ldg(A.tile_nnz + a0);
                }
                if (SEGW && W.table && nW == cs1 - cs0)
                    n_fma += warp_products_seg<ACC>(S, W, A, B, r0, r1, e_a, e_m, e_e, count);
                else if (W.table && nW == cs1 - cs0)
                    n_fma += warp_products<SAFE, false, ACC, NARROW, ACSR>(
                        S, W, A, B, a0, a1, r0, r1, e_a, e_m, e_e, count, ent, enta, cur, ebase,
                        w0 == wbeg);
                else
                    n_fma += warp_products<SAFE, true, ACC, NARROW, ACSR>(
                        S, W, A, B, a0, a1, r0, r1, e_a, e_m, e_e, count, ent, enta, cur, ebase,
                        w0 == wbeg);
            }
            __syncthreads();

            // ---- write-out of the window: each warp its own rows
            if (csr_col != nullptr)
            {
#pragma unroll
                for (int rr = 0; rr < RPW; ++rr)
                {
                    const int r = r0 + rr;
                    if (r >= nrows)
                        break;
                    const int b0 = S.rowacc0[r], b1 = S.rowacc0[r + 1];
                    const long long dst = (long long)S.rowcsr0[r] - b0;
                    if (dst + b1 > nnzC)
                    {
                        if (lane == 0)
                            set_error(err, DERR_NUM_BOUNDS);
                        continue;
                    }
                    for (int p = b0 + lane; p < b1; p += 32)
                    {
                        csr_val[dst + p] = S.acc[p];
                        csr_col[dst + p] = S.ccol[p];
                    }
                }
            }
            if (c_val != nullptr)
            {
                for (int it = tid; it < nW * TD; it += F_THREADS)
                {
                    const int s = it >> 4, r = it & 15;
                    const uint32_t w = S.cm[r * F_CM_STRIDE + s];
                    const uint32_t m = w & 0xFFFFu;
                    const int abase = (int)(w >> 16);
                    const int t = w0 + s;
                    int pre = 0;
                    for (int rr = 0; rr < r; ++rr)
                        pre += __popc(S.cm[rr * F_CM_STRIDE + s] & 0xFFFFu);
                    c_ptr[(size_t)t * TD + r] = (uint8_t)pre;
                    const long long tpos = (long long)__ldg(c_tile_nnz + t) + pre;
                    uint32_t mm = m;
                    int k = 0;
                    while (mm)
                    {
                        const int c = __clz(mm) - 16;
                        mm &= ~(0x8000u >> c);
                        if (tpos + k >= nnzC)
                        {
                            set_error(err, DERR_NUM_BOUNDS);
                            break;
                        }
                        c_colb[tpos + k] = (uint8_t)c;
                        c_val[tpos + k] = S.acc[abase + k];
                        ++k;
                    }
                }
            }
            __syncthreads();
            if (tid < TD)
                S.rowrun[tid] += S.rowtot[tid];
            __syncthreads();
            if (S.rowwin)
            {
                if (S.win_end >= FW)
                    break;
                __syncthreads(); // every thread has read win_end
                if (tid == 0)
                    S.win_begin = S.win_end;
                __syncthreads();
            }
            else
                w0 = w1;
        }
        if (!worker && !PERSIST)
            break;
    }
    if (counters != nullptr)
    {
        // n_fma: each lane counted the B row lengths of its own entries
        const long long nf = warp_sum(n_fma);
        if (lane == 0 && nf)
            atomicAdd((unsigned long long *)&counters[1], (unsigned long long)nf);
    }
}


// Workers of globally accumulated heavy tile rows (NumericConfig::global_rows):
// persistent CTAs take the tasks k_win_plan<..., true> queued - runs of
// consecutive C tiles of a heavy row - and accumulate their products in C's
// CSR value array itself.  Per task, in the CTA's slice of the scratch
// arrays: the tile column -> task tile table, and per (task tile, row) the
// row's entries before that tile (a scan of the masks' popcounts, from the
// task's own per-row start); the task's entries get their columns and a zero
// value.  Then each warp walks its two rows' A entries in column order, each
// B row cut to the task's columns by two binary searches, and adds every
// product at position row start + entries before the tile + entries before
// the column in the tile.  A row belongs to one warp and the warp takes its
// entries in order, with __syncwarp between entries (memory order among its
// lanes): every output is summed in the (K, k) order of the shared-memory
// kernel, by read-modify-write with fma, bitwise that kernel's result.
// Four pieces of an entry's B row have their addresses loaded ahead of their
// adds.
__global__ void __launch_bounds__(F_THREADS)
    k_numeric_glob(DevTiles A, DevTiles B, int tilem, long long nnzC,
                   const int *__restrict__ c_tile_col, const uint16_t *__restrict__ c_mask,
                   const int *__restrict__ csr_rowptr, int *__restrict__ csr_col,
                   double *__restrict__ csr_val, const WinTask *__restrict__ tasks, WinQueue *q,
                   int cap, int tilen, int *__restrict__ slot_all, int *__restrict__ rel_all,
                   int *err)
{
    __shared__ int s_tk, s_I, s_w0, s_w1;
    __shared__ int s_run[TD], s_rp[TD + 1], s_ea[TD + 1];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int *slot = slot_all + (size_t)blockIdx.x * tilen;
    int *rel = rel_all + (size_t)blockIdx.x * GLOB_RELCAP * TD;
    const int ntasks = min(*(volatile int *)&q->count, cap);
    for (;;)
    {
        __syncthreads(); // the previous task is done with the scratch arrays
        if (tid == 0)
            s_tk = atomicAdd(&q->head, 1);
        __syncthreads();
        const int tk = s_tk;
        if (tk >= ntasks)
            break;
        if (tid == 0)
        {
            s_I = __ldg(&tasks[tk].I);
            s_w0 = __ldg(&tasks[tk].w0);
            s_w1 = __ldg(&tasks[tk].w1);
        }
        if (tid < TD)
            s_run[tid] = __ldg(&tasks[tk].run[tid]);
        __syncthreads();
        const int I = s_I, w0 = s_w0, w1 = s_w1, nt = w1 - w0;
        if (I < 0 || I >= tilem || nt <= 0 || nt > GLOB_RELCAP)
        {
            if (tid == 0)
                set_error(err, DERR_WINDOW);
            break; // uniform
        }
        const int nrows = min(TD, A.m - I * TD);
        if (tid <= nrows)
        {
            s_rp[tid] = __ldg(csr_rowptr + I * TD + tid);
            s_ea[tid] = __ldg(A.csr_rowptr + I * TD + tid);
        }
        for (int i = tid; i < nt; i += F_THREADS)
        {
            const int J = __ldg(c_tile_col + w0 + i);
            if ((unsigned)J < (unsigned)tilen)
                slot[J] = i;
        }
        __syncthreads();
        // per (task tile, row): entries of the row before the tile; the task's
        // entries get their columns and a zero value (warp w: rows 2w, 2w + 1)
        for (int rr = 0; rr < RPW; ++rr)
        {
            const int r = warp * RPW + rr;
            if (r >= nrows)
                break; // warp-uniform
            int carry = s_run[r];
            for (int c0 = 0; c0 < nt; c0 += 32)
            {
                const int i = c0 + lane;
                const uint32_t m = i < nt ? (uint32_t)__ldg(c_mask + (size_t)(w0 + i) * TD + r) : 0u;
                const int pc = __popc(m);
                const int incl = warp_incl_scan(pc);
                const int off = carry + incl - pc;
                if (i < nt)
                {
                    rel[i * TD + r] = off;
                    const int J = __ldg(c_tile_col + w0 + i);
                    const long long pos = (long long)s_rp[r] + off;
                    uint32_t mm = m;
                    for (int k = 0; mm != 0u; ++k)
                    {
                        const int c = __clz(mm) - 16;
                        mm &= ~(0x8000u >> c);
                        if (pos + k >= nnzC)
                        {
                            set_error(err, DERR_NUM_BOUNDS);
                            break;
                        }
                        csr_col[pos + k] = J * TD + c;
                        csr_val[pos + k] = 0.0;
                    }
                }
                carry += __shfl_sync(FULL, incl, 31);
            }
        }
        __syncthreads();
        // products: the warp's rows, entries in column order
        const int r0 = warp * RPW, r1 = r0 + RPW - 1;
        if (r0 < nrows)
        {
            const int lo = __ldg(c_tile_col + w0) * TD, hi = (__ldg(c_tile_col + w1 - 1) + 1) * TD;
            const int e_a = s_ea[r0], e_m = s_ea[min(r0 + 1, nrows)], e_e = s_ea[min(r1 + 1, nrows)];
            for (int q0 = e_a; q0 < e_e; q0 += 32)
            {
                const int e = q0 + lane;
                int fs = 0, len = 0, rq = r0;
                double a = 0.0;
                if (e < e_e)
                {
                    const int k = __ldg(A.csr_col + e);
                    a = __ldg(A.csr_val + e);
                    rq = e < e_m ? r0 : r1;
                    if (k >= 0 && k < B.m)
                    {
                        const int f0 = min(max(__ldg(B.csr_rowptr + k), 0), B.nnz);
                        const int f1 = min(max(__ldg(B.csr_rowptr + k + 1), f0), B.nnz);
                        fs = lower_bound(B.csr_col, f0, f1, lo);
                        len = lower_bound(B.csr_col, fs, f1, hi) - fs;
                    }
                }
                // items of at most 32 products: entry j's B row in pieces of 32
                const unsigned live = __ballot_sync(FULL, len > 0);
                for (unsigned lv = live; lv != 0u; lv &= lv - 1u)
                {
                    const int j = __ffs(lv) - 1;
                    const int jfs = __shfl_sync(FULL, fs, j), jlen = __shfl_sync(FULL, len, j);
                    const int jr = __shfl_sync(FULL, rq, j);
                    const double ja = __shfl_sync(FULL, a, j);
                    const long long rbase = s_rp[jr];
                    for (int f0 = 0; f0 < jlen; f0 += 4 * 32)
                    {
                        long long pos[4];
                        double prod[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                        {
                            pos[u] = -1;
                            prod[u] = 0.0;
                            const int f = f0 + u * 32 + lane;
                            if (f < jlen)
                            {
                                const int col = __ldg(B.csr_col + jfs + f);
                                const double b = __ldg(B.csr_val + jfs + f);
                                const int J = col >> 4, c = col & 15;
                                const int sl = (unsigned)J < (unsigned)tilen ? slot[J] : -1;
                                if ((unsigned)sl < (unsigned)nt)
                                {
                                    const uint32_t w = __ldg(c_mask + (size_t)(w0 + sl) * TD + jr);
                                    if (w & (0x8000u >> c))
                                    {
                                        pos[u] = rbase + rel[sl * TD + jr] + __popc(w >> (16 - c));
                                        prod[u] = b;
                                    }
                                }
                                if (pos[u] < 0 || pos[u] >= nnzC)
                                {
                                    set_error(err, DERR_NUM_BOUNDS);
                                    pos[u] = -1;
                                }
                            }
                        }
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            if (pos[u] >= 0)
                                __stcg(csr_val + pos[u], fma(ja, prod[u], __ldcg(csr_val + pos[u])));
                    }
                    __syncwarp(); // this entry's adds before the next entry's
                }
            }
        }
    }
}


// The atomic form of the global-row workers (global_rows = 2): a task's
// tile column -> tile table (a shared-memory hash) and per (tile, row)
// word (entries of the row before the tile within the task << 16 | row mask)
// live in shared memory, so a product costs two shared loads and one atomic
// add into C's value array.  The task's A entries are shared by all warps
// (32 at a time, each entry's row found among the 16 row starts), so a hub
// row does not leave seven warps waiting; products of one output then come
// from several warps in no fixed order, and the values agree with the other
// kernels to the FP64 bound, not bit for bit.
__global__ void __launch_bounds__(F_THREADS)
    k_numeric_glob2(DevTiles A, DevTiles B, int tilem, long long nnzC,
                    const int *__restrict__ c_tile_col, const uint16_t *__restrict__ c_mask,
                    const int *__restrict__ csr_rowptr, int *__restrict__ csr_col,
                    double *__restrict__ csr_val, const WinTask *__restrict__ tasks, WinQueue *q,
                    int cap, int *err)
{
    extern __shared__ __align__(16) unsigned char g2_raw[];
    uint32_t *s_cm = reinterpret_cast<uint32_t *>(g2_raw);  // GNT * TD words
    int *s_hk = reinterpret_cast<int *>(s_cm + GNT * TD);   // GHASH tile columns (-1: empty)
    uint16_t *s_hv = reinterpret_cast<uint16_t *>(s_hk + GHASH); // their task tiles
    __shared__ int s_tk, s_I, s_w0, s_w1, s_jlo;
    __shared__ int s_run[TD], s_rp[TD + 1], s_ea[TD + 1];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ntasks = min(*(volatile int *)&q->count, cap);
    for (;;)
    {
        __syncthreads(); // the previous task is done with shared memory
        if (tid == 0)
            s_tk = atomicAdd(&q->head, 1);
        __syncthreads();
        const int tk = s_tk;
        if (tk >= ntasks)
            break;
        if (tid == 0)
        {
            s_I = __ldg(&tasks[tk].I);
            s_w0 = __ldg(&tasks[tk].w0);
            s_w1 = __ldg(&tasks[tk].w1);
            s_jlo = __ldg(c_tile_col + s_w0);
        }
        if (tid < TD)
            s_run[tid] = __ldg(&tasks[tk].run[tid]);
        __syncthreads();
        const int I = s_I, w0 = s_w0, w1 = s_w1, nt = w1 - w0, jlo = s_jlo;
        const int jspan = nt > 0 ? __ldg(c_tile_col + w1 - 1) - jlo + 1 : 0;
        if (I < 0 || I >= tilem || nt <= 0 || nt > GNT)
        {
            if (tid == 0)
                set_error(err, DERR_WINDOW);
            break; // uniform
        }
        const int nrows = min(TD, A.m - I * TD);
        if (tid <= nrows)
        {
            s_rp[tid] = __ldg(csr_rowptr + I * TD + tid);
            s_ea[tid] = __ldg(A.csr_rowptr + I * TD + tid);
        }
        for (int i = tid; i < GHASH; i += F_THREADS)
            s_hk[i] = -1;
        __syncthreads();
        for (int i = tid; i < nt; i += F_THREADS)
        {
            // the task's tile columns are distinct: linear probing finds a free slot
            const int J = __ldg(c_tile_col + w0 + i);
            int h = glob2_hash(J);
            for (int p = 0; p < GHASH; ++p, h = (h + 1) & (GHASH - 1))
                if (atomicCAS(&s_hk[h], -1, J) == -1)
                {
                    s_hv[h] = (uint16_t)i;
                    break;
                }
        }
        // per (tile, row): entries before the tile in the task and the row
        // mask (a scan per row, warp w: rows 2w, 2w + 1) ...
        for (int rr = 0; rr < RPW; ++rr)
        {
            const int r = warp * RPW + rr;
            if (r >= nrows)
                break; // warp-uniform
            int carry = 0;
            for (int c0 = 0; c0 < nt; c0 += 32)
            {
                const int i = c0 + lane;
                const uint32_t m = i < nt ? (uint32_t)__ldg(c_mask + (size_t)(w0 + i) * TD + r) : 0u;
                const int pc = __popc(m);
                const int incl = warp_incl_scan(pc);
                if (i < nt)
                    s_cm[i * TD + r] = ((uint32_t)(carry + incl - pc) << 16) | m;
                carry += __shfl_sync(FULL, incl, 31);
            }
        }
        __syncthreads();
        // ... then the task's entries get their columns and a zero value,
        // all threads over the (tile, row) pairs (a hub row is shared out)
        for (int x = tid; x < nt * TD; x += F_THREADS)
        {
            const int i = x >> 4, r = x & 15;
            if (r >= nrows)
                continue;
            const uint32_t w = s_cm[i * TD + r];
            uint32_t mm = w & 0xFFFFu;
            if (mm == 0u)
                continue;
            const int J = __ldg(c_tile_col + w0 + i);
            const long long pos = (long long)s_rp[r] + s_run[r] + (w >> 16);
            for (int k = 0; mm != 0u; ++k)
            {
                const int c = __clz(mm) - 16;
                mm &= ~(0x8000u >> c);
                if (pos + k >= nnzC)
                {
                    set_error(err, DERR_NUM_BOUNDS);
                    break;
                }
                csr_col[pos + k] = J * TD + c;
                csr_val[pos + k] = 0.0;
            }
        }
        __syncthreads();
        // products: the task's A entries, 32 per warp at a time
        const int lo = jlo * TD, hi = (jlo + jspan) * TD;
        const int ea = s_ea[0], ee = s_ea[nrows];
        for (int q0 = ea + warp * 32; q0 < ee; q0 += F_THREADS)
        {
            const int e = q0 + lane;
            int fs = 0, len = 0, r = 0;
            double a = 0.0;
            if (e < ee)
            {
#pragma unroll
                for (int h = 8; h > 0; h >>= 1)
                    if (r + h < nrows && s_ea[r + h] <= e)
                        r += h;
                const int k = __ldg(A.csr_col + e);
                a = __ldg(A.csr_val + e);
                if (k >= 0 && k < B.m)
                {
                    const int f0 = min(max(__ldg(B.csr_rowptr + k), 0), B.nnz);
                    const int f1 = min(max(__ldg(B.csr_rowptr + k + 1), f0), B.nnz);
                    fs = lower_bound(B.csr_col, f0, f1, lo);
                    len = lower_bound(B.csr_col, fs, f1, hi) - fs;
                }
            }
            for (unsigned lv = __ballot_sync(FULL, len > 0); lv != 0u; lv &= lv - 1u)
            {
                const int j = __ffs(lv) - 1;
                const int jfs = __shfl_sync(FULL, fs, j), jlen = __shfl_sync(FULL, len, j);
                const int jr = __shfl_sync(FULL, r, j);
                const double ja = __shfl_sync(FULL, a, j);
                const long long rbase = (long long)s_rp[jr] + s_run[jr];
                for (int f = lane; f < jlen; f += 32)
                {
                    const int col = __ldg(B.csr_col + jfs + f);
                    const double b = __ldg(B.csr_val + jfs + f);
                    const int J = col >> 4, c = col & 15;
                    int sl = -1;
                    int h = glob2_hash(J);
                    for (int p = 0; p < GHASH; ++p, h = (h + 1) & (GHASH - 1))
                    {
                        const int key = s_hk[h];
                        if (key == J)
                        {
                            sl = s_hv[h];
                            break;
                        }
                        if (key < 0)
                            break;
                    }
                    if ((unsigned)sl >= (unsigned)nt) // a column of no task tile: cannot happen
                    {
                        set_error(err, DERR_NUM_BOUNDS);
                        continue;
                    }
                    const uint32_t w = s_cm[sl * TD + jr];
                    const long long pos = rbase + (w >> 16) + __popc((w & 0xFFFFu) >> (16 - c));
                    if ((w & (0x8000u >> c)) == 0u || pos >= nnzC)
                    {
                        set_error(err, DERR_NUM_BOUNDS);
                        continue;
                    }
                    atomicAdd(csr_val + pos, ja * b);
                }
            }
        }
    }
}

} // namespace

int numeric_flat_device(Workspace &ws, const DevTiles &A, const DevTiles &B, SymbolicOut &S,
                        const NumericConfig &cfg)
{
    cudaStream_t s = ws.stream;
    const size_t nnz = (size_t)S.nnz;
    if (cfg.write_tiles)
    {
        RTT_CHECK(S.c_col.ensure(nnz + 16, s));
        RTT_CHECK(S.c_val.ensure(sizeof(double) * nnz + 16, s));
    }
    if (cfg.csr_col != nullptr)
        RTT_CHECK(csr_rowptr_device(ws, S, cfg.csr_rowptr));
    if (S.numtile == 0 || S.tilem == 0)
        return RTT_OK;
    // window tasks of heavy tile rows: at most one per F_SLOT_CAP tiles, plus
    // two per ACC - 256 entries (a cut on the entry count), plus one per row
    const long long cap_ll = (long long)S.tilem + S.numtile / F_SLOT_CAP +
                             2 * S.nnz / (ACC_SMALL - 256) + 16;
    const int cap = (int)std::min<long long>(cap_ll, 1 << 26);
    RTT_CHECK(S.w_task.ensure(sizeof(WinTask) * (size_t)cap, s));
    RTT_CHECK(S.w_heavy.ensure((size_t)S.tilem + 16, s));
    RTT_CHECK(S.w_queue.ensure(sizeof(WinQueue), s));
    if (cfg.ev_begin != nullptr)
        RTT_CUDA(cudaEventRecord(cfg.ev_begin, s));
    const int *fused_rowptr = cfg.csr_col ? cfg.csr_rowptr : nullptr;
    // split and narrowing only matter when some tile row has several windows
    const bool split = cfg.split_target >= 0 && S.multi_window;
    // A's entries straight from its CSR rows when they are given (the device
    // path), else from its tiles
    const bool acsr = A.csr_rowptr != nullptr && A.csr_col != nullptr && A.csr_val != nullptr;
    const long long target = cfg.split_target > 0 ? cfg.split_target : SPLIT_TARGET;
    // heavy tile rows in global memory: fused CSR output, sorted B rows
    // without repeated columns, A from its CSR rows
    // (the per-CTA tile-column table limits it to at most 2^20 tile columns)
    const bool glob = split && cfg.global_rows > 0 && acsr && !cfg.conflict_safe &&
                      cfg.csr_col != nullptr && !cfg.write_tiles &&
                      (cfg.global_rows == 2 || S.tilen <= (1 << 20));
    if (split)
    {
        RTT_CUDA(cudaMemsetAsync(S.w_queue.p, 0, sizeof(WinQueue), s));
        auto plan = !glob                  ? k_win_plan<ACC_SMALL, 0>
                    : cfg.global_rows == 2 ? k_win_plan<ACC_SMALL, 2>
                                           : k_win_plan<ACC_SMALL, 1>;
        plan<<<(S.tilem + PLAN_WARPS - 1) / PLAN_WARPS, PLAN_WARPS * 32, 0, s>>>(
            S.tilem, S.m, A, B, S.c_tile_ptr.as<int>(), S.c_tile_col.as<int>(),
            S.c_tile_nnz.as<int>(),
            S.c_mask.as<uint16_t>(), fused_rowptr, S.w_heavy.as<uint8_t>(),
            S.w_task.as<WinTask>(), cap, target, S.w_queue.as<WinQueue>(), cfg.counters);
        ws.launches++;
    }
    auto launch = [&](auto kern, int grid, cudaStream_t st, size_t smem, int *cursors) -> int {
        RTT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, F_THREADS, smem, st>>>(
            A, B, S.tilem, S.nnz, S.c_tile_ptr.as<int>(), S.c_tile_col.as<int>(),
            S.c_mask.as<uint16_t>(), S.c_tile_nnz.as<int>(), S.c_ptr.as<uint8_t>(),
            cfg.write_tiles ? S.c_col.as<uint8_t>() : nullptr,
            cfg.write_tiles ? S.c_val.as<double>() : nullptr, fused_rowptr, cfg.csr_col,
            cfg.csr_val, cfg.counters, ws.err.as<int>(),
            split ? S.w_heavy.as<uint8_t>() : nullptr, S.w_task.as<WinTask>(),
            S.w_queue.as<WinQueue>(), cursors);
        ws.launches++;
        return RTT_OK;
    };
    const size_t smem = sizeof(FlatSmem<ACC_SMALL>);
    if (glob)
    {
        // the global-row workers, on the side stream beside the tile-row CTAs
        int per_sm = 0, sms = 0;
        RTT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws.device));
        RTT_CUDA(cudaEventRecord(ws.fork_ev, s));
        RTT_CUDA(cudaStreamWaitEvent(ws.side, ws.fork_ev, 0));
        if (cfg.global_rows == 2)
        {
            const size_t gsm = sizeof(uint32_t) * GNT * TD + sizeof(int) * GHASH +
                               sizeof(uint16_t) * GHASH;
            RTT_CUDA(cudaFuncSetAttribute(k_numeric_glob2,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsm));
            RTT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_numeric_glob2,
                                                                   F_THREADS, gsm));
            const int grid = std::max(1, per_sm * sms);
            k_numeric_glob2<<<grid, F_THREADS, gsm, ws.side>>>(
                A, B, S.tilem, S.nnz, S.c_tile_col.as<int>(), S.c_mask.as<uint16_t>(),
                fused_rowptr, cfg.csr_col, cfg.csr_val, S.w_task.as<WinTask>(),
                S.w_queue.as<WinQueue>(), cap, ws.err.as<int>());
        }
        else
        {
            auto gk = k_numeric_glob;
            RTT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gk, F_THREADS, 0));
            const int grid = std::max(1, per_sm * sms);
            const int tilen = std::max(S.tilen, 1);
            RTT_CHECK(S.g_slot.ensure(sizeof(int) * (size_t)grid * tilen, s));
            RTT_CHECK(S.g_rel.ensure(sizeof(int) * (size_t)grid * GLOB_RELCAP * TD, s));
            gk<<<grid, F_THREADS, 0, ws.side>>>(A, B, S.tilem, S.nnz, S.c_tile_col.as<int>(),
                                                S.c_mask.as<uint16_t>(), fused_rowptr, cfg.csr_col,
                                                cfg.csr_val, S.w_task.as<WinTask>(),
                                                S.w_queue.as<WinQueue>(), cap, tilen,
                                                S.g_slot.as<int>(), S.g_rel.as<int>(),
                                                ws.err.as<int>());
        }
        ws.launches++;
        RTT_CUDA(cudaEventRecord(ws.join_ev, ws.side));
    }
    else if (split)
    {
        // The workers go first, on the side stream, so that the split rows'
        // tasks start while the tile-row CTAs run (the reference's heavy grid
        // enqueued before its light grid, src/dmma_tile_early_split.h:13-27).
        // One wave of resident CTAs; with an empty queue they exit at once.
        auto wk = acsr ? (cfg.conflict_safe ? k_numeric_flat<true, ACC_SMALL, CTAS_SMALL, true, true, true>
                                            : k_numeric_flat<false, ACC_SMALL, CTAS_SMALL, true, true, true>)
                       : (cfg.conflict_safe ? k_numeric_flat<true, ACC_SMALL, CTAS_SMALL, true, true, false>
                                            : k_numeric_flat<false, ACC_SMALL, CTAS_SMALL, true, true, false>);
        int per_sm = 0, sms = 0;
        RTT_CUDA(cudaFuncSetAttribute(wk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        RTT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wk, F_THREADS, smem));
        RTT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws.device));
        const int grid = std::max(1, per_sm * sms);
        RTT_CHECK(S.w_cursor.ensure(sizeof(int) * (size_t)grid * cursor_cap(A), s));
        RTT_CUDA(cudaEventRecord(ws.fork_ev, s));
        RTT_CUDA(cudaStreamWaitEvent(ws.side, ws.fork_ev, 0));
        RTT_CHECK(launch(wk, grid, ws.side, smem, S.w_cursor.as<int>()));
        RTT_CUDA(cudaEventRecord(ws.join_ev, ws.side));
    }
    auto light =
        acsr ? (cfg.conflict_safe
                    ? (S.multi_window ? k_numeric_flat<true, ACC_SMALL, CTAS_SMALL, false, true, true>
                                      : k_numeric_flat<true, ACC_SMALL, CTAS_SMALL, false, false, true>)
                    : (S.multi_window ? k_numeric_flat<false, ACC_SMALL, CTAS_SMALL, false, true, true>
                                      : k_numeric_flat<false, ACC_SMALL, CTAS_SMALL, false, false, true>))
             : (cfg.conflict_safe
                    ? (S.multi_window ? k_numeric_flat<true, ACC_SMALL, CTAS_SMALL, false, true, false>
                                      : k_numeric_flat<true, ACC_SMALL, CTAS_SMALL, false, false, false>)
                    : (S.multi_window ? k_numeric_flat<false, ACC_SMALL, CTAS_SMALL, false, true, false>
                                      : k_numeric_flat<false, ACC_SMALL, CTAS_SMALL, false, false, false>));
    // B rows of at most SEGW_MAX segments, one window per tile row, no
    // repeated columns: the segment walk
    if (cfg.segment_walk && acsr && !cfg.conflict_safe && !S.multi_window && B.seg_ptr != nullptr &&
        B.seg != nullptr && B.max_row_segs > 0 && B.max_row_segs <= SEGW_MAX)
        light = k_numeric_flat<false, ACC_SMALL, CTAS_SMALL, false, false, true, true>;
    int light_grid = S.tilem;
    if (cfg.persistent_rows && !cfg.conflict_safe && acsr && light == (S.multi_window
            ? k_numeric_flat<false, ACC_SMALL, CTAS_SMALL, false, true, true>
            : k_numeric_flat<false, ACC_SMALL, CTAS_SMALL, false, false, true>))
    {
        // one wave of resident CTAs taking tile rows from a device queue
        light = S.multi_window
                    ? k_numeric_flat<false, ACC_SMALL, CTAS_SMALL, false, true, true, false, true>
                    : k_numeric_flat<false, ACC_SMALL, CTAS_SMALL, false, false, true, false, true>;
        int per_sm = 0, sms = 0;
        RTT_CUDA(cudaFuncSetAttribute(light, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        RTT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, light, F_THREADS, smem));
        RTT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws.device));
        light_grid = std::max(1, std::min(per_sm * sms, S.tilem));
        if (!split)
            RTT_CUDA(cudaMemsetAsync(S.w_queue.p, 0, sizeof(WinQueue), s));
    }
    RTT_CHECK(launch(light, light_grid, s, smem, nullptr));
    if (split)
        RTT_CUDA(cudaStreamWaitEvent(s, ws.join_ev, 0));
    if (cfg.ev_end != nullptr)
        RTT_CUDA(cudaEventRecord(cfg.ev_end, s));
    return RTT_OK;
}

int numeric_select_device(Workspace &ws, const DevTiles &A, const DevTiles &B, SymbolicOut &S,
                          const NumericConfig &cfg)
{
    if (cfg.dmma_pair_cutoff > 0 || cfg.b_staging)
        return numeric_rows_device(ws, A, B, S, cfg);
    return numeric_flat_device(ws, A, B, S, cfg);
}

} // namespace rtt
