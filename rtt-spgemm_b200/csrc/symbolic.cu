// symbolic.cu - steps 1 and 2 of the tiled SpGEMM on sm_100a.
//
// Step 1 (reference spgemm_cpu step1/step2, src/spgemm-cpu.h:3-96, and the
// Super16 candidate step, src/super16_symbolic.cuh:973-1073): the C tiles of
// tile row I are the union over K in A.row(I) of the tile columns of B.row(K).
// One warp owns a tile row and builds the union as a bitmap over a window of
// tile columns in shared memory; the (A tile, B tile) pairs of the tile row
// are flattened across the 32 lanes so every lane issues independent loads.
// Windows wider than the bitmap are processed in passes.
//
// Step 2 (reference step3, src/spgemm-cpu.h:185-281, and the exact-mask step,
// src/super16_symbolic.cuh:1399-1662): the exact structure of every C tile as
// 16 row masks.  One CTA per tile row I: the CTA rebuilds the tile row's C
// tile list (the step-1 union, as a bitmap, compacted into a column -> slot
// table), then each warp ORs, for its two rows r and every A entry (r, k), the
// columns of B's CSR row k into the row masks of their C tiles - the same
// warp-private walk as the numeric step, with shared atomics on 32-bit words
// that hold the warp's two rows.  Tile rows with more C tiles than the slot
// table holds are processed in column windows.  Per-tile counts, per-row
// counts and the tile row total come out of the masks with popc.
#include "rtt_internal.cuh"

#include <climits>
#include <type_traits>

namespace rtt
{
namespace
{

constexpr int WWORDS = 256;             // bitmap words per warp -> 8192 tile columns
constexpr int WBITS = WWORDS * 32;
constexpr int SYM_WARPS = 4;            // warps per CTA

struct WarpSmem1
{
    uint32_t bitmap[WWORDS];
    int start[32];
    int pre[32];
};

constexpr int S2_WARPS = 8;              // warps per CTA, two rows each
constexpr int S2_THREADS = S2_WARPS * 32;
constexpr int S2_PAIRS = TD / 2;         // row pairs of a tile row
// Heavy tile rows (several windows and an R-MAT hub among their rows: one
// row pair with more than HEAVY_PAIR A entries and 2.5x the mean) run in a
// CTA of S2_HEAVY_WARPS warps that all share the walk.
constexpr int S2_HEAVY_WARPS = 32;
constexpr int HEAVY_PAIR = 1024;
constexpr int S2_SLOTS = 254;            // C tiles per window (slot 255 = none)
// The segment walk shares a tile row's entries over all warps of its CTA,
// so it needs no warp per row pair: 4-warp CTAs, twice as many per SM, hide
// the latency of the per-tile-row set-up phases better.
constexpr int S2_SEG_WARPS = 4;
constexpr int S2_STRIDE = 257;           // odd stride: the pairs' mask rows in distinct banks
// Wide windows: tile rows with more C tiles than S2_SLOTS (an R-MAT row's
// tens of thousands) walk their A entries once per window, so the tile rows
// step 1 lists as such run in CTAs whose slot table holds u16 slots, up to
// S2_WIDE_MAX C tiles per window (rtt_config.sym_window_slots; the mask rows
// after the fixed part of dynamic shared memory).
constexpr int S2_WIDE_DEFAULT = 2045;
constexpr int S2_WIDE_MAX = 6000; // the 32-warp CTA's mask rows within 227 KB

// Shared memory of a step-2 CTA; the mask rows (S2_PAIRS rows of `stride`
// words: per slot, row 2p in the low 16 bits and 2p + 1 in the high 16)
// follow it.
template <int NW, bool WIDE>
struct CtaSmem2
{
    using Slot = typename std::conditional<WIDE, uint16_t, uint8_t>::type;
    static constexpr int NONE = WIDE ? 0xFFFF : 0xFF;
    uint32_t bitmap[WWORDS];
    int wordpre[WWORDS];
    int4 ent[NW][32];                    // per warp: B row start, length, mask shift, mask row
    Slot slot[WBITS];                    // window column -> slot
    int lo, hi, nb, wend;
    int share;                           // the warps share the A entries (unbalanced rows)
    int rp[TD + 1];                      // the tile row's A row pointers (segment walk)
};

template <int NW, bool WIDE>
constexpr size_t smem2_bytes(int stride)
{
    return (sizeof(CtaSmem2<NW, WIDE>) + 15) / 16 * 16 + sizeof(uint32_t) * S2_PAIRS * (size_t)stride;
}

// First segment in [lo, hi) whose tile column is >= J (a row's segments are
// in increasing tile-column order).
__device__ __forceinline__ int seg_lower_bound(const unsigned long long *seg, int lo, int hi, int J)
{
    while (lo < hi)
    {
        const int mid = (lo + hi) >> 1;
        if ((long long)(__ldg(seg + mid) >> 16) < J)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Row pairs with very different A entry counts: with NW warps, the pair
// counts and whether one pair holds > 2.5x the mean (and > min_pair).
__device__ __forceinline__ bool skewed_pairs(const DevTiles &A, int I, int nrows, int lane,
                                             int min_pair)
{
    int pc = 0;
    if (lane < S2_PAIRS && A.csr_rowptr != nullptr)
    {
        const int ra = min(2 * lane, nrows), rb = min(2 * lane + 2, nrows);
        pc = __ldg(A.csr_rowptr + I * TD + rb) - __ldg(A.csr_rowptr + I * TD + ra);
    }
    int tot = pc;
    for (int o = 4; o > 0; o >>= 1)
        tot += __shfl_xor_sync(FULL, tot, o);
    return __any_sync(FULL, lane < S2_PAIRS && pc > min_pair && 2 * S2_PAIRS * pc > 5 * tot);
}

// Window bounds [lo, hi] of the tile columns reachable from tile row I.
// pairs: the (A tile, B tile) pairs of the tile row, the work of its bitmap.
__device__ __forceinline__ void row_window(const DevTiles &A, const DevTiles &B, int a0, int a1,
                                           int &lo, int &hi, long long &pairs)
{
    const int lane = lane_id();
    lo = INT_MAX;
    hi = -1;
    long long np = 0;
    for (int a = a0 + lane; a < a1; a += 32)
    {
        const int K = __ldg(A.tile_col + a);
        const int b0 = __ldg(B.tile_ptr + K), b1 = __ldg(B.tile_ptr + K + 1);
        if (b0 < b1)
        {
            lo = min(lo, __ldg(B.tile_col + b0));
            hi = max(hi, __ldg(B.tile_col + b1 - 1));
            np += b1 - b0;
        }
    }
    lo = warp_min(lo);
    hi = warp_max(hi);
    pairs = warp_sum(np);
}

// Mark in the bitmap every tile column of B.row(K), K in A.row(I), that lies
// in [w, wend).  Pairs are flattened over lanes, 32 A tiles at a time.
__device__ __forceinline__ void fill_bitmap(const DevTiles &A, const DevTiles &B, int a0, int a1,
                                            int w, int wend, bool clip, uint32_t *bitmap,
                                            int *s_start, int *s_pre)
{
    const int lane = lane_id();
    for (int c0 = a0; c0 < a1; c0 += 32)
    {
        const int a = c0 + lane;
        int s = 0, len = 0;
        if (a < a1)
        {
            const int K = __ldg(A.tile_col + a);
            const int b0 = __ldg(B.tile_ptr + K), b1 = __ldg(B.tile_ptr + K + 1);
            s = clip ? lower_bound(B.tile_col, b0, b1, w) : b0;
            const int e = clip ? lower_bound(B.tile_col, s, b1, wend) : b1;
            len = e - s;
        }
        const int incl = warp_incl_scan(len);
        s_start[lane] = s;
        s_pre[lane] = incl - len;
        const int total = __shfl_sync(FULL, incl, 31);
        __syncwarp();
        for (int p = lane; p < total; p += 32)
        {
            int lo = 0, hi = 31;
            while (lo < hi)
            {
                const int mid = (lo + hi + 1) >> 1;
                if (s_pre[mid] <= p)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const int J = __ldg(B.tile_col + s_start[lo] + (p - s_pre[lo]));
            const int off = J - w;
            atomicOr(&bitmap[off >> 5], 1u << (off & 31));
        }
        __syncwarp();
    }
}

// Step 1 of a tile row with more pairs than this goes to k_sym_count_wide:
// one warp would walk them alone while the rest of the grid has finished.
constexpr long long S1_WIDE_PAIRS = 1 << 16;
constexpr int S1_WIDE_WARPS = 16;

// Step-1 outcome of tile row I: C tiles, the step-2 window flag and the
// step-2 lists: heavy rows (heavy[I] = 1) and rows with more C tiles than
// one 254-slot window (heavy[I] = 2, for the wide-window CTAs).
__device__ __forceinline__ void step1_out(const DevTiles &A, int I, int count, int lo, int hi,
                                          int lane, int *cnt, int *multi, uint8_t *heavy,
                                          int *list, int *list_count, int *wlist,
                                          int *wlist_count)
{
    // step 2 will need more than one window for this tile row; with an
    // unbalanced row pair it becomes a heavy row (a wide CTA of its own)
    const bool multi_win = count > S2_SLOTS || (hi >= 0 && (long long)hi - lo + 1 > WBITS);
    const bool hv = multi_win && heavy != nullptr &&
                    skewed_pairs(A, I, min(TD, A.m - I * TD), lane, HEAVY_PAIR);
    const bool wide = !hv && count > S2_SLOTS && wlist != nullptr;
    if (lane == 0)
    {
        cnt[I] = count;
        if (multi_win)
            atomicOr(multi, 1);
        if (heavy != nullptr)
        {
            heavy[I] = hv ? 1 : wide ? 2 : 0;
            if (hv)
                list[atomicAdd(list_count, 1)] = I;
            else if (wide)
                wlist[atomicAdd(wlist_count, 1)] = I;
        }
    }
}

__global__ void __launch_bounds__(SYM_WARPS * 32)
    k_sym_count(DevTiles A, DevTiles B, int *cnt, int *multi, uint8_t *heavy, int *list,
                int *list_count, int *wide, int *wide_count, int *wlist, int *wlist_count)
{
    __shared__ WarpSmem1 sm[SYM_WARPS];
    const int lane = lane_id(), wi = threadIdx.x >> 5;
    const int I = blockIdx.x * SYM_WARPS + wi;
    if (I >= A.tilem)
        return;
    WarpSmem1 &S = sm[wi];
    const int a0 = __ldg(A.tile_ptr + I), a1 = __ldg(A.tile_ptr + I + 1);
    int lo, hi;
    long long pairs;
    row_window(A, B, a0, a1, lo, hi, pairs);
    if (pairs > S1_WIDE_PAIRS)
    {
        if (lane == 0)
            wide[atomicAdd(wide_count, 1)] = I;
        return;
    }
    int count = 0;
    if (hi >= 0)
    {
        const bool multi = (long long)hi - lo + 1 > WBITS;
        for (long long w = lo; w <= hi; w += WBITS)
        {
            const int wend = (int)min((long long)hi + 1, w + WBITS);
            const int nwords = (int)((wend - w + 31) >> 5);
            for (int i = lane; i < nwords; i += 32)
                S.bitmap[i] = 0;
            __syncwarp();
            fill_bitmap(A, B, a0, a1, (int)w, wend, multi, S.bitmap, S.start, S.pre);
            int c = 0;
            for (int i = lane; i < nwords; i += 32)
                c += __popc(S.bitmap[i]);
            count += warp_sum(c);
            __syncwarp();
        }
    }
    step1_out(A, I, count, lo, hi, lane, cnt, multi, heavy, list, list_count, wlist, wlist_count);
}

// Step 1 of the tile rows k_sym_count listed as wide: one CTA of
// S1_WIDE_WARPS warps per tile row (persistent CTAs over the list), the
// warps splitting its A tiles and OR-ing into one shared bitmap per window.
__global__ void __launch_bounds__(S1_WIDE_WARPS * 32)
    k_sym_count_wide(DevTiles A, DevTiles B, int *cnt, int *multi, uint8_t *heavy, int *list,
                     int *list_count, const int *wide, const int *wide_count, int *wlist,
                     int *wlist_count)
{
    __shared__ uint32_t bitmap[WWORDS];
    __shared__ int s_start[S1_WIDE_WARPS][32], s_pre[S1_WIDE_WARPS][32];
    __shared__ int s_lo, s_hi, s_count;
    const int tid = threadIdx.x, lane = lane_id(), wi = tid >> 5;
    const int n = *wide_count;
    for (int li = blockIdx.x; li < n; li += gridDim.x)
    {
        const int I = wide[li];
        const int a0 = __ldg(A.tile_ptr + I), a1 = __ldg(A.tile_ptr + I + 1);
        if (tid == 0)
        {
            s_lo = INT_MAX;
            s_hi = -1;
            s_count = 0;
        }
        __syncthreads();
        // this warp's share of the A tiles
        const int per = (a1 - a0 + S1_WIDE_WARPS - 1) / S1_WIDE_WARPS;
        const int b0 = min(a1, a0 + wi * per), b1 = min(a1, b0 + per);
        {
            int lo, hi;
            long long pairs;
            row_window(A, B, b0, b1, lo, hi, pairs);
            if (lane == 0 && hi >= 0)
            {
                atomicMin(&s_lo, lo);
                atomicMax(&s_hi, hi);
            }
        }
        __syncthreads();
        const int lo = s_lo, hi = s_hi;
        if (hi >= 0)
        {
            const bool clip = (long long)hi - lo + 1 > WBITS;
            for (long long w = lo; w <= hi; w += WBITS)
            {
                const int wend = (int)min((long long)hi + 1, w + WBITS);
                const int nwords = (int)((wend - w + 31) >> 5);
                for (int i = tid; i < nwords; i += S1_WIDE_WARPS * 32)
                    bitmap[i] = 0;
                __syncthreads();
                fill_bitmap(A, B, b0, b1, (int)w, wend, clip, bitmap, s_start[wi], s_pre[wi]);
                __syncthreads();
                int c = 0;
                for (int i = tid; i < nwords; i += S1_WIDE_WARPS * 32)
                    c += __popc(bitmap[i]);
                c = warp_sum(c);
                if (lane == 0 && c)
                    atomicAdd(&s_count, c);
                __syncthreads();
            }
        }
        if (wi == 0)
            step1_out(A, I, s_count, lo, hi, lane, cnt, multi, heavy, list, list_count, wlist,
                      wlist_count);
        __syncthreads(); // s_* are reset for the next tile row
    }
}

// Step 2.  Outputs per C tile: column, tile row, 16 row masks and entry
// count; per scalar row: entry count; per tile row: entry total.  NARROW:
// some tile row has several windows and B's rows are sorted, so long B rows
// are cut to each window's columns (compiled out otherwise: it costs the
// single-window walk registers and issue slots).  NW warps per CTA: 8 for
// the tile rows in order (a heavy one is skipped when heavy[] marks it), or
// S2_HEAVY_WARPS for the heavy rows of list[] (all warps share the walk).
template <bool NARROW, int NW, bool SEGS, bool WIDE = false>
__global__ void __launch_bounds__(NW * 32, NW == S2_WARPS ? (WIDE ? 2 : 5) : NW == S2_SEG_WARPS ? 10 : 1)
    k_sym_rows(DevTiles A, DevTiles B, const int *__restrict__ c_tile_ptr,
               int *__restrict__ c_tile_col, int *__restrict__ c_tile_row,
               uint16_t *__restrict__ c_mask, int *__restrict__ c_tile_cnt,
               int *__restrict__ c_row_cnt, int *__restrict__ c_tr_nnz, int *multi, int *err,
               const uint8_t *__restrict__ heavy, const int *__restrict__ list, int wide_slots)
{
    static_assert(NW == S2_WARPS || NW == S2_HEAVY_WARPS || (SEGS && NW == S2_SEG_WARPS),
                  "CTA shapes");
    constexpr int PPW = (S2_PAIRS + NW - 1) / NW; // row pairs each warp counts
    constexpr int NT = NW * 32;
    using Smem = CtaSmem2<NW, WIDE>;
    using Slot = typename Smem::Slot;
    constexpr int NONE = Smem::NONE;
    // slots per window and the odd stride of the mask rows
    const int NSLOT = WIDE ? wide_slots : S2_SLOTS;
    const int STRIDE = WIDE ? (wide_slots + 2) | 1 : S2_STRIDE;
    extern __shared__ __align__(16) unsigned char s2_raw[];
    Smem &S = *reinterpret_cast<Smem *>(s2_raw);
    uint32_t *const MW = reinterpret_cast<uint32_t *>(s2_raw + (sizeof(Smem) + 15) / 16 * 16);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int I = list != nullptr ? list[blockIdx.x] : (int)blockIdx.x;
    if (I >= A.tilem || (list == nullptr && heavy != nullptr && heavy[I]))
        return;
    const int a0 = __ldg(A.tile_ptr + I), a1 = __ldg(A.tile_ptr + I + 1);
    const int cbeg = __ldg(c_tile_ptr + I), cend = __ldg(c_tile_ptr + I + 1);
    const int nrows = min(TD, A.m - I * TD);
    const int r0 = warp * 2, r1 = r0 + 1; // warp-private walk (NW == S2_WARPS) and counts
    uint32_t *mw = MW + min(warp, S2_PAIRS - 1) * STRIDE;
    int4 *ent = S.ent[warp];
    int run[PPW][2] = {}; // entries so far of rows 2p, 2p + 1, pair p = warp + q * NW

    // tile-column range reachable from the tile row
    if (tid == 0)
    {
        S.lo = INT_MAX;
        S.hi = -1;
    }
    __syncthreads();
    {
        int lo = INT_MAX, hi = -1;
        for (int a = a0 + tid; a < a1; a += NT)
        {
            const int K = __ldg(A.tile_col + a);
            const int b0 = __ldg(B.tile_ptr + K), b1 = __ldg(B.tile_ptr + K + 1);
            if (b0 < b1)
            {
                lo = min(lo, __ldg(B.tile_col + b0));
                hi = max(hi, __ldg(B.tile_col + b1 - 1));
            }
        }
        lo = warp_min(lo);
        hi = warp_max(hi);
        if (lane == 0)
        {
            atomicMin(&S.lo, lo);
            atomicMax(&S.hi, hi);
        }
    }
    if (SEGS && tid <= nrows)
        S.rp[tid] = __ldg(A.csr_rowptr + I * TD + tid);
    __syncthreads();
    const int lo = S.lo, hi = S.hi;
    const bool clip = hi >= 0 && (long long)hi - lo + 1 > WBITS;
    if (!SEGS && NARROW && NW == S2_WARPS)
    {
        // Row pairs with very different A entry counts (an R-MAT hub row):
        // all warps share the walk.  Balanced rows keep the warp-private walk,
        // whose mask words no other warp touches.
        if (warp == 0)
        {
            const bool skew = skewed_pairs(A, I, nrows, lane, 32);
            if (lane == 0)
                S.share = skew;
        }
    }
    if (!SEGS && NW != S2_WARPS && tid == 0)
        S.share = 1;
    int cbase = cbeg;
    for (long long wl = lo; hi >= 0 && wl <= hi;)
    {
        const int w = (int)wl;
        int wend = (int)min((long long)hi + 1, wl + WBITS);
        const int nwords = (wend - w + 31) >> 5; // bitmap words the window can touch
        // ---- C tiles of the window: bitmap of the B tile columns in [w, wend)
        for (int i = tid; i < nwords; i += NT)
            S.bitmap[i] = 0u;
        __syncthreads();
        for (int a = a0 + warp; a < a1; a += NW)
        {
            const int K = __ldg(A.tile_col + a);
            int b0 = __ldg(B.tile_ptr + K), b1 = __ldg(B.tile_ptr + K + 1);
            if (clip)
            {
                b0 = lower_bound(B.tile_col, b0, b1, w);
                b1 = lower_bound(B.tile_col, b0, b1, wend);
            }
            for (int j = b0 + lane; j < b1; j += 32)
            {
                const int off = __ldg(B.tile_col + j) - w;
                atomicOr(&S.bitmap[off >> 5], 1u << (off & 31));
            }
        }
        __syncthreads();
        if (warp == 0)
        {
            int run = 0;
            for (int q0 = 0; q0 < nwords; q0 += 32)
            {
                const int v = q0 + lane < nwords ? __popc(S.bitmap[q0 + lane]) : 0;
                const int incl = warp_incl_scan(v);
                if (q0 + lane < nwords)
                    S.wordpre[q0 + lane] = run + incl - v;
                run += __shfl_sync(FULL, incl, 31);
            }
            if (lane == 0)
            {
                int nb = run, we = wend;
                if (nb > NSLOT)
                {
                    // cut the window after its NSLOT-th tile column
                    int q = 0;
                    while (S.wordpre[q] + __popc(S.bitmap[q]) < NSLOT)
                        ++q;
                    uint32_t bits = S.bitmap[q];
                    for (int k = S.wordpre[q]; k < NSLOT - 1; ++k)
                        bits &= bits - 1;
                    we = w + q * 32 + __ffs(bits); // one past the last kept column
                    nb = NSLOT;
                }
                S.nb = nb;
                S.wend = we;
            }
        }
        __syncthreads();
        const int nb = S.nb;
        wend = S.wend;
        const int wlen = wend - w;
        // one window of several: long sorted B rows are cut to its columns
        const bool narrow = NARROW && (w > lo || wend <= hi);
        if (cbase + nb > cend)
        {
            if (tid == 0)
                set_error(err, DERR_SYM_OVERFLOW);
            return;
        }
        constexpr int SPW = 4 / sizeof(Slot); // slots per 32-bit word
        for (int i = tid; i < (wlen + SPW - 1) / SPW; i += NT)
            reinterpret_cast<uint32_t *>(S.slot)[i] = 0xFFFFFFFFu;
        __syncthreads();
        for (int q = tid; q < nwords; q += NT)
        {
            uint32_t bits = S.bitmap[q];
            int slot = S.wordpre[q];
            while (bits)
            {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1;
                const int d = q * 32 + b;
                if (d < wlen)
                {
                    S.slot[d] = (Slot)slot;
                    c_tile_col[cbase + slot] = w + d;
                    c_tile_row[cbase + slot] = I;
                }
                ++slot;
            }
        }
        for (int p = warp; p < S2_PAIRS; p += NW) // the window's slots of every row pair
            for (int i = lane; i < nb; i += 32)
                MW[p * STRIDE + i] = 0u;
        __syncthreads();

        // ---- masks
        if (SEGS)
        {
            // Each A entry (r, k) of the tile row ORs the row segments of B's
            // row k - its 16-bit row masks, one per tile column - into row
            // r's masks: one shared atomic per (entry, B tile) instead of
            // one per (entry, B entry).  The warps share the tile row's
            // entries, 32 at a time (masks combine by OR, in any order).  A
            // lane walks its own entry's segments; lane l starts at segment
            // l mod ns, since neighbouring entries of a row (k - 1, k, k + 1)
            // list almost the same tile columns and would otherwise hit the
            // same mask word in the same step.  Entries with more than 32
            // segments (hub rows) are walked by the whole warp, one by one.
            const bool cut = w > lo || wend <= hi; // a window of several
            const int eb = S.rp[0], ee = S.rp[nrows];
            auto mark = [&](unsigned long long sg, int r) {
                const int d = (int)(sg >> 16) - w;
                if ((unsigned)d < (unsigned)wlen)
                {
                    const int sl = S.slot[d];
                    if (sl != NONE)
                        atomicOr(&MW[(r >> 1) * STRIDE + sl],
                                 ((unsigned)sg & 0xFFFFu) << ((r & 1) * 16));
                }
            };
            for (int c0 = eb + warp * 32; c0 < ee; c0 += NW * 32)
            {
                const int e = c0 + lane;
                int s0 = 0, ns = 0, r = 0;
                if (e < ee)
                {
                    // the entry's row: the last r with rp[r] <= e
#pragma unroll
                    for (int h = 8; h > 0; h >>= 1)
                        if (r + h < nrows && S.rp[r + h] <= e)
                            r += h;
                    const int k = __ldg(A.csr_col + e);
                    if (k >= 0 && k < B.m)
                    {
                        s0 = __ldg(B.seg_ptr + k);
                        int s1 = __ldg(B.seg_ptr + k + 1);
                        if (cut)
                        {
                            s0 = seg_lower_bound(B.seg, s0, s1, w);
                            s1 = seg_lower_bound(B.seg, s0, s1, wend);
                        }
                        ns = max(s1 - s0, 0);
                    }
                }
                const bool lng = ns > 32;
                const int nsh = lng ? 0 : ns;
                const int off = nsh > 0 ? lane % nsh : 0;
                const int steps = __reduce_max_sync(FULL, (unsigned)nsh);
                // four segments' loads in flight before their marks
                constexpr int U = 4;
                for (int i = 0; i < steps; i += U)
                {
                    unsigned long long sg[U];
#pragma unroll
                    for (int u = 0; u < U; ++u)
                    {
                        int x = off + i + u;
                        x -= x >= nsh ? nsh : 0;
                        sg[u] = i + u < nsh ? __ldg(B.seg + s0 + x) : 0ull;
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        if (i + u < nsh)
                            mark(sg[u], r);
                }
                for (unsigned lm = __ballot_sync(FULL, lng); lm != 0u; lm &= lm - 1u)
                {
                    const int j = __ffs(lm) - 1;
                    const int js0 = __shfl_sync(FULL, s0, j), jns = __shfl_sync(FULL, ns, j);
                    const int jr = __shfl_sync(FULL, r, j);
                    for (int t = lane; t < jns; t += 32)
                        mark(__ldg(B.seg + js0 + t), jr);
                }
            }
            __syncthreads(); // every warp's marks are in
        }
        else if ((NARROW || NW != S2_WARPS) && S.share)
        {
            // several windows: a hub row would leave one warp walking while
            // seven wait, so all warps share the tile row's A entries (the
            // masks combine by OR, in any order); warp w takes every
            // NW-th A tile, so short tile rows are shared too
            for (int t0 = a0; t0 < a1; t0 += NW * 32)
            {
                const int t = t0 + lane * NW + warp;
                int n = 0, tn0 = 0, K = 0;
                if (t < a1)
                {
                    tn0 = __ldg(A.tile_nnz + t);
                    n = __ldg(A.tile_nnz + t + 1) - tn0;
                    K = __ldg(A.tile_col + t);
                }
                const int incl = warp_incl_scan(n);
                const int total = __shfl_sync(FULL, incl, 31);
                for (int q0 = 0; q0 < total; q0 += 32)
                {
                    const int q = q0 + lane;
                    int own = 0;
#pragma unroll
                    for (int b = 16; b > 0; b >>= 1)
                        if (__shfl_sync(FULL, incl, own + b - 1) <= q)
                            own += b;
                    own = min(own, 31);
                    const int o_incl = __shfl_sync(FULL, incl, own);
                    const int o_n = __shfl_sync(FULL, n, own);
                    const int o_tn0 = __shfl_sync(FULL, tn0, own);
                    const int o_K = __shfl_sync(FULL, K, own);
                    int fs = 0, len = 0, sh = 0, rb = 0;
                    if (q < total)
                    {
                        const int pc = A.col[o_tn0 + q - (o_incl - o_n)]; // (row << 4) | col
                        const int r = pc >> 4, k = o_K * TD + (pc & 15);
                        if (r < nrows && k < B.m)
                        {
                            fs = min(max(__ldg(B.csr_rowptr + k), 0), B.nnz);
                            len = min(max(__ldg(B.csr_rowptr + k + 1), fs), B.nnz) - fs;
                            if (narrow && len > NARROW_MIN)
                            {
                                const int sb = lower_bound(B.csr_col, fs, fs + len, w * TD);
                                len = lower_bound(B.csr_col, sb, fs + len, wend * TD) - sb;
                                fs = sb;
                            }
                            sh = (r & 1) * 16;
                            rb = (r >> 1) * STRIDE;
                        }
                    }
                    int nbat = min(32, total - q0);
                    if (NARROW)
                    {
                        // B rows with nothing in this window leave the list
                        const unsigned live = __ballot_sync(FULL, len > 0);
                        if (len > 0)
                            ent[__popc(live & ((1u << lane) - 1u))] = make_int4(fs, len, sh, rb);
                        nbat = __popc(live);
                    }
                    else
                        ent[lane] = make_int4(fs, len, sh, rb);
                    __syncwarp();
                    auto mark = [&](int col, int sh, int rb) {
                        const int d = (col >> 4) - w;
                        if ((unsigned)d < (unsigned)wlen)
                        {
                            const int sl = S.slot[d];
                            if (sl != NONE)
                                atomicOr(&MW[rb + sl], (0x8000u >> (col & 15)) << sh);
                        }
                    };
                    for (int j = 0; j < nbat; j += 2)
                    {
                        int4 e0 = ent[j], e1 = ent[(j + 1) & 31];
                        if (j + 1 >= nbat)
                            e1.y = 0;
                        const int c0 = lane < e0.y ? __ldg(B.csr_col + e0.x + lane) : -1;
                        const int c1 = lane < e1.y ? __ldg(B.csr_col + e1.x + lane) : -1;
                        if (c0 >= 0)
                            mark(c0, e0.z, e0.w);
                        if (e0.y > 32) // rows longer than a warp (uniform branch)
                            for (int f = 32 + lane; f < e0.y; f += 32)
                                mark(__ldg(B.csr_col + e0.x + f), e0.z, e0.w);
                        if (c1 >= 0)
                            mark(c1, e1.z, e1.w);
                        if (e1.y > 32)
                            for (int f = 32 + lane; f < e1.y; f += 32)
                                mark(__ldg(B.csr_col + e1.x + f), e1.z, e1.w);
                    }
                    __syncwarp(); // the next batch overwrites this warp's list
                }
            }
            __syncthreads(); // every warp's rows are complete
        }
        else if (NW == S2_WARPS && r0 < nrows)
        {
            // one window: warp-private walk over the warp's own A entries
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
                    em = pp[r1];
                    const int ee = r1 + 1 < TD ? (int)pp[r1 + 1] : tcnt;
                    n = max(ee - eb, 0);
                    K = __ldg(A.tile_col + t);
                }
                const int incl = warp_incl_scan(n);
                const int total = __shfl_sync(FULL, incl, 31);
                for (int q0 = 0; q0 < total; q0 += 32)
                {
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
                    int fs = 0, len = 0, sh = 0;
                    if (q < total)
                    {
                        const int e = o_eb + (q - (o_incl - o_n));
                        sh = e < o_em ? 0 : 16;
                        const int k = o_K * TD + (A.col[o_tn0 + e] & 15);
                        if (k < B.m)
                        {
                            fs = min(max(__ldg(B.csr_rowptr + k), 0), B.nnz);
                            len = min(max(__ldg(B.csr_rowptr + k + 1), fs), B.nnz) - fs;
                        }
                        if (narrow && len > NARROW_MIN)
                        {
                            const int sb = lower_bound(B.csr_col, fs, fs + len, w * TD);
                            len = lower_bound(B.csr_col, sb, fs + len, wend * TD) - sb;
                            fs = sb;
                        }
                    }
                    int nbat = min(32, total - q0);
                    if (NARROW)
                    {
                        // B rows with nothing in this window leave the list
                        const unsigned live = __ballot_sync(FULL, len > 0);
                        if (len > 0)
                            ent[__popc(live & ((1u << lane) - 1u))] = make_int4(fs, len, sh, 0);
                        nbat = __popc(live);
                    }
                    else
                        ent[lane] = make_int4(fs, len, sh, 0);
                    __syncwarp();
                    // one column of B row k into the mask of row r's C tile
                    auto mark = [&](int col, int sh) {
                        const int d = (col >> 4) - w;
                        if ((unsigned)d < (unsigned)wlen)
                        {
                            const int sl = S.slot[d];
                            if (sl != NONE)
                                atomicOr(&mw[sl], (0x8000u >> (col & 15)) << sh);
                        }
                    };
                    for (int j = 0; j < nbat; j += 2)
                    {
                        int4 e0 = ent[j], e1 = ent[(j + 1) & 31];
                        if (j + 1 >= nbat)
                            e1.y = 0;
                        const int c0 = lane < e0.y ? __ldg(B.csr_col + e0.x + lane) : -1;
                        const int c1 = lane < e1.y ? __ldg(B.csr_col + e1.x + lane) : -1;
                        if (c0 >= 0)
                            mark(c0, e0.z);
                        if (e0.y > 32) // rows longer than a warp (uniform branch)
                            for (int f = 32 + lane; f < e0.y; f += 32)
                                mark(__ldg(B.csr_col + e0.x + f), e0.z);
                        if (c1 >= 0)
                            mark(c1, e1.z);
                        if (e1.y > 32)
                            for (int f = 32 + lane; f < e1.y; f += 32)
                                mark(__ldg(B.csr_col + e1.x + f), e1.z);
                    }
                    __syncwarp(); // the next batch overwrites this warp's list
                }
            }
        }
        // per-row counts of the window (pair p: rows 2p, 2p + 1)
#pragma unroll
        for (int q = 0; q < PPW; ++q)
        {
            const int p = warp + q * NW;
            if (p < S2_PAIRS)
            {
                int c0 = 0, c1 = 0;
                for (int i = lane; i < nb; i += 32)
                {
                    const uint32_t v = MW[p * STRIDE + i];
                    c0 += __popc(v & 0xFFFFu);
                    c1 += __popc(v >> 16);
                }
                run[q][0] += warp_sum(c0);
                run[q][1] += warp_sum(c1);
            }
        }
        __syncthreads();
        // ---- outputs of the window: masks (a row pair per 32-bit word: row
        // 2p in the low half is the lower address), tile counts
        uint32_t *c_mask2 = reinterpret_cast<uint32_t *>(c_mask);
        for (int i = tid; i < nb * S2_PAIRS; i += NT)
        {
            const int sl = i >> 3, p = i & 7;
            c_mask2[(size_t)(cbase + sl) * S2_PAIRS + p] = MW[p * STRIDE + sl];
        }
        for (int sl = tid; sl < nb; sl += NT)
        {
            int c = 0;
#pragma unroll
            for (int wv = 0; wv < S2_PAIRS; ++wv)
                c += __popc(MW[wv * STRIDE + sl]);
            c_tile_cnt[cbase + sl] = c;
        }
        __syncthreads();
        cbase += nb;
        wl = wend;
    }
    if (cbase != cend)
    {
        if (tid == 0)
            set_error(err, DERR_SYM_OVERFLOW);
        return;
    }
    int mine = 0;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < PPW; ++q)
        {
            const int p = warp + q * NW;
            if (p < S2_PAIRS)
            {
                if (2 * p < nrows)
                    c_row_cnt[I * TD + 2 * p] = run[q][0];
                if (2 * p + 1 < nrows)
                    c_row_cnt[I * TD + 2 * p + 1] = run[q][1];
                mine += run[q][0] + run[q][1];
            }
        }
    // tile row total
    __shared__ int tot;
    if (tid == 0)
        tot = 0;
    __syncthreads();
    if (lane == 0 && mine)
        atomicAdd(&tot, mine);
    __syncthreads();
    if (tid == 0)
    {
        c_tr_nnz[I] = tot;
        // the numeric step needs more than one window of C tiles here
        if (cend - cbeg > FLAT_SLOT_CAP || tot > FLAT_ACC)
            atomicOr(multi, 1);
    }
}

} // namespace

int symbolic_tile_counts(Workspace &ws, const DevTiles &A, const DevTiles &B, SymbolicOut &S,
                         int *cnt)
{
    cudaStream_t s = ws.stream;
    const int tilem = A.tilem;
    // flags: [0] some tile row needs several step-2 windows, [1] several
    // numeric windows, [2] heavy tile rows listed for the wide step-2 CTA,
    // [3] tile rows listed for the wide step-1 CTA, [4] tile rows listed for
    // the wide-window step-2 CTAs
    RTT_CHECK(S.w_flag.ensure(sizeof(int) * 8, s));
    RTT_CUDA(cudaMemsetAsync(S.w_flag.p, 0, sizeof(int) * 8, s));
    RTT_CHECK(S.s2_heavy.ensure((size_t)tilem + 16, s));
    RTT_CHECK(S.s2_list.ensure(sizeof(int) * (size_t)tilem + 16, s));
    RTT_CHECK(S.s1_list.ensure(sizeof(int) * (size_t)tilem + 16, s));
    const bool wide = S.sym_window_slots >= 0;
    if (wide)
        RTT_CHECK(S.s2_wlist.ensure(sizeof(int) * (size_t)tilem + 16, s));
    if (tilem > 0)
    {
        int *flag = S.w_flag.as<int>();
        int *wlist = wide ? S.s2_wlist.as<int>() : nullptr;
        k_sym_count<<<ceil_div(tilem, SYM_WARPS), SYM_WARPS * 32, 0, s>>>(
            A, B, cnt, flag, S.s2_heavy.as<uint8_t>(), S.s2_list.as<int>(), flag + 2,
            S.s1_list.as<int>(), flag + 3, wlist, flag + 4);
        int sms = 0;
        RTT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws.device));
        // persistent CTAs over the wide list (empty: they exit at once)
        k_sym_count_wide<<<std::min(tilem, 2 * sms), S1_WIDE_WARPS * 32, 0, s>>>(
            A, B, cnt, flag, S.s2_heavy.as<uint8_t>(), S.s2_list.as<int>(), flag + 2,
            S.s1_list.as<int>(), flag + 3, wlist, flag + 4);
        ws.launches += 2;
    }
    return RTT_OK;
}

int symbolic_device(Workspace &ws, const DevTiles &A, const DevTiles &B, SymbolicOut &S,
                    bool b_sorted)
{
    cudaStream_t s = ws.stream;
    if (A.n != B.m)
        return fail(RTT_ERR_SHAPE_MISMATCH, "symbolic: inner dimensions differ");
    S.m = A.m;
    S.n = B.n;
    S.tilem = A.tilem;
    S.tilen = B.tilen;
    const int tilem = A.tilem;
    RTT_CHECK(S.count_tmp.ensure(sizeof(int) * (size_t)(tilem + 1), s));
    RTT_CHECK(S.c_tile_ptr.ensure(sizeof(int) * (size_t)(tilem + 1), s));
    int *cnt = S.count_tmp.as<int>();
    RTT_CHECK(symbolic_tile_counts(ws, A, B, S, cnt));
    RTT_CHECK(scan_exclusive_int(ws, cnt, S.c_tile_ptr.as<int>(), tilem));
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars + 16, S.w_flag.p, sizeof(int) * 5,
                             cudaMemcpyDeviceToHost, s));
    int numtile = 0;
    RTT_CHECK(read_int_checked(ws, S.c_tile_ptr.as<int>() + tilem, &numtile, "symbolic step 1"));
    const bool sym_multi = ws.h_scalars[16] != 0;
    const int n_heavy = ws.h_scalars[18];
    const int n_wide = S.sym_window_slots >= 0 ? ws.h_scalars[20] : 0;
    const int wslots = S.sym_window_slots > 0 ? S.sym_window_slots : S2_WIDE_DEFAULT;
    const int wstride = (wslots + 2) | 1;
    S.numtile = numtile;
    const size_t nt = (size_t)numtile;
    RTT_CHECK(S.c_tile_col.ensure(sizeof(int) * nt, s));
    RTT_CHECK(S.c_tile_row.ensure(sizeof(int) * nt, s));
    RTT_CHECK(S.c_mask.ensure(sizeof(uint16_t) * nt * TD, s));
    RTT_CHECK(S.c_ptr.ensure(nt * TD, s));
    RTT_CHECK(S.c_tile_nnz.ensure(sizeof(int) * (nt + 1), s));
    RTT_CHECK(S.c_row_cnt.ensure(sizeof(int) * (size_t)(S.m + 1), s));
    RTT_CHECK(S.c_rowptr.ensure(sizeof(long long) * (size_t)(tilem + 1), s));
    RTT_CHECK(S.c_tr_nnz.ensure(sizeof(int) * (size_t)(tilem + 1), s));
    RTT_CHECK(S.tile_cnt.ensure(sizeof(int) * (nt + 1), s));
    // step 2 from B's row segments when they and A's CSR rows are at hand
    const bool segs = B.seg_ptr != nullptr && B.seg != nullptr && A.csr_rowptr != nullptr &&
                      A.csr_col != nullptr;
    if (tilem > 0)
    {
        auto go = [&](auto kern, int grid, int threads, size_t smem, cudaStream_t st,
                      const uint8_t *heavy, const int *list, int slots) -> int {
            if (smem > 48 * 1024)
                RTT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem));
            kern<<<grid, threads, smem, st>>>(
                A, B, S.c_tile_ptr.as<int>(), S.c_tile_col.as<int>(), S.c_tile_row.as<int>(),
                S.c_mask.as<uint16_t>(), S.tile_cnt.as<int>(), S.c_row_cnt.as<int>(),
                S.c_tr_nnz.as<int>(), S.w_flag.as<int>() + 1, ws.err.as<int>(), heavy, list,
                slots);
            ws.launches++;
            return RTT_OK;
        };
        if (n_heavy > 0 || n_wide > 0)
        {
            // heavy rows (one 32-warp CTA each) and rows with many C tiles
            // (wide-window CTAs) on the side stream, alongside the tile-row
            // CTAs (which skip them)
            RTT_CUDA(cudaEventRecord(ws.fork_ev, s));
            RTT_CUDA(cudaStreamWaitEvent(ws.side, ws.fork_ev, 0));
        }
        if (n_heavy > 0 && S.sym_window_slots >= 0)
        {
            auto hk = segs ? k_sym_rows<false, S2_HEAVY_WARPS, true, true>
                           : b_sorted ? k_sym_rows<true, S2_HEAVY_WARPS, false, true>
                                      : k_sym_rows<false, S2_HEAVY_WARPS, false, true>;
            RTT_CHECK(go(hk, n_heavy, S2_HEAVY_WARPS * 32, smem2_bytes<S2_HEAVY_WARPS, true>(wstride),
                         ws.side, nullptr, S.s2_list.as<int>(), wslots));
        }
        else if (n_heavy > 0)
        {
            auto hk = segs ? k_sym_rows<false, S2_HEAVY_WARPS, true>
                           : b_sorted ? k_sym_rows<true, S2_HEAVY_WARPS, false>
                                      : k_sym_rows<false, S2_HEAVY_WARPS, false>;
            RTT_CHECK(go(hk, n_heavy, S2_HEAVY_WARPS * 32,
                         smem2_bytes<S2_HEAVY_WARPS, false>(S2_STRIDE), ws.side, nullptr,
                         S.s2_list.as<int>(), 0));
        }
        if (n_wide > 0)
        {
            auto wk = segs ? k_sym_rows<false, S2_WARPS, true, true>
                           : b_sorted ? k_sym_rows<true, S2_WARPS, false, true>
                                      : k_sym_rows<false, S2_WARPS, false, true>;
            RTT_CHECK(go(wk, n_wide, S2_THREADS, smem2_bytes<S2_WARPS, true>(wstride), ws.side,
                         nullptr, S.s2_wlist.as<int>(), wslots));
        }
        if (n_heavy > 0 || n_wide > 0)
            RTT_CUDA(cudaEventRecord(ws.join_ev, ws.side));
        // 4-warp CTAs when every tile row fits one window; a tile row with
        // several windows walks its entries once per window, so it keeps 8
        const bool small = segs && !sym_multi;
        const uint8_t *skip = n_heavy > 0 || n_wide > 0 ? S.s2_heavy.as<uint8_t>() : nullptr;
        if (small)
            RTT_CHECK(go(k_sym_rows<false, S2_SEG_WARPS, true>, tilem, S2_SEG_WARPS * 32,
                         smem2_bytes<S2_SEG_WARPS, false>(S2_STRIDE), s, skip, nullptr, 0));
        else
        {
            auto kern = segs ? k_sym_rows<false, S2_WARPS, true>
                             : b_sorted && sym_multi ? k_sym_rows<true, S2_WARPS, false>
                                                     : k_sym_rows<false, S2_WARPS, false>;
            RTT_CHECK(go(kern, tilem, S2_THREADS, smem2_bytes<S2_WARPS, false>(S2_STRIDE), s, skip,
                         nullptr, 0));
        }
        if (n_heavy > 0 || n_wide > 0)
            RTT_CUDA(cudaStreamWaitEvent(s, ws.join_ev, 0));
    }
    // read with nnz(C) below (one synchronisation for both)
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars + 12, S.w_flag.as<int>() + 1, sizeof(int),
                             cudaMemcpyDeviceToHost, s));
    // exact sizes: nnz(C) as int64 over tile rows first (int32 overflow check)
    long long *tr64 = S.c_rowptr.as<long long>();
    RTT_CHECK(scan_exclusive_i64(ws, S.c_tr_nnz.as<int>(), tr64, tilem));
    long long nnz = 0;
    RTT_CHECK(read_i64_checked(ws, tr64 + tilem, &nnz, "symbolic step 2"));
    S.nnz = nnz;
    S.multi_window = ws.h_scalars[12] != 0;
    if (nnz > (long long)INT_MAX)
        return fail(RTT_ERR_UNREPRESENTABLE, "nnz(C) = " + std::to_string(nnz) +
                                                 " exceeds the int32 offsets of SMatrix / CSR");
    RTT_CHECK(scan_exclusive_int(ws, S.tile_cnt.as<int>(), S.c_tile_nnz.as<int>(), numtile));
    return RTT_OK;
}

} // namespace rtt
