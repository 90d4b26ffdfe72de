// csr2tile.cu - CSR -> 16x16 tile CSR on sm_100a.
//
// Semantics follow csr2tile_row_major (reference src/csr2tile.h:196-259):
// tiles of a tile row in ascending column order, per-tile exclusive row
// offsets (u8), entries of a (tile, row) in CSR order, packed column byte
// (row << 4) | col, mask bit (15 - col); and csr2tile_col_major (:261-478):
// the same tiles with per-tile data in tile-CSC order and plain column bytes.
//
// Fast path (every row's tile column index non-decreasing, i.e. sorted CSR):
// a half-warp owns one tile row, one lane per scalar row.  Each lane walks
// its row with a cursor; the half-warp takes the minimum pending tile column
// (4 xor-shuffles), every lane consumes its entries of that tile, a
// half-warp scan turns per-row counts into the tile's row offsets, and the
// lanes write their entries at tile base + row offset.  Reads of col/val are
// sequential per lane and the 16 rows of a tile row are contiguous in
// memory, so the half-warp streams one contiguous CSR slice.
// Generic path (unsorted rows): a warp per tile row extracts tile columns in
// ascending order and places entries with match_any ranking, which keeps CSR
// order inside each (tile, row).
#include "rtt_internal.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <climits>

namespace rtt
{
namespace
{

// ------------------------------------------------------------ validation
// flags[0]: some row's tile column decreases (needs the generic path)
// flags[1]: some row's column decreases (entries not sorted inside rows)
// flags[2]: some row repeats a column
// One warp per 32 consecutive rows.  Rows of at most 256 entries: each lane
// walks its own row.  A warp with a longer row walks the rows' entries, one
// contiguous range, 32 at a time instead (a hub row costs len / 32 steps, not
// len): a lane compares its entry with the one before unless the entry starts
// a row; the row starts inside a step are one OR-reduced bit mask.
__global__ void k_validate_csr(int m, int n, int nnz, const int *__restrict__ rowptr,
                               const int *__restrict__ col, int *err, int *flags)
{
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw == 0 && lane == 0 && (rowptr[0] != 0 || rowptr[m] != nnz))
        set_error(err, DERR_CSR_ROWPTR);
    if (gw * 32 >= m)
        return; // whole warp
    const int r = (int)(gw * 32) + lane;
    int b = 0, e = 0;
    bool bad = false;
    if (r < m)
    {
        b = rowptr[r];
        e = rowptr[r + 1];
        bad = b < 0 || e < b || e > nnz;
    }
    if (__any_sync(FULL, bad))
    {
        if (lane == 0)
            set_error(err, DERR_CSR_ROWPTR);
        return;
    }
    const int rows = min(32, m - (int)(gw * 32));
    const int lo = __shfl_sync(FULL, b, 0), hi = __shfl_sync(FULL, e, rows - 1);
    bool col_bad = false, tile_dec = false, col_dec = false, col_dup = false;
    if (__reduce_max_sync(FULL, (unsigned)(e - b)) <= 256)
    {
        // short rows: each lane walks its own row (the warp's rows share
        // their cache lines)
        int prev = -1;
        for (int j = b; j < e; ++j)
        {
            const int c = __ldg(col + j);
            if (c < 0 || c >= n)
            {
                col_bad = true;
                break;
            }
            if (prev >= 0)
            {
                tile_dec |= (c >> 4) < (prev >> 4);
                col_dec |= c < prev;
                col_dup |= c == prev;
            }
            prev = c;
        }
    }
    else
    {
        // a long row: the warp walks its rows' entry range 32 at a time
        for (long long c0 = lo; c0 < hi; c0 += 32)
        {
            const bool here = r < m && b >= c0 && b < c0 + 32;
            const unsigned starts = __reduce_or_sync(FULL, here ? 1u << (int)(b - c0) : 0u);
            const int j = (int)c0 + lane;
            if (j < hi)
            {
                const int c = __ldg(col + j);
                if (c < 0 || c >= n)
                    col_bad = true;
                else if (((starts >> lane) & 1u) == 0)
                {
                    const int p = __ldg(col + j - 1); // same row, j - 1 >= lo
                    tile_dec |= (c >> 4) < (p >> 4);
                    col_dec |= c < p;
                    col_dup |= c == p;
                }
            }
        }
    }
    if (__any_sync(FULL, col_bad) && lane == 0)
        set_error(err, DERR_CSR_COL);
    const bool td = __any_sync(FULL, tile_dec), cd = __any_sync(FULL, col_dec),
               dp = __any_sync(FULL, col_dup);
    if (lane == 0)
    {
        if (td)
            atomicOr(&flags[0], 1);
        if (cd)
            atomicOr(&flags[1], 1);
        if (dp)
            atomicOr(&flags[2], 1);
    }
}

// -------------------------------------------------------------- fast path
__global__ void __launch_bounds__(256) k_c2t_count(int m, int tilem, const int *__restrict__ rowptr,
                                                   const int *__restrict__ col, int *__restrict__ cnt,
                                                   const uint8_t *__restrict__ heavy)
{
    const int lane = threadIdx.x & 31, hl = lane & 15;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int I = gw * 2 + (lane >> 4);
    // heavy tile rows are counted by k_c2t_heavy_count
    const bool mine = I < tilem && !(heavy != nullptr && heavy[I]);
    int p = 0, e = 0;
    if (mine && I * TD + hl < m)
    {
        p = rowptr[I * TD + hl];
        e = rowptr[I * TD + hl + 1];
    }
    int cur = p < e ? (__ldg(col + p) >> 4) : INT_MAX;
    int count = 0;
    for (;;)
    {
        const int T = half_min(cur);
        const bool has = T != INT_MAX;
        if (!__any_sync(FULL, has))
            break;
        if (has)
        {
            ++count;
            while (p < e && (__ldg(col + p) >> 4) == T)
                ++p;
            cur = p < e ? (__ldg(col + p) >> 4) : INT_MAX;
        }
    }
    if (mine && hl == 0)
        cnt[I] = count;
}

__global__ void __launch_bounds__(256) k_c2t_fill(int m, int tilem, const int *__restrict__ rowptr,
                                                  const int *__restrict__ col,
                                                  const double *__restrict__ val,
                                                  const int *__restrict__ tile_ptr,
                                                  int *__restrict__ o_tcol, int *__restrict__ o_trow,
                                                  int *__restrict__ o_tnnz, uint8_t *__restrict__ o_ptr,
                                                  uint8_t *__restrict__ o_col,
                                                  double *__restrict__ o_val,
                                                  uint16_t *__restrict__ o_mask, int packed, int *err,
                                                  const uint8_t *__restrict__ heavy)
{
    const int lane = threadIdx.x & 31, hl = lane & 15;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int I = gw * 2 + (lane >> 4);
    // heavy tile rows are filled by k_c2t_heavy_fill
    const bool tr_ok = I < tilem && !(heavy != nullptr && heavy[I]);
    int p = 0, e = 0, base = 0, t = 0, tend = 0;
    if (tr_ok)
    {
        base = rowptr[min(I * TD, m)];
        t = tile_ptr[I];
        tend = tile_ptr[I + 1];
        if (I * TD + hl < m)
        {
            p = rowptr[I * TD + hl];
            e = rowptr[I * TD + hl + 1];
        }
    }
    int cur = p < e ? (__ldg(col + p) >> 4) : INT_MAX;
    for (;;)
    {
        const int T = half_min(cur);
        const bool has = T != INT_MAX;
        if (!__any_sync(FULL, has))
            break;
        int q = p;
        if (has)
            while (q < e && (__ldg(col + q) >> 4) == T)
                ++q;
        const int c = q - p;
        const int incl = half_incl_scan(c);
        const int excl = incl - c;
        const int total = __shfl_sync(FULL, incl, (lane & 16) | 15);
        if (has)
        {
            if (t >= tend)
            {
                set_error(err, DERR_C2T_OVERFLOW);
            }
            else
            {
                o_ptr[(size_t)t * TD + hl] = (uint8_t)excl;
                uint16_t mk = 0;
                int dst = base + excl;
                for (int j = p; j < q; ++j, ++dst)
                {
                    const int cc = __ldg(col + j) & 15;
                    mk |= (uint16_t)(0x8000u >> cc);
                    o_col[dst] = (uint8_t)(packed ? ((hl << 4) | cc) : cc);
                    o_val[dst] = __ldg(val + j);
                }
                o_mask[(size_t)t * TD + hl] = mk;
                if (hl == 0)
                {
                    o_tcol[t] = T;
                    o_trow[t] = I;
                    o_tnnz[t] = base;
                }
            }
            base += total;
            ++t;
            p = q;
            cur = p < e ? (__ldg(col + p) >> 4) : INT_MAX;
        }
    }
}

// ------------------------------------------------------------ row segments
// Row segments of a CSR whose rows have non-decreasing tile columns: every
// maximal run of a row's entries inside one tile column J becomes the segment
// (J << 16) | mask, mask bit (15 - c) for each column c of the run - the row's
// 16-bit row mask in tile J, as csr2tile writes it into mask[].  One warp per
// 32 consecutive rows (as k_validate_csr): each lane walks its own row when
// the warp's rows are short; a warp holding a long row walks its rows one
// after another, 32 entries at a time, and a segment is counted (and written)
// by the lane that holds its first entry.
__device__ __forceinline__ unsigned long long seg_pack(int T, unsigned mk)
{
    return ((unsigned long long)T << 16) | (mk & 0xFFFFu);
}

template <bool FILL>
__global__ void __launch_bounds__(256)
    k_row_segments(int m, const int *__restrict__ rowptr, const int *__restrict__ col,
                   int *__restrict__ seg_cnt, const int *__restrict__ seg_ptr,
                   unsigned long long *__restrict__ seg)
{
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw * 32 >= m)
        return; // whole warp
    const int r0 = (int)(gw * 32), r = r0 + lane;
    int b = 0, e = 0;
    if (r < m)
    {
        b = rowptr[r];
        e = rowptr[r + 1];
    }
    if (__reduce_max_sync(FULL, (unsigned)(e - b)) <= 256)
    {
        const int out = FILL && r < m ? seg_ptr[r] : 0;
        int n = 0, T = -1;
        unsigned mk = 0;
        for (int j = b; j < e; ++j)
        {
            const int c = __ldg(col + j);
            if ((c >> 4) != T)
            {
                if (T >= 0)
                {
                    if (FILL)
                        seg[out + n] = seg_pack(T, mk);
                    ++n;
                }
                T = c >> 4;
                mk = 0;
            }
            mk |= 0x8000u >> (c & 15);
        }
        if (T >= 0)
        {
            if (FILL)
                seg[out + n] = seg_pack(T, mk);
            ++n;
        }
        if (!FILL)
        {
            if (r < m)
                seg_cnt[r] = n;
            // seg_cnt[m]: the most segments of a row
            const unsigned wmax = __reduce_max_sync(FULL, r < m ? (unsigned)n : 0u);
            if (lane == 0 && wmax > 0)
                atomicMax(seg_cnt + m, (int)wmax);
        }
        return;
    }
    const int rows = min(32, m - r0);
    for (int q = 0; q < rows; ++q)
    {
        const int qb = __shfl_sync(FULL, b, q), qe = __shfl_sync(FULL, e, q);
        const int out = FILL ? seg_ptr[r0 + q] : 0;
        int n = 0;
        for (int c0 = qb; c0 < qe; c0 += 32)
        {
            const int j = c0 + lane;
            bool start = false;
            int T = 0;
            if (j < qe)
            {
                T = __ldg(col + j) >> 4;
                start = j == qb || (__ldg(col + j - 1) >> 4) != T;
            }
            const unsigned st = __ballot_sync(FULL, start);
            if (FILL && start)
            {
                unsigned mk = 0;
                for (int t = j; t < qe; ++t)
                {
                    const int c = __ldg(col + t);
                    if ((c >> 4) != T)
                        break;
                    mk |= 0x8000u >> (c & 15);
                }
                seg[out + n + __popc(st & ((1u << lane) - 1u))] = seg_pack(T, mk);
            }
            n += __popc(st);
        }
        if (!FILL && lane == 0)
        {
            seg_cnt[r0 + q] = n;
            atomicMax(seg_cnt + m, n);
        }
    }
}

// Tile structure (no per-entry payload) of a tile row from its rows'
// segments: the tile columns are the union of the 16 rows' segment columns,
// taken in ascending order by a half-warp (a lane per row walks its segment
// list; the half-warp takes the minimum pending column, and the lanes holding
// it step to their next segment).  FILL = false counts the tiles of each
// tile row, FILL = true writes tile_col and tile_row from tile_ptr[I].  Tile
// rows marked heavy are left to k_c2t_heavy_count / k_c2t_heavy_struct.
template <bool FILL>
__global__ void __launch_bounds__(256)
    k_c2t_seg_tiles(int m, int tilem, const int *__restrict__ seg_ptr,
                    const unsigned long long *__restrict__ seg, const int *__restrict__ tile_ptr,
                    int *__restrict__ cnt, int *__restrict__ o_tcol, int *__restrict__ o_trow,
                    int *err, const uint8_t *__restrict__ heavy)
{
    const int lane = threadIdx.x & 31, hl = lane & 15;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int I = gw * 2 + (lane >> 4);
    const bool mine = I < tilem && !(heavy != nullptr && heavy[I]);
    int p = 0, e = 0, t = 0, tend = 0;
    if (mine)
    {
        if (I * TD + hl < m)
        {
            p = seg_ptr[I * TD + hl];
            e = seg_ptr[I * TD + hl + 1];
        }
        if (FILL)
        {
            t = tile_ptr[I];
            tend = tile_ptr[I + 1];
        }
    }
    int cur = p < e ? (int)(__ldg(seg + p) >> 16) : INT_MAX;
    int count = 0;
    for (;;)
    {
        const int T = half_min(cur);
        const bool has = T != INT_MAX;
        if (!__any_sync(FULL, has))
            break;
        if (has)
        {
            if (FILL && hl == 0)
            {
                if (t < tend)
                {
                    o_tcol[t] = T;
                    o_trow[t] = I;
                }
                else
                    set_error(err, DERR_C2T_OVERFLOW);
            }
            ++t;
            ++count;
            if (cur == T)
            {
                ++p;
                cur = p < e ? (int)(__ldg(seg + p) >> 16) : INT_MAX;
            }
        }
    }
    if (!FILL && mine && hl == 0)
        cnt[I] = count;
}

// ------------------------------------------------ fast path, heavy tile rows
// A tile row holding a row with thousands of entries (an R-MAT hub) spans
// thousands of tile columns; the half-warp above takes them one per step and
// becomes the tail of the launch.  Such tile rows get a CTA each: the tile
// columns of the 16 rows become a bitmap, a tile's index is the rank of its
// bit, and since each row's tile columns are non-decreasing, the entries of
// one (tile, row) are one run in the row (at most 16 entries unless columns
// repeat), found and written by the thread that holds its first entry.  Entry
// order inside a (tile, row) stays the CSR order, as on the half-warp path.
constexpr int HV_ENTRIES = 2048;            // tile rows with more entries take this path
constexpr int HV_WORDS = 4096;              // bitmap words: 131072 tile columns
constexpr int HV_THREADS = 256;
constexpr int HV_CHUNK = 2048;              // tiles written per pass

struct HeavySmem
{
    uint32_t bits[HV_WORDS];
    int pre[HV_WORDS + 1];      // set bits before each word
    uint8_t cnt[HV_CHUNK][TD];  // entries per (tile of the pass, row)
    int tbase[HV_CHUNK + 1];    // entries of the pass's tiles before each tile
    int rs[TD + 1], re[TD];     // rows' entry ranges in the pass
    int rpre[TD + 1];           // prefix of the ranges' lengths
    int jlo, count;
};

// First entry of [b, e) whose tile column is >= J (the row's tile columns are
// non-decreasing).
__device__ __forceinline__ int tile_lower_bound(const int *col, int b, int e, int J)
{
    while (b < e)
    {
        const int mid = (b + e) >> 1;
        if ((__ldg(col + mid) >> 4) < J)
            b = mid + 1;
        else
            e = mid;
    }
    return b;
}

// Marks heavy tile rows (flag and list); thread per tile row.
__global__ void k_c2t_heavy_mark(int m, int tilem, const int *__restrict__ rowptr,
                                 const int *__restrict__ col, uint8_t *__restrict__ heavy,
                                 int *__restrict__ list, int *__restrict__ count)
{
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= tilem)
        return;
    const int r0 = I * TD, r1 = min(r0 + TD, m);
    bool hv = rowptr[r1] - rowptr[r0] > HV_ENTRIES;
    if (hv)
    {
        int lo = INT_MAX, hi = -1;
        for (int r = r0; r < r1; ++r)
        {
            const int b = rowptr[r], e = rowptr[r + 1];
            if (b < e)
            {
                lo = min(lo, __ldg(col + b) >> 4);
                hi = max(hi, __ldg(col + e - 1) >> 4);
            }
        }
        hv = hi >= lo && hi - lo < HV_WORDS * 32;
    }
    heavy[I] = hv;
    if (hv)
        list[atomicAdd(count, 1)] = I;
}

// The heavy tile row's tile-column bitmap and the set bits before each word.
__device__ void heavy_bitmap(HeavySmem &S, int I, int m, const int *__restrict__ rowptr,
                             const int *__restrict__ col)
{
    const int tid = threadIdx.x;
    const int r0 = I * TD, r1 = min(r0 + TD, m);
    if (tid == 0)
        S.jlo = INT_MAX;
    for (int i = tid; i < HV_WORDS; i += HV_THREADS)
        S.bits[i] = 0u;
    __syncthreads();
    if (tid < r1 - r0)
    {
        const int b = rowptr[r0 + tid];
        if (b < rowptr[r0 + tid + 1])
            atomicMin(&S.jlo, __ldg(col + b) >> 4);
    }
    __syncthreads();
    const int jlo = S.jlo;
    const int s0 = rowptr[r0], s1 = rowptr[r1];
    for (int j = s0 + tid; j < s1; j += HV_THREADS)
    {
        const int d = (__ldg(col + j) >> 4) - jlo;
        if ((unsigned)d < (unsigned)(HV_WORDS * 32)) // checked by the mark kernel
            atomicOr(&S.bits[d >> 5], 1u << (d & 31));
    }
    __syncthreads();
    if (tid < 32)
    {
        int run = 0;
        for (int q0 = 0; q0 < HV_WORDS; q0 += 32)
        {
            const int v = __popc(S.bits[q0 + tid]);
            const int incl = warp_incl_scan(v);
            S.pre[q0 + tid] = run + incl - v;
            run += __shfl_sync(FULL, incl, 31);
        }
        if (tid == 0)
        {
            S.pre[HV_WORDS] = run;
            S.count = run;
        }
    }
    __syncthreads();
}

// Tile column of the k-th set bit.
__device__ __forceinline__ int heavy_select(const HeavySmem &S, int k)
{
    int lo = 0, hi = HV_WORDS - 1; // last word with pre <= k
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (S.pre[mid] <= k)
            lo = mid;
        else
            hi = mid - 1;
    }
    uint32_t w = S.bits[lo];
    for (int i = S.pre[lo]; i < k; ++i)
        w &= w - 1;
    return S.jlo + lo * 32 + __ffs(w) - 1;
}

__device__ __forceinline__ int heavy_rank(const HeavySmem &S, int J)
{
    const int d = J - S.jlo;
    return S.pre[d >> 5] + __popc(S.bits[d >> 5] & ((1u << (d & 31)) - 1u));
}

__global__ void __launch_bounds__(HV_THREADS)
    k_c2t_heavy_count(int m, const int *__restrict__ list, const int *__restrict__ count,
                      const int *__restrict__ rowptr, const int *__restrict__ col,
                      int *__restrict__ cnt)
{
    extern __shared__ __align__(16) unsigned char hv_dyn[];
    HeavySmem &S = *reinterpret_cast<HeavySmem *>(hv_dyn);
    const int n = *count;
    for (int li = blockIdx.x; li < n; li += gridDim.x)
    {
        const int I = list[li];
        heavy_bitmap(S, I, m, rowptr, col);
        if (threadIdx.x == 0)
            cnt[I] = S.count;
        __syncthreads();
    }
}

// Structure only (no per-entry payload) of the heavy tile rows: tile
// columns are the bitmap's set bits in order.
__global__ void __launch_bounds__(HV_THREADS)
    k_c2t_heavy_struct(int m, const int *__restrict__ list, const int *__restrict__ count,
                       const int *__restrict__ rowptr, const int *__restrict__ col,
                       const int *__restrict__ tile_ptr, int *__restrict__ o_tcol,
                       int *__restrict__ o_trow, int *err)
{
    extern __shared__ __align__(16) unsigned char hv_dyn[];
    HeavySmem &S = *reinterpret_cast<HeavySmem *>(hv_dyn);
    const int n = *count;
    for (int li = blockIdx.x; li < n; li += gridDim.x)
    {
        const int I = list[li];
        heavy_bitmap(S, I, m, rowptr, col);
        const int ntiles = S.count, t0 = tile_ptr[I];
        if (t0 + ntiles != tile_ptr[I + 1])
        {
            if (threadIdx.x == 0)
                set_error(err, DERR_C2T_OVERFLOW);
        }
        else
            for (int k = threadIdx.x; k < ntiles; k += HV_THREADS)
            {
                o_tcol[t0 + k] = heavy_select(S, k);
                o_trow[t0 + k] = I;
            }
        __syncthreads(); // the bitmap is rebuilt for the next tile row
    }
}

__global__ void __launch_bounds__(HV_THREADS)
    k_c2t_heavy_fill(int m, const int *__restrict__ list, const int *__restrict__ count,
                     const int *__restrict__ rowptr, const int *__restrict__ col,
                     const double *__restrict__ val, const int *__restrict__ tile_ptr,
                     int *__restrict__ o_tcol, int *__restrict__ o_trow,
                     int *__restrict__ o_tnnz, uint8_t *__restrict__ o_ptr,
                     uint8_t *__restrict__ o_col, double *__restrict__ o_val,
                     uint16_t *__restrict__ o_mask, int packed, int *err)
{
    extern __shared__ __align__(16) unsigned char hv_dyn[];
    HeavySmem &S = *reinterpret_cast<HeavySmem *>(hv_dyn);
    const int tid = threadIdx.x;
    const int n = *count;
    for (int li = blockIdx.x; li < n; li += gridDim.x)
    {
        const int I = list[li];
        const int r0 = I * TD, nr = min(TD, m - r0);
        heavy_bitmap(S, I, m, rowptr, col);
        const int ntiles = S.count, t0 = tile_ptr[I];
        if (t0 + ntiles != tile_ptr[I + 1])
        {
            if (tid == 0)
                set_error(err, DERR_C2T_OVERFLOW);
            __syncthreads();
            continue;
        }
        int base = rowptr[r0]; // entries of the tile row before the pass
        for (int k0 = 0; k0 < ntiles; k0 += HV_CHUNK)
        {
            const int k1 = min(k0 + HV_CHUNK, ntiles), nk = k1 - k0;
            // the pass's entries: per row, the run of tile columns [Ja, Jb]
            if (tid < TD)
            {
                int b = 0, e = 0;
                if (tid < nr)
                {
                    const int Ja = heavy_select(S, k0), Jb = heavy_select(S, k1 - 1);
                    const int rb = rowptr[r0 + tid], rend = rowptr[r0 + tid + 1];
                    b = tile_lower_bound(col, rb, rend, Ja);
                    e = tile_lower_bound(col, b, rend, Jb + 1);
                }
                S.rs[tid] = b;
                S.re[tid] = e;
            }
            for (int i = tid; i < nk * TD; i += HV_THREADS)
                S.cnt[i >> 4][i & 15] = 0;
            __syncthreads();
            if (tid == 0)
            {
                int t = 0;
                for (int r = 0; r < TD; ++r)
                {
                    S.rpre[r] = t;
                    t += S.re[r] - S.rs[r];
                }
                S.rpre[TD] = t;
            }
            __syncthreads();
            const int total = S.rpre[TD];
            // pass 1: run lengths per (tile, row); a run starts where the
            // tile column changes inside the row
            for (int i = tid; i < total; i += HV_THREADS)
            {
                int r = 0;
                while (S.rpre[r + 1] <= i)
                    ++r;
                const int j = S.rs[r] + (i - S.rpre[r]);
                const int J = __ldg(col + j) >> 4;
                if (j == S.rs[r] || (__ldg(col + j - 1) >> 4) != J)
                {
                    int e = j + 1;
                    while (e < S.re[r] && (__ldg(col + e) >> 4) == J)
                        ++e;
                    if (e - j > 255) // repeated columns beyond a u8 row offset
                        set_error(err, DERR_C2T_OVERFLOW);
                    S.cnt[heavy_rank(S, J) - k0][r] = (uint8_t)min(e - j, 255);
                }
            }
            __syncthreads();
            // per tile: row offsets, size, column, tile row, empty masks
            for (int t = tid; t < nk; t += HV_THREADS)
            {
                int run = 0;
                const size_t g = (size_t)(t0 + k0 + t);
#pragma unroll
                for (int r = 0; r < TD; ++r)
                {
                    o_ptr[g * TD + r] = (uint8_t)run;
                    if (S.cnt[t][r] == 0)
                        o_mask[g * TD + r] = 0;
                    run += S.cnt[t][r];
                }
                S.tbase[t + 1] = run;
                o_tcol[g] = heavy_select(S, k0 + t);
                o_trow[g] = I;
            }
            __syncthreads();
            if (tid < 32)
            {
                int acc = 0;
                for (int q0 = 0; q0 < nk; q0 += 32)
                {
                    const int v = q0 + tid < nk ? S.tbase[q0 + tid + 1] : 0;
                    const int incl = warp_incl_scan(v);
                    if (q0 + tid < nk)
                        S.tbase[q0 + tid] = acc + incl - v;
                    acc += __shfl_sync(FULL, incl, 31);
                }
                if (tid == 0)
                    S.tbase[nk] = acc;
            }
            __syncthreads();
            for (int t = tid; t < nk; t += HV_THREADS)
                o_tnnz[t0 + k0 + t] = base + S.tbase[t];
            // pass 2: each run's first entry writes the run and its mask
            for (int i = tid; i < total; i += HV_THREADS)
            {
                int r = 0;
                while (S.rpre[r + 1] <= i)
                    ++r;
                const int j = S.rs[r] + (i - S.rpre[r]);
                const int J = __ldg(col + j) >> 4;
                if (j == S.rs[r] || (__ldg(col + j - 1) >> 4) != J)
                {
                    const int t = heavy_rank(S, J) - k0;
                    int off = 0;
                    for (int rr = 0; rr < r; ++rr)
                        off += S.cnt[t][rr];
                    int dst = base + S.tbase[t] + off;
                    const int len = S.cnt[t][r]; // the run, as counted in pass 1
                    uint16_t mk = 0;
                    for (int e = j; e < j + len; ++e, ++dst)
                    {
                        const int cc = __ldg(col + e) & 15;
                        mk |= (uint16_t)(0x8000u >> cc);
                        o_col[dst] = (uint8_t)(packed ? ((r << 4) | cc) : cc);
                        o_val[dst] = __ldg(val + e);
                    }
                    o_mask[(size_t)(t0 + k0 + t) * TD + r] = mk;
                }
            }
            base += S.tbase[nk];
            __syncthreads();
        }
    }
}

// ----------------------------------------------------------- generic path
__global__ void __launch_bounds__(256) k_c2t_count_generic(int m, int tilem,
                                                           const int *__restrict__ rowptr,
                                                           const int *__restrict__ col,
                                                           int *__restrict__ cnt)
{
    const int lane = threadIdx.x & 31;
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (I >= tilem)
        return;
    const int s0 = rowptr[I * TD], s1 = rowptr[min(I * TD + TD, m)];
    int prev = -1, count = 0;
    for (;;)
    {
        int mn = INT_MAX;
        for (int j = s0 + lane; j < s1; j += 32)
        {
            int T = __ldg(col + j) >> 4;
            if (T > prev && T < mn)
                mn = T;
        }
        mn = warp_min(mn);
        if (mn == INT_MAX)
            break;
        ++count;
        prev = mn;
    }
    if (lane == 0)
        cnt[I] = count;
}

__global__ void __launch_bounds__(128) k_c2t_fill_generic(
    int m, int tilem, const int *__restrict__ rowptr, const int *__restrict__ col,
    const double *__restrict__ val, const int *__restrict__ tile_ptr, int *__restrict__ o_tcol,
    int *__restrict__ o_trow, int *__restrict__ o_tnnz, uint8_t *__restrict__ o_ptr,
    uint8_t *__restrict__ o_col, double *__restrict__ o_val, uint16_t *__restrict__ o_mask,
    int packed, int *err)
{
    __shared__ int s_rp[4][TD + 1];
    __shared__ int s_cnt[4][TD];
    __shared__ int s_cur[4][TD];
    __shared__ unsigned s_mask[4][TD];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (I >= tilem)
        return;
    const int r0 = I * TD, nrows = min(TD, m - r0);
    if (lane <= TD)
        s_rp[w][lane] = rowptr[r0 + min(lane, nrows)];
    __syncwarp();
    const int s0 = s_rp[w][0], s1 = s_rp[w][nrows];
    int prev = -1, t = tile_ptr[I];
    const int tend = tile_ptr[I + 1];
    int base = s0;
    const unsigned lt = (1u << lane) - 1u;
    for (;;)
    {
        int mn = INT_MAX;
        for (int j = s0 + lane; j < s1; j += 32)
        {
            int T = __ldg(col + j) >> 4;
            if (T > prev && T < mn)
                mn = T;
        }
        const int T = warp_min(mn);
        if (T == INT_MAX)
            break;
        prev = T;
        if (lane < TD)
        {
            s_cnt[w][lane] = 0;
            s_cur[w][lane] = 0;
            s_mask[w][lane] = 0;
        }
        __syncwarp();
        for (int j = s0 + lane; j < s1; j += 32)
        {
            if ((__ldg(col + j) >> 4) == T)
            {
                int r = 0;
                while (r + 1 < nrows && s_rp[w][r + 1] <= j)
                    ++r;
                atomicAdd(&s_cnt[w][r], 1);
            }
        }
        __syncwarp();
        int c = lane < TD ? s_cnt[w][lane] : 0;
        int incl = half_incl_scan(c);
        int excl = incl - c;
        int total = __shfl_sync(FULL, incl, 15);
        if (t >= tend)
        {
            set_error(err, DERR_C2T_OVERFLOW);
            return;
        }
        if (lane < TD)
        {
            o_ptr[(size_t)t * TD + lane] = (uint8_t)excl;
            s_cnt[w][lane] = excl;
        }
        __syncwarp();
        // place entries in CSR order, chunk by chunk
        for (int j0 = s0; j0 < s1; j0 += 32)
        {
            const int j = j0 + lane;
            bool in = false;
            int r = 0, cc = 0;
            if (j < s1)
            {
                const int cj = __ldg(col + j);
                if ((cj >> 4) == T)
                {
                    in = true;
                    cc = cj & 15;
                    while (r + 1 < nrows && s_rp[w][r + 1] <= j)
                        ++r;
                }
            }
            const int key = in ? r : (TD + lane);
            const unsigned peers = __match_any_sync(FULL, key);
            if (in)
            {
                const int rank = __popc(peers & lt);
                const int dst = base + s_cnt[w][r] + s_cur[w][r] + rank;
                o_col[dst] = (uint8_t)(packed ? ((r << 4) | cc) : cc);
                o_val[dst] = __ldg(val + j);
                atomicOr(&s_mask[w][r], 0x8000u >> cc);
            }
            __syncwarp();
            if (in && (peers & lt) == 0)
                s_cur[w][r] += __popc(peers);
            __syncwarp();
        }
        if (lane < TD)
            o_mask[(size_t)t * TD + lane] = (uint16_t)s_mask[w][lane];
        if (lane == 0)
        {
            o_tcol[t] = T;
            o_trow[t] = I;
            o_tnnz[t] = base;
        }
        base += total;
        ++t;
        __syncwarp();
    }
}

// Stable insertion sort of every (tile, row) segment by column byte: the
// in-tile order of csr2tile_col_major for rows whose columns are unsorted.
__global__ void k_sort_tile_rows(int numtile, const int *__restrict__ tnnz,
                                 const uint8_t *__restrict__ ptr, uint8_t *__restrict__ colb,
                                 double *__restrict__ v)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= numtile * TD)
        return;
    int t = x >> 4, r = x & 15;
    int b = tnnz[t] + ptr[(size_t)t * TD + r];
    int e = r == TD - 1 ? tnnz[t + 1] : tnnz[t] + ptr[(size_t)t * TD + r + 1];
    for (int i = b + 1; i < e; ++i)
    {
        uint8_t kc = colb[i];
        double kv = v[i];
        int key = kc & 15;
        int j = i - 1;
        while (j >= b && (colb[j] & 15) > key)
        {
            colb[j + 1] = colb[j];
            v[j + 1] = v[j];
            --j;
        }
        colb[j + 1] = kc;
        v[j + 1] = kv;
    }
}

__global__ void k_set_int(int *p, int v) { *p = v; }

// ------------------------------------------------------ tile CSC / col-major
__global__ void k_iota(int *a, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        a[i] = i;
}

__global__ void k_lower_bound_ptr(const int *__restrict__ sorted_keys, int nkeys, int nbins,
                                  int *__restrict__ ptr)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > nbins)
        return;
    ptr[b] = lower_bound(sorted_keys, 0, nkeys, b);
}

__global__ void k_gather_int(const int *__restrict__ src, const int *__restrict__ idx, int n,
                             int *__restrict__ dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = src[idx[i]];
}

__global__ void k_tile_counts(const int *__restrict__ tnnz, const int *__restrict__ order, int n,
                              int *__restrict__ cnt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        int t = order[i];
        cnt[i] = tnnz[t + 1] - tnnz[t];
    }
}

// warp per destination tile: copy row offsets, mask and entries
__global__ void k_copy_tiles_colmajor(int n, const int *__restrict__ order,
                                      const int *__restrict__ src_tnnz,
                                      const uint8_t *__restrict__ src_ptr,
                                      const uint16_t *__restrict__ src_mask,
                                      const uint8_t *__restrict__ src_col,
                                      const double *__restrict__ src_val,
                                      const int *__restrict__ dst_tnnz, uint8_t *__restrict__ dst_ptr,
                                      uint16_t *__restrict__ dst_mask, uint8_t *__restrict__ dst_col,
                                      double *__restrict__ dst_val)
{
    const int lane = threadIdx.x & 31;
    const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (p >= n)
        return;
    const int t = order[p];
    if (lane < TD)
    {
        dst_ptr[(size_t)p * TD + lane] = src_ptr[(size_t)t * TD + lane];
        dst_mask[(size_t)p * TD + lane] = src_mask[(size_t)t * TD + lane];
    }
    const int sb = src_tnnz[t], cnt = src_tnnz[t + 1] - sb, db = dst_tnnz[p];
    for (int i = lane; i < cnt; i += 32)
    {
        dst_col[db + i] = src_col[sb + i] & 15;
        dst_val[db + i] = src_val[sb + i];
    }
}

// ----------------------------------------------------------- CSR transpose
__global__ void k_row_ids(int m, const int *__restrict__ rowptr, int *__restrict__ rows)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m)
        return;
    for (int j = rowptr[r]; j < rowptr[r + 1]; ++j)
        rows[j] = r;
}

__global__ void k_gather_transpose(int nnz, const int *__restrict__ order,
                                   const int *__restrict__ rows, const double *__restrict__ val,
                                   int *__restrict__ t_col, double *__restrict__ t_val)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnz)
        return;
    int src = order[i];
    t_col[i] = rows[src];
    t_val[i] = val[src];
}

int bits_for(int maxval)
{
    int b = 1;
    while (b < 31 && (1 << b) <= maxval)
        ++b;
    return b;
}

int sort_pairs(Workspace &ws, const int *keys_in, int *keys_out, const int *vals_in, int *vals_out,
               int n, int max_key)
{
    if (n <= 0)
        return RTT_OK;
    size_t bytes = 0;
    const int end_bit = bits_for(max_key);
    RTT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys_in, keys_out, vals_in, vals_out,
                                             n, 0, end_bit, ws.stream));
    RTT_CHECK(ws.scan_tmp.ensure(bytes, ws.stream));
    RTT_CUDA(cub::DeviceRadixSort::SortPairs(ws.scan_tmp.p, bytes, keys_in, keys_out, vals_in,
                                             vals_out, n, 0, end_bit, ws.stream));
    ws.launches += 3;
    return RTT_OK;
}

inline int grid_for(long long threads, int block) { return (int)((threads + block - 1) / block); }

} // namespace

int csr2tile_device(Workspace &ws, int m, int n, int nnz, const int *rowptr, const int *col,
                    const double *val, TileBufs &out, bool packed_col, bool sort_within_rows,
                    bool segments, bool payload)
{
    if (m < 0 || n < 0 || nnz < 0)
        return fail(RTT_ERR_INVALID_ARGUMENT, "csr2tile: negative size");
    cudaStream_t s = ws.stream;
    out.m = m;
    out.n = n;
    out.nnz = nnz;
    out.has_segments = false;
    out.payload = true;
    out.tilem = ceil_div(m, TD);
    out.tilen = ceil_div(n, TD);
    const int tilem = out.tilem;

    RTT_CHECK(out.tile_ptr.ensure(sizeof(int) * (tilem + 1), s));
    RTT_CHECK(out.tmp0.ensure(sizeof(int) * (tilem + 1), s));
    RTT_CHECK(out.tmp1.ensure(sizeof(int) * 4, s));
    int *flags = out.tmp1.as<int>();
    RTT_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * 3, s));
    if (m == 0)
    {
        RTT_CUDA(cudaMemsetAsync(out.tile_ptr.p, 0, sizeof(int), s));
        out.numtile = 0;
        RTT_CHECK(out.tile_nnz.ensure(sizeof(int), s));
        RTT_CUDA(cudaMemsetAsync(out.tile_nnz.p, 0, sizeof(int), s));
        const size_t tiny = 16;
        RTT_CHECK(out.tile_col.ensure(tiny, s));
        RTT_CHECK(out.tile_row.ensure(tiny, s));
        RTT_CHECK(out.ptr.ensure(tiny, s));
        RTT_CHECK(out.mask.ensure(tiny, s));
        RTT_CHECK(out.col.ensure(tiny, s));
        RTT_CHECK(out.val.ensure(tiny, s));
        return RTT_OK;
    }
    k_validate_csr<<<grid_for((long long)ceil_div(m, 32) * 32, 256), 256, 0, s>>>(
        m, n, nnz, rowptr, col, ws.err.as<int>(), flags);
    ws.launches++;
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars + 4, flags, sizeof(int) * 3, cudaMemcpyDeviceToHost, s));
    RTT_CHECK(check_device_error(ws, "csr2tile validate"));
    const bool generic = ws.h_scalars[4] != 0;
    const bool unsorted = ws.h_scalars[5] != 0;
    // rows that are unsorted may hide repeated columns too
    out.dup_cols = ws.h_scalars[6] != 0 || unsorted;
    out.generic = generic;
    out.has_segments = false;
    // the structure alone comes from the row segments, which need rows whose
    // tile columns never decrease; otherwise the whole tile payload is built
    const bool structure_only = !payload && !generic;
    if ((segments || structure_only) && !generic)
    {
        // row segments: count per row, scan, fill
        RTT_CHECK(out.seg_cnt.ensure(sizeof(int) * ((size_t)m + 1), s));
        RTT_CHECK(out.seg_ptr.ensure(sizeof(int) * ((size_t)m + 1), s));
        RTT_CUDA(cudaMemsetAsync(out.seg_cnt.as<int>() + m, 0, sizeof(int), s));
        const int grid = grid_for((long long)ceil_div(m, 32) * 32, 256);
        k_row_segments<false><<<grid, 256, 0, s>>>(m, rowptr, col, out.seg_cnt.as<int>(), nullptr,
                                                   nullptr);
        ws.launches++;
        RTT_CHECK(scan_exclusive_int(ws, out.seg_cnt.as<int>(), out.seg_ptr.as<int>(), m));
        // at most one segment per entry: size by nnz, no host read
        RTT_CHECK(out.seg.ensure(sizeof(unsigned long long) * ((size_t)nnz + 1), s));
        k_row_segments<true><<<grid, 256, 0, s>>>(m, rowptr, col, nullptr, out.seg_ptr.as<int>(),
                                                  out.seg.as<unsigned long long>());
        ws.launches++;
        out.has_segments = true;
    }

    int *cnt = out.tmp0.as<int>();
    // heavy tile rows (a CTA each) are listed on the device; their kernels
    // take the list length from device memory, so no host read is needed
    uint8_t *heavy = nullptr;
    int *hv_list = nullptr, *hv_count = flags + 3;
    int hv_grid = 0;
    const size_t hv_smem = sizeof(HeavySmem);
    if (!generic)
    {
        RTT_CHECK(out.tmp2.ensure((size_t)tilem + 16, s));
        RTT_CHECK(out.tmp3.ensure(sizeof(int) * (size_t)tilem + 16, s));
        heavy = out.tmp2.as<uint8_t>();
        hv_list = out.tmp3.as<int>();
        RTT_CUDA(cudaMemsetAsync(hv_count, 0, sizeof(int), s));
        k_c2t_heavy_mark<<<grid_for(tilem, 256), 256, 0, s>>>(m, tilem, rowptr, col, heavy,
                                                              hv_list, hv_count);
        ws.launches++;
        int sms = 0;
        RTT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws.device));
        hv_grid = std::min(tilem, 2 * sms);
        RTT_CUDA(cudaFuncSetAttribute(k_c2t_heavy_count, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)hv_smem));
        RTT_CUDA(cudaFuncSetAttribute(k_c2t_heavy_fill, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)hv_smem));
        k_c2t_heavy_count<<<hv_grid, HV_THREADS, hv_smem, s>>>(m, hv_list, hv_count, rowptr, col,
                                                               cnt);
        ws.launches++;
    }
    if (structure_only)
    {
        // tile_ptr, tile_col and tile_row only (from the row segments)
        const int grid = grid_for((long long)ceil_div(tilem, 2) * 32, 256);
        k_c2t_seg_tiles<false><<<grid, 256, 0, s>>>(m, tilem, out.seg_ptr.as<int>(),
                                                     out.seg.as<unsigned long long>(), nullptr,
                                                     cnt, nullptr, nullptr, ws.err.as<int>(),
                                                     heavy);
        ws.launches++;
        RTT_CHECK(scan_exclusive_int(ws, cnt, out.tile_ptr.as<int>(), tilem));
        int numtile = 0;
        // the most segments of a row comes back with the tile count (one sync)
        RTT_CUDA(cudaMemcpyAsync(ws.h_scalars + 2, out.seg_cnt.as<int>() + m, sizeof(int),
                                 cudaMemcpyDeviceToHost, s));
        RTT_CHECK(read_int(ws, out.tile_ptr.as<int>() + tilem, &numtile));
        out.max_row_segs = ws.h_scalars[2];
        out.numtile = numtile;
        RTT_CHECK(out.tile_col.ensure(sizeof(int) * (size_t)numtile + 16, s));
        RTT_CHECK(out.tile_row.ensure(sizeof(int) * (size_t)numtile + 16, s));
        k_c2t_seg_tiles<true><<<grid, 256, 0, s>>>(m, tilem, out.seg_ptr.as<int>(),
                                                    out.seg.as<unsigned long long>(),
                                                    out.tile_ptr.as<int>(), nullptr,
                                                    out.tile_col.as<int>(), out.tile_row.as<int>(),
                                                    ws.err.as<int>(), heavy);
        RTT_CUDA(cudaFuncSetAttribute(k_c2t_heavy_struct,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hv_smem));
        k_c2t_heavy_struct<<<hv_grid, HV_THREADS, hv_smem, s>>>(
            m, hv_list, hv_count, rowptr, col, out.tile_ptr.as<int>(), out.tile_col.as<int>(),
            out.tile_row.as<int>(), ws.err.as<int>());
        ws.launches += 2;
        out.payload = false;
        return RTT_OK;
    }
    if (!generic)
        k_c2t_count<<<grid_for((long long)ceil_div(tilem, 2) * 32, 256), 256, 0, s>>>(m, tilem, rowptr,
                                                                                   col, cnt, heavy);
    else
        k_c2t_count_generic<<<grid_for((long long)tilem * 32, 256), 256, 0, s>>>(m, tilem, rowptr,
                                                                               col, cnt);
    ws.launches++;
    RTT_CHECK(scan_exclusive_int(ws, cnt, out.tile_ptr.as<int>(), tilem));
    int numtile = 0;
    RTT_CHECK(read_int(ws, out.tile_ptr.as<int>() + tilem, &numtile));
    out.numtile = numtile;

    RTT_CHECK(out.tile_col.ensure(sizeof(int) * (size_t)numtile, s));
    RTT_CHECK(out.tile_row.ensure(sizeof(int) * (size_t)numtile, s));
    RTT_CHECK(out.tile_nnz.ensure(sizeof(int) * ((size_t)numtile + 1), s));
    RTT_CHECK(out.ptr.ensure((size_t)numtile * TD, s));
    RTT_CHECK(out.mask.ensure(sizeof(uint16_t) * (size_t)numtile * TD, s));
    RTT_CHECK(out.col.ensure((size_t)nnz, s));
    RTT_CHECK(out.val.ensure(sizeof(double) * (size_t)nnz, s));

    if (!generic)
        k_c2t_fill<<<grid_for((long long)ceil_div(tilem, 2) * 32, 256), 256, 0, s>>>(
            m, tilem, rowptr, col, val, out.tile_ptr.as<int>(), out.tile_col.as<int>(),
            out.tile_row.as<int>(), out.tile_nnz.as<int>(), out.ptr.as<uint8_t>(),
            out.col.as<uint8_t>(), out.val.as<double>(), out.mask.as<uint16_t>(), packed_col ? 1 : 0,
            ws.err.as<int>(), heavy);
    else
        k_c2t_fill_generic<<<grid_for((long long)tilem * 32, 128), 128, 0, s>>>(
            m, tilem, rowptr, col, val, out.tile_ptr.as<int>(), out.tile_col.as<int>(),
            out.tile_row.as<int>(), out.tile_nnz.as<int>(), out.ptr.as<uint8_t>(),
            out.col.as<uint8_t>(), out.val.as<double>(), out.mask.as<uint16_t>(), packed_col ? 1 : 0,
            ws.err.as<int>());
    ws.launches++;
    if (!generic)
    {
        k_c2t_heavy_fill<<<hv_grid, HV_THREADS, hv_smem, s>>>(
            m, hv_list, hv_count, rowptr, col, val, out.tile_ptr.as<int>(), out.tile_col.as<int>(),
            out.tile_row.as<int>(), out.tile_nnz.as<int>(), out.ptr.as<uint8_t>(),
            out.col.as<uint8_t>(), out.val.as<double>(), out.mask.as<uint16_t>(),
            packed_col ? 1 : 0, ws.err.as<int>());
        ws.launches++;
    }
    k_set_int<<<1, 1, 0, s>>>(out.tile_nnz.as<int>() + numtile, nnz);
    ws.launches++;
    if (sort_within_rows && unsorted && numtile > 0)
    {
        k_sort_tile_rows<<<grid_for((long long)numtile * TD, 256), 256, 0, s>>>(
            numtile, out.tile_nnz.as<int>(), out.ptr.as<uint8_t>(), out.col.as<uint8_t>(),
            out.val.as<double>());
        ws.launches++;
    }
    return RTT_OK;
}

int csr2tile_refill_device(Workspace &ws, const int *rowptr, const int *col, const double *val,
                           TileBufs &t, bool packed_col)
{
    cudaStream_t s = ws.stream;
    const int m = t.m, tilem = t.tilem;
    if (m == 0 || t.nnz == 0)
        return RTT_OK;
    // the fill kernels of the first build, with the new values: they rewrite
    // the structure arrays with the same bytes and the values in tile order
    if (!t.generic)
    {
        RTT_CHECK(t.tmp1.ensure(sizeof(int) * 4, s));
        RTT_CHECK(t.tmp2.ensure((size_t)tilem + 16, s));
        RTT_CHECK(t.tmp3.ensure(sizeof(int) * (size_t)tilem + 16, s));
        uint8_t *heavy = t.tmp2.as<uint8_t>();
        int *hv_list = t.tmp3.as<int>(), *hv_count = t.tmp1.as<int>() + 3;
        RTT_CUDA(cudaMemsetAsync(hv_count, 0, sizeof(int), s));
        k_c2t_heavy_mark<<<grid_for(tilem, 256), 256, 0, s>>>(m, tilem, rowptr, col, heavy,
                                                              hv_list, hv_count);
        k_c2t_fill<<<grid_for((long long)ceil_div(tilem, 2) * 32, 256), 256, 0, s>>>(
            m, tilem, rowptr, col, val, t.tile_ptr.as<int>(), t.tile_col.as<int>(),
            t.tile_row.as<int>(), t.tile_nnz.as<int>(), t.ptr.as<uint8_t>(), t.col.as<uint8_t>(),
            t.val.as<double>(), t.mask.as<uint16_t>(), packed_col ? 1 : 0, ws.err.as<int>(), heavy);
        int sms = 0;
        RTT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws.device));
        const size_t hv_smem = sizeof(HeavySmem);
        RTT_CUDA(cudaFuncSetAttribute(k_c2t_heavy_fill, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)hv_smem));
        k_c2t_heavy_fill<<<std::min(tilem, 2 * sms), HV_THREADS, hv_smem, s>>>(
            m, hv_list, hv_count, rowptr, col, val, t.tile_ptr.as<int>(), t.tile_col.as<int>(),
            t.tile_row.as<int>(), t.tile_nnz.as<int>(), t.ptr.as<uint8_t>(), t.col.as<uint8_t>(),
            t.val.as<double>(), t.mask.as<uint16_t>(), packed_col ? 1 : 0, ws.err.as<int>());
        ws.launches += 3;
    }
    else
    {
        k_c2t_fill_generic<<<grid_for((long long)tilem * 32, 128), 128, 0, s>>>(
            m, tilem, rowptr, col, val, t.tile_ptr.as<int>(), t.tile_col.as<int>(),
            t.tile_row.as<int>(), t.tile_nnz.as<int>(), t.ptr.as<uint8_t>(), t.col.as<uint8_t>(),
            t.val.as<double>(), t.mask.as<uint16_t>(), packed_col ? 1 : 0, ws.err.as<int>());
        ws.launches++;
    }
    RTT_CUDA(cudaGetLastError());
    return RTT_OK;
}

int validate_csr_device(Workspace &ws, int m, int n, int nnz, const int *rowptr, const int *col,
                        int *flags)
{
    RTT_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * 3, ws.stream));
    if (m > 0)
    {
        k_validate_csr<<<grid_for((long long)ceil_div(m, 32) * 32, 256), 256, 0, ws.stream>>>(
            m, n, nnz, rowptr, col, ws.err.as<int>(), flags);
        ws.launches++;
    }
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars + 4, flags, sizeof(int) * 3, cudaMemcpyDeviceToHost,
                             ws.stream));
    return check_device_error(ws, "csr validate");
}

int build_tile_csc(Workspace &ws, TileBufs &t)
{
    cudaStream_t s = ws.stream;
    const int nt = t.numtile;
    RTT_CHECK(t.csc_ptr.ensure(sizeof(int) * (t.tilen + 1), s));
    RTT_CHECK(t.csc_row.ensure(sizeof(int) * (size_t)(nt + 1), s));
    RTT_CHECK(t.csc_data.ensure(sizeof(int) * (size_t)(nt + 1), s));
    RTT_CHECK(t.tmp2.ensure(sizeof(int) * (size_t)(nt + 1), s));
    RTT_CHECK(t.tmp3.ensure(sizeof(int) * (size_t)(nt + 1), s));
    int *iota = t.tmp2.as<int>();
    int *sorted_keys = t.tmp3.as<int>();
    if (nt > 0)
    {
        k_iota<<<grid_for(nt, 256), 256, 0, s>>>(iota, nt);
        ws.launches++;
        RTT_CHECK(sort_pairs(ws, t.tile_col.as<int>(), sorted_keys, iota, t.csc_data.as<int>(), nt,
                             t.tilen));
        k_gather_int<<<grid_for(nt, 256), 256, 0, s>>>(t.tile_row.as<int>(), t.csc_data.as<int>(),
                                                       nt, t.csc_row.as<int>());
        ws.launches++;
    }
    k_lower_bound_ptr<<<grid_for(t.tilen + 1, 256), 256, 0, s>>>(sorted_keys, nt, t.tilen,
                                                                 t.csc_ptr.as<int>());
    ws.launches++;
    return RTT_OK;
}

int tiles_to_col_major(Workspace &ws, const TileBufs &rm, TileBufs &out)
{
    // rm must carry its CSC index (build_tile_csc)
    cudaStream_t s = ws.stream;
    const int nt = rm.numtile;
    out.m = rm.m;
    out.n = rm.n;
    out.nnz = rm.nnz;
    out.tilem = rm.tilem;
    out.tilen = rm.tilen;
    out.numtile = nt;
    RTT_CHECK(out.tile_nnz.ensure(sizeof(int) * ((size_t)nt + 1), s));
    RTT_CHECK(out.ptr.ensure((size_t)nt * TD + 16, s));
    RTT_CHECK(out.mask.ensure(sizeof(uint16_t) * (size_t)nt * TD + 16, s));
    RTT_CHECK(out.col.ensure((size_t)rm.nnz + 16, s));
    RTT_CHECK(out.val.ensure(sizeof(double) * (size_t)rm.nnz + 16, s));
    RTT_CHECK(out.tmp0.ensure(sizeof(int) * ((size_t)nt + 1), s));
    int *cnt = out.tmp0.as<int>();
    if (nt > 0)
    {
        k_tile_counts<<<grid_for(nt, 256), 256, 0, s>>>(rm.tile_nnz.as<int>(), rm.csc_data.as<int>(),
                                                         nt, cnt);
        ws.launches++;
    }
    RTT_CHECK(scan_exclusive_int(ws, cnt, out.tile_nnz.as<int>(), nt));
    if (nt > 0)
    {
        k_copy_tiles_colmajor<<<grid_for((long long)nt * 32, 256), 256, 0, s>>>(
            nt, rm.csc_data.as<int>(), rm.tile_nnz.as<int>(), rm.ptr.as<uint8_t>(),
            rm.mask.as<uint16_t>(), rm.col.as<uint8_t>(), rm.val.as<double>(),
            out.tile_nnz.as<int>(), out.ptr.as<uint8_t>(), out.mask.as<uint16_t>(),
            out.col.as<uint8_t>(), out.val.as<double>());
        ws.launches++;
    }
    return RTT_OK;
}

int csr_transpose_device(Workspace &ws, int m, int n, int nnz, const int *rowptr, const int *col,
                         const double *val, int *t_rowptr, int *t_col, double *t_val)
{
    cudaStream_t s = ws.stream;
    // grow-only scratch of the workspace: no cudaMalloc / cudaFree (which
    // would wait for every stream of the device) once it has grown
    const size_t bytes = sizeof(int) * (size_t)nnz + 16;
    for (DevBuf &b : ws.tmp)
        RTT_CHECK(b.ensure(bytes, s));
    int *rows = ws.tmp[0].as<int>(), *iota = ws.tmp[1].as<int>();
    int *keys = ws.tmp[2].as<int>(), *order = ws.tmp[3].as<int>();
    if (m > 0)
    {
        k_row_ids<<<grid_for(m, 256), 256, 0, s>>>(m, rowptr, rows);
        ws.launches++;
    }
    if (nnz > 0)
    {
        k_iota<<<grid_for(nnz, 256), 256, 0, s>>>(iota, nnz);
        ws.launches++;
        RTT_CHECK(sort_pairs(ws, col, keys, iota, order, nnz, n));
        k_gather_transpose<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, order, rows, val, t_col, t_val);
        ws.launches++;
    }
    k_lower_bound_ptr<<<grid_for(n + 1, 256), 256, 0, s>>>(keys, nnz, n, t_rowptr);
    ws.launches++;
    return RTT_OK;
}

} // namespace rtt
