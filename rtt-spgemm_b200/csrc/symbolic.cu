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
// src/super16_symbolic.cuh:1399-1662): exact structure of every C tile as 16
// row masks, C(I,J)[r] = OR over K, over k in A(I,K)[r] of B(K,J)[k].  For each
// K of the tile row, the lanes take the B tiles of B.row(K) (one per lane),
// stage their 16 row masks in shared memory and OR them over A(I,K)'s entries
// row by row; results are OR-ed into the window's slot masks with shared
// atomics.  Per-tile counts, per-(tile,row) CSR prefixes, per-row counts and
// the tile row total come straight out of the masks with popc.
#include "rtt_internal.cuh"

#include <climits>

namespace rtt
{
namespace
{

constexpr int WWORDS = 256;             // bitmap words per warp -> 8192 tile columns
constexpr int WBITS = WWORDS * 32;
constexpr int SCAP = 256;               // C tiles per window in step 2
constexpr int SYM_WARPS = 4;            // warps per CTA

struct WarpSmem1
{
    uint32_t bitmap[WWORDS];
    int start[32];
    int pre[32];
};

struct WarpSmem2
{
    uint32_t bitmap[WWORDS];
    int wordpre[WWORDS];
    int start[32];
    int pre[32];
    uint32_t smask[SCAP * 8];           // 16 u16 rows per slot
    uint32_t bmask[32 * 17];            // per-lane staged B masks, stride 17
    int rowcnt[TD];
};

// Window bounds [lo, hi] of the tile columns reachable from tile row I.
__device__ __forceinline__ void row_window(const DevTiles &A, const DevTiles &B, int a0, int a1,
                                           int &lo, int &hi)
{
    const int lane = lane_id();
    lo = INT_MAX;
    hi = -1;
    for (int a = a0 + lane; a < a1; a += 32)
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

__global__ void __launch_bounds__(SYM_WARPS * 32) k_sym_count(DevTiles A, DevTiles B, int *cnt)
{
    __shared__ WarpSmem1 sm[SYM_WARPS];
    const int lane = lane_id(), wi = threadIdx.x >> 5;
    const int I = blockIdx.x * SYM_WARPS + wi;
    if (I >= A.tilem)
        return;
    WarpSmem1 &S = sm[wi];
    const int a0 = __ldg(A.tile_ptr + I), a1 = __ldg(A.tile_ptr + I + 1);
    int lo, hi;
    row_window(A, B, a0, a1, lo, hi);
    int count = 0;
    if (hi >= 0)
    {
        const bool multi = (long long)hi - lo + 1 > WBITS;
        for (long long w = lo; w <= hi; w += WBITS)
        {
            for (int i = lane; i < WWORDS; i += 32)
                S.bitmap[i] = 0;
            __syncwarp();
            const int wend = (int)min((long long)hi + 1, w + WBITS);
            fill_bitmap(A, B, a0, a1, (int)w, wend, multi, S.bitmap, S.start, S.pre);
            int c = 0;
            for (int i = lane; i < WWORDS; i += 32)
                c += __popc(S.bitmap[i]);
            count += warp_sum(c);
            __syncwarp();
        }
    }
    if (lane == 0)
        cnt[I] = count;
}

// Step 2.  Outputs per C tile: column, tile row, 16 row masks, entry count and
// the per-row CSR prefix within the tile row; per scalar row: entry count;
// per tile row: entry total.
__global__ void __launch_bounds__(SYM_WARPS * 32)
    k_sym_struct(DevTiles A, DevTiles B, const int *__restrict__ c_tile_ptr,
                 int *__restrict__ c_tile_col, int *__restrict__ c_tile_row,
                 uint32_t *__restrict__ c_mask32, int *__restrict__ c_tile_cnt,
                 int *__restrict__ c_row_prefix, int *__restrict__ c_row_cnt,
                 int *__restrict__ c_tr_nnz, int *err)
{
    extern __shared__ __align__(16) unsigned char dyn[];
    WarpSmem2 &S = reinterpret_cast<WarpSmem2 *>(dyn)[threadIdx.x >> 5];
    const int lane = lane_id();
    const int I = blockIdx.x * SYM_WARPS + (threadIdx.x >> 5);
    if (I >= A.tilem)
        return;
    const int a0 = __ldg(A.tile_ptr + I), a1 = __ldg(A.tile_ptr + I + 1);
    const int cbeg = c_tile_ptr[I], cend = c_tile_ptr[I + 1];
    if (lane < TD)
        S.rowcnt[lane] = 0;
    int lo, hi;
    row_window(A, B, a0, a1, lo, hi);
    int cbase = cbeg;
    int rowrun = 0; // lane r (< 16): running CSR prefix of row r over the row's tiles
    const bool multi = hi >= 0 && ((long long)hi - lo + 1 > SCAP);
    long long w = lo;
    while (hi >= 0 && w <= hi)
    {
        // choose a window [w, wend) with at most SCAP C tiles
        int width = WBITS;
        int nW = 0;
        int wend = 0;
        for (;;)
        {
            wend = (int)min((long long)hi + 1, w + width);
            for (int i = lane; i < WWORDS; i += 32)
                S.bitmap[i] = 0;
            __syncwarp();
            fill_bitmap(A, B, a0, a1, (int)w, wend, multi, S.bitmap, S.start, S.pre);
            int c = 0;
            for (int i = lane; i < WWORDS; i += 32)
                c += __popc(S.bitmap[i]);
            nW = warp_sum(c);
            if (nW <= SCAP || width <= SCAP)
                break;
            width >>= 1;
            __syncwarp();
        }
        // word prefix of the bitmap (slot rank lookup)
        {
            int run = 0;
            for (int base = 0; base < WWORDS; base += 32)
            {
                const int v = __popc(S.bitmap[base + lane]);
                const int incl = warp_incl_scan(v);
                S.wordpre[base + lane] = run + incl - v;
                run += __shfl_sync(FULL, incl, 31);
            }
        }
        for (int i = lane; i < nW * 8; i += 32)
            S.smask[i] = 0;
        __syncwarp();
        if (cbase + nW > cend)
        {
            set_error(err, DERR_SYM_OVERFLOW);
            return;
        }
        // C tile columns of this window
        for (int wi = lane; wi < WWORDS; wi += 32)
        {
            uint32_t bits = S.bitmap[wi];
            int slot = S.wordpre[wi];
            while (bits)
            {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1;
                c_tile_col[cbase + slot] = (int)w + wi * 32 + b;
                c_tile_row[cbase + slot] = I;
                ++slot;
            }
        }
        // mask products, one B tile per lane, K by K
        for (int a = a0; a < a1; ++a)
        {
            const int K = __ldg(A.tile_col + a);
            const int b0 = __ldg(B.tile_ptr + K), b1 = __ldg(B.tile_ptr + K + 1);
            int s = b0, e = b1;
            if (multi)
            {
                s = lower_bound(B.tile_col, b0, b1, (int)w);
                e = lower_bound(B.tile_col, s, b1, wend);
            }
            if (s >= e)
                continue;
            const int an = __ldg(A.tile_nnz + a);
            const uint4 ap = *reinterpret_cast<const uint4 *>(A.ptr + (size_t)a * TD);
            const int aend = __ldg(A.tile_nnz + a + 1) - an;
            for (int jb0 = s; jb0 < e; jb0 += 32)
            {
                const int jb = jb0 + lane;
                const bool act = jb < e;
                int slot = 0;
                if (act)
                {
                    const int J = __ldg(B.tile_col + jb);
                    const int tb = B.row_data ? __ldg(B.row_data + jb) : jb;
                    const int off = J - (int)w;
                    const uint32_t word = S.bitmap[off >> 5];
                    slot = S.wordpre[off >> 5] + __popc(word & ((1u << (off & 31)) - 1u));
                    const uint4 *bm = reinterpret_cast<const uint4 *>(B.mask + (size_t)tb * TD);
                    const uint4 m0 = __ldg(bm), m1 = __ldg(bm + 1);
                    uint32_t *dst = &S.bmask[lane * 17];
                    const uint32_t wv[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                    {
                        dst[2 * q] = wv[q] & 0xFFFFu;
                        dst[2 * q + 1] = wv[q] >> 16;
                    }
                }
                __syncwarp();
                if (act)
                {
                    const uint32_t *bml = &S.bmask[lane * 17];
                    const uint32_t pw[4] = {ap.x, ap.y, ap.z, ap.w};
                    uint32_t prod[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        prod[q] = 0;
#pragma unroll
                    for (int r = 0; r < TD; ++r)
                    {
                        const int i0 = (pw[r >> 2] >> ((r & 3) * 8)) & 0xFF;
                        const int i1 = r == TD - 1 ? aend : ((pw[(r + 1) >> 2] >> (((r + 1) & 3) * 8)) & 0xFF);
                        uint32_t pr = 0;
                        for (int i = i0; i < i1; ++i)
                            pr |= bml[__ldg(A.col + an + i) & 15];
                        prod[r >> 1] |= pr << ((r & 1) * 16);
                    }
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        if (prod[q])
                            atomicOr(&S.smask[slot * 8 + q], prod[q]);
                }
                __syncwarp();
            }
        }
        __syncwarp();
        // write masks, tile counts and per-row prefixes; accumulate row counts
        for (int q = lane; q < nW * 8; q += 32)
            c_mask32[(size_t)(cbase + q / 8) * 8 + (q & 7)] = S.smask[q];
        for (int sl = lane; sl < nW; sl += 32)
        {
            int c = 0;
#pragma unroll
            for (int q = 0; q < 8; ++q)
                c += __popc(S.smask[sl * 8 + q]);
            c_tile_cnt[cbase + sl] = c;
        }
        // per-row running prefix across the window's tiles (lanes = rows)
        if (lane < TD)
        {
            const int r = lane;
            for (int sl = 0; sl < nW; ++sl)
            {
                c_row_prefix[(size_t)(cbase + sl) * TD + r] = rowrun;
                rowrun += __popc((S.smask[sl * 8 + (r >> 1)] >> ((r & 1) * 16)) & 0xFFFFu);
            }
        }
        __syncwarp();
        cbase += nW;
        w = wend;
    }
    if (cbase != cend)
        set_error(err, DERR_SYM_OVERFLOW);
    const int nrows = min(TD, A.m - I * TD);
    int total = 0;
    if (lane < TD)
    {
        if (lane < nrows)
            c_row_cnt[I * TD + lane] = rowrun;
        total = rowrun;
    }
    total = warp_sum(total);
    if (lane == 0)
        c_tr_nnz[I] = total;
}

__global__ void k_set_i64(long long *p, long long v) { *p = v; }

inline int grid_for(long long threads, int block) { return (int)((threads + block - 1) / block); }

} // namespace

int symbolic_device(Workspace &ws, const DevTiles &A, const DevTiles &B, SymbolicOut &S)
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
    if (tilem > 0)
    {
        k_sym_count<<<ceil_div(tilem, SYM_WARPS), SYM_WARPS * 32, 0, s>>>(A, B, cnt);
        ws.launches++;
    }
    RTT_CHECK(scan_exclusive_int(ws, cnt, S.c_tile_ptr.as<int>(), tilem));
    int numtile = 0;
    RTT_CHECK(read_int(ws, S.c_tile_ptr.as<int>() + tilem, &numtile));
    RTT_CHECK(check_device_error(ws, "symbolic step 1"));
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
    RTT_CHECK(S.row_prefix.ensure(sizeof(int) * nt * TD, s));
    if (tilem > 0)
    {
        const size_t smem = sizeof(WarpSmem2) * SYM_WARPS;
        RTT_CUDA(cudaFuncSetAttribute(k_sym_struct, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        k_sym_struct<<<ceil_div(tilem, SYM_WARPS), SYM_WARPS * 32, smem, s>>>(
            A, B, S.c_tile_ptr.as<int>(), S.c_tile_col.as<int>(), S.c_tile_row.as<int>(),
            S.c_mask.as<uint32_t>(), S.tile_cnt.as<int>(), S.row_prefix.as<int>(),
            S.c_row_cnt.as<int>(), S.c_tr_nnz.as<int>(), ws.err.as<int>());
        ws.launches++;
    }
    // exact sizes: nnz(C) as int64 over tile rows first (int32 overflow check)
    long long *tr64 = S.c_rowptr.as<long long>();
    RTT_CHECK(scan_exclusive_i64(ws, S.c_tr_nnz.as<int>(), tr64, tilem));
    long long nnz = 0;
    RTT_CHECK(read_i64(ws, tr64 + tilem, &nnz));
    RTT_CHECK(check_device_error(ws, "symbolic step 2"));
    S.nnz = nnz;
    if (nnz > (long long)INT_MAX)
        return fail(RTT_ERR_UNREPRESENTABLE, "nnz(C) = " + std::to_string(nnz) +
                                                 " exceeds the int32 offsets of SMatrix / CSR");
    RTT_CHECK(scan_exclusive_int(ws, S.tile_cnt.as<int>(), S.c_tile_nnz.as<int>(), numtile));
    return RTT_OK;
}

} // namespace rtt
