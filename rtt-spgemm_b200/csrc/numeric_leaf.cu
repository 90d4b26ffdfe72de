// numeric_leaf.cu - the numeric step on the FP64 tensor cores, straight from
// hybrid leaf tiles (A as 8x4 leaves, B as 4x8 leaves with their CSC).
//
// The reference's DMMA numeric (dmma_numeric_kernel, src/dmma_spgemm.h:
// 4164-4304, with dmma_decode_value, :4148-4162) computes every 8x8 C tile as
// a sum over K of 8x4 A leaf times 4x8 B leaf products.  The leaf layouts are
// chosen so that the physical index of an element is the lane that holds it
// in the mma.sync.m8n8k4.f64 fragments: A leaf (r, k) at r * 4 + k = lane
// (row lane / 4, column lane % 4), B leaf (k, n) at n * 4 + k = lane (row
// lane % 4, column lane / 4).  A dense leaf (span 32) is one coalesced load
// per lane; a sparse leaf gives the lane its value at the popcount of the
// mask bits below its own, or zero.
//
// Here one warp owns one 16x16 C tile of the symbolic structure and walks
// its four 8x8 quadrants that hold entries: the A leaves of 8-row block I8
// (sorted by K4) are intersected with the B leaves of 8-column block J8 (its
// CSC, sorted by K4) - 32 A leaves at a time, each lane binary-searching its
// K4 in the B column's list - and every match is one DMMA into the lane's
// two accumulators (row lane / 4, columns (lane % 4) * 2 + {0, 1}), in K
// order.  The results go to C's 16x16 tile arrays at the positions the
// symbolic masks give (row offset + entries before the column), and tile2csr
// turns them into CSR.  FP64 throughout; the sums run over whole 4-wide K
// blocks, so values differ from the scalar kernels' in the last bits only
// (within the FP64 bound of the oracle).
#include "rtt_internal.cuh"

#include <climits>

namespace rtt
{
namespace
{

struct LeafView
{
    const int *row_ptr, *col_idx, *value_off, *csc_ptr, *csc_row, *csc_ids;
    const unsigned *mask;
    const double *values;
    int trc, tcc;
};

LeafView leaf_view(const HybridDev &H)
{
    LeafView v{};
    v.row_ptr = H.row_ptr.as<int>();
    v.col_idx = H.col_idx.as<int>();
    v.value_off = H.value_off.as<int>();
    v.csc_ptr = H.has_csc ? H.csc_ptr.as<int>() : nullptr;
    v.csc_row = H.has_csc ? H.csc_row.as<int>() : nullptr;
    v.csc_ids = H.has_csc ? H.csc_ids.as<int>() : nullptr;
    v.mask = H.mask.as<unsigned>();
    v.values = H.values.as<double>();
    v.trc = H.trc;
    v.tcc = H.tcc;
    return v;
}

// The lane's element of leaf t (physical index = lane).
__device__ __forceinline__ double leaf_elem(const LeafView &L, int t, int lane)
{
    const int b = __ldg(L.value_off + t);
    if (__ldg(L.value_off + t + 1) - b == 32)
        return __ldg(L.values + b + lane);
    const unsigned m = __ldg(L.mask + t);
    if (((m >> lane) & 1u) == 0u)
        return 0.0;
    return __ldg(L.values + b + __popc(m & ((1u << lane) - 1u)));
}

__device__ __forceinline__ void leaf_dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

constexpr int LEAF_WARPS = 8;

__global__ void __launch_bounds__(LEAF_WARPS * 32)
    k_numeric_leaf(int numtile, const int *__restrict__ c_tile_row, const int *__restrict__ c_tile_col,
                   const uint16_t *__restrict__ c_mask, const int *__restrict__ c_tile_nnz,
                   long long nnzC, uint8_t *__restrict__ c_ptr, uint8_t *__restrict__ c_colb,
                   double *__restrict__ c_val, LeafView A, LeafView B, long long *counters,
                   int *err)
{
    const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= numtile)
        return;
    const int I = __ldg(c_tile_row + t), J = __ldg(c_tile_col + t);
    // the tile's 16 row masks (bit 15 - c) and each row's first entry
    const uint32_t mrow = lane < TD ? (uint32_t)__ldg(c_mask + t * TD + lane) : 0u;
    const int pc = __popc(mrow);
    const int pre = warp_incl_scan(pc) - pc;
    if (lane < TD)
        c_ptr[t * TD + lane] = (uint8_t)pre;
    const long long tbase = __ldg(c_tile_nnz + t);
    long long n_dmma = 0;
#pragma unroll 1
    for (int q = 0; q < 4; ++q)
    {
        const int dr = q >> 1, dc = q & 1;
        const uint32_t qbits =
            (lane >> 3) == dr && lane < TD ? (mrow >> (dc ? 0 : 8)) & 0xFFu : 0u;
        if (!__any_sync(FULL, qbits != 0u))
            continue;
        const int I8 = 2 * I + dr, J8 = 2 * J + dc;
        if (I8 >= A.trc || J8 >= B.tcc)
            continue; // rows / columns past the matrix: no entries (uniform)
        const int a0 = __ldg(A.row_ptr + I8), a1 = __ldg(A.row_ptr + I8 + 1);
        const int b0 = __ldg(B.csc_ptr + J8), b1 = __ldg(B.csc_ptr + J8 + 1);
        double d0 = 0.0, d1 = 0.0;
        for (int c0 = a0; c0 < a1 && b0 < b1; c0 += 32)
        {
            const int a = c0 + lane;
            int bt = -1;
            if (a < a1)
            {
                const int K = __ldg(A.col_idx + a);
                int lo = b0, hi = b1;
                while (lo < hi)
                {
                    const int mid = (lo + hi) >> 1;
                    if (__ldg(B.csc_row + mid) < K)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                if (lo < b1 && __ldg(B.csc_row + lo) == K)
                    bt = __ldg(B.csc_ids + lo);
            }
            // the matches in K order: one DMMA each
            for (unsigned hits = __ballot_sync(FULL, bt >= 0); hits != 0u; hits &= hits - 1u)
            {
                const int j = __ffs(hits) - 1;
                const int at = c0 + j, btj = __shfl_sync(FULL, bt, j);
                leaf_dmma(d0, d1, leaf_elem(A, at, lane), leaf_elem(B, btj, lane));
                ++n_dmma;
            }
        }
        // lane: row dr * 8 + lane / 4, columns dc * 8 + (lane % 4) * 2 + {0, 1}
        const int r = dr * 8 + (lane >> 2);
        const uint32_t mr = __shfl_sync(FULL, mrow, r);
        const int rpre = __shfl_sync(FULL, pre, r);
#pragma unroll
        for (int u = 0; u < 2; ++u)
        {
            const int c = dc * 8 + (lane & 3) * 2 + u;
            if (mr & (0x8000u >> c))
            {
                const long long pos = tbase + rpre + __popc(mr >> (16 - c));
                if (pos >= nnzC)
                {
                    set_error(err, DERR_NUM_BOUNDS);
                    continue;
                }
                c_colb[pos] = (uint8_t)c;
                c_val[pos] = u ? d1 : d0;
            }
        }
    }
    if (lane == 0 && counters != nullptr && n_dmma > 0)
        atomicAdd((unsigned long long *)&counters[0], (unsigned long long)n_dmma);
}

// nnzCub = sum over A's entries (i, k) of nnz(B row k): one warp per row of A.
__global__ void k_leaf_cub(int m, const int *__restrict__ a_rp, const int *__restrict__ a_ci,
                           int b_m, const int *__restrict__ b_rp, long long *counters)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= m)
        return;
    long long s = 0;
    for (int e = __ldg(a_rp + w) + lane; e < __ldg(a_rp + w + 1); e += 32)
    {
        const int k = __ldg(a_ci + e);
        if (k >= 0 && k < b_m)
            s += __ldg(b_rp + k + 1) - __ldg(b_rp + k);
    }
    s = warp_sum(s);
    if (lane == 0 && s > 0)
        atomicAdd((unsigned long long *)&counters[1], (unsigned long long)s);
}

} // namespace

int numeric_leaf_device(Workspace &ws, const DevTiles &A, const DevTiles &B, HybridDev &LA,
                        HybridDev &LB, SymbolicOut &S, const NumericConfig &cfg)
{
    cudaStream_t s = ws.stream;
    const size_t nnz = (size_t)S.nnz;
    RTT_CHECK(S.c_col.ensure(nnz + 16, s));
    RTT_CHECK(S.c_val.ensure(sizeof(double) * nnz + 16, s));
    // the leaves of this product's operands (the values as they are now)
    RTT_CHECK(csr_to_hybrid_device(ws, A.m, A.n, A.nnz, A.csr_rowptr, A.csr_col, A.csr_val, 8, 4,
                                   0, LEAF_DENSE_THRESHOLD, 0, LA));
    RTT_CHECK(csr_to_hybrid_device(ws, B.m, B.n, B.nnz, B.csr_rowptr, B.csr_col, B.csr_val, 4, 8,
                                   1, LEAF_DENSE_THRESHOLD, 1, LB));
    if (cfg.counters != nullptr && A.m > 0)
    {
        k_leaf_cub<<<(int)(((long long)A.m * 32 + 255) / 256), 256, 0, s>>>(
            A.m, A.csr_rowptr, A.csr_col, B.m, B.csr_rowptr, cfg.counters);
        ws.launches++;
    }
    if (cfg.ev_begin != nullptr)
        RTT_CUDA(cudaEventRecord(cfg.ev_begin, s));
    if (S.numtile > 0)
    {
        const long long threads = (long long)S.numtile * 32;
        k_numeric_leaf<<<(int)((threads + LEAF_WARPS * 32 - 1) / (LEAF_WARPS * 32)),
                         LEAF_WARPS * 32, 0, s>>>(
            S.numtile, S.c_tile_row.as<int>(), S.c_tile_col.as<int>(), S.c_mask.as<uint16_t>(),
            S.c_tile_nnz.as<int>(), S.nnz, S.c_ptr.as<uint8_t>(), S.c_col.as<uint8_t>(),
            S.c_val.as<double>(), leaf_view(LA), leaf_view(LB), cfg.counters, ws.err.as<int>());
        ws.launches++;
    }
    if (cfg.ev_end != nullptr)
        RTT_CUDA(cudaEventRecord(cfg.ev_end, s));
    RTT_CUDA(cudaGetLastError());
    return RTT_OK;
}

} // namespace rtt
