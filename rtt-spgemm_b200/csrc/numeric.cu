// numeric.cu - step 3 (values) of the tiled SpGEMM on sm_100a.
//
// One warp per C tile (I, J) (reference step4, src/spgemm-cpu.h:284-367, and
// the per-task numeric kernels, src/dmma_spgemm.h:4164-4410, :5385-5465).
//  1. Tile pairs: the K lists A.row(I) and B.col(J) are intersected by binary
//     search - each lane takes one K of B.col(J) and searches A.row(I) - and
//     the matches are compacted with a ballot, in ascending K, 32 at a time.
//  2. Sparse pairs: lanes 0-15 take even pairs, lanes 16-31 odd pairs; lane r
//     walks A(I,K)'s row r and, for each entry (k, a), B(K,J)'s row k,
//     accumulating into a private 16x16 FP64 accumulator row in shared memory
//     (no atomics; the summation order per output is fixed, so the result is
//     bitwise reproducible run to run and independent of other work).
//  3. Dense pairs (nnz(A tile) * nnz(B tile) >= cutoff): both tiles are
//     expanded to dense 16x16 in shared memory and multiplied on the FP64
//     tensor cores with 16 mma.sync.m8n8k4 (2x2 output quadrants x 4 k-steps;
//     A in 8x4 sub-tiles, B in 4x8 sub-tiles).  tcgen05 has no FP64 kind, so
//     the warp-level DMMA is the Blackwell FP64 tensor-core instruction.
//  4. Output: the C mask (from the symbolic step) orders the entries; lanes
//     write the tile format (row offsets, column bytes, values) and/or the
//     final CSR (row pointer + per-(tile,row) prefix from the symbolic step),
//     i.e. tile2csr fused into the numeric pass.
#include "rtt_internal.cuh"

#include <climits>

namespace rtt
{
namespace
{

constexpr int NUM_WARPS = 8;

struct NumSmem
{
    double acc[2][TD * TD];
    int pa[32];
    int pb[32];
    int pd[32];
};

struct NumSmemDense
{
    double acc[2][TD * TD];
    int pa[32];
    int pb[32];
    int pd[32];
    double da[TD * TD];
    double db[TD * TD];
};

__device__ __forceinline__ void dmma_m8n8k4(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <bool DMMA, typename Smem>
__global__ void __launch_bounds__(NUM_WARPS * 32)
    k_numeric(DevTiles A, DevTiles B, int numtileC, long long nnzC,
              const int *__restrict__ c_tile_row, const int *__restrict__ c_tile_col,
              const uint16_t *__restrict__ c_mask, const int *__restrict__ c_tile_nnz,
              uint8_t *__restrict__ c_ptr, uint8_t *__restrict__ c_colb, double *__restrict__ c_val,
              const int *__restrict__ c_row_prefix, const int *__restrict__ csr_rowptr,
              int *__restrict__ csr_col, double *__restrict__ csr_val, int cutoff,
              long long *counters, int *err)
{
    extern __shared__ __align__(16) unsigned char dyn[];
    Smem &S = reinterpret_cast<Smem *>(dyn)[threadIdx.x >> 5];
    const int lane = lane_id();
    const int s = blockIdx.x * NUM_WARPS + (threadIdx.x >> 5);
    if (s >= numtileC)
        return;
    const int r = lane & 15, h = lane >> 4;
    const unsigned lt = (1u << lane) - 1u;
    const int I = __ldg(c_tile_row + s), J = __ldg(c_tile_col + s);

    double *acc_flat = &S.acc[0][0];
    for (int i = lane; i < 2 * TD * TD; i += 32)
        acc_flat[i] = 0.0;
    double d[8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
        d[i] = 0.0;
    long long n_dense = 0, n_pairs = 0;

    const int a0 = __ldg(A.tile_ptr + I), a1 = __ldg(A.tile_ptr + I + 1);
    const int b0 = __ldg(B.csc_ptr + J), b1 = __ldg(B.csc_ptr + J + 1);
    __syncwarp();
    for (int p0 = b0; p0 < b1; p0 += 32)
    {
        const int p = p0 + lane;
        bool found = false;
        int ia = 0, tb = 0, dense = 0;
        if (p < b1 && a0 < a1)
        {
            const int K = __ldg(B.csc_row + p);
            ia = lower_bound(A.tile_col, a0, a1, K);
            found = ia < a1 && __ldg(A.tile_col + ia) == K;
            if (found)
            {
                tb = B.csc_data ? __ldg(B.csc_data + p) : p;
                if (DMMA)
                {
                    const long long na = __ldg(A.tile_nnz + ia + 1) - __ldg(A.tile_nnz + ia);
                    const long long nb = __ldg(B.tile_nnz + tb + 1) - __ldg(B.tile_nnz + tb);
                    dense = na * nb >= (long long)cutoff ? 1 : 0;
                }
            }
        }
        const unsigned bal = __ballot_sync(FULL, found);
        const int nq = __popc(bal);
        n_pairs += nq;
        n_dense += __popc(__ballot_sync(FULL, found && dense));
        if (found)
        {
            const int idx = __popc(bal & lt);
            S.pa[idx] = ia;
            S.pb[idx] = tb;
            S.pd[idx] = dense;
        }
        __syncwarp();
        // sparse pairs: half h takes pairs h, h+2, ...; lane r owns row r
        double *accr = &S.acc[h][r * TD];
        for (int q = h; q < nq; q += 2)
        {
            if (DMMA && S.pd[q])
                continue;
            const int ta = S.pa[q], tbq = S.pb[q];
            const int an = __ldg(A.tile_nnz + ta);
            const int i0 = an + A.ptr[(size_t)ta * TD + r];
            const int i1 = r == TD - 1 ? __ldg(A.tile_nnz + ta + 1) : an + A.ptr[(size_t)ta * TD + r + 1];
            if (i0 >= i1)
                continue;
            const int bn = __ldg(B.tile_nnz + tbq), bend = __ldg(B.tile_nnz + tbq + 1);
            const uint8_t *bptr = B.ptr + (size_t)tbq * TD;
            for (int i = i0; i < i1; ++i)
            {
                const int kk = __ldg(A.col + i) & 15;
                const double a = __ldg(A.val + i);
                const int f0 = bn + bptr[kk];
                const int f1 = kk == TD - 1 ? bend : bn + bptr[kk + 1];
                for (int f = f0; f < f1; ++f)
                {
                    const int c = __ldg(B.col + f) & 15;
                    accr[c] = fma(a, __ldg(B.val + f), accr[c]);
                }
            }
        }
        __syncwarp();
        if constexpr (DMMA)
        {
            NumSmemDense &D = reinterpret_cast<NumSmemDense &>(S);
            for (int q = 0; q < nq; ++q)
            {
                if (!D.pd[q])
                    continue;
                const int ta = D.pa[q], tbq = D.pb[q];
                for (int i = lane; i < TD * TD; i += 32)
                {
                    D.da[i] = 0.0;
                    D.db[i] = 0.0;
                }
                __syncwarp();
                if (lane < TD)
                {
                    const int an = __ldg(A.tile_nnz + ta);
                    const int i0 = an + A.ptr[(size_t)ta * TD + r];
                    const int i1 = r == TD - 1 ? __ldg(A.tile_nnz + ta + 1)
                                               : an + A.ptr[(size_t)ta * TD + r + 1];
                    for (int i = i0; i < i1; ++i)
                        D.da[r * TD + (__ldg(A.col + i) & 15)] += __ldg(A.val + i);
                }
                else
                {
                    const int bn = __ldg(B.tile_nnz + tbq);
                    const int f0 = bn + B.ptr[(size_t)tbq * TD + r];
                    const int f1 = r == TD - 1 ? __ldg(B.tile_nnz + tbq + 1)
                                               : bn + B.ptr[(size_t)tbq * TD + r + 1];
                    for (int f = f0; f < f1; ++f)
                        D.db[r * TD + (__ldg(B.col + f) & 15)] += __ldg(B.val + f);
                }
                __syncwarp();
                const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
                for (int qr = 0; qr < 2; ++qr)
#pragma unroll
                    for (int qc = 0; qc < 2; ++qc)
#pragma unroll
                        for (int kb = 0; kb < 4; ++kb)
                        {
                            const double av = D.da[(qr * 8 + g) * TD + kb * 4 + t4];
                            const double bv = D.db[(kb * 4 + t4) * TD + qc * 8 + g];
                            dmma_m8n8k4(d[(qr * 2 + qc) * 2], d[(qr * 2 + qc) * 2 + 1], av, bv);
                        }
                __syncwarp();
            }
        }
    }
    if constexpr (DMMA)
    {
        __syncwarp();
        const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
        for (int qr = 0; qr < 2; ++qr)
#pragma unroll
            for (int qc = 0; qc < 2; ++qc)
#pragma unroll
                for (int i = 0; i < 2; ++i)
                    S.acc[0][(qr * 8 + g) * TD + qc * 8 + t4 * 2 + i] += d[(qr * 2 + qc) * 2 + i];
    }
    __syncwarp();
    if (counters != nullptr && lane == 0)
    {
        atomicAdd((unsigned long long *)&counters[0], (unsigned long long)n_dense);
        atomicAdd((unsigned long long *)&counters[1], (unsigned long long)(n_pairs - n_dense));
    }
    // ---- output
    const uint32_t mr = __ldg(c_mask + (size_t)s * TD + r);
    const int cnt = __popc(mr);
    const int excl = half_incl_scan(cnt) - cnt;
    uint32_t sub = (mr >> (8 - 8 * h)) & 0xFFu;
    int rank = h ? __popc(mr >> 8) : 0;
    const double *a0r = &S.acc[0][r * TD];
    const double *a1r = &S.acc[1][r * TD];
    if (c_val != nullptr)
    {
        const int toff = __ldg(c_tile_nnz + s);
        if (h == 0)
            c_ptr[(size_t)s * TD + r] = (uint8_t)excl;
        uint32_t b = sub;
        int k = rank;
        while (b)
        {
            const int lead = __clz(b) - 24;
            b &= ~(0x80u >> lead);
            const int c = 8 * h + lead;
            const long long pos = (long long)toff + excl + k;
            ++k;
            if (pos < 0 || pos >= nnzC)
            {
                set_error(err, DERR_NUM_BOUNDS);
                break;
            }
            c_colb[pos] = (uint8_t)c;
            c_val[pos] = a0r[c] + a1r[c];
        }
    }
    if (csr_col != nullptr)
    {
        const int row = I * TD + r;
        if (row < A.m)
        {
            const long long base = (long long)__ldg(csr_rowptr + row) + __ldg(c_row_prefix + (size_t)s * TD + r);
            uint32_t b = sub;
            int k = rank;
            while (b)
            {
                const int lead = __clz(b) - 24;
                b &= ~(0x80u >> lead);
                const int c = 8 * h + lead;
                const long long pos = base + k;
                ++k;
                if (pos < 0 || pos >= nnzC)
                {
                    set_error(err, DERR_NUM_BOUNDS);
                    break;
                }
                csr_col[pos] = J * TD + c;
                csr_val[pos] = a0r[c] + a1r[c];
            }
        }
    }
}

// CSR row pointer of C from per-row counts and the int64 tile-row bases.
__global__ void k_csr_rowptr(int tilem, int m, const long long *__restrict__ tr_base,
                             const int *__restrict__ row_cnt, int *__restrict__ rowptr)
{
    const int lane = threadIdx.x & 31, hl = lane & 15;
    const int I = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 2 + (lane >> 4);
    const int row = I * TD + hl;
    const int c = (I < tilem && row < m) ? row_cnt[row] : 0;
    const int excl = half_incl_scan(c) - c;
    if (I < tilem && row < m)
        rowptr[row] = (int)(tr_base[I] + excl);
    if (I == tilem - 1 && hl == 0)
        rowptr[m] = (int)tr_base[tilem];
}

inline int grid_for(long long threads, int block) { return (int)((threads + block - 1) / block); }

} // namespace

int csr_rowptr_device(Workspace &ws, SymbolicOut &S, int *rowptr)
{
    if (S.tilem == 0)
    {
        RTT_CUDA(cudaMemsetAsync(rowptr, 0, sizeof(int), ws.stream));
        return RTT_OK;
    }
    k_csr_rowptr<<<grid_for((long long)ceil_div(S.tilem, 2) * 32, 256), 256, 0, ws.stream>>>(
        S.tilem, S.m, S.c_rowptr.as<long long>(), S.c_row_cnt.as<int>(), rowptr);
    ws.launches++;
    return RTT_OK;
}

int numeric_device(Workspace &ws, const DevTiles &A, const DevTiles &B, SymbolicOut &S,
                   const NumericConfig &cfg)
{
    cudaStream_t s = ws.stream;
    const size_t nt = (size_t)S.numtile;
    const size_t nnz = (size_t)S.nnz;
    if (cfg.write_tiles)
    {
        RTT_CHECK(S.c_col.ensure(nnz + 16, s));
        RTT_CHECK(S.c_val.ensure(sizeof(double) * nnz + 16, s));
    }
    if (cfg.csr_col != nullptr)
        RTT_CHECK(csr_rowptr_device(ws, S, cfg.csr_rowptr));
    if (nt == 0)
        return RTT_OK;
    const int grid = (int)((nt + NUM_WARPS - 1) / NUM_WARPS);
    if (cfg.ev_begin != nullptr)
        RTT_CUDA(cudaEventRecord(cfg.ev_begin, s));
    if (cfg.dmma_pair_cutoff > 0)
    {
        const size_t smem = sizeof(NumSmemDense) * NUM_WARPS;
        RTT_CUDA(cudaFuncSetAttribute(k_numeric<true, NumSmemDense>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_numeric<true, NumSmemDense><<<grid, NUM_WARPS * 32, smem, s>>>(
            A, B, (int)nt, S.nnz, S.c_tile_row.as<int>(), S.c_tile_col.as<int>(),
            S.c_mask.as<uint16_t>(), S.c_tile_nnz.as<int>(), S.c_ptr.as<uint8_t>(),
            cfg.write_tiles ? S.c_col.as<uint8_t>() : nullptr,
            cfg.write_tiles ? S.c_val.as<double>() : nullptr, S.row_prefix.as<int>(), cfg.csr_rowptr,
            cfg.csr_col, cfg.csr_val, cfg.dmma_pair_cutoff, cfg.counters, ws.err.as<int>());
    }
    else
    {
        const size_t smem = sizeof(NumSmem) * NUM_WARPS;
        RTT_CUDA(cudaFuncSetAttribute(k_numeric<false, NumSmem>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_numeric<false, NumSmem><<<grid, NUM_WARPS * 32, smem, s>>>(
            A, B, (int)nt, S.nnz, S.c_tile_row.as<int>(), S.c_tile_col.as<int>(),
            S.c_mask.as<uint16_t>(), S.c_tile_nnz.as<int>(), S.c_ptr.as<uint8_t>(),
            cfg.write_tiles ? S.c_col.as<uint8_t>() : nullptr,
            cfg.write_tiles ? S.c_val.as<double>() : nullptr, S.row_prefix.as<int>(), cfg.csr_rowptr,
            cfg.csr_col, cfg.csr_val, 0, cfg.counters, ws.err.as<int>());
    }
    ws.launches++;
    if (cfg.ev_end != nullptr)
        RTT_CUDA(cudaEventRecord(cfg.ev_end, s));
    return RTT_OK;
}

} // namespace rtt
