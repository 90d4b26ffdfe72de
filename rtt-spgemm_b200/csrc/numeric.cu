// numeric.cu - C's CSR row pointer from the symbolic counts.
//
// rowptr[16 I + r] = base(I) + sum of the counts of rows 16 I .. 16 I + r - 1,
// with base(I) the int64 exclusive scan of the tile-row totals (the symbolic
// step checked that nnz(C) fits int32).  Two tile rows per warp, one half-warp
// scan each.
#include "rtt_internal.cuh"

namespace rtt
{
namespace
{

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

} // namespace rtt
