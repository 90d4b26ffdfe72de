// batched.cu - many independent products through one pipeline run.
//
// A batch of products C_i = A_i * B_i is one product of block-diagonal
// matrices: diag(A_1, ..., A_k) * diag(B_1, ..., B_k) = diag(C_1, ..., C_k).
// Every block starts on a 16-row and 16-column boundary (each instance's
// dimensions are padded up to a multiple of the tile edge with empty rows),
// so no 16x16 tile mixes two instances and the tile rows of all instances are
// the work items of one launch of each stage: csr2tile, the two symbolic
// steps and the numeric step each run once for the whole batch, the hardware
// block scheduler acting as the cross-instance work queue.  Kernels here
// assemble the block-diagonal operands from per-instance device arrays, sum
// each instance's output count, and split the product back into per-instance
// CSR (row pointers from 0, instance-local columns).
#include "rtt_internal.cuh"

#include <algorithm>

namespace rtt
{
namespace
{

// instance owning big row r: last i with row_off[i] <= r
__device__ __forceinline__ int instance_of(const int *__restrict__ off, int count, int r)
{
    int lo = 0, hi = count; // invariant off[lo] <= r < off[hi]
    while (hi - lo > 1)
    {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= r)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// One warp per row of the block-diagonal matrix.  Every instance's row
// pointer is checked against its own entry count and every column against its
// own width before anything is written: a broken instance sets the device
// error word (the batch fails as a whole) and cannot write outside its part.
__global__ void k_batch_assemble(int count, int total_rows, const int *const *__restrict__ rp_tab,
                                 const int *const *__restrict__ ci_tab,
                                 const double *const *__restrict__ va_tab,
                                 const int *__restrict__ rows, const int *__restrict__ cols,
                                 const int *__restrict__ row_off,
                                 const int *__restrict__ col_add, const int *__restrict__ nnz_off,
                                 int *__restrict__ out_rp, int *__restrict__ out_col,
                                 double *__restrict__ out_val, int *err)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w > total_rows)
        return;
    const int r = (int)w;
    if (r == total_rows)
    {
        if (lane == 0)
            out_rp[r] = nnz_off[count];
        return;
    }
    const int i = instance_of(row_off, count, r);
    const int j = r - row_off[i];
    if (j >= rows[i])
    {
        if (lane == 0)
            out_rp[r] = nnz_off[i + 1]; // padding row: empty
        return;
    }
    const int *rp = rp_tab[i];
    const int base = nnz_off[i], nnz_i = nnz_off[i + 1] - base;
    int b = rp[j], e = rp[j + 1];
    if (b < 0 || e < b || e > nnz_i)
    {
        if (lane == 0)
            set_error(err, DERR_CSR_ROWPTR);
        b = e = min(max(b, 0), nnz_i);
    }
    if (lane == 0)
        out_rp[r] = base + b;
    const int *ci = ci_tab[i];
    const double *va = va_tab[i];
    const int add = col_add[i], ncols = cols[i];
    for (int k = b + lane; k < e; k += 32)
    {
        int cc = ci[k];
        if ((unsigned)cc >= (unsigned)ncols)
        {
            set_error(err, DERR_CSR_COL);
            cc = 0;
        }
        out_col[base + k] = cc + add;
        out_val[base + k] = va[k];
    }
}

// One CTA per instance: entries of C_i = sum of its rows' counts.
__global__ void k_batch_count(int count, const int *__restrict__ row_off,
                              const int *__restrict__ rows, const int *__restrict__ row_cnt,
                              long long *__restrict__ nnz)
{
    const int i = blockIdx.x;
    if (i >= count)
        return;
    long long s = 0;
    for (int j = threadIdx.x; j < rows[i]; j += blockDim.x)
        s += row_cnt[row_off[i] + j];
    s = warp_sum(s);
    __shared__ long long part[32];
    if ((threadIdx.x & 31) == 0)
        part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        long long t = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q)
            t += part[q];
        nnz[i] = t;
    }
}

// One warp per big row: per-instance row pointer and instance-local columns.
__global__ void k_batch_split(int count, int total_rows, const int *__restrict__ row_off,
                              const int *__restrict__ rows, const int *__restrict__ sec_off,
                              const int *__restrict__ col_sub, const int *__restrict__ big_rp,
                              int *__restrict__ out_rp, int *__restrict__ col)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= total_rows)
        return;
    const int r = (int)w;
    const int i = instance_of(row_off, count, r);
    const int j = r - row_off[i];
    if (j >= rows[i])
        return;
    const int r0 = row_off[i];
    const int base = big_rp[r0];
    if (lane == 0)
    {
        out_rp[sec_off[i] + j] = big_rp[r] - base;
        if (j == rows[i] - 1)
            out_rp[sec_off[i] + j + 1] = big_rp[r + 1] - base;
    }
    const int sub = col_sub[i];
    for (int e = big_rp[r] + lane; e < big_rp[r + 1]; e += 32)
        col[e] -= sub;
}

// instances without rows: their row pointer section is the single entry 0
__global__ void k_batch_empty(int count, const int *__restrict__ rows,
                              const int *__restrict__ sec_off, int *__restrict__ out_rp)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count && rows[i] == 0)
        out_rp[sec_off[i]] = 0;
}

// New values of every instance into the block-diagonal value array (the
// structure assembled by k_batch_assemble stays): blockIdx.y is the instance,
// the x blocks stride over its entries.
__global__ void k_batch_values(int count, const double *const *__restrict__ va_tab,
                               const int *__restrict__ nnz_off, double *__restrict__ out_val)
{
    const int i = blockIdx.y;
    if (i >= count)
        return;
    const int b = nnz_off[i], n = nnz_off[i + 1] - b;
    const double *src = va_tab[i];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        out_val[b + j] = src[j];
}

inline int warps_grid(long long warps) { return (int)((warps * 32 + 255) / 256); }

} // namespace

int batch_assemble_device(Workspace &ws, int count, int total_rows, const int *const *rp_tab,
                          const int *const *ci_tab, const double *const *va_tab, const int *rows,
                          const int *cols, const int *row_off, const int *col_add,
                          const int *nnz_off, int *out_rp, int *out_col, double *out_val)
{
    k_batch_assemble<<<warps_grid((long long)total_rows + 1), 256, 0, ws.stream>>>(
        count, total_rows, rp_tab, ci_tab, va_tab, rows, cols, row_off, col_add, nnz_off, out_rp,
        out_col, out_val, ws.err.as<int>());
    ws.launches++;
    RTT_CUDA(cudaGetLastError());
    return RTT_OK;
}

int batch_count_device(Workspace &ws, int count, const int *row_off, const int *rows,
                       const int *row_cnt, long long *nnz)
{
    if (count > 0)
    {
        k_batch_count<<<count, 256, 0, ws.stream>>>(count, row_off, rows, row_cnt, nnz);
        ws.launches++;
        RTT_CUDA(cudaGetLastError());
    }
    return RTT_OK;
}

int batch_values_device(Workspace &ws, int count, int max_nnz, const double *const *va_tab,
                        const int *nnz_off, double *out_val)
{
    if (count > 0 && max_nnz > 0)
    {
        const int xb = std::min((max_nnz + 255) / 256, 64);
        for (int y0 = 0; y0 < count; y0 += 65535) // gridDim.y limit
        {
            const int ny = std::min(count - y0, 65535);
            k_batch_values<<<dim3(xb, ny), 256, 0, ws.stream>>>(ny, va_tab + y0, nnz_off + y0,
                                                                out_val);
            ws.launches++;
        }
        RTT_CUDA(cudaGetLastError());
    }
    return RTT_OK;
}

int batch_split_device(Workspace &ws, int count, int total_rows, const int *row_off,
                       const int *rows, const int *sec_off, const int *col_sub, const int *big_rp,
                       int *out_rp, int *col)
{
    if (total_rows > 0)
    {
        k_batch_split<<<warps_grid(total_rows), 256, 0, ws.stream>>>(
            count, total_rows, row_off, rows, sec_off, col_sub, big_rp, out_rp, col);
        ws.launches++;
    }
    if (count > 0)
    {
        k_batch_empty<<<(count + 255) / 256, 256, 0, ws.stream>>>(count, rows, sec_off, out_rp);
        ws.launches++;
    }
    RTT_CUDA(cudaGetLastError());
    return RTT_OK;
}

} // namespace rtt
