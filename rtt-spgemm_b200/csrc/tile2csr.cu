// tile2csr.cu - square tiles (edge 8 or 16) -> CSR on sm_100a.
//
// Semantics of tile2csr / tile2csr_restore_rows (reference
// src/tile2csr.h:232-329, :337-523): per tile row, per local row, the row's
// entries of each tile in tile order; row bounds clamped into [0, tile nnz];
// entries whose column lies past the tile edge or past n are dropped; an
// optional new->old row map sends reordered row i to original row
// new_to_old[i] (rows at or past the map's size must be empty).  Without the
// canonical promise each row is sorted by column with the same heap sort the
// reference uses, so even duplicate columns come out in the same order.
//
// One thread per (tile row, local row): it walks the tiles of its tile row,
// which keeps the per-row output cursor in a register, exactly like the
// reference's per-tile-row local offsets.
#include "rtt_internal.cuh"

namespace rtt
{
namespace
{

__device__ __forceinline__ void t2c_bounds(const uint8_t *ptr, size_t off, int lr, int rc, int tnz,
                                           int &s, int &e)
{
    int a = ptr[off + lr];
    int b = lr + 1 == rc ? tnz : ptr[off + lr + 1];
    a = min(a, tnz);
    b = max(b, a);
    b = min(b, tnz);
    s = a;
    e = b;
}

__global__ void k_t2c_count(const int *__restrict__ tile_ptr, const int *__restrict__ tile_col,
                            const int *__restrict__ tile_nnz, const uint8_t *__restrict__ ptr,
                            const uint8_t *__restrict__ col, int m, int n, int tilem, int td,
                            const int *__restrict__ new_to_old, int perm_size,
                            const int *__restrict__ row_data, int *__restrict__ row_cnt, int *err)
{
    const long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int tr = (int)(x / td), lr = (int)(x % td);
    if (tr >= tilem)
        return;
    const int row = tr * td + lr;
    if (row >= m)
        return;
    const int rc = min(td, m - tr * td);
    int cnt = 0;
    for (int t = tile_ptr[tr]; t < tile_ptr[tr + 1]; ++t)
    {
        const int d = row_data ? row_data[t] : t; // data index of row-major tile t
        const int tnz = tile_nnz[d + 1] - tile_nnz[d], off = tile_nnz[d];
        const int tc = tile_col[t];
        int s, e;
        t2c_bounds(ptr, (size_t)d * td, lr, rc, tnz, s, e);
        for (int i = s; i < e; ++i)
        {
            const int lc = col[off + i];
            if (lc < td && tc >= 0 && (long long)tc * td + lc < n)
                ++cnt;
        }
    }
    if (perm_size < 0)
        row_cnt[row] = cnt;
    else if (row >= perm_size)
    {
        if (cnt != 0)
            set_error(err, DERR_T2C_TAIL);
    }
    else
        row_cnt[new_to_old[row]] = cnt;
}

__global__ void k_t2c_fill(const int *__restrict__ tile_ptr, const int *__restrict__ tile_col,
                           const int *__restrict__ tile_nnz, const uint8_t *__restrict__ ptr,
                           const uint8_t *__restrict__ col, const double *__restrict__ val, int m,
                           int n, int tilem, int td, const int *__restrict__ new_to_old,
                           int perm_size, const int *__restrict__ row_data,
                           const int *__restrict__ rowptr, long long nnz,
                           int *__restrict__ out_col, double *__restrict__ out_val, int *err)
{
    const long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int tr = (int)(x / td), lr = (int)(x % td);
    if (tr >= tilem)
        return;
    const int row = tr * td + lr;
    if (row >= m)
        return;
    int dst_row = row;
    if (perm_size >= 0)
    {
        if (row >= perm_size)
            return;
        dst_row = new_to_old[row];
    }
    const int rc = min(td, m - tr * td);
    long long o = rowptr[dst_row];
    const long long oend = rowptr[dst_row + 1];
    for (int t = tile_ptr[tr]; t < tile_ptr[tr + 1]; ++t)
    {
        const int d = row_data ? row_data[t] : t; // data index of row-major tile t
        const int tnz = tile_nnz[d + 1] - tile_nnz[d], off = tile_nnz[d];
        const int tc = tile_col[t];
        int s, e;
        t2c_bounds(ptr, (size_t)d * td, lr, rc, tnz, s, e);
        for (int i = s; i < e; ++i)
        {
            const int lc = col[off + i];
            if (lc < td && tc >= 0 && (long long)tc * td + lc < n)
            {
                if (o >= oend || o >= nnz)
                {
                    set_error(err, DERR_T2C_BOUNDS);
                    return;
                }
                out_col[o] = tc * td + lc;
                out_val[o] = val[off + i];
                ++o;
            }
        }
    }
}

// Heap sort of one row by column carrying values (the reference's
// tile2csr_sort_rows, src/tile2csr.h:179-223), one thread per row.
__device__ __forceinline__ void hs_swap(int *c, double *v, long long x, long long y)
{
    int tc = c[x];
    double tv = v[x];
    c[x] = c[y];
    v[x] = v[y];
    c[y] = tc;
    v[y] = tv;
}

__device__ void hs_sift(int *c, double *v, long long b, long long root, long long count)
{
    for (;;)
    {
        long long child = root * 2 + 1;
        if (child >= count)
            return;
        if (child + 1 < count && c[b + child] < c[b + child + 1])
            ++child;
        if (c[b + root] >= c[b + child])
            return;
        hs_swap(c, v, b + root, b + child);
        root = child;
    }
}

__global__ void k_sort_rows(int m, const int *__restrict__ rowptr, int *c, double *v)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m)
        return;
    const long long b = rowptr[r], cnt = rowptr[r + 1] - b;
    for (long long root = cnt / 2; root > 0; --root)
        hs_sift(c, v, b, root - 1, cnt);
    for (long long rem = cnt; rem > 1; --rem)
    {
        hs_swap(c, v, b, b + rem - 1);
        hs_sift(c, v, b, 0, rem - 1);
    }
}

inline int grid_for(long long threads, int block) { return (int)((threads + block - 1) / block); }

} // namespace

int tile2csr_count_device(Workspace &ws, const int *tile_ptr, const int *tile_col,
                          const int *tile_nnz, const uint8_t *ptr, const uint8_t *col, int m,
                          int n, int tilem, int td, const int *new_to_old, int perm_size,
                          int *row_cnt, const int *row_data)
{
    RTT_CUDA(cudaMemsetAsync(row_cnt, 0, sizeof(int) * (size_t)(m + 1), ws.stream));
    if (tilem > 0)
    {
        k_t2c_count<<<grid_for((long long)tilem * td, 256), 256, 0, ws.stream>>>(
            tile_ptr, tile_col, tile_nnz, ptr, col, m, n, tilem, td, new_to_old, perm_size,
            row_data, row_cnt, ws.err.as<int>());
        ws.launches++;
    }
    return RTT_OK;
}

int tile2csr_fill_device(Workspace &ws, const int *tile_ptr, const int *tile_col,
                         const int *tile_nnz, const uint8_t *ptr, const uint8_t *col,
                         const double *val, int m, int n, int tilem, int td,
                         const int *new_to_old, int perm_size, const int *rowptr, int *out_col,
                         double *out_val, bool sort_rows, const int *row_data)
{
    int total = 0;
    RTT_CHECK(read_int(ws, rowptr + m, &total));
    const long long nnz = total;
    if (tilem > 0)
    {
        k_t2c_fill<<<grid_for((long long)tilem * td, 256), 256, 0, ws.stream>>>(
            tile_ptr, tile_col, tile_nnz, ptr, col, val, m, n, tilem, td, new_to_old, perm_size,
            row_data, rowptr, nnz, out_col, out_val, ws.err.as<int>());
        ws.launches++;
    }
    if (sort_rows && m > 0)
    {
        k_sort_rows<<<grid_for(m, 128), 128, 0, ws.stream>>>(m, rowptr, out_col, out_val);
        ws.launches++;
    }
    return RTT_OK;
}

int tile2csr_count_launch(cudaStream_t s, const int *tile_ptr, const int *tile_col,
                          const int *tile_nnz, const uint8_t *ptr, const uint8_t *col, int m,
                          int n, int tilem, int td, int *row_cnt, int *err)
{
    if (tilem > 0)
    {
        k_t2c_count<<<grid_for((long long)tilem * td, 256), 256, 0, s>>>(
            tile_ptr, tile_col, tile_nnz, ptr, col, m, n, tilem, td, nullptr, -1, nullptr,
            row_cnt, err);
        RTT_CUDA(cudaGetLastError());
    }
    return RTT_OK;
}

int tile2csr_fill_launch(cudaStream_t s, const int *tile_ptr, const int *tile_col,
                         const int *tile_nnz, const uint8_t *ptr, const uint8_t *col,
                         const double *val, int m, int n, int tilem, int td, const int *rowptr,
                         long long nnz, int *out_col, double *out_val, bool sort_rows, int *err)
{
    if (tilem > 0)
    {
        k_t2c_fill<<<grid_for((long long)tilem * td, 256), 256, 0, s>>>(
            tile_ptr, tile_col, tile_nnz, ptr, col, val, m, n, tilem, td, nullptr, -1, nullptr,
            rowptr, nnz, out_col, out_val, err);
        RTT_CUDA(cudaGetLastError());
    }
    if (sort_rows && m > 0)
    {
        k_sort_rows<<<grid_for(m, 128), 128, 0, s>>>(m, rowptr, out_col, out_val);
        RTT_CUDA(cudaGetLastError());
    }
    return RTT_OK;
}

} // namespace rtt
