// noalloc.cu - tile2csr from device-resident tiles into caller-owned device
// CSR buffers, allocating nothing: no cudaMalloc / cudaFree, no pinned host
// memory, no growing workspace.  Its only working memory is one static device
// array per device, found once with cudaGetSymbolAddress.
//
// Same kernels and results as rtt_tile2csr (the reference's tile2csr,
// src/tile2csr.h:232-329): per row the entries of its tiles in tile order,
// row bounds clamped, out-of-range columns dropped, rows heap-sorted by
// column unless the caller promises canonical tiles.
#include "rtt_internal.cuh"

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <climits>
#include <mutex>
#include <string>

namespace
{
constexpr size_t kScratchBytes = size_t(1) << 20; // 1 MiB per device
constexpr size_t kHeaderBytes = 256;              // counters; CUB temp storage follows
constexpr int kMaxRows = 1 << 25;                 // 33,554,432 rows
constexpr int kMaxDevices = 64;
constexpr int kErrTiles = 110;                    // malformed tile lists
} // namespace

// Per-device scratch.  Layout:
//   [0, 8)            unsigned long long: CSR entry total of this call
//   [8, 12)           int: first device error code of this call
//   [256, 1 MiB)      CUB temp storage of the row-pointer scan
// The first 16 bytes must be zero when a call's first kernel starts; every
// call clears them with cudaMemsetAsync on its own stream before launching.
// The CUB region needs no initial value.
static __device__ __align__(256) unsigned char g_tile2csr_scratch[kScratchBytes];

namespace
{
using namespace rtt;

struct ScratchHeader
{
    unsigned long long total;
    int err;
    int pad;
};

std::mutex g_noalloc_mutex;
void *g_scratch_addr[kMaxDevices] = {};

__global__ void k_noalloc_check_lists(int tilem, const int *__restrict__ tile_ptr, int nt,
                                      const int *__restrict__ tile_nnz, int nent, int *err)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= tilem)
    {
        const int v = tile_ptr[i];
        if (v < 0 || v > nt || (i < tilem && tile_ptr[i + 1] < v))
            set_error(err, kErrTiles);
    }
    if (i <= nt)
    {
        const int v = tile_nnz[i];
        if (v < 0 || v > nent || (i < nt && tile_nnz[i + 1] < v))
            set_error(err, kErrTiles);
    }
}

__global__ void k_noalloc_total(const int *__restrict__ cnt, int m, unsigned long long *total)
{
    unsigned long long s = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (long long)gridDim.x * blockDim.x)
        s += (unsigned)cnt[i];
    s = warp_sum(s);
    if (lane_id() == 0 && s != 0)
        atomicAdd(total, s);
}

int read_header(void *scratch, cudaStream_t s, ScratchHeader &h)
{
    RTT_CUDA(cudaMemcpyAsync(&h, scratch, sizeof(h), cudaMemcpyDeviceToHost, s));
    RTT_CUDA(cudaStreamSynchronize(s));
    return RTT_OK;
}

int map_err(int code)
{
    if (code == kErrTiles)
        return fail(RTT_ERR_INVALID_ARGUMENT, "tile2csr_device_noalloc: malformed tile lists");
    if (code == DERR_T2C_BOUNDS)
        return fail(RTT_ERR_DEVICE_CHECK, "tile2csr_device_noalloc: output index out of range");
    return fail(RTT_ERR_DEVICE_CHECK,
                "tile2csr_device_noalloc: device check failed, code " + std::to_string(code));
}

} // namespace

extern "C" int rtt_tile2csr_device_noalloc(const SMatrix *M, int tile_dim, int canonical,
                                           long long out_capacity, long long *out_nnz,
                                           void *stream)
{
    if (M == nullptr || out_nnz == nullptr)
        return fail(RTT_ERR_INVALID_ARGUMENT, "tile2csr_device_noalloc: NULL argument");
    *out_nnz = -1;
    if (tile_dim != 8 && tile_dim != 16)
        return fail(RTT_ERR_INVALID_ARGUMENT, "tile2csr_device_noalloc: tile_dim must be 8 or 16");
    const int m = M->m, n = M->n, tilem = M->tilem, nt = M->numtile, nent = M->nnz;
    if (m < 0 || n < 0 || nt < 0 || nent < 0 || tilem != (m + tile_dim - 1) / tile_dim ||
        out_capacity < 0)
        return fail(RTT_ERR_INVALID_ARGUMENT, "tile2csr_device_noalloc: bad sizes");
    if (m > kMaxRows)
        return fail(RTT_ERR_INVALID_ARGUMENT,
                    "tile2csr_device_noalloc: m = " + std::to_string(m) +
                        " rows exceeds the allocation-free limit of 33554432 rows");
    if (M->rowpointer == nullptr || M->tile_ptr == nullptr || M->tile_nnz == nullptr ||
        (nt > 0 && (M->tile_columnidx == nullptr || M->tile_csr_Ptr == nullptr)) ||
        (nent > 0 && (M->tile_csr_Col == nullptr || M->tile_csr_Value == nullptr)))
        return fail(RTT_ERR_INVALID_ARGUMENT, "tile2csr_device_noalloc: NULL device array");
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    int dev = 0;
    RTT_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(RTT_ERR_INVALID_ARGUMENT, "tile2csr_device_noalloc: device index out of range");
    if (g_scratch_addr[dev] == nullptr)
        RTT_CUDA(cudaGetSymbolAddress(&g_scratch_addr[dev], g_tile2csr_scratch));
    unsigned char *scratch = static_cast<unsigned char *>(g_scratch_addr[dev]);
    auto *total = reinterpret_cast<unsigned long long *>(scratch);
    int *err = reinterpret_cast<int *>(scratch + 8);
    void *cub_tmp = scratch + kHeaderBytes;

    int *rowptr = M->rowpointer;
    size_t cub_bytes = 0;
    if (m > 0)
    {
        RTT_CUDA(cub::DeviceScan::InclusiveSum(nullptr, cub_bytes, rowptr + 1, rowptr + 1, m, s));
        if (cub_bytes > kScratchBytes - kHeaderBytes)
            return fail(RTT_ERR_INVALID_ARGUMENT,
                        "tile2csr_device_noalloc: the row-pointer scan needs " +
                            std::to_string(cub_bytes) + " bytes of scratch, more than the " +
                            std::to_string(kScratchBytes - kHeaderBytes) + " available");
    }

    RTT_CUDA(cudaMemsetAsync(scratch, 0, sizeof(ScratchHeader), s));
    RTT_CUDA(cudaMemsetAsync(rowptr, 0, sizeof(int) * ((size_t)m + 1), s));
    {
        const long long th = (long long)std::max(tilem, nt) + 1;
        k_noalloc_check_lists<<<(int)((th + 255) / 256), 256, 0, s>>>(tilem, M->tile_ptr, nt,
                                                                      M->tile_nnz, nent, err);
        RTT_CUDA(cudaGetLastError());
    }
    ScratchHeader h{};
    // the tile lists are bounds-checked before any kernel walks them
    RTT_CHECK(read_header(scratch, s, h));
    if (h.err != 0)
        return map_err(h.err);
    const uint8_t *tptr = M->tile_csr_Ptr, *tcol = M->tile_csr_Col;
    RTT_CHECK(tile2csr_count_launch(s, M->tile_ptr, M->tile_columnidx, M->tile_nnz, tptr, tcol, m,
                                    n, tilem, tile_dim, rowptr + 1, err));
    if (m > 0)
    {
        const int blocks = std::min((m + 255) / 256, 148 * 4);
        k_noalloc_total<<<blocks, 256, 0, s>>>(rowptr + 1, m, total);
        RTT_CUDA(cudaGetLastError());
        RTT_CUDA(cub::DeviceScan::InclusiveSum(cub_tmp, cub_bytes, rowptr + 1, rowptr + 1, m, s));
    }
    RTT_CHECK(read_header(scratch, s, h));
    if (h.err != 0)
        return map_err(h.err);
    if (h.total > (unsigned long long)INT_MAX)
        return fail(RTT_ERR_UNREPRESENTABLE, "tile2csr_device_noalloc: nnz exceeds int32");
    *out_nnz = (long long)h.total;
    if (M->columnindex == nullptr && M->value == nullptr)
        return RTT_OK; // size query: rowpointer and nnz written
    if ((long long)h.total > out_capacity ||
        (h.total > 0 && (M->columnindex == nullptr || M->value == nullptr)))
        return fail(RTT_ERR_INVALID_ARGUMENT,
                    "tile2csr_device_noalloc: output capacity " + std::to_string(out_capacity) +
                        " is below the " + std::to_string(h.total) + " entries of the result");
    RTT_CHECK(tile2csr_fill_launch(s, M->tile_ptr, M->tile_columnidx, M->tile_nnz, tptr, tcol,
                                   M->tile_csr_Value, m, n, tilem, tile_dim, rowptr,
                                   (long long)h.total, M->columnindex, M->value, canonical == 0,
                                   err));
    RTT_CHECK(read_header(scratch, s, h));
    if (h.err != 0)
        return map_err(h.err);
    return RTT_OK;
}
