// runtime.cu - workspace, device buffers, scans and error plumbing.
#include "rtt_internal.cuh"

#include <cub/device/device_scan.cuh>
#include <cub/iterator/transform_input_iterator.cuh>

#include <algorithm>
#include <cstdio>
#include <mutex>

namespace rtt
{

std::string &last_error_ref()
{
    static thread_local std::string msg;
    return msg;
}

int fail(int status, const std::string &msg)
{
    last_error_ref() = msg;
    return status;
}

int cuda_fail(cudaError_t e, const char *what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (e == cudaErrorMemoryAllocation)
        return fail(RTT_ERR_OUT_OF_MEMORY, m);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return fail(RTT_ERR_NO_DEVICE, m);
    return fail(RTT_ERR_CUDA, m);
}

// Growth is refused on a thread that is capturing a CUDA graph (a captured
// cudaMallocAsync would hand the buffer to the graph).
namespace
{
thread_local bool g_growth_frozen = false;
} // namespace

void freeze_growth(bool on) { g_growth_frozen = on; }

// Grow-only buffers from the device's stream-ordered pool: a regrow frees
// and allocates in the order of stream s, without the device-wide
// synchronisation of cudaFree / cudaMalloc, so contexts that run on other
// streams (the serving loop's workers) do not wait for each other's kernels.
// The pool keeps freed memory for reuse (release threshold raised in
// Workspace::init).
int DevBuf::ensure(size_t bytes, cudaStream_t s)
{
    if (bytes == 0)
        bytes = 16;
    if (bytes <= cap)
        return RTT_OK;
    if (g_growth_frozen)
        return fail(RTT_ERR_STATE, "device buffer growth inside a CUDA graph capture");
    if (p != nullptr)
    {
        if (cudaFreeAsync(p, s) != cudaSuccess)
        {
            cudaGetLastError();
            cudaFree(p);
        }
        p = nullptr;
        cap = 0;
    }
    // round up so that repeated slightly-larger requests do not thrash
    size_t want = bytes + bytes / 8 + 256;
    cudaError_t e = cudaMallocAsync(&p, want, s);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        e = cudaMalloc(&p, want);
    }
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        e = cudaMalloc(&p, bytes);
        want = bytes;
    }
    if (e != cudaSuccess)
    {
        p = nullptr;
        cudaGetLastError();
        return cuda_fail(e, "cudaMalloc");
    }
    cap = want;
    return RTT_OK;
}

void DevBuf::release()
{
    if (p != nullptr)
        cudaFree(p);
    p = nullptr;
    cap = 0;
}

int Workspace::init(int dev)
{
    device = dev;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
    {
        cudaGetLastError();
        return fail(RTT_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (dev < 0 || dev >= count)
        return fail(RTT_ERR_INVALID_ARGUMENT, "device index out of range");
    RTT_CUDA(cudaSetDevice(dev));
    cudaDeviceProp prop;
    RTT_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10)
        return fail(RTT_ERR_NO_DEVICE, "this library is built for sm_100a (B200); found sm_" +
                                           std::to_string(prop.major * 10 + prop.minor));
    {
        // the default pool keeps up to 8 GiB of freed memory for reuse (a
        // regrow then costs no driver allocation); above that it returns
        // memory at synchronisations, so it does not starve other
        // allocators of the process (a framework's caching allocator)
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
        {
            uint64_t keep = 8ull << 30;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    }
    RTT_CHECK(err.ensure(sizeof(int) * 4, stream));
    RTT_CUDA(cudaMemset(err.p, 0, sizeof(int) * 4));
    if (h_scalars == nullptr)
    {
        RTT_CUDA(cudaMallocHost(&h_scalars, sizeof(int) * 32));
        RTT_CUDA(cudaMallocHost(&h_scalars64, sizeof(long long) * 8));
    }
    for (cudaEvent_t &e : ev)
        if (e == nullptr)
            RTT_CUDA(cudaEventCreate(&e));
    if (side == nullptr)
        RTT_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    for (cudaEvent_t *e : {&fork_ev, &join_ev})
        if (*e == nullptr)
            RTT_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return RTT_OK;
}

void Workspace::destroy()
{
    err.release();
    scan_tmp.release();
    for (DevBuf &b : tmp)
        b.release();
    if (h_scalars != nullptr)
        cudaFreeHost(h_scalars);
    if (h_scalars64 != nullptr)
        cudaFreeHost(h_scalars64);
    h_scalars = nullptr;
    h_scalars64 = nullptr;
    for (cudaEvent_t &e : ev)
        if (e != nullptr)
        {
            cudaEventDestroy(e);
            e = nullptr;
        }
    for (cudaEvent_t *e : {&fork_ev, &join_ev})
        if (*e != nullptr)
        {
            cudaEventDestroy(*e);
            *e = nullptr;
        }
    if (side != nullptr)
        cudaStreamDestroy(side);
    side = nullptr;
}

namespace
{
__global__ void k_zero_first_int(int *p) { p[0] = 0; }
__global__ void k_zero_first_i64(long long *p) { p[0] = 0; }

struct ToI64
{
    __host__ __device__ long long operator()(int v) const { return (long long)v; }
};
} // namespace

int scan_exclusive_int(Workspace &ws, const int *in, int *out, int n)
{
    k_zero_first_int<<<1, 1, 0, ws.stream>>>(out);
    ws.launches++;
    if (n <= 0)
        return RTT_OK;
    size_t bytes = 0;
    RTT_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, in, out + 1, n, ws.stream));
    RTT_CHECK(ws.scan_tmp.ensure(bytes, ws.stream));
    RTT_CUDA(cub::DeviceScan::InclusiveSum(ws.scan_tmp.p, bytes, in, out + 1, n, ws.stream));
    ws.launches++;
    return RTT_OK;
}

int scan_exclusive_i64(Workspace &ws, const int *in, long long *out, int n)
{
    k_zero_first_i64<<<1, 1, 0, ws.stream>>>(out);
    ws.launches++;
    if (n <= 0)
        return RTT_OK;
    cub::TransformInputIterator<long long, ToI64, const int *> it(in, ToI64());
    size_t bytes = 0;
    RTT_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, it, out + 1, n, ws.stream));
    RTT_CHECK(ws.scan_tmp.ensure(bytes, ws.stream));
    RTT_CUDA(cub::DeviceScan::InclusiveSum(ws.scan_tmp.p, bytes, it, out + 1, n, ws.stream));
    ws.launches++;
    return RTT_OK;
}

namespace
{
// The error word copied to ws.h_scalars[8] before the last synchronisation.
int error_word_seen(Workspace &ws, const char *stage)
{
    int code = ws.h_scalars[8];
    if (code != 0)
    {
        cudaMemsetAsync(ws.err.p, 0, sizeof(int), ws.stream);
        return fail(RTT_ERR_DEVICE_CHECK,
                    std::string(stage) + ": device check failed, code " + std::to_string(code));
    }
    return RTT_OK;
}
} // namespace

int check_device_error(Workspace &ws, const char *stage)
{
    RTT_CUDA(cudaGetLastError());
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars + 8, ws.err.p, sizeof(int), cudaMemcpyDeviceToHost,
                             ws.stream));
    RTT_CUDA(cudaStreamSynchronize(ws.stream));
    ws.syncs++;
    return error_word_seen(ws, stage);
}

int read_int_checked(Workspace &ws, const int *d, int *h, const char *stage)
{
    RTT_CUDA(cudaGetLastError());
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars + 8, ws.err.p, sizeof(int), cudaMemcpyDeviceToHost,
                             ws.stream));
    RTT_CHECK(read_int(ws, d, h));
    return error_word_seen(ws, stage);
}

int read_i64_checked(Workspace &ws, const long long *d, long long *h, const char *stage)
{
    RTT_CUDA(cudaGetLastError());
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars + 8, ws.err.p, sizeof(int), cudaMemcpyDeviceToHost,
                             ws.stream));
    RTT_CHECK(read_i64(ws, d, h));
    return error_word_seen(ws, stage);
}

int read_int(Workspace &ws, const int *d, int *h)
{
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars, d, sizeof(int), cudaMemcpyDeviceToHost, ws.stream));
    RTT_CUDA(cudaStreamSynchronize(ws.stream));
    ws.syncs++;
    *h = ws.h_scalars[0];
    return RTT_OK;
}

int read_i64(Workspace &ws, const long long *d, long long *h)
{
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars64, d, sizeof(long long), cudaMemcpyDeviceToHost,
                             ws.stream));
    RTT_CUDA(cudaStreamSynchronize(ws.stream));
    ws.syncs++;
    *h = ws.h_scalars64[0];
    return RTT_OK;
}

void TileBufs::release()
{
    each([](const DevBuf &b) { const_cast<DevBuf &>(b).release(); });
}

DevTiles TileBufs::view() const
{
    DevTiles t{};
    t.m = m;
    t.n = n;
    t.tilem = tilem;
    t.tilen = tilen;
    t.numtile = numtile;
    t.nnz = nnz;
    t.tile_ptr = tile_ptr.as<int>();
    t.tile_col = tile_col.as<int>();
    // the per-entry arrays only when built (null views otherwise)
    t.tile_nnz = payload ? tile_nnz.as<int>() : nullptr;
    t.ptr = payload ? ptr.as<uint8_t>() : nullptr;
    t.col = payload ? col.as<uint8_t>() : nullptr;
    t.val = payload ? val.as<double>() : nullptr;
    t.mask = payload ? mask.as<uint16_t>() : nullptr;
    t.row_data = nullptr;
    t.csc_ptr = csc_ptr.as<int>();
    t.csc_row = csc_row.as<int>();
    t.csc_data = csc_data.as<int>();
    t.csr_rowptr = nullptr;
    t.csr_col = nullptr;
    t.csr_val = nullptr;
    t.seg_ptr = has_segments ? seg_ptr.as<int>() : nullptr;
    t.seg = has_segments ? seg.as<unsigned long long>() : nullptr;
    t.max_row_segs = has_segments ? max_row_segs : 0;
    return t;
}

DevTiles tile_row_slice(const DevTiles &A, int I0, int I1)
{
    DevTiles t = A;
    t.tile_ptr = A.tile_ptr + I0;
    t.tilem = I1 - I0;
    t.m = std::min(A.m, I1 * TD) - I0 * TD;
    if (A.csr_rowptr != nullptr)
        t.csr_rowptr = A.csr_rowptr + (size_t)I0 * TD;
    if (A.seg_ptr != nullptr)
        t.seg_ptr = A.seg_ptr + (size_t)I0 * TD;
    return t;
}

void SymbolicOut::release()
{
    each([](const DevBuf &b) { const_cast<DevBuf &>(b).release(); });
}

DevCTiles SymbolicOut::view()
{
    DevCTiles c{};
    c.tilem = tilem;
    c.tilen = tilen;
    c.m = m;
    c.n = n;
    c.tile_ptr = c_tile_ptr.as<int>();
    c.tile_col = c_tile_col.as<int>();
    c.tile_row = c_tile_row.as<int>();
    c.tile_nnz = c_tile_nnz.as<int>();
    c.mask = c_mask.as<uint16_t>();
    c.ptr = c_ptr.as<uint8_t>();
    c.col = c_col.as<uint8_t>();
    c.val = c_val.as<double>();
    return c;
}

} // namespace rtt
