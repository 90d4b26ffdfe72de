// api.cu - the extern "C" entry points declared in include/rtt_spgemm.h.
//
// Host-buffer drop-ins (csr2tile_row_major, csr2tile_col_major, spgemm_cpu,
// tile2csr, tile2csr_restore_rows replacements) upload the SMatrix arrays,
// run the sm_100a kernels and copy results into malloc'd host arrays.  They
// share one lazily created context per device, serialised by a mutex (the
// reference functions are not re-entrant either).  Outputs are committed to
// the caller's SMatrix only after every copy succeeded.
#include "rtt_internal.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <mutex>
#include <vector>

#include <sys/mman.h>

namespace rtt
{
// One captured numeric phase.  The key lists every host-side input that its
// launches baked in: shapes and flags of the tiles and of C, the operand and
// output pointers, the configuration, the stream and the allocation epoch
// (which covers every workspace pointer).
struct GraphSlot
{
    std::vector<long long> key;
    bool warm = false; // the last call ran eagerly with this key
    cudaGraphExec_t exec = nullptr;
    int launches = 0; // kernels in the graph
    void reset()
    {
        if (exec != nullptr)
            cudaGraphExecDestroy(exec);
        exec = nullptr;
        key.clear();
        warm = false;
        launches = 0;
    }
};
} // namespace rtt

struct rtt_context_s
{
    rtt::Workspace ws;
    rtt_config cfg;
    rtt::TileBufs A, B;
    rtt::DevBuf bt_rowptr, bt_col, bt_val; // B = A^T for RTT_OP_AAT
    rtt::DevBuf bp_rowptr, bp_col, bp_val; // B with permuted rows (rtt_spgemm_update_b)
    rtt::DevBuf diag_hist;                 // rtt_tile_heatmap
    rtt::DevBuf in_rp, in_col, in_val;     // host-buffer uploads
    rtt::DevBuf in2_rp, in2_col, in2_val;
    rtt::DevBuf out_rp, out_col, out_val;  // host-buffer product output
    rtt::DevBuf counters;
    rtt::DevBuf maxnnz;
    rtt::DevBuf vflags; // flags of the values-only update's CSR validation
    rtt::SymbolicOut S;
    rtt_stats stats;
    bool have_symbolic = false;
    bool b_alias = false;
    bool owns_stream = false;
    // B as scalar CSR rows for the numeric step (borrowed or owned above)
    const int *b_rp = nullptr;
    const int *b_ci = nullptr;
    const double *b_va = nullptr;
    long long b_nnz = 0;
    bool b_dups = false;
    // A's structure as given to the last symbolic (values-only updates)
    const int *a_rp = nullptr;
    const int *a_ci = nullptr;
    const double *a_va = nullptr; // A's values of the current numeric step
    bool op_aat = false;
    // page-locked staging of the host-buffer entry points (created on first use)
    void *hstage[2] = {};
    cudaEvent_t hstage_ev[2] = {};
    // batched products: block-diagonal operands and per-instance bookkeeping
    rtt::DevBuf bat_a_rp, bat_a_col, bat_a_val, bat_b_rp, bat_b_col, bat_b_val;
    rtt::DevBuf bat_meta, bat_big_rp, bat_nnz;
    bool bat_active = false;
    int bat_count = 0, bat_rows = 0;
    // entry offsets of the instances in the block-diagonal A (and B), their
    // largest entry count, and the device pointer table of a values-only update
    std::vector<int> bat_a_off, bat_b_off;
    int bat_a_max = 0, bat_b_max = 0;
    rtt::DevBuf bat_vtab;
    // offsets (in ints) of the device meta arrays inside bat_meta
    size_t bat_rows_off = 0, bat_rowoff_off = 0, bat_sec_off = 0, bat_colsub_off = 0;
    // CUDA graphs of the numeric phase
    rtt::GraphSlot graph[4]; // numeric, values-only, batched, batched values-only
    cudaStream_t cap_stream = nullptr; // capture stream (never the legacy one)
    int cut_cached = -1; // effective DMMA cutoff of the current tiles (-1: unknown)
    // 64-bit products: step-1 counts, per-row counts of C, its int64 row
    // pointer, a chunk's local row pointer; chunks of A's tile rows
    rtt::DevBuf w_cnt, w_rowcnt, w_rowptr, w_local;
    std::vector<int> w_bounds;      // chunk c is tile rows [w_bounds[c], w_bounds[c + 1])
    std::vector<long long> w_base;  // first entry of chunk c in C
    rtt::DevTiles w_dA{}, w_dB{};
    bool have_sym64 = false;
    long long w_nnz = 0;
    // hybrid leaves of A and B for the leaf DMMA numeric step (leaf_dmma)
    rtt::HybridDev leaf_a, leaf_b;
};

namespace
{
using namespace rtt;

// The context's own device buffers (tiles, C and workspace aside).
std::vector<DevBuf *> own_buffers(rtt_context c)
{
    return {&c->bt_rowptr, &c->bt_col,    &c->bt_val,     &c->in_rp,     &c->in_col,
            &c->in_val,    &c->in2_rp,    &c->in2_col,    &c->in2_val,   &c->out_rp,
            &c->out_col,   &c->out_val,   &c->counters,   &c->maxnnz,    &c->bat_a_rp,
            &c->bat_a_col, &c->bat_a_val, &c->bat_b_rp,   &c->bat_b_col, &c->bat_b_val,
            &c->bat_meta,  &c->bat_big_rp, &c->bat_nnz,  &c->vflags,    &c->bat_vtab,
            &c->w_cnt,     &c->w_rowcnt,  &c->w_rowptr,   &c->w_local,   &c->bp_rowptr,
            &c->bp_col,    &c->bp_val,    &c->diag_hist};
}

std::mutex g_mutex;
int g_device = 0;
rtt_context g_ctx[16] = {};

int default_context(rtt_context *out)
{
    if (g_device < 0 || g_device >= 16)
        return fail(RTT_ERR_INVALID_ARGUMENT, "device index out of range");
    if (g_ctx[g_device] == nullptr)
    {
        rtt_context c = nullptr;
        int st = rtt_context_create(&c, g_device);
        if (st != RTT_OK)
            return st;
        g_ctx[g_device] = c;
    }
    RTT_CUDA(cudaSetDevice(g_device));
    *out = g_ctx[g_device];
    return RTT_OK;
}

// Host <-> device copies of the host-buffer entry points.  Page-locked host
// memory is copied directly.  Pageable memory goes through two page-locked
// staging buffers of the context: the DMA of one chunk overlaps the
// multi-threaded host copy of the other (which also takes the first-touch page
// faults of freshly malloc'd outputs on all cores instead of one).
constexpr size_t kStageBytes = size_t(32) << 20;
constexpr size_t kDirectBytes = size_t(4) << 20; // below this a plain copy is as fast

void par_memcpy(void *dst, const void *src, size_t bytes)
{
    const size_t piece = size_t(1) << 20;
    const long long n = (long long)((bytes + piece - 1) / piece);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; ++i)
    {
        const size_t off = (size_t)i * piece;
        std::memcpy(static_cast<char *>(dst) + off, static_cast<const char *>(src) + off,
                    std::min(piece, bytes - off));
    }
}

bool is_pageable(const void *p)
{
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess)
    {
        cudaGetLastError(); // clear the sticky-free error of an unknown pointer
        return true;
    }
    return at.type == cudaMemoryTypeUnregistered;
}

int ensure_stage(rtt_context c)
{
    for (int b = 0; b < 2; ++b)
    {
        if (c->hstage[b] == nullptr)
            RTT_CUDA(cudaMallocHost(&c->hstage[b], kStageBytes));
        if (c->hstage_ev[b] == nullptr)
            RTT_CUDA(cudaEventCreateWithFlags(&c->hstage_ev[b], cudaEventDisableTiming));
    }
    return RTT_OK;
}

int h2d(rtt_context c, void *dst, const void *src, size_t bytes, cudaStream_t s)
{
    if (bytes < kDirectBytes || !is_pageable(src))
    {
        RTT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        return RTT_OK;
    }
    RTT_CHECK(ensure_stage(c));
    for (size_t off = 0, i = 0; off < bytes; off += kStageBytes, ++i)
    {
        const int b = (int)(i & 1);
        const size_t n = std::min(kStageBytes, bytes - off);
        RTT_CUDA(cudaEventSynchronize(c->hstage_ev[b])); // previous copy out of this buffer
        par_memcpy(c->hstage[b], static_cast<const char *>(src) + off, n);
        RTT_CUDA(cudaMemcpyAsync(static_cast<char *>(dst) + off, c->hstage[b], n,
                                 cudaMemcpyHostToDevice, s));
        RTT_CUDA(cudaEventRecord(c->hstage_ev[b], s));
    }
    return RTT_OK;
}

int d2h(rtt_context c, void *dst, const void *src, size_t bytes, cudaStream_t s)
{
    if (bytes < kDirectBytes || !is_pageable(dst))
    {
        RTT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        RTT_CUDA(cudaStreamSynchronize(s));
        return RTT_OK;
    }
    RTT_CHECK(ensure_stage(c));
    const size_t nch = (bytes + kStageBytes - 1) / kStageBytes;
    auto issue = [&](size_t i) -> int {
        const int b = (int)(i & 1);
        const size_t off = i * kStageBytes, n = std::min(kStageBytes, bytes - off);
        RTT_CUDA(cudaMemcpyAsync(c->hstage[b], static_cast<const char *>(src) + off, n,
                                 cudaMemcpyDeviceToHost, s));
        RTT_CUDA(cudaEventRecord(c->hstage_ev[b], s));
        return RTT_OK;
    };
    RTT_CUDA(cudaStreamSynchronize(s)); // staging buffers free of earlier uploads
    RTT_CHECK(issue(0));
    for (size_t i = 0; i < nch; ++i)
    {
        if (i + 1 < nch)
            RTT_CHECK(issue(i + 1)); // its buffer's previous chunk was copied out below
        const int b = (int)(i & 1);
        RTT_CUDA(cudaEventSynchronize(c->hstage_ev[b]));
        const size_t off = i * kStageBytes;
        par_memcpy(static_cast<char *>(dst) + off, c->hstage[b], std::min(kStageBytes, bytes - off));
    }
    return RTT_OK;
}

template <typename T>
int upload(rtt_context c, DevBuf &b, const T *h, size_t n, cudaStream_t s)
{
    RTT_CHECK(b.ensure(sizeof(T) * n + 16, s));
    if (n > 0)
    {
        if (h == nullptr)
            return fail(RTT_ERR_INVALID_ARGUMENT, "NULL host array with nonzero length");
        RTT_CHECK(h2d(c, b.p, h, sizeof(T) * n, s));
    }
    return RTT_OK;
}

// Host output arrays of the host-buffer entry points are malloc'd: the
// caller frees them with free(), as with the reference.  Large ones start on
// a 2 MiB boundary and are advised to use transparent huge pages where the
// kernel offers them, so that their first touch (inside d2h) takes one page
// fault per 2 MiB instead of one per 4 KiB.
void *host_alloc(size_t bytes)
{
    constexpr size_t huge = size_t(2) << 20;
    if (bytes < 2 * huge)
        return std::malloc(bytes);
    void *p = nullptr;
    if (posix_memalign(&p, huge, bytes) != 0)
        return nullptr;
    madvise(p, bytes, MADV_HUGEPAGE); // advice only: a kernel without THP ignores it
    return p;
}

template <typename T>
int download(rtt_context c, T **out, const void *d, size_t n, cudaStream_t s)
{
    T *h = static_cast<T *>(host_alloc(sizeof(T) * (n > 0 ? n : 1)));
    if (h == nullptr)
        return fail(RTT_ERR_OUT_OF_MEMORY, "host malloc failed");
    if (n > 0)
    {
        const int st = d2h(c, h, d, sizeof(T) * n, s);
        if (st != RTT_OK)
        {
            std::free(h);
            return st;
        }
    }
    *out = h;
    return RTT_OK;
}

// Free a set of host arrays on failure paths.  Slots live in a fixed array so
// the pointers handed out stay valid while more slots are taken.
struct HostArrays
{
    static constexpr int kMax = 16;
    void *ptrs[kMax] = {};
    int used = 0;
    bool committed = false;
    template <typename T>
    T **slot()
    {
        if (used >= kMax)
            std::abort(); // programming error: raise kMax
        return reinterpret_cast<T **>(&ptrs[used++]);
    }
    ~HostArrays()
    {
        if (!committed)
            for (int i = 0; i < used; ++i)
                std::free(ptrs[i]);
    }
};

int map_device_error(int st)
{
    if (st == RTT_ERR_DEVICE_CHECK)
    {
        const std::string &m = last_error_ref();
        if (m.find("code 101") != std::string::npos || m.find("code 102") != std::string::npos)
            return fail(RTT_ERR_INVALID_CSR, "invalid CSR input: " + m);
        if (m.find("code 109") != std::string::npos)
            return fail(RTT_ERR_TAIL_NONEMPTY, "row past the permutation prefix is not empty");
    }
    return st;
}

__global__ void k_masks_from_entries(int numtile, const int *__restrict__ tnnz,
                                     const uint8_t *__restrict__ ptr,
                                     const uint8_t *__restrict__ col, uint16_t *__restrict__ mask)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= numtile * TD)
        return;
    const int t = x >> 4, r = x & 15;
    const int b = tnnz[t], cnt = tnnz[t + 1] - b;
    int s = ptr[(size_t)t * TD + r];
    int e = r == TD - 1 ? cnt : ptr[(size_t)t * TD + r + 1];
    s = min(s, cnt);
    e = min(max(e, s), cnt);
    uint32_t m = 0;
    for (int i = s; i < e; ++i)
        m |= 0x8000u >> (col[b + i] & 15);
    mask[x] = (uint16_t)m;
}

__global__ void k_expand_ptr(int nbins, const int *__restrict__ ptr, int *__restrict__ owner)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbins)
        return;
    for (int p = ptr[b]; p < ptr[b + 1]; ++p)
        owner[p] = b;
}

__global__ void k_iota_i(int *a, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        a[i] = i;
}

__global__ void k_gather_i(const int *__restrict__ src, const int *__restrict__ idx, int n,
                           int *__restrict__ dst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = src[idx[i]];
}

__global__ void k_lower_bound(const int *__restrict__ keys, int nkeys, int nbins, int *__restrict__ ptr)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > nbins)
        return;
    ptr[b] = lower_bound(keys, 0, nkeys, b);
}

// Structure checks of caller-provided tiles, run before any kernel indexes
// through them: list pointers monotone and ending at the entry count, list
// indices in range and strictly increasing inside a list, per-tile entry
// offsets monotone and in range, per-tile row offsets non-decreasing.
constexpr int DERR_TILES = 110;

__global__ void k_validate_lists(int nlists, const int *__restrict__ ptr, const int *__restrict__ idx,
                                 int nidx, int max_idx, int *err)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l == 0 && (ptr[0] != 0 || ptr[nlists] != nidx))
        set_error(err, DERR_TILES);
    if (l >= nlists)
        return;
    const int b = ptr[l], e = ptr[l + 1];
    if (b < 0 || e < b || e > nidx)
    {
        set_error(err, DERR_TILES);
        return;
    }
    int prev = -1;
    for (int i = b; i < e; ++i)
    {
        const int v = idx[i];
        if (v < 0 || v >= max_idx || v <= prev)
        {
            set_error(err, DERR_TILES);
            return;
        }
        prev = v;
    }
}

__global__ void k_validate_tile_data(int nt, const int *__restrict__ tnnz, int nent, int ptr_stride,
                                     const uint8_t *__restrict__ ptr, int *err)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt)
        return;
    const int b = tnnz[t], e = tnnz[t + 1];
    if (b < 0 || e < b || e > nent)
    {
        set_error(err, DERR_TILES);
        return;
    }
    int prev = 0;
    for (int r = 0; r < ptr_stride; ++r)
    {
        const int p = ptr[(size_t)t * ptr_stride + r];
        if (p < prev || p > e - b)
        {
            set_error(err, DERR_TILES);
            return;
        }
        prev = p;
    }
}

__global__ void k_validate_ptr(int n, const int *__restrict__ ptr, int maxv, int *err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n)
        return;
    const int v = ptr[i];
    if (v < 0 || v > maxv || (i < n && ptr[i + 1] < v))
        set_error(err, DERR_TILES);
}

inline int grid_for(long long threads, int block) { return (int)((threads + block - 1) / block); }

int check_tiles(Workspace &ws, const char *what)
{
    int st = check_device_error(ws, what);
    if (st == RTT_ERR_DEVICE_CHECK && last_error_ref().find("code 110") != std::string::npos)
        return fail(RTT_ERR_INVALID_ARGUMENT, std::string(what) + ": malformed tile structure");
    return st;
}

int bits_for(int maxval)
{
    int b = 1;
    while (b < 31 && (1 << b) <= maxval)
        ++b;
    return b;
}

bool csr_args_ok(const SMatrix *M)
{
    return M != nullptr && M->m >= 0 && M->n >= 0 && M->nnz >= 0 &&
           (M->m == 0 || M->rowpointer != nullptr) &&
           (M->nnz == 0 || (M->columnindex != nullptr && M->value != nullptr));
}

// Upload a host CSR and tile it (row-major) into T.
int tile_host_csr(rtt_context c, const SMatrix *M, TileBufs &T, bool packed, bool sorted_rows)
{
    cudaStream_t s = c->ws.stream;
    RTT_CHECK(upload(c, c->in_rp, M->rowpointer, (size_t)M->m + (M->m > 0 ? 1 : 0), s));
    RTT_CHECK(upload(c, c->in_col, M->columnindex, (size_t)M->nnz, s));
    RTT_CHECK(upload(c, c->in_val, M->value, (size_t)M->nnz, s));
    int st = csr2tile_device(c->ws, M->m, M->n, M->nnz, c->in_rp.as<int>(), c->in_col.as<int>(),
                             c->in_val.as<double>(), T, packed, sorted_rows);
    st = map_device_error(st);
    if (st != RTT_OK)
        return st;
    return map_device_error(check_device_error(c->ws, "csr2tile"));
}

// Upload legacy tiles (row-major A or column-major B) and build the views the
// kernels need.  For column-major input the per-tile arrays are in tile-CSC
// order: the CSC index is taken as given and a row index is derived from it.
int upload_tiles(rtt_context c, const SMatrix *M, bool col_major, TileBufs &T)
{
    cudaStream_t s = c->ws.stream;
    const int tilem = ceil_div(M->m, TD), tilen = ceil_div(M->n, TD);
    if (M->numtile < 0 || M->nnz < 0 || M->tile_nnz == nullptr)
        return fail(RTT_ERR_INVALID_ARGUMENT, "tile matrix without tile_nnz");
    const int nt = M->numtile;
    const int nnz = M->tile_nnz[nt];
    if (nnz < 0 || nnz > M->nnz)
        return fail(RTT_ERR_INVALID_ARGUMENT, "tile_nnz[numtile] exceeds nnz");
    if (nt > 0 && (M->tile_csr_Ptr == nullptr))
        return fail(RTT_ERR_INVALID_ARGUMENT, "tile matrix without tile_csr_Ptr");
    if (nnz > 0 && (M->tile_csr_Col == nullptr || M->tile_csr_Value == nullptr))
        return fail(RTT_ERR_INVALID_ARGUMENT, "tile matrix without entries");
    T.m = M->m;
    T.n = M->n;
    T.tilem = tilem;
    T.tilen = tilen;
    T.numtile = nt;
    T.nnz = nnz;
    RTT_CHECK(upload(c, T.tile_nnz, M->tile_nnz, (size_t)nt + 1, s));
    RTT_CHECK(upload(c, T.ptr, M->tile_csr_Ptr, (size_t)nt * TD, s));
    RTT_CHECK(upload(c, T.col, M->tile_csr_Col, (size_t)nnz, s));
    RTT_CHECK(upload(c, T.val, M->tile_csr_Value, (size_t)nnz, s));
    RTT_CHECK(T.mask.ensure(sizeof(uint16_t) * (size_t)nt * TD + 16, s));
    if (nt > 0)
    {
        k_validate_tile_data<<<grid_for(nt, 256), 256, 0, s>>>(nt, T.tile_nnz.as<int>(), nnz, TD,
                                                               T.ptr.as<uint8_t>(), c->ws.err.as<int>());
        c->ws.launches++;
        RTT_CHECK(check_tiles(c->ws, "tile data"));
        k_masks_from_entries<<<grid_for((long long)nt * TD, 256), 256, 0, s>>>(
            nt, T.tile_nnz.as<int>(), T.ptr.as<uint8_t>(), T.col.as<uint8_t>(),
            T.mask.as<uint16_t>());
        c->ws.launches++;
    }
    if (!col_major)
    {
        if (M->tile_ptr == nullptr || (nt > 0 && M->tile_columnidx == nullptr))
            return fail(RTT_ERR_INVALID_ARGUMENT, "row-major tiles without tile_ptr/tile_columnidx");
        RTT_CHECK(upload(c, T.tile_ptr, M->tile_ptr, (size_t)tilem + 1, s));
        RTT_CHECK(upload(c, T.tile_col, M->tile_columnidx, (size_t)nt, s));
        T.row_data.release();
        k_validate_lists<<<grid_for(tilem + 1, 256), 256, 0, s>>>(
            tilem, T.tile_ptr.as<int>(), T.tile_col.as<int>(), nt, tilen, c->ws.err.as<int>());
        c->ws.launches++;
        return check_tiles(c->ws, "row-major tile lists");
    }
    if (M->csc_tile_ptr == nullptr || (nt > 0 && M->csc_tile_rowidx == nullptr))
        return fail(RTT_ERR_INVALID_ARGUMENT, "column-major tiles without csc_tile_ptr/csc_tile_rowidx");
    RTT_CHECK(upload(c, T.csc_ptr, M->csc_tile_ptr, (size_t)tilen + 1, s));
    RTT_CHECK(upload(c, T.csc_row, M->csc_tile_rowidx, (size_t)nt, s));
    T.csc_data.release();
    k_validate_lists<<<grid_for(tilen + 1, 256), 256, 0, s>>>(
        tilen, T.csc_ptr.as<int>(), T.csc_row.as<int>(), nt, tilem, c->ws.err.as<int>());
    c->ws.launches++;
    RTT_CHECK(check_tiles(c->ws, "column-major tile lists"));
    // row view: stable sort of CSC positions by tile row
    RTT_CHECK(T.tile_ptr.ensure(sizeof(int) * ((size_t)tilem + 1), s));
    RTT_CHECK(T.tile_col.ensure(sizeof(int) * (size_t)nt + 16, s));
    RTT_CHECK(T.row_data.ensure(sizeof(int) * (size_t)nt + 16, s));
    RTT_CHECK(T.tmp0.ensure(sizeof(int) * (size_t)nt + 16, s));
    RTT_CHECK(T.tmp1.ensure(sizeof(int) * (size_t)nt + 16, s));
    RTT_CHECK(T.tmp2.ensure(sizeof(int) * (size_t)nt + 16, s));
    int *owner = T.tmp0.as<int>(), *iota = T.tmp1.as<int>(), *keys = T.tmp2.as<int>();
    if (nt > 0)
    {
        k_expand_ptr<<<grid_for(tilen, 256), 256, 0, s>>>(tilen, T.csc_ptr.as<int>(), owner);
        k_iota_i<<<grid_for(nt, 256), 256, 0, s>>>(iota, nt);
        size_t bytes = 0;
        const int eb = bits_for(tilem);
        RTT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, T.csc_row.as<int>(), keys, iota,
                                                 T.row_data.as<int>(), nt, 0, eb, s));
        RTT_CHECK(c->ws.scan_tmp.ensure(bytes, s));
        RTT_CUDA(cub::DeviceRadixSort::SortPairs(c->ws.scan_tmp.p, bytes, T.csc_row.as<int>(), keys,
                                                 iota, T.row_data.as<int>(), nt, 0, eb, s));
        k_gather_i<<<grid_for(nt, 256), 256, 0, s>>>(owner, T.row_data.as<int>(), nt,
                                                     T.tile_col.as<int>());
        c->ws.launches += 6;
    }
    k_lower_bound<<<grid_for(tilem + 1, 256), 256, 0, s>>>(keys, nt, tilem, T.tile_ptr.as<int>());
    c->ws.launches++;
    return RTT_OK;
}

// The DMMA variant of the numeric kernel reserves extra shared memory; use it
// only when some tile pair can reach the configured cutoff.
int effective_cutoff(rtt_context c, const DevTiles &A, const DevTiles &B, int *cutoff)
{
    *cutoff = c->cfg.dmma_pair_cutoff;
    if (*cutoff <= 0 || !A.tile_nnz || !B.tile_nnz)
    {
        *cutoff = 0;
        return RTT_OK;
    }
    if (c->cut_cached >= 0)
    {
        *cutoff = c->cut_cached;
        return RTT_OK;
    }
    RTT_CHECK(c->counters.ensure(sizeof(long long) * 4, c->ws.stream));
    RTT_CHECK(c->maxnnz.ensure(sizeof(int) * 2, c->ws.stream));
    RTT_CHECK(max_tile_nnz_device(c->ws, A.tile_nnz, A.numtile, c->maxnnz.as<int>()));
    RTT_CHECK(max_tile_nnz_device(c->ws, B.tile_nnz, B.numtile, c->maxnnz.as<int>() + 1));
    RTT_CUDA(cudaMemcpyAsync(c->ws.h_scalars + 10, c->maxnnz.p, sizeof(int) * 2,
                             cudaMemcpyDeviceToHost, c->ws.stream));
    RTT_CUDA(cudaStreamSynchronize(c->ws.stream));
    c->ws.syncs++;
    if ((long long)c->ws.h_scalars[10] * c->ws.h_scalars[11] < (long long)*cutoff)
        *cutoff = 0;
    c->cut_cached = *cutoff; // tile sizes change only with a new symbolic
    return RTT_OK;
}

DevTiles view_with_rowdata(const TileBufs &T)
{
    DevTiles v = T.view();
    v.row_data = T.row_data.p ? T.row_data.as<int>() : nullptr;
    v.csc_data = T.csc_data.p ? T.csc_data.as<int>() : nullptr;
    return v;
}

inline long long as_key(const void *p) { return (long long)(intptr_t)p; }

// Host-side inputs of the numeric launches (GraphSlot::key), outputs excluded.
void numeric_key(rtt_context c, std::vector<long long> &k)
{
    const TileBufs &TB = c->b_alias ? c->A : c->B;
    const TileBufs *both[2] = {&c->A, &TB};
    for (const TileBufs *T : both)
        for (long long v : {(long long)T->m, (long long)T->n, (long long)T->tilem,
                            (long long)T->tilen, (long long)T->numtile, (long long)T->nnz,
                            (long long)T->dup_cols, (long long)T->generic,
                            (long long)T->payload})
            k.push_back(v);
    const SymbolicOut &S = c->S;
    for (long long v : {(long long)S.numtile, S.nnz, (long long)S.tilem, (long long)S.tilen,
                        (long long)S.m, (long long)S.n, (long long)S.multi_window})
        k.push_back(v);
    for (long long v : {as_key(c->b_rp), as_key(c->b_ci), as_key(c->b_va), c->b_nnz,
                        (long long)c->b_dups, (long long)c->b_alias, (long long)c->op_aat,
                        as_key(c->a_rp), as_key(c->a_ci), as_key(c->a_va),
                        (long long)c->cut_cached,
                        (long long)c->bat_active, (long long)c->bat_count,
                        (long long)c->bat_rows})
        k.push_back(v);
    const int *cfg = reinterpret_cast<const int *>(&c->cfg);
    k.insert(k.end(), cfg, cfg + sizeof(rtt_config) / sizeof(int));
    // every device buffer of the context: a regrown one changes its address
    auto put = [&](const DevBuf &b) { k.push_back(as_key(b.p)); };
    c->A.each(put);
    c->B.each(put);
    c->S.each(put);
    for (const DevBuf *b : own_buffers(c))
        put(*b);
    const Workspace &ws = c->ws;
    put(ws.err);
    put(ws.scan_tmp);
    for (const DevBuf &b : ws.tmp)
        put(b);
    for (long long v : {as_key(ws.h_scalars), as_key(ws.h_scalars64), as_key(ws.side)})
        k.push_back(v);
}

// The numeric phase can be captured: CSR written by the numeric kernel, and
// no leaf DMMA step (its leaf build reads sizes on the host).
bool graphs_allowed(rtt_context c)
{
    return c->cfg.fused_csr_output != 0 && c->cfg.leaf_dmma == 0;
}

// Runs enqueue (device work on ws.stream, with no host read and no sync)
// either eagerly or as a CUDA graph: the second call in a row with the same
// key captures it (on a private stream: the legacy default stream cannot
// capture) and launches the graph; later calls with that key replay it.
// A capture that fails, because a workspace buffer had to grow, runs eagerly.
template <class F>
int run_phase(rtt_context c, int slot, const std::vector<long long> &head, bool allow,
              F &&enqueue)
{
    Workspace &ws = c->ws;
    GraphSlot &g = c->graph[slot];
    // the call's own inputs (head), then the context's state
    auto make_key = [&]() {
        std::vector<long long> k = head;
        numeric_key(c, k);
        k.push_back(as_key(ws.stream));
        return k;
    };
    c->stats.graph_launched = 0;
    if (!allow || c->cfg.cuda_graphs == 0 || c->cfg.stage_timing != 0)
    {
        g.reset();
        return enqueue();
    }
    std::vector<long long> key = make_key();
    if (g.exec != nullptr && key == g.key)
    {
        RTT_CUDA(cudaGraphLaunch(g.exec, ws.stream));
        ws.launches += g.launches;
        c->stats.graph_launched = 1;
        return RTT_OK;
    }
    auto eager = [&]() -> int {
        g.reset();
        RTT_CHECK(enqueue());
        g.key = make_key(); // with the addresses of buffers that grew inside enqueue
        g.warm = true;
        return RTT_OK;
    };
    if (!g.warm || key != g.key)
        return eager();
    if (c->cap_stream == nullptr)
        RTT_CUDA(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
    cudaStream_t user = ws.stream;
    const int launches0 = ws.launches;
    ws.stream = c->cap_stream;
    freeze_growth(true);
    cudaGraph_t graph = nullptr;
    int rc = RTT_ERR_CUDA;
    cudaError_t e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess)
    {
        rc = enqueue();
        e = cudaStreamEndCapture(c->cap_stream, &graph);
    }
    freeze_growth(false);
    ws.stream = user;
    const int captured = ws.launches - launches0;
    ws.launches = launches0;
    cudaGraphExec_t exec = nullptr;
    if (rc == RTT_OK && e == cudaSuccess && graph != nullptr)
        e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph != nullptr)
        cudaGraphDestroy(graph);
    if (rc != RTT_OK || e != cudaSuccess || exec == nullptr)
    {
        if (exec != nullptr)
            cudaGraphExecDestroy(exec);
        cudaGetLastError();
        cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(ws.side, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone)
            return fail(RTT_ERR_CUDA, "side stream left in a failed graph capture");
        return eager();
    }
    g.exec = exec;
    g.key = std::move(key);
    g.launches = captured;
    g.warm = false;
    RTT_CUDA(cudaGraphLaunch(exec, user));
    ws.launches += captured;
    c->stats.graph_launched = 1;
    return RTT_OK;
}

// Device work of the numeric step into C's CSR (c_row_ptr, c_col_idx,
// c_values), counters copied to ws.h_scalars64[2..5]; no host reads unless
// fused_csr_output == 0 (tile2csr sizes its output on the host).
int numeric_enqueue(rtt_context c, int *c_row_ptr, int *c_col_idx, double *c_values, int cutoff)
{
    Workspace &ws = c->ws;
    const TileBufs &TB = c->b_alias ? c->A : c->B;
    RTT_CHECK(c->counters.ensure(sizeof(long long) * 4, ws.stream));
    RTT_CUDA(cudaMemsetAsync(c->counters.p, 0, sizeof(long long) * 4, ws.stream));
    NumericConfig nc;
    nc.dmma_pair_cutoff = cutoff;
    nc.counters = c->counters.as<long long>();
    // TMA staging reads the tile arrays: only when they were built
    nc.b_staging = c->cfg.b_staging != 0 && c->A.payload && TB.payload;
    nc.split_target = c->cfg.split_target;
    if (c->cfg.stage_timing)
    {
        nc.ev_begin = ws.ev[3];
        nc.ev_end = ws.ev[4];
    }
    // the leaf DMMA step writes C's tiles; tile2csr makes the CSR
    const bool leaf = c->cfg.leaf_dmma != 0;
    const bool fused = c->cfg.fused_csr_output != 0 && !leaf;
    nc.write_tiles = !fused || c->cfg.keep_tiles != 0;
    if (fused)
    {
        nc.csr_rowptr = c_row_ptr;
        nc.csr_col = c_col_idx;
        nc.csr_val = c_values;
    }
    DevTiles dB = TB.view();
    dB.csr_rowptr = c->b_rp;
    dB.csr_col = c->b_ci;
    dB.csr_val = c->b_va;
    dB.nnz = (int)c->b_nnz;
    nc.conflict_safe = c->b_dups;
    nc.segment_walk = c->cfg.segment_walk != 0;
    nc.persistent_rows = c->cfg.persistent_rows != 0;
    nc.global_rows = c->cfg.global_rows;
    // the numeric step reads A's entries from its CSR rows
    DevTiles dA = c->A.view();
    dA.csr_rowptr = c->a_rp;
    dA.csr_col = c->a_ci;
    dA.csr_val = c->a_va;
    if (leaf)
        RTT_CHECK(numeric_leaf_device(ws, dA, dB, c->leaf_a, c->leaf_b, c->S, nc));
    else
        RTT_CHECK(numeric_select_device(ws, dA, dB, c->S, nc));
    if (!fused)
    {
        SymbolicOut &S = c->S;
        RTT_CHECK(csr_rowptr_device(ws, S, c_row_ptr));
        RTT_CHECK(tile2csr_fill_device(ws, S.c_tile_ptr.as<int>(), S.c_tile_col.as<int>(),
                                       S.c_tile_nnz.as<int>(), S.c_ptr.as<uint8_t>(),
                                       S.c_col.as<uint8_t>(), S.c_val.as<double>(), S.m, S.n,
                                       S.tilem, TD, nullptr, -1, c_row_ptr, c_col_idx, c_values,
                                       false));
    }
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars64 + 2, c->counters.p, sizeof(long long) * 4,
                             cudaMemcpyDeviceToHost, ws.stream));
    return RTT_OK;
}

// After numeric_enqueue (eager or graph): device checks, then the statistics.
int numeric_finish(rtt_context c)
{
    Workspace &ws = c->ws;
    RTT_CHECK(check_device_error(ws, "numeric"));
    if (c->cfg.stage_timing && c->S.numtile > 0)
    {
        float tn = 0.f;
        RTT_CUDA(cudaEventElapsedTime(&tn, ws.ev[3], ws.ev[4]));
        c->stats.numeric_kernel_ms = tn;
    }
    c->stats.dmma_pairs = ws.h_scalars64[2];
    c->stats.sparse_pairs = ws.h_scalars64[3];
    // the numeric kernels count every (a_ik, b_kj) pair once: sum over A
    // entries of nnz(B(k, :)), the reference's nnzCub
    c->stats.nnz_cub = ws.h_scalars64[3];
    c->stats.split_windows = ws.h_scalars64[4];
    c->stats.split_multi_window_tasks = ws.h_scalars64[5];
    c->stats.kernel_launches = ws.launches;
    c->stats.host_syncs = ws.syncs;
    return RTT_OK;
}

int numeric_args_ok(rtt_context c, const int *c_row_ptr, const int *c_col_idx,
                    const double *c_values)
{
    if (c_row_ptr == nullptr || (c->S.nnz > 0 && (c_col_idx == nullptr || c_values == nullptr)))
        return fail(RTT_ERR_INVALID_ARGUMENT, "NULL output buffer");
    return RTT_OK;
}

} // namespace

// csr2tile of A (and B: A's own tiles for A*A, A^T's for A*A^T), B's scalar
// CSR rows, and the device views the symbolic and numeric steps take.  The
// shape checks of the entry points come first.  Shared by the 32-bit product
// and the 64-bit (chunked) one.
int prepare_operands(rtt_context c, const rtt_csr_view *A, const rtt_csr_view *B, int op,
                     DevTiles &dA, DevTiles &dB)
{
    Workspace &ws = c->ws;
    // The flat numeric step reads A and B from their CSR rows, so only the
    // tile index and B's row segments are built; the per-entry tile arrays
    // are built for the kernels that read them (DMMA pairs, TMA staging).
    const bool payload = c->cfg.dmma_pair_cutoff > 0 || c->cfg.b_staging != 0;
    // B's row segments drive symbolic step 2: A's own when B is A
    RTT_CHECK(map_device_error(csr2tile_device(ws, A->rows, A->cols, (int)A->nnz, A->row_ptr,
                                               A->col_idx, A->values, c->A, true, false,
                                               op == RTT_OP_AB && B == nullptr, payload)));
    c->a_rp = A->row_ptr;
    c->a_ci = A->col_idx;
    c->a_va = A->values;
    c->op_aat = op == RTT_OP_AAT;
    if (op == RTT_OP_AB && B == nullptr)
    {
        if (A->rows != A->cols)
            return rtt::fail(RTT_ERR_SHAPE_MISMATCH, "A*A needs a square A");
        c->b_alias = true;
        c->b_rp = A->row_ptr;
        c->b_ci = A->col_idx;
        c->b_va = A->values;
        c->b_nnz = A->nnz;
        c->b_dups = c->A.dup_cols;
    }
    else
    {
        c->b_alias = false;
        if (op == RTT_OP_AAT)
        {
            RTT_CHECK(c->bt_rowptr.ensure(sizeof(int) * ((size_t)A->cols + 1), ws.stream));
            RTT_CHECK(c->bt_col.ensure(sizeof(int) * (size_t)A->nnz + 16, ws.stream));
            RTT_CHECK(c->bt_val.ensure(sizeof(double) * (size_t)A->nnz + 16, ws.stream));
            RTT_CHECK(csr_transpose_device(ws, A->rows, A->cols, (int)A->nnz, A->row_ptr,
                                           A->col_idx, A->values, c->bt_rowptr.as<int>(),
                                           c->bt_col.as<int>(), c->bt_val.as<double>()));
            RTT_CHECK(map_device_error(csr2tile_device(ws, A->cols, A->rows, (int)A->nnz,
                                                       c->bt_rowptr.as<int>(), c->bt_col.as<int>(),
                                                       c->bt_val.as<double>(), c->B, true, false,
                                                       true, payload)));
            c->b_rp = c->bt_rowptr.as<int>();
            c->b_ci = c->bt_col.as<int>();
            c->b_va = c->bt_val.as<double>();
            c->b_nnz = A->nnz;
        }
        else
        {
            if (B->rows != A->cols)
                return rtt::fail(RTT_ERR_SHAPE_MISMATCH, "A->cols != B->rows");
            if (B->nnz < 0 || B->nnz > INT_MAX)
                return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "bad B shape");
            RTT_CHECK(map_device_error(csr2tile_device(ws, B->rows, B->cols, (int)B->nnz,
                                                       B->row_ptr, B->col_idx, B->values, c->B,
                                                       true, false, true, payload)));
            c->b_rp = B->row_ptr;
            c->b_ci = B->col_idx;
            c->b_va = B->values;
            c->b_nnz = B->nnz;
        }
        c->b_dups = c->B.dup_cols;
    }
    const TileBufs &TB = c->b_alias ? c->A : c->B;
    dB = TB.view();
    dB.csr_rowptr = c->b_rp;
    dB.csr_col = c->b_ci;
    dB.csr_val = c->b_va;
    dB.nnz = (int)c->b_nnz;
    dA = c->A.view();
    // A's CSR rows: step 2 walks the tile row's entries straight from them
    dA.csr_rowptr = A->row_ptr;
    dA.csr_col = A->col_idx;
    return RTT_OK;
}

extern "C" {

const char *rtt_status_string(int status)
{
    switch (status)
    {
    case RTT_OK:
        return "ok";
    case RTT_ERR_INVALID_ARGUMENT:
        return "invalid argument";
    case RTT_ERR_INVALID_CSR:
        return "invalid CSR";
    case RTT_ERR_SHAPE_MISMATCH:
        return "shape mismatch";
    case RTT_ERR_OUT_OF_MEMORY:
        return "out of memory";
    case RTT_ERR_CUDA:
        return "CUDA error";
    case RTT_ERR_UNREPRESENTABLE:
        return "output not representable in int32";
    case RTT_ERR_NO_DEVICE:
        return "no usable CUDA device";
    case RTT_ERR_DEVICE_CHECK:
        return "device-side check failed";
    case RTT_ERR_INVALID_PERMUTATION:
        return "invalid permutation";
    case RTT_ERR_TAIL_NONEMPTY:
        return "row past the permutation prefix is not empty";
    case RTT_ERR_STATE:
        return "invalid call order";
    default:
        return "unknown status";
    }
}

const char *rtt_last_error(void) { return rtt::last_error_ref().c_str(); }

const char *rtt_version(void) { return "rtt-spgemm-b200 0.1 (sm_100a)"; }

void rtt_config_default(rtt_config *config)
{
    if (config == nullptr)
        return;
    std::memset(config, 0, sizeof(*config));
    config->dmma_pair_cutoff = 0;
    config->fused_csr_output = 1;
    config->keep_tiles = 0;
    config->b_staging = 0;
    config->cuda_graphs = 1;
}

int rtt_set_device(int device)
{
    std::lock_guard<std::mutex> lock(g_mutex);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    {
        cudaGetLastError();
        return rtt::fail(RTT_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= count || device >= 16)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "device index out of range");
    g_device = device;
    return RTT_OK;
}

int rtt_context_create(rtt_context *ctx, int device)
{
    if (ctx == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "ctx is NULL");
    rtt_context c = new (std::nothrow) rtt_context_s();
    if (c == nullptr)
        return rtt::fail(RTT_ERR_OUT_OF_MEMORY, "context allocation failed");
    int st = c->ws.init(device);
    if (st != RTT_OK)
    {
        c->ws.destroy();
        delete c;
        return st;
    }
    rtt_config_default(&c->cfg);
    std::memset(&c->stats, 0, sizeof(c->stats));
    *ctx = c;
    return RTT_OK;
}

void rtt_context_destroy(rtt_context c)
{
    if (c == nullptr)
        return;
    cudaSetDevice(c->ws.device);
    cudaStreamSynchronize(c->ws.stream);
    for (rtt::GraphSlot &g : c->graph)
        g.reset();
    if (c->cap_stream != nullptr)
        cudaStreamDestroy(c->cap_stream);
    c->A.release();
    c->B.release();
    c->S.release();
    c->leaf_a.release();
    c->leaf_b.release();
    for (rtt::DevBuf *b : own_buffers(c))
        b->release();
    for (int b = 0; b < 2; ++b)
    {
        if (c->hstage[b] != nullptr)
            cudaFreeHost(c->hstage[b]);
        if (c->hstage_ev[b] != nullptr)
            cudaEventDestroy(c->hstage_ev[b]);
    }
    const int dev = c->ws.device;
    c->ws.destroy();
    delete c;
    // hand the memory this context freed back to the driver
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
        cudaMemPoolTrimTo(pool, 0);
    cudaGetLastError();
}

int rtt_context_trim(rtt_context c)
{
    if (c == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "ctx is NULL");
    RTT_CUDA(cudaSetDevice(c->ws.device));
    RTT_CUDA(cudaStreamSynchronize(c->ws.stream));
    if (c->ws.side != nullptr)
        RTT_CUDA(cudaStreamSynchronize(c->ws.side));
    for (rtt::GraphSlot &g : c->graph)
        g.reset();
    c->A.release();
    c->B.release();
    c->S.release();
    c->leaf_a.release();
    c->leaf_b.release();
    for (rtt::DevBuf *b : own_buffers(c))
        b->release();
    c->ws.scan_tmp.release();
    for (rtt::DevBuf &b : c->ws.tmp)
        b.release();
    c->have_symbolic = false;
    c->have_sym64 = false;
    c->bat_active = false;
    c->cut_cached = -1;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, c->ws.device) == cudaSuccess)
        cudaMemPoolTrimTo(pool, 0);
    cudaGetLastError();
    return RTT_OK;
}

int rtt_context_set_stream(rtt_context c, void *stream)
{
    if (c == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "ctx is NULL");
    // buffers allocated in the order of the old stream are complete before
    // the new stream uses them
    RTT_CUDA(cudaStreamSynchronize(c->ws.stream));
    c->ws.stream = static_cast<cudaStream_t>(stream);
    return RTT_OK;
}

int rtt_context_set_config(rtt_context c, const rtt_config *config)
{
    if (c == nullptr || config == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (config->dmma_pair_cutoff < 0)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "dmma_pair_cutoff must be >= 0");
    if (config->chunk_tiles < 0 || config->chunk_nnz < 0 || config->segment_walk < 0 ||
        config->segment_walk > 1 || config->persistent_rows < 0 || config->persistent_rows > 1)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT,
                         "chunk_tiles, chunk_nnz >= 0, segment_walk and persistent_rows 0 or 1");
    if (config->leaf_dmma < 0 || config->leaf_dmma > 1)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "leaf_dmma must be 0 or 1");
    if (config->global_rows < 0 || config->global_rows > 2)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "global_rows must be 0, 1 or 2");
    if (config->sym_window_slots < -1 ||
        (config->sym_window_slots > 0 &&
         (config->sym_window_slots < 255 || config->sym_window_slots > 6000)))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "sym_window_slots must be -1, 0 or 255..6000");
    c->cfg = *config;
    c->S.sym_window_slots = config->sym_window_slots;
    c->cut_cached = -1;
    return RTT_OK;
}

int rtt_context_get_stats(rtt_context c, rtt_stats *stats)
{
    if (c == nullptr || stats == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "NULL argument");
    *stats = c->stats;
    return RTT_OK;
}

// ---------------------------------------------------------------- drop-ins
int rtt_csr2tile_row_major(SMatrix *M)
{
    if (!csr_args_ok(M))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "csr2tile_row_major: bad CSR arguments");
    std::lock_guard<std::mutex> lock(g_mutex);
    rtt_context c = nullptr;
    RTT_CHECK(default_context(&c));
    TileBufs &T = c->A;
    RTT_CHECK(tile_host_csr(c, M, T, true, false));
    cudaStream_t s = c->ws.stream;
    const size_t nt = (size_t)T.numtile;
    HostArrays h;
    int **tp = h.slot<int>(), **tc = h.slot<int>(), **tr = h.slot<int>(), **tn = h.slot<int>();
    unsigned char **P = h.slot<unsigned char>(), **Cb = h.slot<unsigned char>();
    double **V = h.slot<double>();
    unsigned short **Mk = h.slot<unsigned short>();
    RTT_CHECK(download(c, tp, T.tile_ptr.p, (size_t)T.tilem + 1, s));
    RTT_CHECK(download(c, tc, T.tile_col.p, nt, s));
    RTT_CHECK(download(c, tr, T.tile_row.p, nt, s));
    RTT_CHECK(download(c, tn, T.tile_nnz.p, nt + 1, s));
    RTT_CHECK(download(c, P, T.ptr.p, nt * TD, s));
    RTT_CHECK(download(c, Cb, T.col.p, (size_t)M->nnz, s));
    RTT_CHECK(download(c, V, T.val.p, (size_t)M->nnz, s));
    RTT_CHECK(download(c, Mk, T.mask.p, nt * TD, s));
    M->tilem = T.tilem;
    M->tilen = T.tilen;
    M->numtile = T.numtile;
    M->tile_ptr = *tp;
    M->tile_columnidx = *tc;
    M->tile_rowidx = *tr;
    M->tile_nnz = *tn;
    M->tile_csr_Ptr = *P;
    M->tile_csr_Col = *Cb;
    M->tile_csr_Value = *V;
    M->mask = *Mk;
    h.committed = true;
    return RTT_OK;
}

int rtt_csr2tile_col_major(SMatrix *M)
{
    if (!csr_args_ok(M))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "csr2tile_col_major: bad CSR arguments");
    std::lock_guard<std::mutex> lock(g_mutex);
    rtt_context c = nullptr;
    RTT_CHECK(default_context(&c));
    TileBufs &T = c->A;
    TileBufs &U = c->B;
    RTT_CHECK(tile_host_csr(c, M, T, false, true));
    RTT_CHECK(build_tile_csc(c->ws, T));
    RTT_CHECK(tiles_to_col_major(c->ws, T, U));
    RTT_CHECK(check_device_error(c->ws, "csr2tile_col_major"));
    cudaStream_t s = c->ws.stream;
    const size_t nt = (size_t)T.numtile;
    HostArrays h;
    int **tp = h.slot<int>(), **tc = h.slot<int>(), **tn = h.slot<int>();
    int **cp = h.slot<int>(), **cr = h.slot<int>();
    unsigned char **P = h.slot<unsigned char>(), **Cb = h.slot<unsigned char>();
    double **V = h.slot<double>();
    unsigned short **Mk = h.slot<unsigned short>();
    int **tr = h.slot<int>();
    RTT_CHECK(download(c, tp, T.tile_ptr.p, (size_t)T.tilem + 1, s));
    RTT_CHECK(download(c, tc, T.tile_col.p, nt, s));
    RTT_CHECK(download(c, tn, U.tile_nnz.p, nt + 1, s));
    RTT_CHECK(download(c, cp, T.csc_ptr.p, (size_t)T.tilen + 1, s));
    RTT_CHECK(download(c, cr, T.csc_row.p, nt, s));
    RTT_CHECK(download(c, P, U.ptr.p, nt * TD, s));
    RTT_CHECK(download(c, Cb, U.col.p, (size_t)M->nnz, s));
    RTT_CHECK(download(c, V, U.val.p, (size_t)M->nnz, s));
    RTT_CHECK(download(c, Mk, U.mask.p, nt * TD, s));
    *tr = static_cast<int *>(std::calloc(nt > 0 ? nt : 1, sizeof(int)));
    if (*tr == nullptr)
        return rtt::fail(RTT_ERR_OUT_OF_MEMORY, "host calloc failed");
    M->tilem = T.tilem;
    M->tilen = T.tilen;
    M->numtile = T.numtile;
    M->tile_ptr = *tp;
    M->tile_columnidx = *tc;
    M->tile_rowidx = *tr;
    M->tile_nnz = *tn;
    M->csc_tile_ptr = *cp;
    M->csc_tile_rowidx = *cr;
    M->tile_csr_Ptr = *P;
    M->tile_csr_Col = *Cb;
    M->tile_csr_Value = *V;
    M->mask = *Mk;
    h.committed = true;
    return RTT_OK;
}

int rtt_spgemm_tile(SMatrix *A, SMatrix *B, SMatrix *C)
{
    if (A == nullptr || B == nullptr || C == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "spgemm_tile: NULL matrix");
    if (A->m < 0 || A->n < 0 || B->m < 0 || B->n < 0)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "spgemm_tile: negative shape");
    if (A->n != B->m)
        return rtt::fail(RTT_ERR_SHAPE_MISMATCH, "spgemm_tile: A->n != B->m");
    std::lock_guard<std::mutex> lock(g_mutex);
    rtt_context c = nullptr;
    RTT_CHECK(default_context(&c));
    RTT_CHECK(upload_tiles(c, A, false, c->A));
    RTT_CHECK(upload_tiles(c, B, true, c->B));
    const DevTiles dA = view_with_rowdata(c->A);
    DevTiles dB = view_with_rowdata(c->B);
    // B's scalar CSR rows for the symbolic and numeric steps, assembled on the
    // device from the column-major tiles (tile2csr through the row->data index)
    {
        cudaStream_t s = c->ws.stream;
        const int mb = B->m;
        RTT_CHECK(c->in2_rp.ensure(sizeof(int) * ((size_t)mb + 2), s));
        RTT_CHECK(c->in_col.ensure(sizeof(int) * ((size_t)mb + 2), s));
        int *cnt = c->in_col.as<int>();
        RTT_CHECK(tile2csr_count_device(c->ws, dB.tile_ptr, dB.tile_col, dB.tile_nnz, dB.ptr,
                                        dB.col, mb, B->n, dB.tilem, TD, nullptr, -1, cnt,
                                        dB.row_data));
        RTT_CHECK(scan_exclusive_int(c->ws, cnt, c->in2_rp.as<int>(), mb));
        int bnnz = 0;
        RTT_CHECK(read_int(c->ws, c->in2_rp.as<int>() + mb, &bnnz));
        RTT_CHECK(c->in2_col.ensure(sizeof(int) * (size_t)bnnz + 16, s));
        RTT_CHECK(c->in2_val.ensure(sizeof(double) * (size_t)bnnz + 16, s));
        RTT_CHECK(tile2csr_fill_device(c->ws, dB.tile_ptr, dB.tile_col, dB.tile_nnz, dB.ptr, dB.col,
                                       dB.val, mb, B->n, dB.tilem, TD, nullptr, -1,
                                       c->in2_rp.as<int>(), c->in2_col.as<int>(),
                                       c->in2_val.as<double>(), false, dB.row_data));
        dB.csr_rowptr = c->in2_rp.as<int>();
        dB.csr_col = c->in2_col.as<int>();
        dB.csr_val = c->in2_val.as<double>();
        dB.nnz = bnnz;
    }
    RTT_CHECK(map_device_error(symbolic_device(c->ws, dA, dB, c->S)));
    NumericConfig nc;
    RTT_CHECK(effective_cutoff(c, dA, dB, &nc.dmma_pair_cutoff));
    nc.write_tiles = true;
    nc.conflict_safe = true; // caller tiles may repeat a coordinate
    nc.b_staging = c->cfg.b_staging != 0;
    nc.split_target = c->cfg.split_target;
    RTT_CHECK(numeric_select_device(c->ws, dA, dB, c->S, nc));
    RTT_CHECK(check_device_error(c->ws, "spgemm_tile numeric"));
    cudaStream_t s = c->ws.stream;
    SymbolicOut &S = c->S;
    const size_t nt = (size_t)S.numtile, nnz = (size_t)S.nnz;
    HostArrays h;
    int **tp = h.slot<int>(), **tc = h.slot<int>(), **tr = h.slot<int>(), **tn = h.slot<int>();
    unsigned char **P = h.slot<unsigned char>(), **Cb = h.slot<unsigned char>();
    double **V = h.slot<double>();
    unsigned short **Mk = h.slot<unsigned short>();
    RTT_CHECK(download(c, tp, S.c_tile_ptr.p, (size_t)S.tilem + 1, s));
    RTT_CHECK(download(c, tc, S.c_tile_col.p, nt, s));
    RTT_CHECK(download(c, tr, S.c_tile_row.p, nt, s));
    RTT_CHECK(download(c, tn, S.c_tile_nnz.p, nt + 1, s));
    RTT_CHECK(download(c, P, S.c_ptr.p, nt * TD, s));
    RTT_CHECK(download(c, Cb, S.c_col.p, nnz, s));
    RTT_CHECK(download(c, V, S.c_val.p, nnz, s));
    RTT_CHECK(download(c, Mk, S.c_mask.p, nt * TD, s));
    C->m = A->m;
    C->n = B->n;
    C->tilem = S.tilem;
    C->tilen = S.tilen;
    C->numtile = S.numtile;
    C->nnz = (int)S.nnz;
    C->tile_ptr = *tp;
    C->tile_columnidx = *tc;
    C->tile_rowidx = *tr;
    C->tile_nnz = *tn;
    C->tile_csr_Ptr = *P;
    C->tile_csr_Col = *Cb;
    C->tile_csr_Value = *V;
    C->mask = *Mk;
    h.committed = true;
    return RTT_OK;
}

int rtt_tile2csr_restore_rows(SMatrix *M, const int *new_to_old, int perm_size, int tile_dim,
                              int canonical)
{
    if (M == nullptr || M->m < 0 || M->n < 0 || M->tilem < 0 || M->numtile < 0 ||
        M->tile_ptr == nullptr || M->tile_nnz == nullptr ||
        (M->numtile > 0 && (M->tile_columnidx == nullptr || M->tile_csr_Ptr == nullptr)) ||
        (M->nnz > 0 && (M->tile_csr_Col == nullptr || M->tile_csr_Value == nullptr)))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "tile2csr: malformed tile matrix");
    if (tile_dim != 8 && tile_dim != 16)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "tile2csr: tile_dim must be 8 or 16");
    const bool identity = new_to_old == nullptr && perm_size < 0;
    if (!identity)
    {
        if (perm_size < 0 || perm_size > M->m || (perm_size > 0 && new_to_old == nullptr))
            return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "tile2csr_restore_rows: bad permutation size");
        std::vector<unsigned char> seen((size_t)M->m, 0);
        for (int i = 0; i < perm_size; ++i)
        {
            const int o = new_to_old[i];
            if (o < 0 || o >= M->m || seen[(size_t)o])
                return rtt::fail(RTT_ERR_INVALID_PERMUTATION,
                                 "tile2csr_restore_rows: permutation is not one-to-one");
            seen[(size_t)o] = 1;
        }
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    rtt_context c = nullptr;
    RTT_CHECK(default_context(&c));
    cudaStream_t s = c->ws.stream;
    TileBufs &T = c->A;
    const int nt = M->numtile, tilem = M->tilem, m = M->m;
    const int tnz = nt >= 0 ? M->tile_nnz[nt] : 0;
    RTT_CHECK(upload(c, T.tile_ptr, M->tile_ptr, (size_t)tilem + 1, s));
    RTT_CHECK(upload(c, T.tile_col, M->tile_columnidx, (size_t)nt, s));
    RTT_CHECK(upload(c, T.tile_nnz, M->tile_nnz, (size_t)nt + 1, s));
    RTT_CHECK(upload(c, T.ptr, M->tile_csr_Ptr, (size_t)nt * tile_dim, s));
    const size_t nent = (size_t)std::max(tnz, M->nnz);
    RTT_CHECK(upload(c, T.col, M->tile_csr_Col, nent, s));
    RTT_CHECK(upload(c, T.val, M->tile_csr_Value, nent, s));
    {
        // tile lists: monotone pointers, in-range entry offsets (columns are
        // range-checked per entry by the kernels, as the reference does)
        // row offsets are clamped per row by the kernels (as the reference
        // does), so only the per-tile entry ranges are checked here
        k_validate_tile_data<<<grid_for(nt > 0 ? nt : 1, 256), 256, 0, s>>>(
            nt, T.tile_nnz.as<int>(), (int)nent, 0, T.ptr.as<uint8_t>(), c->ws.err.as<int>());
        k_validate_ptr<<<grid_for(tilem + 1, 256), 256, 0, s>>>(tilem, T.tile_ptr.as<int>(), nt,
                                                                c->ws.err.as<int>());
        c->ws.launches += 2;
        RTT_CHECK(check_tiles(c->ws, "tile2csr input"));
    }
    RTT_CHECK(upload(c, c->in2_rp, new_to_old, identity ? 0 : (size_t)perm_size, s));
    const int *perm = identity ? nullptr : c->in2_rp.as<int>();
    const int psize = identity ? -1 : perm_size;
    RTT_CHECK(c->out_rp.ensure(sizeof(int) * ((size_t)m + 2), s));
    RTT_CHECK(c->in_col.ensure(sizeof(int) * ((size_t)m + 2), s));
    int *row_cnt = c->in_col.as<int>();
    RTT_CHECK(tile2csr_count_device(c->ws, T.tile_ptr.as<int>(), T.tile_col.as<int>(),
                                    T.tile_nnz.as<int>(), T.ptr.as<uint8_t>(), T.col.as<uint8_t>(),
                                    m, M->n, tilem, tile_dim, perm, psize, row_cnt));
    RTT_CHECK(map_device_error(check_device_error(c->ws, "tile2csr count")));
    // int64 total first (overflow check), then the int32 row pointer
    RTT_CHECK(c->in_val.ensure(sizeof(long long) * ((size_t)m + 2), s));
    RTT_CHECK(scan_exclusive_i64(c->ws, row_cnt, c->in_val.as<long long>(), m));
    long long total = 0;
    RTT_CHECK(read_i64(c->ws, c->in_val.as<long long>() + m, &total));
    if (total > (long long)INT_MAX)
        return rtt::fail(RTT_ERR_UNREPRESENTABLE, "tile2csr: nnz exceeds int32");
    RTT_CHECK(scan_exclusive_int(c->ws, row_cnt, c->out_rp.as<int>(), m));
    RTT_CHECK(c->out_col.ensure(sizeof(int) * (size_t)total + 16, s));
    RTT_CHECK(c->out_val.ensure(sizeof(double) * (size_t)total + 16, s));
    RTT_CHECK(tile2csr_fill_device(c->ws, T.tile_ptr.as<int>(), T.tile_col.as<int>(),
                                   T.tile_nnz.as<int>(), T.ptr.as<uint8_t>(), T.col.as<uint8_t>(),
                                   T.val.as<double>(), m, M->n, tilem, tile_dim, perm, psize,
                                   c->out_rp.as<int>(), c->out_col.as<int>(),
                                   c->out_val.as<double>(), canonical == 0));
    RTT_CHECK(map_device_error(check_device_error(c->ws, "tile2csr fill")));
    HostArrays h;
    int **rp = h.slot<int>(), **ci = h.slot<int>();
    double **v = h.slot<double>();
    RTT_CHECK(download(c, rp, c->out_rp.p, (size_t)m + 1, s));
    RTT_CHECK(download(c, ci, c->out_col.p, (size_t)total, s));
    RTT_CHECK(download(c, v, c->out_val.p, (size_t)total, s));
    M->rowpointer = *rp;
    M->columnindex = *ci;
    M->value = *v;
    M->nnz = (int)total;
    h.committed = true;
    return RTT_OK;
}

int rtt_csr_to_hybrid_tiles(const SMatrix *M, int tile_rows, int tile_cols, int col_major,
                            int dense_threshold, int build_csc, rtt_hybrid_tiles *out)
{
    if (M == nullptr || out == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "hybrid tiles: NULL argument");
    if (tile_rows <= 0 || tile_cols <= 0 || tile_rows * tile_cols != 32 || dense_threshold < 1 ||
        dense_threshold > 32)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT,
                         "hybrid tiles: tile_rows * tile_cols must be 32, 1 <= threshold <= 32");
    if (M->m < 0 || M->n < 0 || M->nnz < 0 || (M->m == 0 && M->nnz != 0) ||
        (M->m > 0 && M->rowpointer == nullptr) ||
        (M->nnz > 0 && (M->columnindex == nullptr || M->value == nullptr)))
        return rtt::fail(RTT_ERR_INVALID_CSR, "hybrid tiles: malformed CSR");
    if ((long long)M->n / tile_cols >= (1ll << 30) || (long long)M->m / tile_rows >= (1ll << 29))
        return rtt::fail(RTT_ERR_UNREPRESENTABLE, "hybrid tiles: tile grid too large");
    std::lock_guard<std::mutex> lock(g_mutex);
    rtt_context c = nullptr;
    RTT_CHECK(default_context(&c));
    return map_device_error(csr_to_hybrid_host(c->ws, M, tile_rows, tile_cols, col_major,
                                               dense_threshold, build_csc, out));
}

int rtt_super16_index_build(const rtt_hybrid_tiles *L, unsigned int role, rtt_super16_index *out)
{
    if (L == nullptr || out == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "super16 index: NULL argument");
    // leaf geometry and arrays (the checks of build_device_index,
    // src/super16_symbolic.cuh:2128-2143, plus the sorted leaf rows its merge assumes)
    const bool a_role = role == RTT_SUPER16_A8X4;
    if (!a_role && role != RTT_SUPER16_B4X8)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "super16 index: role must be A8x4 or B4x8");
    if ((a_role && (L->tile_rows != 8 || L->tile_cols != 4)) ||
        (!a_role && (L->tile_rows != 4 || L->tile_cols != 8)))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "super16 index: leaf geometry does not fit the role");
    if (L->rows < 0 || L->cols < 0 || L->tile_row_count < 0 || L->tile_col_count < 0 ||
        L->num_tiles < 0 || L->tile_row_ptr == nullptr ||
        (L->num_tiles > 0 && (L->tile_col_idx == nullptr || L->masks == nullptr ||
                              L->tile_row_count == 0 || L->tile_col_count == 0)))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "super16 index: malformed leaf tiles");
    if (L->tile_row_ptr[0] != 0 || L->tile_row_ptr[L->tile_row_count] != L->num_tiles)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "super16 index: bad leaf row pointer");
    for (int r = 0; r < L->tile_row_count; ++r)
    {
        const int b = L->tile_row_ptr[r], e = L->tile_row_ptr[r + 1];
        if (b > e || e > L->num_tiles)
            return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "super16 index: bad leaf row pointer");
        for (int t = b; t < e; ++t)
        {
            const int col = L->tile_col_idx[t];
            if (col < 0 || col >= L->tile_col_count || (t > b && col <= L->tile_col_idx[t - 1]))
                return rtt::fail(RTT_ERR_INVALID_ARGUMENT,
                                 "super16 index: leaf columns must increase inside a leaf row");
        }
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    rtt_context c = nullptr;
    RTT_CHECK(default_context(&c));
    return super16_index_host(c->ws, L, role, out);
}

void rtt_super16_index_destroy(rtt_super16_index *x)
{
    if (x == nullptr)
        return;
    std::free(x->row_ptr);
    std::free(x->col_idx);
    std::free(x->child_ptr);
    std::free(x->child_mask);
    std::free(x->child_leaf_ids);
    std::free(x->boolean_row_masks);
    std::free(x->col_ptr);
    std::free(x->row_idx);
    std::free(x->csc_parent_ids);
    std::memset(x, 0, sizeof(*x));
}

int rtt_plan_tail_queue(int ntasks, const int *scans, const int *matches, const int *output_nnz,
                        const rtt_tail_policy *policy, const rtt_tail_cost_model *model,
                        int *chunks_out, rtt_tail_plan *plan)
{
    if (ntasks < 0 || policy == nullptr || model == nullptr || plan == nullptr ||
        (ntasks > 0 && (scans == nullptr || matches == nullptr || output_nnz == nullptr ||
                        chunks_out == nullptr)))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "plan_tail_queue: bad arguments");
    std::lock_guard<std::mutex> lock(g_mutex);
    rtt_context c = nullptr;
    RTT_CHECK(default_context(&c));
    cudaStream_t s = c->ws.stream;
    const size_t n = (size_t)ntasks;
    RTT_CHECK(upload(c, c->in_rp, scans, n, s));
    RTT_CHECK(upload(c, c->in_col, matches, n, s));
    RTT_CHECK(upload(c, c->in2_rp, output_nnz, n, s));
    RTT_CHECK(c->out_rp.ensure(sizeof(int) * (n + 1), s));
    RTT_CHECK(plan_tail_queue_device(c->ws, ntasks, c->in_rp.as<int>(), c->in_col.as<int>(),
                                     c->in2_rp.as<int>(), *policy, *model, c->out_rp.as<int>(),
                                     plan));
    if (ntasks > 0)
    {
        RTT_CUDA(cudaMemcpyAsync(chunks_out, c->out_rp.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
        RTT_CUDA(cudaStreamSynchronize(s));
    }
    return RTT_OK;
}

void rtt_early_split_policy_default(rtt_tail_policy *p)
{
    if (p == nullptr)
        return;
    std::memset(p, 0, sizeof(*p));
    p->enabled = 0;
    p->admission_threshold = 684947.875;
    p->chunk_target = 342473.938;
    p->max_chunks = 8;
    p->max_heavy_fraction = 0.001;
    p->record_capacity = 131072;
    p->workspace_limit_bytes = 512ll * 1024 * 1024;
    p->workspace_reduction = 1;
}

int rtt_plan_early_split(int ntasks, const int *scans, const int *matches,
                         const int *output_nnz, const rtt_tail_policy *policy,
                         const rtt_tail_cost_model *model, int sm_count, int *chunks_out,
                         rtt_early_split_plan *plan)
{
    if (ntasks < 0 || policy == nullptr || model == nullptr || plan == nullptr ||
        (ntasks > 0 && chunks_out == nullptr))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "plan_early_split: bad arguments");
    std::memset(plan, 0, sizeof(*plan));
    plan->output_tasks = ntasks;
    plan->ordinary_tasks = ntasks;
    plan->sm_count = sm_count;
    plan->exact_parent_partition = 1;
    auto all_ordinary = [&]() {
        for (int i = 0; i < ntasks; ++i)
            chunks_out[i] = 0;
    };
    all_ordinary();
    if (!policy->enabled)
        return RTT_OK; // default off
    if (sm_count <= 0)
    {
        plan->reason = 2; // invalid topology
        return RTT_OK;
    }
    // the partition is the tail-queue plan's, with the policy switched on
    rtt_tail_policy base = *policy;
    base.enabled = 1;
    rtt_tail_plan tp;
    RTT_CHECK(rtt_plan_tail_queue(ntasks, scans, matches, output_nnz, &base, model, chunks_out,
                                  &tp));
    plan->base_reason = tp.reason;
    if (tp.reason != 1)
    {
        plan->reason = 3; // base fallback: the all-ordinary partition, no heavy records
        all_ordinary();
        return RTT_OK;
    }
    // at most ceil(sm_count / 2) persistent heavy CTAs (a pressure bound)
    const long long cap = ((long long)sm_count + 1) / 2;
    if (cap <= 0 || cap > INT_MAX)
    {
        plan->reason = 4;
        all_ordinary();
        return RTT_OK;
    }
    plan->reason = 1;
    plan->ordinary_tasks = tp.ordinary_tasks;
    plan->heavy_tasks = tp.heavy_tasks;
    plan->chunks = tp.chunks;
    plan->global_heavy_worker_block_cap = (int)cap;
    plan->heavy_worker_blocks = (int)std::min<long long>(tp.chunks, cap);
    plan->reduction_worker_blocks =
        policy->workspace_reduction ? (int)std::min<long long>(tp.heavy_tasks, cap) : 0;
    plan->descriptor_bytes = tp.descriptor_bytes;
    plan->heavy_flag_bytes = tp.heavy_flag_bytes;
    plan->partial_workspace_bytes = tp.partial_workspace_bytes;
    // each heavy task owns >= 2 chunks and the parts cover every task once
    long long heavy = 0;
    bool ok = plan->ordinary_tasks + plan->heavy_tasks == plan->output_tasks;
    for (int i = 0; i < ntasks; ++i)
    {
        heavy += chunks_out[i] > 0;
        ok = ok && chunks_out[i] != 1;
    }
    ok = ok && heavy == plan->heavy_tasks;
    plan->exact_parent_partition = ok ? 1 : 0;
    if (!ok || plan->heavy_worker_blocks <= 0)
    {
        plan->reason = 3;
        plan->ordinary_tasks = ntasks;
        plan->heavy_tasks = plan->chunks = 0;
        plan->heavy_worker_blocks = plan->reduction_worker_blocks = 0;
        plan->descriptor_bytes = plan->heavy_flag_bytes = plan->partial_workspace_bytes = 0;
        all_ordinary();
    }
    return RTT_OK;
}

void rtt_hybrid_tiles_destroy(rtt_hybrid_tiles *h)
{
    if (h == nullptr)
        return;
    std::free(h->tile_row_ptr);
    std::free(h->tile_col_idx);
    std::free(h->value_offsets);
    std::free(h->masks);
    std::free(h->values);
    std::free(h->tile_col_ptr);
    std::free(h->tile_row_idx);
    std::free(h->csc_tile_ids);
    std::memset(h, 0, sizeof(*h));
}

int rtt_tile2csr(SMatrix *M, int tile_dim, int canonical)
{
    return rtt_tile2csr_restore_rows(M, nullptr, -1, tile_dim, canonical);
}

void rtt_matrix_destroy(SMatrix *M, int owned_csr)
{
    if (M == nullptr)
        return;
    std::free(M->tile_ptr);
    std::free(M->tile_columnidx);
    std::free(M->tile_rowidx);
    std::free(M->tile_nnz);
    std::free(M->tile_csr_Value);
    std::free(M->tile_csr_Col);
    std::free(M->tile_csr_Ptr);
    std::free(M->mask);
    std::free(M->csc_tile_ptr);
    std::free(M->csc_tile_rowidx);
    M->tile_ptr = M->tile_columnidx = M->tile_rowidx = M->tile_nnz = nullptr;
    M->csc_tile_ptr = M->csc_tile_rowidx = nullptr;
    M->tile_csr_Value = nullptr;
    M->tile_csr_Col = M->tile_csr_Ptr = nullptr;
    M->mask = nullptr;
    if (owned_csr)
    {
        std::free(M->rowpointer);
        std::free(M->columnindex);
        std::free(M->value);
        M->rowpointer = nullptr;
        M->columnindex = nullptr;
        M->value = nullptr;
    }
}

// ------------------------------------------------------------ device path
int rtt_spgemm_symbolic(rtt_context c, const rtt_csr_view *A, const rtt_csr_view *B, int op,
                        long long *nnz_c, long long *tiles_c)
{
    if (c == nullptr || A == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (op != RTT_OP_AB && op != RTT_OP_AAT)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "op must be RTT_OP_AB or RTT_OP_AAT");
    if (op == RTT_OP_AAT && B != nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "RTT_OP_AAT takes B == NULL");
    if (A->rows < 0 || A->cols < 0 || A->nnz < 0 || A->nnz > INT_MAX)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "bad A shape");
    RTT_CUDA(cudaSetDevice(c->ws.device));
    c->have_symbolic = false;
    c->have_sym64 = false;
    c->bat_active = false;
    c->cut_cached = -1;
    c->ws.launches = 0;
    c->ws.syncs = 0;
    std::memset(&c->stats, 0, sizeof(c->stats));
    Workspace &ws = c->ws;
    const bool timing = c->cfg.stage_timing != 0;
    if (timing)
        RTT_CUDA(cudaEventRecord(ws.ev[0], ws.stream));
    DevTiles dA, dB;
    RTT_CHECK(prepare_operands(c, A, B, op, dA, dB));
    const TileBufs &TB = c->b_alias ? c->A : c->B;
    if (timing)
        RTT_CUDA(cudaEventRecord(ws.ev[1], ws.stream));
    RTT_CHECK(map_device_error(symbolic_device(ws, dA, dB, c->S, !c->b_dups)));
    if (timing)
    {
        float t01 = 0.f, t12 = 0.f;
        RTT_CUDA(cudaEventRecord(ws.ev[2], ws.stream));
        RTT_CUDA(cudaEventSynchronize(ws.ev[2]));
        RTT_CUDA(cudaEventElapsedTime(&t01, ws.ev[0], ws.ev[1]));
        RTT_CUDA(cudaEventElapsedTime(&t12, ws.ev[1], ws.ev[2]));
        c->stats.csr2tile_ms = t01;
        c->stats.symbolic_ms = t12;
    }
    c->stats.nnz_a = c->A.nnz;
    c->stats.nnz_b = TB.nnz;
    c->stats.nnz_c = c->S.nnz;
    c->stats.tiles_a = c->A.numtile;
    c->stats.tiles_b = TB.numtile;
    c->stats.tiles_c = c->S.numtile;
    c->stats.host_syncs = ws.syncs;
    if (nnz_c)
        *nnz_c = c->S.nnz;
    if (tiles_c)
        *tiles_c = c->S.numtile;
    c->have_symbolic = true;
    return RTT_OK;
}

int rtt_spgemm_update_b(rtt_context c, const rtt_csr_view *B, const int *row_new_to_old,
                        long long *nnz_c, long long *tiles_c)
{
    if (c == nullptr || B == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "update_b: NULL argument");
    if (!c->have_symbolic || c->bat_active || c->op_aat)
        return rtt::fail(RTT_ERR_STATE,
                         "rtt_spgemm_update_b needs a C = A*B (or A*A) symbolic phase first");
    if (B->rows < 0 || B->cols < 0 || B->nnz < 0 || B->nnz > INT_MAX)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "bad B shape");
    if (B->rows != c->A.n)
        return rtt::fail(RTT_ERR_SHAPE_MISMATCH, "update_b: B->rows != A->cols");
    RTT_CUDA(cudaSetDevice(c->ws.device));
    Workspace &ws = c->ws;
    cudaStream_t s = ws.stream;
    c->have_symbolic = false;
    c->cut_cached = -1;
    ws.launches = 0;
    ws.syncs = 0;
    rtt_csr_view b = *B;
    if (row_new_to_old != nullptr)
    {
        // permutation mode: B's rows in the given order (the map is checked
        // to be a permutation on the device), columns as they are
        RTT_CHECK(c->bp_rowptr.ensure(sizeof(int) * ((size_t)B->rows + 1), s));
        RTT_CHECK(c->bp_col.ensure(sizeof(int) * (size_t)B->nnz + 16, s));
        RTT_CHECK(c->bp_val.ensure(sizeof(double) * (size_t)B->nnz + 16, s));
        RTT_CHECK(csr_permute_device(ws, *B, row_new_to_old, nullptr, c->bp_rowptr.as<int>(),
                                     c->bp_col.as<int>(), c->bp_val.as<double>()));
        b.row_ptr = c->bp_rowptr.as<int>();
        b.col_idx = c->bp_col.as<int>();
        b.values = c->bp_val.as<double>();
    }
    // A's tiles and CSR stay as the last symbolic phase left them; B is tiled anew
    const bool payload = c->cfg.dmma_pair_cutoff > 0 || c->cfg.b_staging != 0;
    RTT_CHECK(map_device_error(csr2tile_device(ws, b.rows, b.cols, (int)b.nnz, b.row_ptr,
                                               b.col_idx, b.values, c->B, true, false, true,
                                               payload && c->A.payload)));
    c->b_alias = false;
    c->b_rp = b.row_ptr;
    c->b_ci = b.col_idx;
    c->b_va = b.values;
    c->b_nnz = b.nnz;
    c->b_dups = c->B.dup_cols;
    DevTiles dB = c->B.view();
    dB.csr_rowptr = c->b_rp;
    dB.csr_col = c->b_ci;
    dB.csr_val = c->b_va;
    dB.nnz = (int)c->b_nnz;
    DevTiles dA = c->A.view();
    dA.csr_rowptr = c->a_rp;
    dA.csr_col = c->a_ci;
    RTT_CHECK(map_device_error(symbolic_device(ws, dA, dB, c->S, !c->b_dups)));
    c->stats.nnz_b = c->B.nnz;
    c->stats.nnz_c = c->S.nnz;
    c->stats.tiles_b = c->B.numtile;
    c->stats.tiles_c = c->S.numtile;
    c->stats.host_syncs = ws.syncs;
    if (nnz_c)
        *nnz_c = c->S.nnz;
    if (tiles_c)
        *tiles_c = c->S.numtile;
    c->have_symbolic = true;
    return RTT_OK;
}

int rtt_tile_heatmap(rtt_context c, int which, int bins, unsigned long long *hist)
{
    if (c == nullptr || hist == nullptr || bins < 1 || bins > 4096 || which < 0 || which > 2)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "tile_heatmap: bad arguments");
    if (!c->have_symbolic && !c->have_sym64)
        return rtt::fail(RTT_ERR_STATE, "tile_heatmap needs a symbolic phase first");
    RTT_CUDA(cudaSetDevice(c->ws.device));
    Workspace &ws = c->ws;
    const TileBufs &TB = c->b_alias ? c->A : c->B;
    int tilem = 0, tilen = 0;
    const int *tp = nullptr, *tc = nullptr;
    if (which == 2)
    {
        tilem = c->S.tilem;
        tilen = c->S.tilen;
        tp = c->S.c_tile_ptr.as<int>();
        tc = c->S.c_tile_col.as<int>();
    }
    else
    {
        const TileBufs &T = which == 0 ? c->A : TB;
        tilem = T.tilem;
        tilen = T.tilen;
        tp = T.tile_ptr.as<int>();
        tc = T.tile_col.as<int>();
    }
    const size_t cells = (size_t)bins * bins;
    RTT_CHECK(c->diag_hist.ensure(sizeof(unsigned long long) * cells, ws.stream));
    RTT_CHECK(tile_heatmap_device(ws, tilem, tilen, tp, tc, bins,
                                  c->diag_hist.as<unsigned long long>()));
    RTT_CUDA(cudaMemcpyAsync(hist, c->diag_hist.p, sizeof(unsigned long long) * cells,
                             cudaMemcpyDeviceToHost, ws.stream));
    return check_device_error(ws, "tile_heatmap");
}

int rtt_spgemm_numeric_values(rtt_context c, const double *a_values, const double *b_values,
                              int *c_row_ptr, int *c_col_idx, double *c_values)
{
    if (c == nullptr || a_values == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "numeric_values: NULL argument");
    if (!c->have_symbolic || c->bat_active)
        return rtt::fail(RTT_ERR_STATE, "rtt_spgemm_numeric_values before rtt_spgemm_symbolic");
    RTT_CHECK(numeric_args_ok(c, c_row_ptr, c_col_idx, c_values));
    RTT_CUDA(cudaSetDevice(c->ws.device));
    Workspace &ws = c->ws;
    // The kernels below index by the structure arrays given to symbolic,
    // which the caller keeps unchanged: check once more on the device that
    // they still form valid CSRs before anything indexes by them (one sync).
    // The fast csr2tile fill also needs tile columns that never decrease in
    // a row, as at the first build.
    RTT_CHECK(c->vflags.ensure(sizeof(int) * 4, ws.stream));
    const char *changed = "values-only update: the CSR structure changed since symbolic";
    RTT_CHECK(map_device_error(validate_csr_device(ws, c->A.m, c->A.n, c->A.nnz, c->a_rp,
                                                   c->a_ci, c->vflags.as<int>())));
    if (!c->A.generic && ws.h_scalars[4] != 0)
        return rtt::fail(RTT_ERR_INVALID_CSR, changed);
    if (!c->b_alias && !c->op_aat)
    {
        RTT_CHECK(map_device_error(validate_csr_device(ws, c->B.m, c->B.n, c->B.nnz, c->b_rp,
                                                       c->b_ci, c->vflags.as<int>())));
        if (!c->B.generic && ws.h_scalars[4] != 0)
            return rtt::fail(RTT_ERR_INVALID_CSR, changed);
    }
    // B's values for the numeric step: A's (A*A), A^T's (rebuilt below) or new
    c->a_va = a_values;
    if (c->b_alias)
        c->b_va = a_values;
    else if (c->op_aat)
        c->b_va = c->bt_val.as<double>();
    else if (b_values != nullptr)
        c->b_va = b_values;
    int cutoff = 0;
    const TileBufs &TB = c->b_alias ? c->A : c->B;
    RTT_CHECK(effective_cutoff(c, c->A.view(), TB.view(), &cutoff));
    std::vector<long long> key{1, as_key(a_values), as_key(b_values), as_key(c_row_ptr),
                               as_key(c_col_idx), as_key(c_values)};
    RTT_CHECK(run_phase(c, 1, key, graphs_allowed(c), [&]() -> int {
        // A's tiles take the new values (same structure, same tile order);
        // without tile arrays the numeric step reads the new values directly
        if (c->A.payload)
            RTT_CHECK(map_device_error(
                csr2tile_refill_device(ws, c->a_rp, c->a_ci, a_values, c->A, true)));
        if (!c->b_alias && c->op_aat)
        {
            // B = A^T again, values only (its structure is unchanged)
            RTT_CHECK(csr_transpose_device(ws, c->A.m, c->A.n, c->A.nnz, c->a_rp, c->a_ci,
                                           a_values, c->bt_rowptr.as<int>(), c->bt_col.as<int>(),
                                           c->bt_val.as<double>()));
            if (c->B.payload)
                RTT_CHECK(map_device_error(csr2tile_refill_device(
                    ws, c->bt_rowptr.as<int>(), c->bt_col.as<int>(), c->bt_val.as<double>(),
                    c->B, true)));
        }
        else if (!c->b_alias && b_values != nullptr && c->B.payload)
            RTT_CHECK(map_device_error(
                csr2tile_refill_device(ws, c->b_rp, c->b_ci, b_values, c->B, true)));
        return numeric_enqueue(c, c_row_ptr, c_col_idx, c_values, cutoff);
    }));
    return numeric_finish(c);
}

int rtt_spgemm_numeric(rtt_context c, int *c_row_ptr, int *c_col_idx, double *c_values)
{
    if (c == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (!c->have_symbolic)
        return rtt::fail(RTT_ERR_STATE, "rtt_spgemm_numeric before rtt_spgemm_symbolic");
    RTT_CHECK(numeric_args_ok(c, c_row_ptr, c_col_idx, c_values));
    RTT_CUDA(cudaSetDevice(c->ws.device));
    int cutoff = 0;
    const TileBufs &TB = c->b_alias ? c->A : c->B;
    RTT_CHECK(effective_cutoff(c, c->A.view(), TB.view(), &cutoff));
    std::vector<long long> key{0, as_key(c_row_ptr), as_key(c_col_idx), as_key(c_values)};
    RTT_CHECK(run_phase(c, 0, key, graphs_allowed(c), [&]() -> int {
        return numeric_enqueue(c, c_row_ptr, c_col_idx, c_values, cutoff);
    }));
    return numeric_finish(c);
}

// ------------------------------------------------------------ 64-bit products
// C with more than INT32_MAX entries (R-MAT 2^20 A*A^T: about 9.4e9).  The
// C tile structure of such a product does not fit beside C, so both phases
// run over chunks of A's tile rows (tile_row_slice): the symbolic phase runs
// steps 1-2 per chunk and keeps only the per-row counts of C (their int64
// scan is C's row pointer); the numeric phase runs steps 1-2 of a chunk again
// and its numeric step straight into the chunk's part of C's CSR, through a
// chunk-local int32 row pointer.  Chunks hold at most chunk_tiles C tiles
// (planned from step 1 over all tile rows) and fewer than chunk_nnz entries
// (a chunk past it is halved).
namespace
{
constexpr long long WIDE_CHUNK_TILES = 1ll << 25;

__global__ void k_rowptr_copy(long long n, const long long *__restrict__ src,
                              long long *__restrict__ dst)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[i];
}
} // namespace

int rtt_spgemm_symbolic64(rtt_context c, const rtt_csr_view *A, const rtt_csr_view *B, int op,
                          long long *nnz_c)
{
    if (c == nullptr || A == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (op != RTT_OP_AB && op != RTT_OP_AAT)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "op must be RTT_OP_AB or RTT_OP_AAT");
    if (op == RTT_OP_AAT && B != nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "RTT_OP_AAT takes B == NULL");
    if (A->rows < 0 || A->cols < 0 || A->nnz < 0 || A->nnz > INT_MAX)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "bad A shape");
    RTT_CUDA(cudaSetDevice(c->ws.device));
    c->have_symbolic = false;
    c->have_sym64 = false;
    c->bat_active = false;
    c->cut_cached = -1;
    c->ws.launches = 0;
    c->ws.syncs = 0;
    std::memset(&c->stats, 0, sizeof(c->stats));
    Workspace &ws = c->ws;
    cudaStream_t s = ws.stream;
    DevTiles dA, dB;
    RTT_CHECK(prepare_operands(c, A, B, op, dA, dB));
    const int tilem = dA.tilem, m = dA.m;
    // step 1 over every tile row: C tiles per tile row, to plan the chunks
    std::vector<int> tcnt((size_t)tilem);
    if (tilem > 0)
    {
        RTT_CHECK(c->w_cnt.ensure(sizeof(int) * (size_t)tilem, s));
        RTT_CHECK(symbolic_tile_counts(ws, dA, dB, c->S, c->w_cnt.as<int>()));
        RTT_CUDA(cudaMemcpyAsync(tcnt.data(), c->w_cnt.p, sizeof(int) * (size_t)tilem,
                                 cudaMemcpyDeviceToHost, s));
        RTT_CHECK(check_device_error(ws, "symbolic64 step 1"));
    }
    const long long budget = c->cfg.chunk_tiles > 0 ? c->cfg.chunk_tiles : WIDE_CHUNK_TILES;
    const long long cap = c->cfg.chunk_nnz > 0 ? c->cfg.chunk_nnz : (long long)INT_MAX;
    std::vector<int> bounds{0};
    long long run = 0;
    for (int I = 0; I < tilem; ++I)
    {
        if (run + tcnt[I] > budget && I > bounds.back())
        {
            bounds.push_back(I);
            run = 0;
        }
        run += tcnt[I];
    }
    if (tilem > 0)
        bounds.push_back(tilem);
    // steps 1-2 per chunk: the per-row counts of C
    RTT_CHECK(c->w_rowcnt.ensure(sizeof(int) * ((size_t)m + 1), s));
    RTT_CHECK(c->w_rowptr.ensure(sizeof(long long) * ((size_t)m + 1), s));
    std::vector<int> done{0};
    std::vector<long long> base{0};
    long long tiles = 0;
    for (size_t k = 0; k + 1 < bounds.size();)
    {
        const int I0 = bounds[k], I1 = bounds[k + 1];
        const DevTiles sA = tile_row_slice(dA, I0, I1);
        int st = map_device_error(symbolic_device(ws, sA, dB, c->S, !c->b_dups));
        if ((st == RTT_ERR_UNREPRESENTABLE || (st == RTT_OK && c->S.nnz > cap)) && I1 - I0 > 1)
        {
            bounds.insert(bounds.begin() + (long)k + 1, I0 + (I1 - I0) / 2); // halve it
            continue;
        }
        if (st == RTT_OK && c->S.nnz > cap)
            return rtt::fail(RTT_ERR_UNREPRESENTABLE,
                             "one tile row of C holds more entries than a chunk may");
        RTT_CHECK(st);
        RTT_CUDA(cudaMemcpyAsync(c->w_rowcnt.as<int>() + (size_t)I0 * TD, c->S.c_row_cnt.p,
                                 sizeof(int) * (size_t)sA.m, cudaMemcpyDeviceToDevice, s));
        done.push_back(I1);
        base.push_back(base.back() + c->S.nnz);
        tiles += c->S.numtile;
        ++k;
    }
    RTT_CHECK(scan_exclusive_i64(ws, c->w_rowcnt.as<int>(), c->w_rowptr.as<long long>(), m));
    long long nnz = 0;
    RTT_CHECK(read_i64_checked(ws, c->w_rowptr.as<long long>() + m, &nnz, "symbolic64"));
    if (nnz != base.back())
        return rtt::fail(RTT_ERR_DEVICE_CHECK, "symbolic64: chunk totals disagree with the rows");
    c->w_bounds = done;
    c->w_base = base;
    c->w_dA = dA;
    c->w_dB = dB;
    c->w_nnz = nnz;
    const TileBufs &TB = c->b_alias ? c->A : c->B;
    c->stats.nnz_a = c->A.nnz;
    c->stats.nnz_b = TB.nnz;
    c->stats.nnz_c = nnz;
    c->stats.tiles_a = c->A.numtile;
    c->stats.tiles_b = TB.numtile;
    c->stats.tiles_c = tiles;
    c->stats.host_syncs = ws.syncs;
    c->have_sym64 = true;
    if (nnz_c)
        *nnz_c = nnz;
    return RTT_OK;
}

int rtt_spgemm_numeric64(rtt_context c, long long *c_row_ptr, int *c_col_idx, double *c_values)
{
    if (c == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (!c->have_sym64)
        return rtt::fail(RTT_ERR_STATE, "rtt_spgemm_numeric64 before rtt_spgemm_symbolic64");
    if (c_row_ptr == nullptr || (c->w_nnz > 0 && (c_col_idx == nullptr || c_values == nullptr)))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "NULL output buffer");
    RTT_CUDA(cudaSetDevice(c->ws.device));
    Workspace &ws = c->ws;
    cudaStream_t s = ws.stream;
    ws.launches = 0;
    const DevTiles &dA = c->w_dA, &dB = c->w_dB;
    const long long m = dA.m;
    k_rowptr_copy<<<std::max(1, (int)std::min<long long>((m + 256) / 256, 4096)), 256, 0, s>>>(
        m + 1, c->w_rowptr.as<long long>(), c_row_ptr);
    ws.launches++;
    RTT_CHECK(c->counters.ensure(sizeof(long long) * 4, s));
    RTT_CUDA(cudaMemsetAsync(c->counters.p, 0, sizeof(long long) * 4, s));
    for (size_t k = 0; k + 1 < c->w_bounds.size(); ++k)
    {
        const int I0 = c->w_bounds[k], I1 = c->w_bounds[k + 1];
        DevTiles sA = tile_row_slice(dA, I0, I1);
        RTT_CHECK(map_device_error(symbolic_device(ws, sA, dB, c->S, !c->b_dups)));
        if (c->S.nnz != c->w_base[k + 1] - c->w_base[k])
            return rtt::fail(RTT_ERR_DEVICE_CHECK, "numeric64: a chunk's size changed");
        RTT_CHECK(c->w_local.ensure(sizeof(int) * ((size_t)sA.m + 1), s));
        NumericConfig nc;
        nc.counters = c->counters.as<long long>();
        nc.split_target = c->cfg.split_target;
        nc.write_tiles = false;
        nc.conflict_safe = c->b_dups;
        nc.segment_walk = c->cfg.segment_walk != 0;
        nc.persistent_rows = c->cfg.persistent_rows != 0;
    nc.global_rows = c->cfg.global_rows;
        nc.csr_rowptr = c->w_local.as<int>();
        nc.csr_col = c_col_idx + c->w_base[k];
        nc.csr_val = c_values + c->w_base[k];
        sA.csr_val = c->a_va;
        RTT_CHECK(numeric_flat_device(ws, sA, dB, c->S, nc));
    }
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars64 + 2, c->counters.p, sizeof(long long) * 4,
                             cudaMemcpyDeviceToHost, s));
    RTT_CHECK(check_device_error(ws, "numeric64"));
    c->stats.sparse_pairs = ws.h_scalars64[3];
    c->stats.nnz_cub = ws.h_scalars64[3];
    c->stats.split_windows = ws.h_scalars64[4];
    c->stats.split_multi_window_tasks = ws.h_scalars64[5];
    c->stats.kernel_launches = ws.launches;
    c->stats.host_syncs = ws.syncs;
    return RTT_OK;
}

// ------------------------------------------------------------ batched products
namespace
{
inline long long pad16(long long v) { return (v + 15) / 16 * 16; }

bool view_ok(const rtt_csr_view &v)
{
    return v.rows >= 0 && v.cols >= 0 && v.nnz >= 0 && v.nnz <= INT_MAX &&
           v.row_ptr != nullptr && (v.nnz == 0 || (v.col_idx != nullptr && v.values != nullptr));
}

// Block-diagonal assembly of count instances into (rp, col, val): instance i's
// rows start at row_off[i] (multiples of 16), its columns are shifted by
// col_add[i].  meta_base points at count * 3 pointer slots + int arrays.
int assemble(rtt_context c, int count, const rtt_csr_view *V, const std::vector<int> &row_off,
             const std::vector<int> &col_add, DevBuf &rp, DevBuf &col, DevBuf &val,
             std::vector<int> &nnz_off_out, int &max_nnz)
{
    Workspace &ws = c->ws;
    cudaStream_t s = ws.stream;
    const int total_rows = row_off[(size_t)count];
    std::vector<int> rows((size_t)count), cols((size_t)count), nnz_off((size_t)count + 1, 0);
    std::vector<const void *> tab((size_t)count * 3);
    for (int i = 0; i < count; ++i)
    {
        rows[(size_t)i] = V[i].rows;
        cols[(size_t)i] = V[i].cols;
        nnz_off[(size_t)i + 1] = nnz_off[(size_t)i] + (int)V[i].nnz;
        tab[(size_t)i] = V[i].row_ptr;
        tab[(size_t)count + i] = V[i].col_idx;
        tab[(size_t)2 * count + i] = V[i].values;
    }
    const int nnz = nnz_off[(size_t)count];
    max_nnz = 0;
    for (int i = 0; i < count; ++i)
        max_nnz = std::max(max_nnz, (int)V[i].nnz);
    nnz_off_out = nnz_off;
    // device copy of the tables: pointers first (8-byte aligned), then ints
    // (grow-only scratch: no cudaFree, which would wait for every stream)
    DevBuf &tabd = ws.tmp[0];
    // rows, row_off (count + 1), col_add, nnz_off (count + 1), cols
    const size_t ints = (size_t)count * 5 + 2;
    RTT_CHECK(tabd.ensure(sizeof(void *) * tab.size() + sizeof(int) * ints, s));
    char *base = tabd.as<char>();
    int *d_rows = reinterpret_cast<int *>(base + sizeof(void *) * tab.size());
    int *d_rowoff = d_rows + count, *d_coladd = d_rowoff + count + 1, *d_nnzoff = d_coladd + count;
    int *d_cols = d_nnzoff + count + 1;
    std::vector<int> packed;
    packed.insert(packed.end(), rows.begin(), rows.end());
    packed.insert(packed.end(), row_off.begin(), row_off.end());
    packed.insert(packed.end(), col_add.begin(), col_add.begin() + count);
    packed.insert(packed.end(), nnz_off.begin(), nnz_off.end());
    packed.insert(packed.end(), cols.begin(), cols.end());
    RTT_CUDA(cudaMemcpyAsync(base, tab.data(), sizeof(void *) * tab.size(), cudaMemcpyHostToDevice, s));
    RTT_CUDA(cudaMemcpyAsync(d_rows, packed.data(), sizeof(int) * packed.size(), cudaMemcpyHostToDevice, s));
    RTT_CHECK(rp.ensure(sizeof(int) * ((size_t)total_rows + 1), s));
    RTT_CHECK(col.ensure(sizeof(int) * (size_t)nnz + 16, s));
    RTT_CHECK(val.ensure(sizeof(double) * (size_t)nnz + 16, s));
    const void *const *tp = reinterpret_cast<const void *const *>(base);
    RTT_CHECK(batch_assemble_device(ws, count, total_rows, reinterpret_cast<const int *const *>(tp),
                                    reinterpret_cast<const int *const *>(tp + count),
                                    reinterpret_cast<const double *const *>(tp + 2 * count),
                                    d_rows, d_cols, d_rowoff, d_coladd, d_nnzoff, rp.as<int>(),
                                    col.as<int>(), val.as<double>()));
    return RTT_OK;
}
} // namespace

int rtt_spgemm_batched_symbolic(rtt_context c, int count, const rtt_csr_view *A,
                                const rtt_csr_view *B, long long *nnz_c, long long *nnz_total)
{
    if (c == nullptr || count < 1 || A == nullptr || nnz_c == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "batched: bad arguments");
    long long R = 0, K = 0, P = 0, annz = 0, bnnz = 0, sec = 0;
    std::vector<int> row_off((size_t)count + 1), col_off((size_t)count + 1),
        pcol_off((size_t)count + 1), sec_off((size_t)count), rows((size_t)count);
    for (int i = 0; i < count; ++i)
    {
        if (!view_ok(A[i]) || (B != nullptr && !view_ok(B[i])))
            return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "batched: bad instance " + std::to_string(i));
        if (B == nullptr ? A[i].rows != A[i].cols : B[i].rows != A[i].cols)
            return rtt::fail(RTT_ERR_SHAPE_MISMATCH, "batched: instance " + std::to_string(i) +
                                                         " has mismatched shapes");
        row_off[(size_t)i] = (int)R;
        col_off[(size_t)i] = (int)K;
        pcol_off[(size_t)i] = (int)P;
        sec_off[(size_t)i] = (int)sec;
        rows[(size_t)i] = A[i].rows;
        R += pad16(A[i].rows);
        K += pad16(A[i].cols);
        P += pad16(B ? B[i].cols : A[i].cols);
        annz += A[i].nnz;
        bnnz += B ? B[i].nnz : 0;
        sec += A[i].rows + 1;
        if (R > INT_MAX / 2 || K > INT_MAX / 2 || P > INT_MAX / 2 || annz > INT_MAX ||
            bnnz > INT_MAX || sec > INT_MAX)
            return rtt::fail(RTT_ERR_UNREPRESENTABLE, "batched: batch exceeds int32 sizes");
    }
    row_off[(size_t)count] = (int)R;
    col_off[(size_t)count] = (int)K;
    pcol_off[(size_t)count] = (int)P;
    RTT_CUDA(cudaSetDevice(c->ws.device));
    Workspace &ws = c->ws;
    cudaStream_t s = ws.stream;
    // A's block diagonal (rows at row_off, columns shifted to col_off)
    RTT_CHECK(assemble(c, count, A, row_off, col_off, c->bat_a_rp, c->bat_a_col, c->bat_a_val,
                       c->bat_a_off, c->bat_a_max));
    rtt_csr_view va{(int)R, (int)K, annz, c->bat_a_rp.as<int>(), c->bat_a_col.as<int>(),
                    c->bat_a_val.as<double>()};
    rtt_csr_view vb{};
    if (B != nullptr)
    {
        RTT_CHECK(assemble(c, count, B, col_off, pcol_off, c->bat_b_rp, c->bat_b_col,
                           c->bat_b_val, c->bat_b_off, c->bat_b_max));
        vb = rtt_csr_view{(int)K, (int)P, bnnz, c->bat_b_rp.as<int>(), c->bat_b_col.as<int>(),
                          c->bat_b_val.as<double>()};
    }
    long long nnz = 0, tiles = 0;
    RTT_CHECK(rtt_spgemm_symbolic(c, &va, B ? &vb : nullptr, RTT_OP_AB, &nnz, &tiles));
    // per-instance bookkeeping on the device: rows, row offsets, sections, column shifts
    const size_t meta = (size_t)count * 4 + 1;
    RTT_CHECK(c->bat_meta.ensure(sizeof(int) * meta, s));
    std::vector<int> packed;
    packed.insert(packed.end(), rows.begin(), rows.end());
    packed.insert(packed.end(), row_off.begin(), row_off.end());
    packed.insert(packed.end(), sec_off.begin(), sec_off.end());
    packed.insert(packed.end(), pcol_off.begin(), pcol_off.begin() + count);
    RTT_CUDA(cudaMemcpyAsync(c->bat_meta.p, packed.data(), sizeof(int) * packed.size(),
                             cudaMemcpyHostToDevice, s));
    c->bat_rows_off = 0;
    c->bat_rowoff_off = (size_t)count;
    c->bat_sec_off = (size_t)count * 2 + 1;
    c->bat_colsub_off = (size_t)count * 3 + 1;
    RTT_CHECK(c->bat_nnz.ensure(sizeof(long long) * (size_t)count, s));
    const int *meta_d = c->bat_meta.as<int>();
    RTT_CHECK(batch_count_device(ws, count, meta_d + c->bat_rowoff_off, meta_d + c->bat_rows_off,
                                 c->S.c_row_cnt.as<int>(), c->bat_nnz.as<long long>()));
    RTT_CUDA(cudaMemcpyAsync(nnz_c, c->bat_nnz.p, sizeof(long long) * (size_t)count,
                             cudaMemcpyDeviceToHost, s));
    RTT_CUDA(cudaStreamSynchronize(s));
    if (nnz_total)
        *nnz_total = nnz;
    c->bat_active = true;
    c->bat_count = count;
    c->bat_rows = (int)R;
    if (B == nullptr)
        c->bat_b_off.clear();
    return RTT_OK;
}

int rtt_spgemm_batched_numeric(rtt_context c, int *c_row_ptr, int *c_col_idx, double *c_values)
{
    if (c == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (!c->bat_active || !c->have_symbolic)
        return rtt::fail(RTT_ERR_STATE, "rtt_spgemm_batched_numeric before rtt_spgemm_batched_symbolic");
    if (c_row_ptr == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "NULL output buffer");
    RTT_CHECK(numeric_args_ok(c, c_row_ptr, c_col_idx, c_values));
    RTT_CUDA(cudaSetDevice(c->ws.device));
    cudaStream_t s = c->ws.stream;
    RTT_CHECK(c->bat_big_rp.ensure(sizeof(int) * ((size_t)c->bat_rows + 1), s));
    int cutoff = 0;
    const TileBufs &TB = c->b_alias ? c->A : c->B;
    RTT_CHECK(effective_cutoff(c, c->A.view(), TB.view(), &cutoff));
    std::vector<long long> key{2,
                               as_key(c_row_ptr),
                               as_key(c_col_idx),
                               as_key(c_values),
                               (long long)c->bat_rows_off,
                               (long long)c->bat_rowoff_off,
                               (long long)c->bat_sec_off,
                               (long long)c->bat_colsub_off};
    RTT_CHECK(run_phase(c, 2, key, graphs_allowed(c), [&]() -> int {
        RTT_CHECK(numeric_enqueue(c, c->bat_big_rp.as<int>(), c_col_idx, c_values, cutoff));
        const int *meta_d = c->bat_meta.as<int>();
        return batch_split_device(c->ws, c->bat_count, c->bat_rows, meta_d + c->bat_rowoff_off,
                                  meta_d + c->bat_rows_off, meta_d + c->bat_sec_off,
                                  meta_d + c->bat_colsub_off, c->bat_big_rp.as<int>(),
                                  c_row_ptr, c_col_idx);
    }));
    return numeric_finish(c);
}

int rtt_spgemm_batched_numeric_values(rtt_context c, const double *const *a_values,
                                      const double *const *b_values, int *c_row_ptr,
                                      int *c_col_idx, double *c_values)
{
    if (c == nullptr || a_values == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "batched values: NULL argument");
    if (!c->bat_active || !c->have_symbolic)
        return rtt::fail(RTT_ERR_STATE,
                         "rtt_spgemm_batched_numeric_values before rtt_spgemm_batched_symbolic");
    const int n = c->bat_count;
    const bool with_b = b_values != nullptr;
    if (with_b && c->bat_b_off.empty())
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "batched values: the batch has no B");
    for (int i = 0; i < n; ++i)
        if ((a_values[i] == nullptr && c->bat_a_off[(size_t)i + 1] > c->bat_a_off[(size_t)i]) ||
            (with_b && b_values[i] == nullptr &&
             c->bat_b_off[(size_t)i + 1] > c->bat_b_off[(size_t)i]))
            return rtt::fail(RTT_ERR_INVALID_ARGUMENT,
                             "batched values: NULL values of instance " + std::to_string(i));
    RTT_CHECK(numeric_args_ok(c, c_row_ptr, c_col_idx, c_values));
    RTT_CUDA(cudaSetDevice(c->ws.device));
    Workspace &ws = c->ws;
    cudaStream_t s = ws.stream;
    // device table: A's value pointers [, B's], then A's entry offsets [, B's];
    // written before the (possibly captured) device work that reads it
    const int parts = with_b ? 2 : 1;
    const size_t ptr_bytes = sizeof(void *) * (size_t)n * parts;
    const size_t bytes = ptr_bytes + sizeof(int) * ((size_t)n + 1) * parts;
    std::vector<char> host(bytes);
    std::memcpy(host.data(), a_values, sizeof(void *) * (size_t)n);
    if (with_b)
        std::memcpy(host.data() + sizeof(void *) * n, b_values, sizeof(void *) * (size_t)n);
    std::memcpy(host.data() + ptr_bytes, c->bat_a_off.data(), sizeof(int) * ((size_t)n + 1));
    if (with_b)
        std::memcpy(host.data() + ptr_bytes + sizeof(int) * ((size_t)n + 1), c->bat_b_off.data(),
                    sizeof(int) * ((size_t)n + 1));
    RTT_CHECK(c->bat_vtab.ensure(bytes, s));
    RTT_CHECK(c->bat_big_rp.ensure(sizeof(int) * ((size_t)c->bat_rows + 1), s));
    RTT_CUDA(cudaMemcpyAsync(c->bat_vtab.p, host.data(), bytes, cudaMemcpyHostToDevice, s));
    const char *dt = c->bat_vtab.as<char>();
    const double *const *a_tab = reinterpret_cast<const double *const *>(dt);
    const double *const *b_tab = a_tab + n;
    const int *a_off = reinterpret_cast<const int *>(dt + ptr_bytes);
    const int *b_off = a_off + n + 1;
    int cutoff = 0;
    const TileBufs &TB = c->b_alias ? c->A : c->B;
    RTT_CHECK(effective_cutoff(c, c->A.view(), TB.view(), &cutoff));
    std::vector<long long> key{3, as_key(c_row_ptr), as_key(c_col_idx), as_key(c_values),
                               (long long)with_b};
    RTT_CHECK(run_phase(c, 3, key, graphs_allowed(c), [&]() -> int {
        // the instances' values into the block diagonal, then its tiles
        RTT_CHECK(batch_values_device(ws, n, c->bat_a_max, a_tab, a_off,
                                      c->bat_a_val.as<double>()));
        if (c->A.payload)
            RTT_CHECK(map_device_error(csr2tile_refill_device(
                ws, c->a_rp, c->a_ci, c->bat_a_val.as<double>(), c->A, true)));
        if (with_b && !c->b_alias)
        {
            RTT_CHECK(batch_values_device(ws, n, c->bat_b_max, b_tab, b_off,
                                          c->bat_b_val.as<double>()));
            if (c->B.payload)
                RTT_CHECK(map_device_error(csr2tile_refill_device(
                    ws, c->b_rp, c->b_ci, c->bat_b_val.as<double>(), c->B, true)));
        }
        RTT_CHECK(numeric_enqueue(c, c->bat_big_rp.as<int>(), c_col_idx, c_values, cutoff));
        const int *meta_d = c->bat_meta.as<int>();
        return batch_split_device(ws, n, c->bat_rows, meta_d + c->bat_rowoff_off,
                                  meta_d + c->bat_rows_off, meta_d + c->bat_sec_off,
                                  meta_d + c->bat_colsub_off, c->bat_big_rp.as<int>(), c_row_ptr,
                                  c_col_idx);
    }));
    return numeric_finish(c);
}

int rtt_reorder_plan_build(rtt_context c, const rtt_csr_view *A, rtt_reorder_plan *plan)
{
    return rtt_reorder_plan_build_variant(c, A, RTT_REORDER_FULL, plan);
}

int rtt_reorder_plan_build_variant(rtt_context c, const rtt_csr_view *A, int variant,
                                   rtt_reorder_plan *plan)
{
    if (c == nullptr || A == nullptr || plan == nullptr || !view_ok(*A))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "reorder_plan_build: bad arguments");
    if (variant < RTT_REORDER_FULL || variant > RTT_REORDER_UNGUARDED)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "reorder_plan_build: unknown variant");
    RTT_CUDA(cudaSetDevice(c->ws.device));
    // the traversal trusts A's structure: validate it like csr2tile does
    RTT_CHECK(map_device_error(csr2tile_device(c->ws, A->rows, A->cols, (int)A->nnz, A->row_ptr,
                                               A->col_idx, A->values, c->A, true, false)));
    c->have_symbolic = false; // the context's A tiles were reused as scratch
    return rtt::reorder_plan_device(c->ws, *A, variant, plan);
}

void rtt_reorder_plan_destroy(rtt_reorder_plan *plan)
{
    if (plan == nullptr)
        return;
    std::free(plan->row_old_to_new);
    std::free(plan->row_new_to_old);
    std::free(plan->inner_old_to_new);
    std::free(plan->inner_new_to_old);
    std::memset(plan, 0, sizeof(*plan));
}

int rtt_csr_permute(rtt_context c, const rtt_csr_view *A, const int *row_new_to_old,
                    const int *col_old_to_new, int *out_row_ptr, int *out_col_idx,
                    double *out_values)
{
    if (c == nullptr || A == nullptr || !view_ok(*A) || out_row_ptr == nullptr ||
        (A->nnz > 0 && (out_col_idx == nullptr || out_values == nullptr)))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "csr_permute: bad arguments");
    RTT_CUDA(cudaSetDevice(c->ws.device));
    RTT_CHECK(rtt::csr_permute_device(c->ws, *A, row_new_to_old, col_old_to_new, out_row_ptr,
                                      out_col_idx, out_values));
    RTT_CUDA(cudaStreamSynchronize(c->ws.stream));
    return RTT_OK;
}

int rtt_csr_transpose(rtt_context c, const rtt_csr_view *A, int *t_row_ptr, int *t_col_idx,
                      double *t_values)
{
    if (c == nullptr || A == nullptr || !view_ok(*A) || t_row_ptr == nullptr ||
        (A->nnz > 0 && (t_col_idx == nullptr || t_values == nullptr)))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "csr_transpose: bad arguments");
    RTT_CUDA(cudaSetDevice(c->ws.device));
    Workspace &ws = c->ws;
    cudaStream_t s = ws.stream;
    // straight into the caller's arrays; the scratch is the context's own
    RTT_CHECK(csr_transpose_device(ws, A->rows, A->cols, (int)A->nnz, A->row_ptr, A->col_idx,
                                   A->values, t_row_ptr, t_col_idx, t_values));
    RTT_CUDA(cudaStreamSynchronize(s));
    return RTT_OK;
}

int rtt_spgemm_tiles_view(rtt_context c, SMatrix *out)
{
    if (c == nullptr || out == nullptr)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!c->have_symbolic || (c->cfg.fused_csr_output && !c->cfg.keep_tiles))
        return rtt::fail(RTT_ERR_STATE, "no C tiles kept (set keep_tiles or unfused output)");
    SymbolicOut &S = c->S;
    std::memset(out, 0, sizeof(*out));
    out->m = S.m;
    out->n = S.n;
    out->nnz = (int)S.nnz;
    out->tilem = S.tilem;
    out->tilen = S.tilen;
    out->numtile = S.numtile;
    out->tile_ptr = S.c_tile_ptr.as<int>();
    out->tile_columnidx = S.c_tile_col.as<int>();
    out->tile_rowidx = S.c_tile_row.as<int>();
    out->tile_nnz = S.c_tile_nnz.as<int>();
    out->tile_csr_Ptr = S.c_ptr.as<unsigned char>();
    out->tile_csr_Col = S.c_col.as<unsigned char>();
    out->tile_csr_Value = S.c_val.as<double>();
    out->mask = S.c_mask.as<unsigned short>();
    return RTT_OK;
}

namespace
{
// The host-buffer product up to C on the device (c->out_*): uploads, both
// phases; m, n and nnz of C come back.
int csr_host_product(rtt_context c, const SMatrix *A, const SMatrix *B, int op, int *m_out,
                     int *n_out, long long *nnz_out)
{
    RTT_CUDA(cudaSetDevice(c->ws.device));
    cudaStream_t s = c->ws.stream;
    RTT_CHECK(upload(c, c->in_rp, A->rowpointer, (size_t)A->m + 1, s));
    RTT_CHECK(upload(c, c->in_col, A->columnindex, (size_t)A->nnz, s));
    RTT_CHECK(upload(c, c->in_val, A->value, (size_t)A->nnz, s));
    rtt_csr_view va{A->m, A->n, A->nnz, c->in_rp.as<int>(), c->in_col.as<int>(),
                    c->in_val.as<double>()};
    rtt_csr_view vb{};
    if (B != nullptr)
    {
        RTT_CHECK(upload(c, c->in2_rp, B->rowpointer, (size_t)B->m + 1, s));
        RTT_CHECK(upload(c, c->in2_col, B->columnindex, (size_t)B->nnz, s));
        RTT_CHECK(upload(c, c->in2_val, B->value, (size_t)B->nnz, s));
        vb = rtt_csr_view{B->m, B->n, B->nnz, c->in2_rp.as<int>(), c->in2_col.as<int>(),
                          c->in2_val.as<double>()};
    }
    long long nnz = 0, tiles = 0;
    RTT_CHECK(rtt_spgemm_symbolic(c, &va, B ? &vb : nullptr, op, &nnz, &tiles));
    const int m = A->m;
    RTT_CHECK(c->out_rp.ensure(sizeof(int) * ((size_t)m + 1), s));
    RTT_CHECK(c->out_col.ensure(sizeof(int) * (size_t)nnz + 16, s));
    RTT_CHECK(c->out_val.ensure(sizeof(double) * (size_t)nnz + 16, s));
    RTT_CHECK(rtt_spgemm_numeric(c, c->out_rp.as<int>(), c->out_col.as<int>(),
                                 c->out_val.as<double>()));
    *m_out = m;
    *n_out = op == RTT_OP_AAT ? A->m : (B ? B->n : A->n);
    *nnz_out = nnz;
    return RTT_OK;
}
} // namespace

int rtt_spgemm_csr_host(rtt_context c, const SMatrix *A, const SMatrix *B, int op, SMatrix *C)
{
    if (c == nullptr || !csr_args_ok(A) || C == nullptr || (B != nullptr && !csr_args_ok(B)))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "spgemm_csr_host: bad arguments");
    int m = 0, n = 0;
    long long nnz = 0;
    RTT_CHECK(csr_host_product(c, A, B, op, &m, &n, &nnz));
    cudaStream_t s = c->ws.stream;
    HostArrays h;
    int **rp = h.slot<int>(), **ci = h.slot<int>();
    double **v = h.slot<double>();
    RTT_CHECK(download(c, rp, c->out_rp.p, (size_t)m + 1, s));
    RTT_CHECK(download(c, ci, c->out_col.p, (size_t)nnz, s));
    RTT_CHECK(download(c, v, c->out_val.p, (size_t)nnz, s));
    std::memset(C, 0, sizeof(*C));
    C->m = m;
    C->n = n;
    C->nnz = (int)nnz;
    C->rowpointer = *rp;
    C->columnindex = *ci;
    C->value = *v;
    h.committed = true;
    return RTT_OK;
}

int rtt_spgemm_csr_host_into(rtt_context c, const SMatrix *A, const SMatrix *B, int op,
                             int *c_row_ptr, int *c_col_idx, double *c_values,
                             long long capacity, long long *nnz_c)
{
    if (c == nullptr || !csr_args_ok(A) || (B != nullptr && !csr_args_ok(B)) ||
        c_row_ptr == nullptr || nnz_c == nullptr || capacity < 0 ||
        (capacity > 0 && (c_col_idx == nullptr || c_values == nullptr)))
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT, "spgemm_csr_host_into: bad arguments");
    int m = 0, n = 0;
    long long nnz = 0;
    RTT_CHECK(csr_host_product(c, A, B, op, &m, &n, &nnz));
    *nnz_c = nnz;
    if (nnz > capacity)
        return rtt::fail(RTT_ERR_INVALID_ARGUMENT,
                         "spgemm_csr_host_into: nnz(C) = " + std::to_string(nnz) +
                             " exceeds the capacity of the output arrays (nnz_c holds the size)");
    cudaStream_t s = c->ws.stream;
    RTT_CHECK(d2h(c, c_row_ptr, c->out_rp.p, sizeof(int) * ((size_t)m + 1), s));
    if (nnz > 0)
    {
        RTT_CHECK(d2h(c, c_col_idx, c->out_col.p, sizeof(int) * (size_t)nnz, s));
        RTT_CHECK(d2h(c, c_values, c->out_val.p, sizeof(double) * (size_t)nnz, s));
    }
    RTT_CUDA(cudaStreamSynchronize(s));
    return RTT_OK;
}

} // extern "C"
