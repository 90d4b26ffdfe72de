// hybrid.cu - CSR -> 32-element hybrid leaf tiles (8x4 A / 4x8 B) on sm_100a.
//
// Semantics of csr_to_hybrid_tiles (reference src/dmma_tiles.h:243-438, the
// container at :29-62): tiles of tile_rows x tile_cols (= 32) elements; the
// physical index of a local (r, c) is r * tile_cols + c (row-major payload,
// A) or c * tile_rows + r (column-major payload, B); repeated coordinates are
// summed; a tile whose distinct count reaches dense_threshold stores all 32
// values in physical order (zeros included), any other tile stores its values
// packed in increasing mask-bit order; value_offsets is the running payload
// size, so a tile is dense exactly when its span is 32.  The optional tile
// CSC lists, per tile column, the tile rows and tile-CSR ids in tile-row order.
//
// The reference walks tile rows on the host, sorting each row's entries.  Here
// every entry gets one 64-bit key (tile row, tile column, physical index),
// one device radix sort orders the whole matrix, and the tiles fall out of
// segment heads, scans and one scatter - all on the device.
#include "rtt_internal.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>

#include <climits>
#include <cstdlib>
#include <cstring>

namespace rtt
{
namespace
{

constexpr int ELEMS = 32;
constexpr int TC_BITS = 30; // tile column field width in the key
constexpr int PH_BITS = 5;  // physical index field width

__global__ void k_hyb_validate(int m, int n, int nnz, const int *__restrict__ rowptr,
                               const int *__restrict__ col, int *err)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && (rowptr[0] != 0 || rowptr[m] != nnz))
        set_error(err, DERR_CSR_ROWPTR);
    if (i < m && rowptr[i + 1] < rowptr[i])
        set_error(err, DERR_CSR_ROWPTR);
    if (i < nnz && (col[i] < 0 || col[i] >= n))
        set_error(err, DERR_CSR_COL);
}

// One warp per row: key of every entry (tile row | tile column | physical).
__global__ void k_hyb_keys(int m, const int *__restrict__ rowptr, const int *__restrict__ col,
                           int tr, int tc, int col_major, unsigned long long *__restrict__ keys)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= m)
        return;
    const int row = (int)w;
    const unsigned long long trow = (unsigned long long)(row / tr);
    const int lr = row % tr;
    for (int e = rowptr[row] + lane; e < rowptr[row + 1]; e += 32)
    {
        const int c = col[e];
        const int lc = c % tc;
        const int ph = col_major ? lc * tr + lr : lr * tc + lc;
        keys[e] = (trow << (TC_BITS + PH_BITS)) | ((unsigned long long)(c / tc) << PH_BITS) |
                  (unsigned long long)ph;
    }
}

// Heads of distinct coordinates (entry level) and of tiles (coordinate level).
__global__ void k_hyb_heads(int nnz, const unsigned long long *__restrict__ keys,
                            int *__restrict__ coord_head, int *__restrict__ tile_head)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnz)
        return;
    const unsigned long long k = keys[i];
    const bool newc = i == 0 || keys[i - 1] != k;
    coord_head[i] = newc ? 1 : 0;
    tile_head[i] = (newc && (i == 0 || (keys[i - 1] >> PH_BITS) != (k >> PH_BITS))) ? 1 : 0;
}

// Per distinct coordinate: its value (sum of its run, in sorted = CSR order),
// its tile's mask bit and count; per tile head: column, tile row, first
// coordinate.  coord_id / tile_id are inclusive scans of the heads.
__global__ void k_hyb_tiles(int nnz, const unsigned long long *__restrict__ keys,
                            const double *__restrict__ vals, const int *__restrict__ coord_head,
                            const int *__restrict__ coord_id, const int *__restrict__ tile_id,
                            double *__restrict__ cval, unsigned char *__restrict__ cphys,
                            int *__restrict__ ctile, unsigned int *__restrict__ mask,
                            int *__restrict__ tcount, int *__restrict__ tcol,
                            int *__restrict__ trow, int *__restrict__ tfirst)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnz || !coord_head[i])
        return;
    const unsigned long long k = keys[i];
    double s = vals[i];
    for (long long j = i + 1; j < nnz && keys[j] == k; ++j)
        s += vals[j];
    const int cid = coord_id[i] - 1, t = tile_id[i] - 1;
    const int ph = (int)(k & ((1ull << PH_BITS) - 1));
    cval[cid] = s;
    cphys[cid] = (unsigned char)ph;
    ctile[cid] = t;
    atomicOr(&mask[t], 1u << ph);
    atomicAdd(&tcount[t], 1);
    if (i == 0 || (keys[i - 1] >> PH_BITS) != (k >> PH_BITS))
    {
        tcol[t] = (int)((k >> PH_BITS) & ((1ull << TC_BITS) - 1));
        trow[t] = (int)(k >> (TC_BITS + PH_BITS));
        tfirst[t] = cid;
    }
}

__global__ void k_hyb_sizes(int ntiles, const int *__restrict__ tcount, int thr,
                            int *__restrict__ tsize, int *__restrict__ row_hist,
                            const int *__restrict__ trow, int *__restrict__ ndense)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles)
        return;
    const bool dense = tcount[t] >= thr;
    tsize[t] = dense ? ELEMS : tcount[t];
    atomicAdd(&row_hist[trow[t]], 1);
    if (dense)
        atomicAdd(ndense, 1);
}

__global__ void k_hyb_values(int ncoord, const double *__restrict__ cval,
                             const unsigned char *__restrict__ cphys,
                             const int *__restrict__ ctile, const int *__restrict__ tfirst,
                             const int *__restrict__ toff, const int *__restrict__ tcount, int thr,
                             double *__restrict__ values)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncoord)
        return;
    const int t = ctile[c];
    const int slot = tcount[t] >= thr ? (int)cphys[c] : c - tfirst[t];
    values[toff[t] + slot] = cval[c];
}

__global__ void k_hyb_hist(int n, const int *__restrict__ key, int *__restrict__ hist)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        atomicAdd(&hist[key[i]], 1);
}

__global__ void k_hyb_iota(int n, int *__restrict__ a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        a[i] = i;
}

__global__ void k_hyb_gather(int n, const int *__restrict__ idx, const int *__restrict__ src,
                             int *__restrict__ dst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = src[idx[i]];
}

inline int blocks(long long n, int b) { return (int)((n + b - 1) / b); }

template <typename T>
int alloc_dev(T **p, size_t n)
{
    RTT_CUDA(cudaMalloc((void **)p, sizeof(T) * (n > 0 ? n : 1)));
    return RTT_OK;
}

// Exclusive scan of n ints into out (n + 1 entries).
int scan_into(Workspace &ws, const int *in, int *out, int n)
{
    return scan_exclusive_int(ws, in, out, n);
}

struct DevArrays
{
    static constexpr int kMax = 40;
    void *p[kMax] = {};
    int used = 0;
    template <typename T>
    int get(T **out, size_t n)
    {
        if (used >= kMax)
            return fail(RTT_ERR_STATE, "hybrid tiles: too many device arrays");
        RTT_CHECK(alloc_dev(out, n));
        p[used++] = *out;
        return RTT_OK;
    }
    ~DevArrays()
    {
        for (int i = 0; i < used; ++i)
            cudaFree(p[i]);
    }
};

template <typename T>
int to_host(T **out, const T *d, size_t n, cudaStream_t s)
{
    *out = nullptr;
    if (n == 0)
        return RTT_OK;
    T *h = static_cast<T *>(std::malloc(sizeof(T) * n));
    if (h == nullptr)
        return fail(RTT_ERR_OUT_OF_MEMORY, "host malloc failed");
    cudaError_t e = cudaMemcpyAsync(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
    {
        std::free(h);
        return cuda_fail(e, "hybrid tiles: device to host copy");
    }
    *out = h;
    return RTT_OK;
}

} // namespace

int csr_to_hybrid_device(Workspace &ws, int m, int n, int nnz, const int *rp, const int *ci,
                         const double *va, int tr, int tc, int col_major, int thr, int build_csc,
                         HybridDev &H)
{
    cudaStream_t s = ws.stream;
    RTT_CUDA(cudaMemsetAsync(ws.err.p, 0, sizeof(int), s));
    k_hyb_validate<<<blocks(std::max(m + 1, nnz), 256), 256, 0, s>>>(m, n, nnz, rp, ci, ws.err.as<int>());
    ws.launches++;
    RTT_CHECK(check_device_error(ws, "hybrid tiles: CSR"));

    const int trc = m / tr + (m % tr != 0), tcc = n / tc + (n % tc != 0);
    H.rows = m;
    H.cols = n;
    H.tr = tr;
    H.tc = tc;
    H.trc = trc;
    H.tcc = tcc;
    H.col_major = col_major;
    H.has_csc = build_csc != 0;
    // grow-only scratch: entry level, coordinate level, tile level
    auto get = [&](DevBuf &b, size_t bytes) { return b.ensure(bytes > 0 ? bytes : 16, s); };
    const size_t E = (size_t)nnz;
    RTT_CHECK(get(H.tmp[0], 8 * E));       // keys
    RTT_CHECK(get(H.tmp[1], 8 * E));       // sorted keys
    RTT_CHECK(get(H.tmp[2], 8 * E));       // sorted values
    RTT_CHECK(get(H.tmp[3], 4 * (E + 1))); // coordinate heads
    RTT_CHECK(get(H.tmp[4], 4 * (E + 1))); // tile heads
    RTT_CHECK(get(H.tmp[5], 4 * (E + 1))); // coordinate ids
    RTT_CHECK(get(H.tmp[6], 4 * (E + 1))); // tile ids
    auto *keys = H.tmp[0].as<unsigned long long>(), *skeys = H.tmp[1].as<unsigned long long>();
    double *svals = H.tmp[2].as<double>();
    int *chead = H.tmp[3].as<int>(), *thead = H.tmp[4].as<int>(), *cid = H.tmp[5].as<int>(),
        *tid = H.tmp[6].as<int>();
    int ncoord = 0, ntiles = 0;
    if (nnz > 0)
    {
        k_hyb_keys<<<blocks((long long)m * 32, 256), 256, 0, s>>>(m, rp, ci, tr, tc, col_major, keys);
        int hibit = 0; // key bits in use
        {
            unsigned long long top = ((unsigned long long)trc << (TC_BITS + PH_BITS));
            while (hibit < 64 && (top >> hibit) != 0)
                ++hibit;
            hibit = std::max(hibit, TC_BITS + PH_BITS);
        }
        size_t bytes = 0;
        RTT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys, skeys, va, svals, nnz, 0,
                                                 hibit, s));
        RTT_CHECK(ws.scan_tmp.ensure(bytes, s));
        RTT_CUDA(cub::DeviceRadixSort::SortPairs(ws.scan_tmp.p, bytes, keys, skeys, va, svals, nnz,
                                                 0, hibit, s));
        k_hyb_heads<<<blocks(nnz, 256), 256, 0, s>>>(nnz, skeys, chead, thead);
        ws.launches += 4;
        // inclusive scans: coordinate / tile id of every entry
        RTT_CHECK(scan_into(ws, chead, cid, nnz)); // cid[i + 1] = inclusive count
        RTT_CHECK(scan_into(ws, thead, tid, nnz));
        RTT_CHECK(read_int(ws, cid + nnz, &ncoord));
        RTT_CHECK(read_int(ws, tid + nnz, &ntiles));
    }
    const size_t NC = (size_t)ncoord, NT = (size_t)ntiles;
    RTT_CHECK(get(H.tmp[7], 8 * NC));      // coordinate values
    RTT_CHECK(get(H.tmp[8], NC));          // coordinate physical index
    RTT_CHECK(get(H.tmp[9], 4 * NC));      // coordinate tile
    RTT_CHECK(get(H.tmp[10], 4 * NT));     // tile counts
    RTT_CHECK(get(H.tmp[11], 4 * NT));     // tile rows
    RTT_CHECK(get(H.tmp[12], 4 * NT));     // tile first coordinate
    RTT_CHECK(get(H.tmp[13], 4 * NT));     // tile payload sizes
    RTT_CHECK(get(H.tmp[14], 4 * ((size_t)std::max(trc, tcc) + 1))); // row / column histogram
    RTT_CHECK(get(H.tmp[15], 16));         // dense count
    RTT_CHECK(get(H.row_ptr, 4 * ((size_t)trc + 1)));
    RTT_CHECK(get(H.col_idx, 4 * NT));
    RTT_CHECK(get(H.value_off, 4 * (NT + 1)));
    RTT_CHECK(get(H.mask, 4 * NT));
    double *cval = H.tmp[7].as<double>();
    unsigned char *cphys = H.tmp[8].as<unsigned char>();
    int *ctile = H.tmp[9].as<int>(), *tcount = H.tmp[10].as<int>(), *trow = H.tmp[11].as<int>(),
        *tfirst = H.tmp[12].as<int>(), *tsize = H.tmp[13].as<int>(), *hist = H.tmp[14].as<int>(),
        *ndense = H.tmp[15].as<int>();
    int *tcol = H.col_idx.as<int>(), *toff = H.value_off.as<int>(), *rowptr = H.row_ptr.as<int>();
    unsigned int *mask = H.mask.as<unsigned int>();
    RTT_CUDA(cudaMemsetAsync(mask, 0, sizeof(unsigned) * std::max(NT, (size_t)1), s));
    RTT_CUDA(cudaMemsetAsync(tcount, 0, sizeof(int) * std::max(NT, (size_t)1), s));
    RTT_CUDA(cudaMemsetAsync(hist, 0, sizeof(int) * ((size_t)trc + 1), s));
    RTT_CUDA(cudaMemsetAsync(ndense, 0, sizeof(int), s));
    int payload = 0, ndense_h = 0;
    if (nnz > 0)
    {
        k_hyb_tiles<<<blocks(nnz, 256), 256, 0, s>>>(nnz, skeys, svals, chead, cid + 1, tid + 1,
                                                     cval, cphys, ctile, mask, tcount, tcol, trow,
                                                     tfirst);
        k_hyb_sizes<<<blocks(ntiles, 256), 256, 0, s>>>(ntiles, tcount, thr, tsize, hist, trow,
                                                       ndense);
        ws.launches += 2;
        RTT_CHECK(scan_into(ws, tsize, toff, ntiles));
        RTT_CHECK(read_int(ws, toff + ntiles, &payload));
        RTT_CHECK(read_int(ws, ndense, &ndense_h));
    }
    else
    {
        RTT_CUDA(cudaMemsetAsync(toff, 0, sizeof(int), s));
    }
    RTT_CHECK(scan_into(ws, hist, rowptr, trc));
    RTT_CHECK(get(H.values, 8 * (size_t)payload));
    double *values = H.values.as<double>();
    RTT_CUDA(cudaMemsetAsync(values, 0, sizeof(double) * (size_t)std::max(payload, 1), s));
    if (ncoord > 0)
    {
        k_hyb_values<<<blocks(ncoord, 256), 256, 0, s>>>(ncoord, cval, cphys, ctile, tfirst, toff,
                                                         tcount, thr, values);
        ws.launches++;
    }
    H.ntiles = ntiles;
    H.payload = payload;
    H.ndense = ndense_h;

    if (build_csc)
    {
        RTT_CHECK(get(H.csc_ptr, 4 * ((size_t)tcc + 1)));
        RTT_CHECK(get(H.csc_row, 4 * NT));
        RTT_CHECK(get(H.csc_ids, 4 * NT));
        RTT_CHECK(get(H.tmp[16], 4 * NT)); // iota
        RTT_CHECK(get(H.tmp[17], 4 * NT)); // sorted column keys
        int *iota = H.tmp[16].as<int>(), *skey = H.tmp[17].as<int>();
        int *csc_ptr = H.csc_ptr.as<int>(), *csc_row = H.csc_row.as<int>(),
            *csc_ids = H.csc_ids.as<int>();
        if (ntiles > 0)
        {
            // stable sort of tile ids by tile column keeps tile-row order per column
            k_hyb_iota<<<blocks(ntiles, 256), 256, 0, s>>>(ntiles, iota);
            int cbits = 1;
            while (cbits < 31 && (tcc >> cbits) != 0)
                ++cbits;
            size_t bytes = 0;
            RTT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, tcol, skey, iota, csc_ids,
                                                     ntiles, 0, cbits, s));
            RTT_CHECK(ws.scan_tmp.ensure(bytes, s));
            RTT_CUDA(cub::DeviceRadixSort::SortPairs(ws.scan_tmp.p, bytes, tcol, skey, iota,
                                                     csc_ids, ntiles, 0, cbits, s));
            k_hyb_gather<<<blocks(ntiles, 256), 256, 0, s>>>(ntiles, csc_ids, trow, csc_row);
            ws.launches += 4;
        }
        // column pointer: scan of the tiles per tile column
        RTT_CUDA(cudaMemsetAsync(hist, 0, sizeof(int) * ((size_t)tcc + 1), s));
        if (ntiles > 0)
        {
            k_hyb_hist<<<blocks(ntiles, 256), 256, 0, s>>>(ntiles, tcol, hist);
            ws.launches++;
        }
        RTT_CHECK(scan_into(ws, hist, csc_ptr, tcc));
    }
    return check_device_error(ws, "hybrid tiles");
}

void HybridDev::release()
{
    DevBuf *all[] = {&row_ptr, &col_idx, &value_off, &mask, &values, &csc_ptr, &csc_row, &csc_ids};
    for (DevBuf *b : all)
        b->release();
    for (DevBuf &b : tmp)
        b.release();
}

int csr_to_hybrid_host(Workspace &ws, const SMatrix *M, int tr, int tc, int col_major, int thr,
                       int build_csc, rtt_hybrid_tiles *out)
{
    cudaStream_t s = ws.stream;
    const int m = M->m, n = M->n, nnz = M->nnz;
    DevArrays D;
    int *rp = nullptr, *ci = nullptr;
    double *va = nullptr;
    RTT_CHECK(D.get(&rp, (size_t)m + 1));
    RTT_CHECK(D.get(&ci, (size_t)nnz));
    RTT_CHECK(D.get(&va, (size_t)nnz));
    RTT_CUDA(cudaMemcpyAsync(rp, M->rowpointer, sizeof(int) * ((size_t)m + 1), cudaMemcpyHostToDevice, s));
    if (nnz > 0)
    {
        RTT_CUDA(cudaMemcpyAsync(ci, M->columnindex, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, s));
        RTT_CUDA(cudaMemcpyAsync(va, M->value, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice, s));
    }
    HybridDev H;
    int st = csr_to_hybrid_device(ws, m, n, nnz, rp, ci, va, tr, tc, col_major, thr, build_csc, H);
    // host copies (malloc'd, caller frees with rtt_hybrid_tiles_destroy)
    rtt_hybrid_tiles h{};
    if (st == RTT_OK)
    {
        h.rows = m;
        h.cols = n;
        h.tile_rows = tr;
        h.tile_cols = tc;
        h.tile_row_count = H.trc;
        h.tile_col_count = H.tcc;
        h.num_tiles = H.ntiles;
        h.payload_size = H.payload;
        h.dense_tiles = H.ndense;
        h.sparse_tiles = H.ntiles - H.ndense;
        st = to_host(&h.tile_row_ptr, H.row_ptr.as<int>(), (size_t)H.trc + 1, s);
    }
    if (st == RTT_OK)
        st = to_host(&h.tile_col_idx, H.col_idx.as<int>(), (size_t)H.ntiles, s);
    if (st == RTT_OK)
        st = to_host(&h.value_offsets, H.value_off.as<int>(), (size_t)H.ntiles + 1, s);
    if (st == RTT_OK)
        st = to_host(&h.masks, H.mask.as<unsigned int>(), (size_t)H.ntiles, s);
    if (st == RTT_OK)
        st = to_host(&h.values, H.values.as<double>(), (size_t)H.payload, s);
    if (st == RTT_OK && build_csc)
    {
        st = to_host(&h.tile_col_ptr, H.csc_ptr.as<int>(), (size_t)H.tcc + 1, s);
        if (st == RTT_OK)
            st = to_host(&h.tile_row_idx, H.csc_row.as<int>(), (size_t)H.ntiles, s);
        if (st == RTT_OK)
            st = to_host(&h.csc_tile_ids, H.csc_ids.as<int>(), (size_t)H.ntiles, s);
    }
    cudaStreamSynchronize(s);
    H.release();
    if (st != RTT_OK)
    {
        rtt_hybrid_tiles_destroy(&h);
        return st;
    }
    *out = h;
    return RTT_OK;
}

// ------------------------------------------------------------- Super16 index
// The 16x16 parent index over leaf tiles (reference build_device_index,
// src/super16_symbolic.cuh:2123-2323).  A parent row covers RG leaf rows (2
// for 8x4 A leaves, 4 for 4x8 B leaves) and a parent column CG leaf columns
// (4 for A, 2 for B).  Each leaf row lists strictly increasing leaf columns,
// so a parent row's parents are the merged quotients leaf column / CG of its
// RG lists: one thread per parent row keeps one cursor per list.
namespace
{

template <int RG, int CG>
__device__ __forceinline__ int s16_next(const int *__restrict__ tcol, const int (&cur)[RG],
                                        const int (&end)[RG])
{
    int nxt = INT_MAX;
#pragma unroll
    for (int c = 0; c < RG; ++c)
        if (cur[c] < end[c])
            nxt = min(nxt, tcol[cur[c]] / CG);
    return nxt;
}

template <int RG>
__device__ __forceinline__ void s16_open(int P, int lrows, const int *__restrict__ tptr, int (&cur)[RG],
                                         int (&end)[RG])
{
#pragma unroll
    for (int c = 0; c < RG; ++c)
    {
        const int lr = P * RG + c;
        cur[c] = lr < lrows ? tptr[lr] : 0;
        end[c] = lr < lrows ? tptr[lr + 1] : 0;
    }
}

// parents per parent row
template <int RG, int CG>
__global__ void k_s16_count(int prows, int lrows, const int *__restrict__ tptr,
                            const int *__restrict__ tcol, unsigned long long *__restrict__ cnt)
{
    const int P = blockIdx.x * blockDim.x + threadIdx.x;
    if (P >= prows)
        return;
    int cur[RG], end[RG];
    s16_open<RG>(P, lrows, tptr, cur, end);
    unsigned long long n = 0;
    for (int J = s16_next<RG, CG>(tcol, cur, end); J != INT_MAX; J = s16_next<RG, CG>(tcol, cur, end))
    {
        ++n;
#pragma unroll
        for (int c = 0; c < RG; ++c)
            while (cur[c] < end[c] && tcol[cur[c]] / CG == J)
                ++cur[c];
    }
    cnt[P] = n;
}

// parent columns, child pointers and masks, leaf ids (leaf row by leaf row)
template <int RG, int CG>
__global__ void k_s16_fill(int prows, int lrows, const int *__restrict__ tptr,
                           const int *__restrict__ tcol, const unsigned long long *__restrict__ rowptr,
                           unsigned *__restrict__ pcol, unsigned long long *__restrict__ cptr,
                           unsigned char *__restrict__ cmask, unsigned *__restrict__ leaf_ids)
{
    const int P = blockIdx.x * blockDim.x + threadIdx.x;
    if (P >= prows)
        return;
    int cur[RG], end[RG];
    s16_open<RG>(P, lrows, tptr, cur, end);
    unsigned long long p = rowptr[P];
    // the parent row's leaves are the ids tptr[RG P] .. of its leaf rows
    unsigned long long out = (unsigned long long)cur[0];
    for (int J = s16_next<RG, CG>(tcol, cur, end); J != INT_MAX; J = s16_next<RG, CG>(tcol, cur, end))
    {
        unsigned mk = 0;
        pcol[p] = (unsigned)J;
        cptr[p] = out;
#pragma unroll
        for (int c = 0; c < RG; ++c)
            while (cur[c] < end[c] && tcol[cur[c]] / CG == J)
            {
                const int id = cur[c]++;
                mk |= 1u << (c * CG + tcol[id] % CG);
                leaf_ids[out++] = (unsigned)id;
            }
        cmask[p] = (unsigned char)mk;
        ++p;
    }
}

__global__ void k_s16_set(unsigned long long *p, unsigned long long v) { *p = v; }

// The 16 Boolean rows of every parent (thread per parent row r).  A leaves
// are 8x4 with bit r * 4 + c; B leaves 4x8 with bit c * 4 + r.
template <bool A_ROLE>
__global__ void k_s16_rows(long long n, const unsigned long long *__restrict__ cptr,
                           const unsigned char *__restrict__ cmask,
                           const unsigned *__restrict__ leaf_ids, const unsigned *__restrict__ lmask,
                           unsigned short *__restrict__ rows)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const long long p = i >> 4;
    const int r = (int)(i & 15);
    const unsigned occ = cmask[p];
    const unsigned long long base = cptr[p];
    unsigned res = 0;
    if (A_ROLE)
    {
        // leaf (r / 8, t): its row r % 8 is 4 bits, columns 4 t .. 4 t + 3
#pragma unroll
        for (int t = 0; t < 4; ++t)
        {
            const int slot = (r >> 3) * 4 + t;
            if ((occ >> slot) & 1u)
            {
                const unsigned m = lmask[leaf_ids[base + __popc(occ & ((1u << slot) - 1u))]];
                res |= ((m >> ((r & 7) * 4)) & 0xFu) << (4 * t);
            }
        }
    }
    else
    {
        // leaf (r / 4, h): its row k = r % 4 is every fourth bit from k,
        // columns 8 h .. 8 h + 7
        const int k = r & 3;
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            const int slot = (r >> 2) * 2 + h;
            if ((occ >> slot) & 1u)
            {
                const unsigned m = lmask[leaf_ids[base + __popc(occ & ((1u << slot) - 1u))]] >> k;
                unsigned row8 = 0;
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    row8 |= ((m >> (4 * c)) & 1u) << c;
                res |= row8 << (8 * h);
            }
        }
    }
    rows[i] = (unsigned short)res;
}

// parent CSC of B: keys column * prows + row, sorted, then split
__global__ void k_s16_csc_keys(int prows, const unsigned long long *__restrict__ rowptr,
                               const unsigned *__restrict__ pcol,
                               unsigned long long *__restrict__ keys, unsigned *__restrict__ ids)
{
    const int P = blockIdx.x * blockDim.x + threadIdx.x;
    if (P >= prows)
        return;
    for (unsigned long long id = rowptr[P]; id < rowptr[P + 1]; ++id)
    {
        keys[id] = (unsigned long long)pcol[id] * (unsigned long long)prows + (unsigned long long)P;
        ids[id] = (unsigned)id;
    }
}

__global__ void k_s16_csc_rows(long long n, int prows, const unsigned long long *__restrict__ keys,
                               unsigned *__restrict__ row_idx)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        row_idx[i] = (unsigned)(keys[i] % (unsigned long long)prows);
}

// col_ptr[c] = first sorted key of column c or later
__global__ void k_s16_col_ptr(int pcols, int prows, long long n,
                              const unsigned long long *__restrict__ keys,
                              unsigned long long *__restrict__ col_ptr)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > pcols)
        return;
    const unsigned long long want = (unsigned long long)c * (unsigned long long)prows;
    long long lo = 0, hi = n;
    while (lo < hi)
    {
        const long long mid = (lo + hi) >> 1;
        if (keys[mid] < want)
            lo = mid + 1;
        else
            hi = mid;
    }
    col_ptr[c] = (unsigned long long)lo;
}

} // namespace

int super16_index_host(Workspace &ws, const rtt_hybrid_tiles *L, unsigned role,
                       rtt_super16_index *out)
{
    cudaStream_t s = ws.stream;
    const bool a_role = role == RTT_SUPER16_A8X4;
    const int RG = a_role ? 2 : 4, CG = a_role ? 4 : 2;
    const int lrows = L->tile_row_count, nt = L->num_tiles;
    const int prows = lrows == 0 ? 0 : 1 + (lrows - 1) / RG;
    const int pcols = L->tile_col_count == 0 ? 0 : 1 + (L->tile_col_count - 1) / CG;
    DevArrays D;
    int *tptr = nullptr, *tcol = nullptr;
    unsigned *lmask = nullptr;
    unsigned long long *cnt = nullptr, *rowptr = nullptr;
    RTT_CHECK(D.get(&tptr, (size_t)lrows + 1));
    RTT_CHECK(D.get(&tcol, (size_t)nt));
    RTT_CHECK(D.get(&lmask, (size_t)nt));
    RTT_CHECK(D.get(&cnt, (size_t)prows + 1));
    RTT_CHECK(D.get(&rowptr, (size_t)prows + 1));
    RTT_CUDA(cudaMemcpyAsync(tptr, L->tile_row_ptr, sizeof(int) * ((size_t)lrows + 1),
                             cudaMemcpyHostToDevice, s));
    if (nt > 0)
    {
        RTT_CUDA(cudaMemcpyAsync(tcol, L->tile_col_idx, sizeof(int) * (size_t)nt,
                                 cudaMemcpyHostToDevice, s));
        RTT_CUDA(cudaMemcpyAsync(lmask, L->masks, sizeof(unsigned) * (size_t)nt,
                                 cudaMemcpyHostToDevice, s));
    }
    RTT_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * ((size_t)prows + 1), s));
    if (prows > 0)
    {
        if (a_role)
            k_s16_count<2, 4><<<blocks(prows, 128), 128, 0, s>>>(prows, lrows, tptr, tcol, cnt);
        else
            k_s16_count<4, 2><<<blocks(prows, 128), 128, 0, s>>>(prows, lrows, tptr, tcol, cnt);
    }
    size_t bytes = 0;
    RTT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt, rowptr, prows + 1, s));
    RTT_CHECK(ws.scan_tmp.ensure(bytes, s));
    RTT_CUDA(cub::DeviceScan::ExclusiveSum(ws.scan_tmp.p, bytes, cnt, rowptr, prows + 1, s));
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars64, rowptr + prows, sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, s));
    RTT_CUDA(cudaStreamSynchronize(s));
    const unsigned long long pc64 = (unsigned long long)ws.h_scalars64[0];
    if (pc64 > 0xFFFFFFFFull || (!a_role && pc64 > (unsigned long long)INT_MAX))
        return fail(RTT_ERR_UNREPRESENTABLE, "super16 index: too many parents");
    const long long pc = (long long)pc64;

    unsigned *pcol = nullptr, *leaf_ids = nullptr;
    unsigned long long *cptr = nullptr;
    unsigned char *cmask = nullptr;
    unsigned short *brows = nullptr;
    RTT_CHECK(D.get(&pcol, (size_t)pc));
    RTT_CHECK(D.get(&cptr, (size_t)pc + 1));
    RTT_CHECK(D.get(&cmask, (size_t)pc));
    RTT_CHECK(D.get(&leaf_ids, (size_t)nt));
    RTT_CHECK(D.get(&brows, (size_t)pc * 16));
    if (prows > 0)
    {
        if (a_role)
            k_s16_fill<2, 4><<<blocks(prows, 128), 128, 0, s>>>(prows, lrows, tptr, tcol, rowptr,
                                                               pcol, cptr, cmask, leaf_ids);
        else
            k_s16_fill<4, 2><<<blocks(prows, 128), 128, 0, s>>>(prows, lrows, tptr, tcol, rowptr,
                                                               pcol, cptr, cmask, leaf_ids);
    }
    k_s16_set<<<1, 1, 0, s>>>(cptr + pc, (unsigned long long)nt);
    if (pc > 0)
    {
        if (a_role)
            k_s16_rows<true><<<blocks(pc * 16, 256), 256, 0, s>>>(pc * 16, cptr, cmask, leaf_ids,
                                                                 lmask, brows);
        else
            k_s16_rows<false><<<blocks(pc * 16, 256), 256, 0, s>>>(pc * 16, cptr, cmask, leaf_ids,
                                                                  lmask, brows);
    }
    unsigned long long *col_ptr = nullptr;
    unsigned *row_idx = nullptr, *csc_ids = nullptr;
    if (!a_role)
    {
        unsigned long long *keys = nullptr, *skeys = nullptr;
        unsigned *ids = nullptr;
        RTT_CHECK(D.get(&keys, (size_t)pc));
        RTT_CHECK(D.get(&skeys, (size_t)pc));
        RTT_CHECK(D.get(&ids, (size_t)pc));
        RTT_CHECK(D.get(&csc_ids, (size_t)pc));
        RTT_CHECK(D.get(&row_idx, (size_t)pc));
        RTT_CHECK(D.get(&col_ptr, (size_t)pcols + 1));
        if (pc > 0)
        {
            k_s16_csc_keys<<<blocks(prows, 128), 128, 0, s>>>(prows, rowptr, pcol, keys, ids);
            int kbits = 1;
            const unsigned long long top = (unsigned long long)pcols * (unsigned long long)prows;
            while (kbits < 64 && (top >> kbits) != 0)
                ++kbits;
            bytes = 0;
            RTT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys, skeys, ids, csc_ids,
                                                     (int)pc, 0, kbits, s));
            RTT_CHECK(ws.scan_tmp.ensure(bytes, s));
            RTT_CUDA(cub::DeviceRadixSort::SortPairs(ws.scan_tmp.p, bytes, keys, skeys, ids,
                                                     csc_ids, (int)pc, 0, kbits, s));
            k_s16_csc_rows<<<blocks(pc, 256), 256, 0, s>>>(pc, prows, skeys, row_idx);
        }
        k_s16_col_ptr<<<blocks((long long)pcols + 1, 256), 256, 0, s>>>(pcols, prows, pc, skeys,
                                                                       col_ptr);
    }
    RTT_CUDA(cudaGetLastError());

    rtt_super16_index h{};
    h.role = role;
    h.rows = L->rows;
    h.cols = L->cols;
    h.parent_row_count = (unsigned)prows;
    h.parent_col_count = (unsigned)pcols;
    h.parent_count = (unsigned)pc;
    int st = to_host(&h.row_ptr, rowptr, (size_t)prows + 1, s);
    if (st == RTT_OK)
        st = to_host(&h.col_idx, pcol, (size_t)pc, s);
    if (st == RTT_OK)
        st = to_host(&h.child_ptr, cptr, (size_t)pc + 1, s);
    if (st == RTT_OK)
        st = to_host(&h.child_mask, cmask, (size_t)pc, s);
    if (st == RTT_OK)
        st = to_host(&h.child_leaf_ids, leaf_ids, (size_t)nt, s);
    if (st == RTT_OK)
        st = to_host(&h.boolean_row_masks, brows, (size_t)pc * 16, s);
    if (st == RTT_OK && !a_role)
    {
        st = to_host(&h.col_ptr, col_ptr, (size_t)pcols + 1, s);
        if (st == RTT_OK)
            st = to_host(&h.row_idx, row_idx, (size_t)pc, s);
        if (st == RTT_OK)
            st = to_host(&h.csc_parent_ids, csc_ids, (size_t)pc, s);
    }
    if (st != RTT_OK)
    {
        rtt_super16_index_destroy(&h);
        return st;
    }
    *out = h;
    return RTT_OK;
}

} // namespace rtt
