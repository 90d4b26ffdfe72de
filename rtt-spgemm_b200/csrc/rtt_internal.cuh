// rtt_internal.cuh - shared device/host helpers of the sm_100a tiled SpGEMM.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <string>

#include "rtt_spgemm.h"

namespace rtt
{

constexpr int TD = 16;          // tile edge (reference BLOCK_SIZE)
constexpr int WARP = 32;
constexpr unsigned FULL = 0xffffffffu;

// Device-side error words.  Kernels record the first failure with atomicCAS
// and skip the offending access; the host reads the word after a sync.
enum DeviceError : int
{
    DERR_NONE = 0,
    DERR_CSR_ROWPTR = 101,      // row_ptr not monotone / out of range
    DERR_CSR_COL = 102,         // column out of range
    DERR_C2T_OVERFLOW = 103,    // csr2tile wrote past a tile row
    DERR_SYM_OVERFLOW = 104,    // symbolic produced more tiles than counted
    DERR_NUM_PAIRS = 105,       // numeric pair buffer overflow
    DERR_NUM_BOUNDS = 106,      // numeric output index out of range
    DERR_T2C_BOUNDS = 107,      // tile2csr output index out of range
    DERR_WINDOW = 108,          // symbolic window bookkeeping failed
    DERR_T2C_TAIL = 109,        // tile2csr: row past the permutation prefix not empty
};

__device__ __forceinline__ void set_error(int *err, int code)
{
    if (err != nullptr)
        atomicCAS(err, 0, code);
}

// Row-major 16x16 tile CSR on the device (SMatrix semantics).  col bytes may
// be packed (row << 4) | col (A from csr2tile_row_major) or plain (B from
// csr2tile_col_major, C): the kernels only use the low nibble.
struct DevTiles
{
    int m, n, tilem, tilen, numtile, nnz;
    const int *tile_ptr;    // tilem + 1 (row-major structure)
    const int *tile_col;    // numtile
    const int *tile_nnz;    // numtile + 1, offsets into col/val (data order)
    const uint8_t *ptr;     // numtile * 16, exclusive row offsets (data order)
    const uint8_t *col;     // nnz
    const double *val;      // nnz
    const uint16_t *mask;   // numtile * 16, bit (15 - c) (data order)
    const int *row_data;    // row-major position -> data index (nullptr = identity)
    // tile CSC (column lists of K), data index per entry
    const int *csc_ptr;     // tilen + 1
    const int *csc_row;     // numtile
    const int *csc_data;    // numtile (nullptr = identity)
    // the same matrix as scalar CSR rows (B side of the numeric step; the
    // row-k segments of B tile row K concatenated in column order)
    const int *csr_rowptr;  // m + 1
    const int *csr_col;     // nnz
    const double *csr_val;  // nnz
    // row segments of the scalar CSR rows (nullptr when not built): the runs
    // of a row's entries inside one tile column, in column order, each as
    // (tile column << 16) | 16-bit column mask (bit 15 - c) - a B row's part
    // of every 16-bit tile row mask, listed per scalar row
    const int *seg_ptr;               // m + 1
    const unsigned long long *seg;    // seg_ptr[m]
    int max_row_segs;                 // most segments of one row (when seg_ptr is set)
};

// C tile structure produced by the symbolic phase.
struct DevCTiles
{
    int tilem, tilen, m, n;
    int *tile_ptr;      // tilem + 1
    int *tile_col;      // numtile
    int *tile_row;      // numtile
    int *tile_nnz;      // numtile + 1 (exclusive offsets)
    uint16_t *mask;     // numtile * 16
    uint8_t *ptr;       // numtile * 16
    uint8_t *col;       // nnz
    double *val;        // nnz
};

// ---------------------------------------------------------------- warp utils
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(FULL, v, o);
    return v;
}

__device__ __forceinline__ int warp_min(int v)
{
    return __reduce_min_sync(FULL, v);
}

__device__ __forceinline__ int warp_max(int v)
{
    return __reduce_max_sync(FULL, v);
}

// inclusive scan over the warp
template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v)
{
    const int l = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        T u = __shfl_up_sync(FULL, v, o);
        if (l >= o)
            v += u;
    }
    return v;
}

// inclusive scan inside each 16-lane half (width-16 shuffles)
template <typename T>
__device__ __forceinline__ T half_incl_scan(T v)
{
    const int l = lane_id() & 15;
#pragma unroll
    for (int o = 1; o < 16; o <<= 1)
    {
        T u = __shfl_up_sync(FULL, v, o, 16);
        if (l >= o)
            v += u;
    }
    return v;
}

__device__ __forceinline__ int half_min(int v)
{
#pragma unroll
    for (int o = 8; o > 0; o >>= 1)
        v = min(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

template <typename T>
__device__ __forceinline__ T half_sum(T v)
{
#pragma unroll
    for (int o = 8; o > 0; o >>= 1)
        v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// first index in [lo, hi) with a[i] >= key
__device__ __forceinline__ int lower_bound(const int *a, int lo, int hi, int key)
{
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (a[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__host__ __device__ __forceinline__ int ceil_div(int a, int b) { return a / b + (a % b != 0); }

// --------------------------------------------------------------- host side
std::string &last_error_ref();
int fail(int status, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define RTT_CUDA(call)                                                        \
    do                                                                        \
    {                                                                         \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess)                                                \
            return ::rtt::cuda_fail(e_, #call);                               \
    } while (0)

#define RTT_CHECK(call)                                                       \
    do                                                                        \
    {                                                                         \
        int s_ = (call);                                                      \
        if (s_ != RTT_OK)                                                     \
            return s_;                                                        \
    } while (0)

// Grow-only device buffer owned by a workspace.
struct DevBuf
{
    void *p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes, cudaStream_t s);
    void release();
    template <typename T>
    T *as() const { return static_cast<T *>(p); }
};

// Device workspace: named grow-only buffers plus pinned host scalars.
struct Workspace
{
    int device = 0;
    cudaStream_t stream = nullptr;
    DevBuf err;        // int device error word
    DevBuf scan_tmp;   // CUB temp storage
    DevBuf tmp[4];     // grow-only scratch of the transpose and the batch tables
    int *h_scalars = nullptr; // pinned, 32 ints
    long long *h_scalars64 = nullptr; // pinned, 8 long long
    int launches = 0;
    int syncs = 0;
    cudaEvent_t ev[6] = {};  // stage timing events (recorded on stream)
    // second stream for work that overlaps the main one (forked and joined
    // with the two events inside one call)
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    int init(int dev);
    void destroy();
};

// exclusive scan of n ints in place into out (n + 1 entries: out[n] = total)
int scan_exclusive_int(Workspace &ws, const int *in, int *out, int n);
// exclusive scan of n ints into int64 offsets (n + 1 entries)
int scan_exclusive_i64(Workspace &ws, const int *in, long long *out, int n);
// read the device error word (syncs the stream); returns RTT_ERR_DEVICE_CHECK on error
int check_device_error(Workspace &ws, const char *stage);
// copy one int / int64 from device to host (syncs)
int read_int(Workspace &ws, const int *d, int *h);
int read_i64(Workspace &ws, const long long *d, long long *h);
// the same reads with the device error word checked in the same synchronisation
int read_int_checked(Workspace &ws, const int *d, int *h, const char *stage);
int read_i64_checked(Workspace &ws, const long long *d, long long *h, const char *stage);
// while on, DevBuf growth on this thread fails with RTT_ERR_STATE (graph capture)
void freeze_growth(bool on);

// ------------------------------------------------------------- kernel hosts
// csr2tile: row-major tiles of a device CSR.  Output arrays allocated from bufs.
struct TileBufs
{
    DevBuf tile_ptr, tile_col, tile_row, tile_nnz, ptr, col, val, mask;
    DevBuf csc_ptr, csc_row, csc_data, row_data;
    DevBuf tmp0, tmp1, tmp2, tmp3;
    DevBuf seg_ptr, seg, seg_cnt; // row segments (csr2tile_device with segments = true)
    int m = 0, n = 0, tilem = 0, tilen = 0, numtile = 0, nnz = 0;
    bool has_segments = false;
    int max_row_segs = 0; // most segments of one row (structure-only builds; else 0 = unknown)
    bool payload = true;  // per-entry arrays (tile_nnz, ptr, col, val, mask) built
    bool dup_cols = false; // some row may repeat a column (set by csr2tile_device)
    bool generic = false;  // built by the generic (unsorted tile columns) path
    void release();
    DevTiles view() const;
    // every device buffer of the struct (release, CUDA-graph keys)
    template <class F>
    void each(F &&f) const
    {
        const DevBuf *all[] = {&tile_ptr, &tile_col, &tile_row, &tile_nnz, &ptr,  &col,
                               &val,      &mask,     &csc_ptr,  &csc_row,  &csc_data,
                               &row_data, &tmp0,     &tmp1,     &tmp2,     &tmp3,
                               &seg_ptr,  &seg,      &seg_cnt};
        for (const DevBuf *b : all)
            f(*b);
    }
};

// segments: also list the row segments of the CSR (seg_ptr, seg; only when
// every row's tile columns are non-decreasing, else has_segments stays false).
// payload = false: only the tile index (tile_ptr, tile_col, tile_row) and the
// row segments, when the rows allow it (out.payload tells what was built)
int csr2tile_device(Workspace &ws, int m, int n, int nnz, const int *rowptr, const int *col,
                    const double *val, TileBufs &out, bool packed_col, bool sort_within_rows,
                    bool segments = false, bool payload = true);
// values-only update: tiles built by csr2tile_device (sort_within_rows false)
// from a CSR of the same structure get the values val (no host round trip)
int csr2tile_refill_device(Workspace &ws, const int *rowptr, const int *col, const double *val,
                           TileBufs &t, bool packed_col);
// k_validate_csr on the device, then the host reads the error word (syncs):
// RTT_ERR_DEVICE_CHECK code 101/102 for a malformed CSR; flags: 3 device ints
// (tile column / column decreases in a row, repeated column), copied to
// ws.h_scalars[4..6]
int validate_csr_device(Workspace &ws, int m, int n, int nnz, const int *rowptr, const int *col,
                        int *flags);
// tile CSC index (column lists) over row-major tiles
int build_tile_csc(Workspace &ws, TileBufs &t);
// rearrange row-major tiles into the csr2tile_col_major layout (data in CSC order)
int tiles_to_col_major(Workspace &ws, const TileBufs &rowmajor, TileBufs &out);
// CSR transpose on the device
// bipartite Cuthill-McKee reorder plan of a device CSR (host maps malloc'd)
int reorder_plan_device(Workspace &ws, const rtt_csr_view &A, int variant, rtt_reorder_plan *plan);
// device CSR with permuted rows and remapped (then sorted) columns
int csr_permute_device(Workspace &ws, const rtt_csr_view &A, const int *row_new_to_old,
                       const int *col_old_to_new, int *out_rp, int *out_col, double *out_val);
// A^T of a device CSR into caller-sized arrays (n + 1, nnz, nnz), sorted rows;
// enqueued on ws.stream, scratch from ws.tmp
int csr_transpose_device(Workspace &ws, int m, int n, int nnz, const int *rowptr, const int *col,
                         const double *val, int *t_rowptr, int *t_col, double *t_val);

// Accumulator slots and C tiles per window of the flat numeric kernel (the
// symbolic step flags tile rows beyond either).
constexpr int FLAT_ACC = 2048;
constexpr int FLAT_SLOT_CAP = 128;
// In a tile row with several windows, a sorted B row longer than this is cut
// to the window's columns by binary search before its entries are walked
// (shorter rows are loaded whole and their entries outside the window skipped).
// 0 cuts every row: on B200 that beat 4, 12 and 32 by 3-5% on R-MAT and banded
// products, since even a short row's search skips loads of whole tiles' worth
// of out-of-window entries, and left the one-window stencil unchanged.
#ifndef NARROW_MIN
#define NARROW_MIN 0
#endif

struct SymbolicOut
{
    DevBuf c_tile_ptr, c_tile_col, c_tile_row, c_tile_nnz, c_mask, c_ptr, c_col, c_val;
    DevBuf c_row_cnt;   // m ints, per-row nnz of C
    DevBuf c_rowptr;    // tilem + 1 int64: exclusive scan of nnz per C tile row
    DevBuf c_tr_nnz;    // tilem ints, nnz per C tile row
    DevBuf count_tmp;   // tilem + 1 ints
    DevBuf tile_cnt;    // numtile ints, nnz per C tile
    // numeric split of heavy tile rows: window tasks, per-tile-row flag, queue
    DevBuf w_task, w_heavy, w_queue, w_flag;
    DevBuf w_cursor; // per worker CTA: window cursors of its task's A entries
    DevBuf g_slot, g_rel; // per global-row worker CTA: tile column table, row offsets
    // symbolic step 2: heavy tile rows (flag per tile row, list) and the
    // list of tile rows for the wide-window CTAs
    DevBuf s2_heavy, s2_list, s2_wlist;
    // symbolic step 1: tile rows with many tile pairs (list for a wide CTA)
    DevBuf s1_list;
    // some C tile row needs more than one window of the flat numeric kernel
    // (set by the symbolic step; true when unknown)
    bool multi_window = true;
    // C tiles per window of the wide-window step-2 CTAs (0: the default,
    // -1: tile rows with many C tiles stay in the 254-slot CTAs)
    int sym_window_slots = 0;
    int numtile = 0;
    long long nnz = 0;
    int tilem = 0, tilen = 0, m = 0, n = 0;
    void release();
    DevCTiles view();
    // every device buffer of the struct (release, CUDA-graph keys)
    template <class F>
    void each(F &&f) const
    {
        const DevBuf *all[] = {&c_tile_ptr, &c_tile_col, &c_tile_row, &c_tile_nnz, &c_mask,
                               &c_ptr,      &c_col,      &c_val,      &c_row_cnt,  &c_rowptr,
                               &c_tr_nnz,   &count_tmp,  &tile_cnt,   &w_task,     &w_heavy,
                               &w_queue,    &w_flag,     &s2_heavy,   &s2_list,
                               &s2_wlist,   &s1_list,    &w_cursor,   &g_slot,
                               &g_rel};
        for (const DevBuf *b : all)
            f(*b);
    }
};

// step 1 only: C tiles per tile row of A * B into cnt (A.tilem ints)
int symbolic_tile_counts(Workspace &ws, const DevTiles &A, const DevTiles &B, SymbolicOut &S,
                         int *cnt);
// tile counts of a tile grid on a bins x bins histogram (device, cleared first)
int tile_heatmap_device(Workspace &ws, int tilem, int tilen, const int *tile_ptr,
                        const int *tile_col, int bins, unsigned long long *d_hist);
// tile rows [I0, I1) of a device tile matrix with its CSR rows (the 64-bit
// products run A in such slices; B stays whole)
DevTiles tile_row_slice(const DevTiles &A, int I0, int I1);
// b_sorted: B's CSR rows have strictly increasing columns (lets the walk of a
// wide tile row's windows cut long B rows to each window)
int symbolic_device(Workspace &ws, const DevTiles &A, const DevTiles &B, SymbolicOut &S,
                    bool b_sorted = false);

struct NumericConfig
{
    // the defaults of rtt_config_default: no DMMA pairs, the flat kernel
    int dmma_pair_cutoff = 0;
    bool b_staging = false;         // TMA staging of B tile rows in the numeric step
    int split_target = 0;           // products per window task (0 = default, < 0 = no split)
    bool write_tiles = true;
    int *csr_rowptr = nullptr;  // fused CSR output when csr_col != nullptr
    int *csr_col = nullptr;
    double *csr_val = nullptr;
    long long *counters = nullptr; // device [0] dmma pairs, [1] sparse pairs, [2] split windows
    cudaEvent_t ev_begin = nullptr; // recorded around the numeric kernel when set
    cudaEvent_t ev_end = nullptr;
    bool conflict_safe = false;     // B rows may repeat a column: accumulate with shared atomics
    bool segment_walk = false;      // the numeric step may walk B's row segments
    bool persistent_rows = false;   // tile-row CTAs as one resident wave over a device queue
    // heavy tile rows accumulated in C's CSR values in global memory: 0 off,
    // 1 read-modify-write (bitwise the shared-memory result), 2 atomic adds
    int global_rows = 0;
};

// CSR row pointer of C (m + 1 ints) from the symbolic counts
int csr_rowptr_device(Workspace &ws, SymbolicOut &S, int *rowptr);
// numeric step, one CTA per C tile row (TMA-staged B tile rows)
int numeric_rows_device(Workspace &ws, const DevTiles &A, const DevTiles &B, SymbolicOut &S,
                        const NumericConfig &cfg);
// numeric step without a copy pipeline: warp-private Gustavson per row pair
int numeric_flat_device(Workspace &ws, const DevTiles &A, const DevTiles &B, SymbolicOut &S,
                        const NumericConfig &cfg);
struct HybridDev;
// numeric step on the FP64 tensor cores from hybrid leaves of A's and B's CSR
// (A.csr_*, B.csr_*; the leaves are built into LA / LB): C's 16x16 tiles
int numeric_leaf_device(Workspace &ws, const DevTiles &A, const DevTiles &B, HybridDev &LA,
                        HybridDev &LB, SymbolicOut &S, const NumericConfig &cfg);
// the flat kernel unless DMMA pairs exist or TMA staging of B is asked for
int numeric_select_device(Workspace &ws, const DevTiles &A, const DevTiles &B, SymbolicOut &S,
                          const NumericConfig &cfg);
// largest per-tile entry count of a tile matrix (device scalar *out)
int max_tile_nnz_device(Workspace &ws, const int *tile_nnz, int numtile, int *out);

// tile2csr on device tiles of edge td.  Writes rowptr (m + 1) then col/val.
int tile2csr_count_device(Workspace &ws, const int *tile_ptr, const int *tile_col,
                          const int *tile_nnz, const uint8_t *ptr, const uint8_t *col, int m,
                          int n, int tilem, int td, const int *new_to_old, int perm_size,
                          int *rowptr_out, const int *row_data = nullptr);
int tile2csr_fill_device(Workspace &ws, const int *tile_ptr, const int *tile_col,
                         const int *tile_nnz, const uint8_t *ptr, const uint8_t *col,
                         const double *val, int m, int n, int tilem, int td,
                         const int *new_to_old, int perm_size, const int *rowptr, int *out_col,
                         double *out_val, bool sort_rows, const int *row_data = nullptr);
// batched products (block-diagonal operands)
int batch_assemble_device(Workspace &ws, int count, int total_rows, const int *const *rp_tab,
                          const int *const *ci_tab, const double *const *va_tab, const int *rows,
                          const int *cols, const int *row_off, const int *col_add,
                          const int *nnz_off, int *out_rp, int *out_col, double *out_val);
int batch_count_device(Workspace &ws, int count, const int *row_off, const int *rows,
                       const int *row_cnt, long long *nnz);
// values-only update of a batch: instance i's nnz_off[i+1] - nnz_off[i]
// values from va_tab[i] into out_val at nnz_off[i] (max_nnz: the largest)
int batch_values_device(Workspace &ws, int count, int max_nnz, const double *const *va_tab,
                        const int *nnz_off, double *out_val);
int batch_split_device(Workspace &ws, int count, int total_rows, const int *row_off,
                       const int *rows, const int *sec_off, const int *col_sub, const int *big_rp,
                       int *out_rp, int *col);
// tail-queue admission plan of n tasks (device arrays); chunks per task into d_chunks
int plan_tail_queue_device(Workspace &ws, int n, const int *d_scans, const int *d_matches,
                           const int *d_out, const rtt_tail_policy &policy,
                           const rtt_tail_cost_model &model, int *d_chunks, rtt_tail_plan *plan);
// Hybrid leaf tiles on the device (the reference's HybridTileMatrix as
// DmmaDeviceTiles, src/dmma_tiles.h:29-62, src/dmma_spgemm.h:178-221): CSR
// over leaf rows (row_ptr, col_idx), value_off (a tile is dense exactly when
// its span is 32), u32 masks, values, and the optional CSC (csc_ptr over leaf
// columns, csc_row, csc_ids = CSR tile ids).  Buffers grow only.
struct HybridDev
{
    int rows = 0, cols = 0, tr = 0, tc = 0, trc = 0, tcc = 0;
    int ntiles = 0, payload = 0, ndense = 0, col_major = 0;
    bool has_csc = false;
    DevBuf row_ptr, col_idx, value_off, mask, values, csc_ptr, csc_row, csc_ids;
    DevBuf tmp[18]; // build scratch
    void release();
};
// device CSR -> hybrid leaf tiles of tile_rows x tile_cols (32 elements) in H
int csr_to_hybrid_device(Workspace &ws, int m, int n, int nnz, const int *rowptr, const int *col,
                         const double *val, int tile_rows, int tile_cols, int col_major,
                         int dense_threshold, int build_csc, HybridDev &H);
// Leaves with at least this many of their 32 entries are stored dense (the
// reference's default dense threshold).
constexpr int LEAF_DENSE_THRESHOLD = 24;
// CSR (host arrays) -> hybrid leaf tiles on the device, results malloc'd into out
int csr_to_hybrid_host(Workspace &ws, const SMatrix *M, int tile_rows, int tile_cols,
                       int col_major, int dense_threshold, int build_csc, rtt_hybrid_tiles *out);
// Super16 parent index of validated host leaf tiles (role 1 = A8x4, 2 = B4x8)
int super16_index_host(Workspace &ws, const rtt_hybrid_tiles *leaf, unsigned role,
                       rtt_super16_index *out);
// launch-only forms (no workspace, identity row order): the caller owns the
// stream and the error word; row_cnt needs m entries cleared to zero
int tile2csr_count_launch(cudaStream_t s, const int *tile_ptr, const int *tile_col,
                          const int *tile_nnz, const uint8_t *ptr, const uint8_t *col, int m,
                          int n, int tilem, int td, int *row_cnt, int *err);
int tile2csr_fill_launch(cudaStream_t s, const int *tile_ptr, const int *tile_col,
                         const int *tile_nnz, const uint8_t *ptr, const uint8_t *col,
                         const double *val, int m, int n, int tilem, int td, const int *rowptr,
                         long long nnz, int *out_col, double *out_val, bool sort_rows, int *err);

} // namespace rtt
