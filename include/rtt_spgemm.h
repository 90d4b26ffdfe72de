/*
 * rtt_spgemm.h - C ABI of the B200 (sm_100a) tiled FP64 SpGEMM.
 *
 * This library replaces the tiled SpGEMM path of for-the-juan/RTT-SpGEMM:
 * CSR -> 16x16 tiles (csr2tile) -> three-step tile SpGEMM (C = A*B, A*A,
 * A*A^T) -> tiles -> CSR (tile2csr).  Every entry point below does its work
 * with hand-written CUDA kernels on one GPU; there is no CPU fallback.  When
 * no usable GPU is present an entry point returns RTT_ERR_NO_DEVICE.
 *
 * Conventions kept from the reference so that existing callers drop in:
 *   - SMatrix is byte-for-byte the struct of src/common.h:50-72
 *     (MAT_VAL_TYPE = double, MAT_PTR_TYPE = int).
 *   - Tile geometry is 16x16 (BLOCK_SIZE, src/common.h:30-33).
 *   - Row-major tiles (csr2tile_row_major): tile_csr_Col holds the packed
 *     byte (row << 4) | col, mask[tile*16 + row] has bit (15 - col) set,
 *     tile_csr_Ptr holds exclusive per-row offsets inside the tile and
 *     tile_nnz is the exclusive scan of per-tile counts (numtile + 1 entries).
 *   - Column-major tiles (csr2tile_col_major): per-tile data stored in tile
 *     CSC order, plain column bytes, rows past a partial edge padded with the
 *     tile's entry count.
 *   - Outputs are allocated with malloc() into the SMatrix and are owned by
 *     the caller (free() them, or call rtt_matrix_destroy).
 *
 * Differences from the reference, all deliberate:
 *   - Functions return an rtt_status code instead of void/bool and never
 *     abort; on failure the output SMatrix is left unchanged.
 *   - rtt_spgemm_tile reads A's in-tile column as (byte & 0xF).  The
 *     reference spgemm_cpu uses the packed byte directly as a column
 *     (src/spgemm-cpu.h:231, :324), which is wrong for every A row but row 0.
 *   - rtt_spgemm_tile also fills C->m, C->n, C->tilem, C->tilen, C->mask and
 *     C->tile_rowidx, which spgemm_cpu leaves untouched.
 */
#ifndef RTT_SPGEMM_H_
#define RTT_SPGEMM_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RTT_API __attribute__((visibility("default")))
#else
#define RTT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#ifndef MAT_VAL_TYPE
#define MAT_VAL_TYPE double
#endif
#ifndef MAT_PTR_TYPE
#define MAT_PTR_TYPE int
#endif

/* Edge of the legacy square tile (reference BLOCK_SIZE). */
#define RTT_TILE_DIM 16
/* Edge of the reference's native 8x8 output tile (DMMA_TILE_M/N). */
#define RTT_OUTPUT_TILE_DIM 8

#ifndef SMATRIX
#define SMATRIX
/* Identical layout to the reference SMatrix (src/common.h:50-72). */
typedef struct
{
    int m;
    int n;
    int nnz;
    int isSymmetric;
    MAT_VAL_TYPE *value;
    int *columnindex;
    MAT_PTR_TYPE *rowpointer;
    int tilem;
    int tilen;
    MAT_PTR_TYPE *tile_ptr;
    int *tile_columnidx;
    int *tile_rowidx;
    int *tile_nnz;
    int numtile;
    MAT_VAL_TYPE *tile_csr_Value;
    unsigned char *tile_csr_Col;
    unsigned char *tile_csr_Ptr;
    unsigned short *mask;
    int *csc_tile_ptr;
    int *csc_tile_rowidx;
} SMatrix;
#endif

/* Status codes.  RTT_ERR_UNREPRESENTABLE mirrors the reference's
 * WIDE_OUTPUT_UNREPRESENTABLE status (src/main.cu:2203-2219): the result does
 * not fit the int32 fields of SMatrix / the int32 CSR of the device path. */
typedef enum
{
    RTT_OK = 0,
    RTT_ERR_INVALID_ARGUMENT = 1,
    RTT_ERR_INVALID_CSR = 2,
    RTT_ERR_SHAPE_MISMATCH = 3,
    RTT_ERR_OUT_OF_MEMORY = 4,
    RTT_ERR_CUDA = 5,
    RTT_ERR_UNREPRESENTABLE = 6,
    RTT_ERR_NO_DEVICE = 7,
    RTT_ERR_DEVICE_CHECK = 8,
    RTT_ERR_INVALID_PERMUTATION = 9,
    RTT_ERR_TAIL_NONEMPTY = 10,
    RTT_ERR_STATE = 11
} rtt_status;

/* Human-readable name of a status code. */
RTT_API const char *rtt_status_string(int status);
/* Message of the most recent failure on the calling thread ("" if none). */
RTT_API const char *rtt_last_error(void);
/* Library version string. */
RTT_API const char *rtt_version(void);

/* ------------------------------------------------------------------------
 * Host-buffer drop-ins.  SMatrix arrays live in host memory; the work runs on
 * the current CUDA device (device 0 unless rtt_set_device was called).
 * ------------------------------------------------------------------------ */

/* Replaces mmio_allinone (src/mmio_highlevel.h:593-760), the reference's
 * Matrix Market reader: a coordinate file (real, integer, pattern -> 1.0,
 * complex -> real part; general, symmetric, hermitian or skew-symmetric) into
 * a CSR SMatrix: m, n, nnz, isSymmetric and malloc'd rowpointer, columnindex,
 * value (free them, or rtt_matrix_destroy(out, 1)).  0-based; entries neither
 * sorted nor merged; a symmetric or hermitian file also stores each
 * off-diagonal entry mirrored, placed as it is read - the reference's exact
 * layout.  value_mode 1 sets entry i's value to i % 10 as the reference's
 * benchmark does after reading (src/main.cu:1109-1110); 0 keeps the file's.
 * Unlike the reference, indices outside the declared shape and short files
 * are errors (RTT_ERR_INVALID_CSR); a bad banner or a missing file gives
 * RTT_ERR_INVALID_ARGUMENT.  Host only: no GPU is needed. */
RTT_API int rtt_mmio_read(const char *path, int value_mode, SMatrix *out);

/* Select the CUDA device used by the host-buffer entry points. */
RTT_API int rtt_set_device(int device);

/* Replaces csr2tile_row_major(SMatrix*) (src/csr2tile.h:196-259).
 * Reads m, n, nnz, rowpointer, columnindex, value; allocates and fills
 * tilem, tilen, numtile, tile_ptr, tile_columnidx, tile_rowidx, tile_nnz,
 * tile_csr_Ptr, tile_csr_Col, tile_csr_Value, mask. */
RTT_API int rtt_csr2tile_row_major(SMatrix *matrix);

/* Replaces csr2tile_col_major(SMatrix*) (src/csr2tile.h:261-478).
 * Additionally fills csc_tile_ptr and csc_tile_rowidx; the per-tile arrays
 * (tile_nnz, tile_csr_*, mask) are in tile-CSC order, tile_rowidx is zeroed
 * as in the reference. */
RTT_API int rtt_csr2tile_col_major(SMatrix *matrix);

/* Replaces spgemm_cpu(SMatrix*A, SMatrix*B, SMatrix*C) (src/spgemm-cpu.h:369-455).
 * A: output of csr2tile_row_major; B: output of csr2tile_col_major (B may
 * describe A itself for C = A*A, or A^T for C = A*A^T).  C receives the
 * legacy 16x16 tile CSR: tile_ptr, tile_columnidx, tile_nnz, tile_csr_Ptr,
 * tile_csr_Col (plain column), tile_csr_Value, nnz, numtile, plus m, n,
 * tilem, tilen, tile_rowidx and mask (bit 15 - col). */
RTT_API int rtt_spgemm_tile(SMatrix *A, SMatrix *B, SMatrix *C);

/* Replaces tile2csr(SMatrix*, bool canonical) (src/tile2csr.h:232-329) for
 * square tiles of edge tile_dim (8: the reference's native output tiles;
 * 16: the legacy tiles produced by rtt_spgemm_tile).  Fills rowpointer,
 * columnindex, value and nnz.  Entries with an out-of-range column are
 * dropped and row bounds are clamped exactly as the reference does.  With
 * canonical == 0 each row is sorted by column (stable). */
RTT_API int rtt_tile2csr(SMatrix *matrix, int tile_dim, int canonical);

/* Replaces tile2csr_restore_rows (src/tile2csr.h:337-523): tile2csr that
 * writes reordered row new_row of C to original row row_new_to_old[new_row]
 * for new_row < permutation_size.  Rows at or past permutation_size must be
 * empty (RTT_ERR_TAIL_NONEMPTY otherwise); an illegal permutation returns
 * RTT_ERR_INVALID_PERMUTATION. */
RTT_API int rtt_tile2csr_restore_rows(SMatrix *matrix, const int *row_new_to_old,
                              int permutation_size, int tile_dim,
                              int canonical);

/* tile2csr on DEVICE tiles into caller-owned DEVICE CSR buffers, allocating
 * nothing (no cudaMalloc/cudaFree, no pinned host memory).  No counterpart in
 * the reference: its tile2csr (src/tile2csr.h:232) mallocs its output.  For
 * callers that may not allocate while they run: code whose device memory is
 * owned by an outer framework's pool or arena, and serving loops that must not
 * take cudaMalloc's device-wide synchronisation.
 * matrix: m, n, tilem, numtile, nnz (entries in tile_csr_Col/Value) and the
 * device arrays tile_ptr, tile_columnidx, tile_nnz, tile_csr_Ptr, tile_csr_Col,
 * tile_csr_Value on the CURRENT device, tiles of edge tile_dim (8 or 16) as
 * rtt_tile2csr takes them; rowpointer: caller's device array of m + 1 ints,
 * always written; columnindex, value: caller's device arrays with room for
 * out_capacity entries, or both NULL to ask only for the size.  *out_nnz
 * receives the entry count of the result.  Results equal rtt_tile2csr's.
 * Runs on stream (a cudaStream_t; NULL = legacy default stream) and returns
 * after its work there has finished.
 * Limits: m <= 33,554,432 rows (larger m returns RTT_ERR_INVALID_ARGUMENT
 * with a message naming the limit); its working memory is a 1 MiB static
 * device array per device.  The first call on a device looks that array up
 * (cudaGetSymbolAddress) and may load the module.  Calls that overlapped on
 * one device would share the array and race, so calls through this process
 * are serialised by a lock. */
RTT_API int rtt_tile2csr_device_noalloc(const SMatrix *matrix, int tile_dim, int canonical,
                                        long long out_capacity, long long *out_nnz,
                                        void *stream);

/* Split a legacy 16x16 tile C (as produced by rtt_spgemm_tile) into the
 * reference's native 8x8 output layout: the SMatrix that dmma_tilespgemm
 * exports (src/dmma_spgemm.h:6399-6488) - tile_ptr over 8-row tile rows,
 * tile_columnidx over 8-column tile columns, tile_nnz offsets, 8 row-offset
 * bytes per tile, column byte = col % 8.  Empty 8x8 quadrants are dropped. */
RTT_API int rtt_tile16_to_tile8(const SMatrix *c16, SMatrix *c8);

/* The reference's HybridTileMatrix (src/dmma_tiles.h:29-62), field for field
 * (MAT_PTR_TYPE = int): 32-element leaf tiles, 8x4 for A and 4x8 for B. */
typedef struct
{
    int rows, cols, tile_rows, tile_cols, tile_row_count, tile_col_count;
    int num_tiles, payload_size, dense_tiles, sparse_tiles;
    int *tile_row_ptr;      /* tile_row_count + 1 */
    int *tile_col_idx;      /* num_tiles */
    int *value_offsets;     /* num_tiles + 1; span 32 <=> dense tile */
    unsigned int *masks;    /* num_tiles, bit = physical index */
    double *values;         /* payload_size */
    int *tile_col_ptr;      /* optional tile CSC: tile_col_count + 1 */
    int *tile_row_idx;      /* num_tiles */
    int *csc_tile_ids;      /* num_tiles, ids in the tile CSR */
} rtt_hybrid_tiles;

/* Replaces csr_to_hybrid_tiles (src/dmma_tiles.h:243-438): host CSR in, hybrid
 * leaf tiles out (malloc'd arrays; free with rtt_hybrid_tiles_destroy).  A
 * uses (8, 4, col_major = 0), B uses (4, 8, col_major = 1); tile_rows *
 * tile_cols must be 32 and 1 <= dense_threshold <= 32.  Repeated coordinates
 * are summed.  Invalid CSR returns RTT_ERR_INVALID_CSR, other bad arguments
 * RTT_ERR_INVALID_ARGUMENT; out is untouched on failure (the reference's
 * transactional contract). */
RTT_API int rtt_csr_to_hybrid_tiles(const SMatrix *csr, int tile_rows, int tile_cols,
                                    int col_major, int dense_threshold, int build_csc,
                                    rtt_hybrid_tiles *out);

/* Operand roles of the Super16 index (the reference's rtt::super16::OperandRole,
 * src/super16_symbolic.cuh:64-68). */
#define RTT_SUPER16_A8X4 1
#define RTT_SUPER16_B4X8 2

/* The reference's Super16 16x16 parent index over hybrid leaf tiles
 * (rtt::super16::DeviceIndexView, src/super16_symbolic.cuh:85-106), field for
 * field, as host arrays.  A parent is the 16x16 block of 2 x 4 A leaves (8x4)
 * or 4 x 2 B leaves (4x8).  Parents of a parent row are in increasing column
 * order; a parent's leaves (child_leaf_ids[child_ptr[p] ..]) are listed leaf
 * row by leaf row, each in leaf-column order; child_mask bit
 * child_row * col_group + leaf_col % col_group marks a present leaf
 * (col_group 4 for A, 2 for B); boolean_row_masks[16 p + r] has bit c set when
 * (r, c) of the parent is structurally nonzero (LSB = column 0).  B also gets
 * the parent CSC (rows in increasing order per column), NULL for A. */
typedef struct
{
    unsigned int role;
    int rows, cols;
    unsigned int parent_row_count, parent_col_count, parent_count;
    unsigned long long *row_ptr;       /* parent_row_count + 1 */
    unsigned int *col_idx;             /* parent_count */
    unsigned long long *child_ptr;     /* parent_count + 1 */
    unsigned char *child_mask;         /* parent_count */
    unsigned int *child_leaf_ids;      /* num_tiles of the leaves */
    unsigned short *boolean_row_masks; /* parent_count * 16 */
    unsigned long long *col_ptr;       /* B4x8: parent_col_count + 1 */
    unsigned int *row_idx;             /* B4x8: parent_count */
    unsigned int *csc_parent_ids;      /* B4x8: parent_count */
} rtt_super16_index;

/* Replaces build_device_index (src/super16_symbolic.cuh:2123-2323): the
 * Super16 index of leaf tiles from rtt_csr_to_hybrid_tiles (8x4 for
 * RTT_SUPER16_A8X4, 4x8 for RTT_SUPER16_B4X8), built on the GPU, returned in
 * malloc'd arrays (free with rtt_super16_index_destroy).  Leaf rows must list
 * strictly increasing tile columns inside [0, tile_col_count) (as
 * rtt_csr_to_hybrid_tiles writes them); otherwise RTT_ERR_INVALID_ARGUMENT.
 * out is untouched on failure. */
RTT_API int rtt_super16_index_build(const rtt_hybrid_tiles *leaf, unsigned int role,
                                    rtt_super16_index *out);
RTT_API void rtt_super16_index_destroy(rtt_super16_index *index);

/* Tail-queue admission (the reference's DmmaTileTailQueuePolicy / CostModel /
 * Plan, src/dmma_tile_tail_queue.h:20-121; enabled is the policy switch). */
typedef struct
{
    int enabled;
    double admission_threshold; /* FP32 work above this admits a task (256) */
    double chunk_target;        /* work per chunk (256) */
    int max_chunks;             /* 2..32 (8) */
    double max_heavy_fraction;  /* (0.01) */
    int record_capacity;        /* (1 << 20) */
    long long workspace_limit_bytes; /* (1 GiB) */
    int workspace_reduction;    /* (1) */
} rtt_tail_policy;

typedef struct
{
    double intercept, scan, match, output; /* (0, 1, 8, 0.25) */
} rtt_tail_cost_model;

typedef struct
{
    int reason; /* DmmaTileTailQueueGateReason: 0 off, 1 enabled, 2 invalid policy,
                   3 invalid task, 4 zero heavy, 5 record capacity, 6 heavy fraction,
                   7 workspace capacity */
    long long output_tasks, ordinary_tasks, heavy_tasks, chunks;
    long long descriptor_bytes, heavy_flag_bytes, partial_workspace_bytes;
    double heavy_fraction, average_chunks;
} rtt_tail_plan;

/* Replaces dmma_plan_tile_tail_queue (src/dmma_tile_tail_queue.h:190-291),
 * planned on the GPU: task i is described by scans[i], matches[i] and
 * output_nnz[i] (host arrays of ntasks); chunks_out[i] receives the task's
 * chunk count (0 = ordinary task), and plan the summary and gate reason,
 * exactly as the reference computes them (FP32 admission arithmetic). */
RTT_API int rtt_plan_tail_queue(int ntasks, const int *scans, const int *matches,
                                const int *output_nnz, const rtt_tail_policy *policy,
                                const rtt_tail_cost_model *model, int *chunks_out,
                                rtt_tail_plan *plan);

/* Early split (the reference's DmmaTileEarlySplitPlan,
 * src/dmma_tile_early_split.h:72-97): the tail-queue partition exposed as a
 * bounded grid of persistent heavy CTAs, at most ceil(sm_count / 2) of them,
 * enqueued before the light grid. */
typedef struct
{
    int reason;      /* DmmaTileEarlySplitGateReason: 0 default off, 1 enabled,
                        2 invalid topology, 3 base fallback, 4 worker cap overflow */
    int base_reason; /* the tail-queue planner's reason (rtt_tail_plan.reason) */
    long long output_tasks, ordinary_tasks, heavy_tasks, chunks;
    int sm_count;
    int global_heavy_worker_block_cap; /* ceil(sm_count / 2) */
    int heavy_worker_blocks;           /* min(chunks, cap) */
    int reduction_worker_blocks;       /* min(heavy_tasks, cap) with workspace reduction */
    long long descriptor_bytes, heavy_flag_bytes, partial_workspace_bytes;
    int exact_parent_partition;        /* every task is ordinary or heavy exactly once */
} rtt_early_split_plan;

/* The reference's early-split policy defaults (DmmaTileEarlySplitPolicy,
 * src/dmma_tile_early_split.h:33-43): enabled = 0, admission 684947.875,
 * chunk target 342473.938, 8 chunks, heavy fraction 0.001, 131072 records,
 * 512 MiB of partial workspace, workspace reduction on. */
RTT_API void rtt_early_split_policy_default(rtt_tail_policy *policy);

/* Replaces dmma_plan_tile_early_split (src/dmma_tile_early_split.h:152-229):
 * the tail-queue plan of rtt_plan_tail_queue (with the policy forced on) plus
 * the heavy-worker bound.  chunks_out[i] receives task i's chunk count (0 =
 * ordinary; all 0 unless reason == 1).  sm_count <= 0 gives reason 2. */
RTT_API int rtt_plan_early_split(int ntasks, const int *scans, const int *matches,
                                 const int *output_nnz, const rtt_tail_policy *policy,
                                 const rtt_tail_cost_model *model, int sm_count,
                                 int *chunks_out, rtt_early_split_plan *plan);

/* Row / inner (K) reorder plan of A (the reference's DmmaReorderPlan,
 * src/dmma_reorder.h:173-224, reduced to its maps and counters).  Maps are
 * host arrays malloc'd by rtt_reorder_plan_build (rtt_reorder_plan_destroy
 * frees them); new = old_to_new[old], old = new_to_old[new]. */
typedef struct
{
    int rows, cols, nnz;
    int active_rows, active_inner; /* rows / columns reached by the traversal */
    int components, levels;        /* components traversed, traversal levels */
    int accepted;                  /* 1: the coarse proposal has fewer 8x4 A tiles and was
                                      taken; 0: the coarse stage left A's order */
    long long tiles_before;        /* distinct 8x4 tiles of A as given */
    long long tiles_after;         /* ... under the plan (never more than tiles_before,
                                      except in RTT_REORDER_UNGUARDED) */
    long long proposal_tiles;      /* ... under the coarse traversal's proposal */
    long long moved_rows, moved_inner;
    int *row_old_to_new, *row_new_to_old;
    int *inner_old_to_new, *inner_new_to_old;
    int variant;                   /* RTT_REORDER_* the plan was built with */
    /* Fine passes: windows of 32 rows (4 groups of 8) and of 16 inner
     * indices (4 groups of 4), and the windows whose packing was committed. */
    int row_windows, accepted_row_windows;
    int inner_windows, accepted_inner_windows;
    long long row_tile_reduction, inner_tile_reduction; /* 8x4 tiles the committed windows removed */
    /* Fan-out proxy: over the windows' groups (8 rows, or 4 inner indices),
     * the span of the opposite axis's tiles they touch, before and after. */
    long long row_fanout_before, row_fanout_after;
    long long inner_fanout_before, inner_fanout_after;
} rtt_reorder_plan;

/* Frees the arrays of a hybrid tile matrix and zeroes it (the reference's
 * destroy_hybrid_tile_matrix, src/dmma_tiles.h:64-79). */
RTT_API void rtt_hybrid_tiles_destroy(rtt_hybrid_tiles *tiles);

/* Frees every array the library allocated into matrix (tile fields, the csc
 * fields and, when owned_csr != 0, rowpointer/columnindex/value) and sets the
 * pointers to NULL.  The reference matrix_destroy (src/csr2tile.h:481-492)
 * frees the tile fields only. */
RTT_API void rtt_matrix_destroy(SMatrix *matrix, int owned_csr);

/* ------------------------------------------------------------------------
 * Device-resident product: device CSR(A) [, CSR(B)] in -> device CSR(C) out,
 * through 16x16 tiles.  This is the path the reference times
 * (src/main.cu:2171-2382: B csr2tile + symbolic + allocation + numeric),
 * extended with csr2tile of A and tile2csr of C.
 * ------------------------------------------------------------------------ */

typedef struct rtt_context_s *rtt_context;

/* C = A * B (B == NULL means B = A), C = A * A^T. */
enum
{
    RTT_OP_AB = 0,
    RTT_OP_AAT = 1
};

/* Device CSR operand (int32 offsets, 0-based, FP64 values). */
typedef struct
{
    int rows;
    int cols;
    long long nnz;
    const int *row_ptr; /* rows + 1 */
    const int *col_idx; /* nnz */
    const double *values; /* nnz */
} rtt_csr_view;

/* Tuning knobs of one context.  Zero-initialise and call
 * rtt_config_default() to get the defaults. */
typedef struct
{
    /* A tile pair (A(I,K), B(K,J)) goes to the FP64 DMMA tensor-core path
     * when nnz(A(I,K)) * nnz(B(K,J)) >= dmma_pair_cutoff; 0 disables DMMA
     * (the default: the flat scalar kernel measured faster on every workload
     * tried, banded batches with dense tiles included; 3072 is a typical
     * value for brick-ordered stencils). */
    int dmma_pair_cutoff;
    /* Numeric writes C's CSR directly (fused tile2csr) when nonzero;
     * otherwise C is written as 16x16 tiles and converted by tile2csr. */
    int fused_csr_output;
    /* Keep C's 16x16 tile arrays on the device after numeric (needed for
     * rtt_spgemm_tiles_view); implied when fused_csr_output == 0. */
    int keep_tiles;
    /* Record CUDA events around the stages (csr2tile, symbolic, numeric
     * kernel) on the context's stream; results land in rtt_stats. */
    int stage_timing;
    /* Numeric kernel without DMMA pairs: 0 = warp-private Gustavson with
     * direct loads of B's rows (default, fastest on B200), 1 = B tile rows
     * streamed by TMA bulk copies through a shared-memory stage ring (the
     * kernel that also runs the DMMA pairs). */
    int b_staging;
    /* Early split of heavy C tile rows.  A tile row that needs several
     * windows of C tiles walks all its products once per window; when that
     * walk exceeds split_target products the row is cut into tasks of
     * consecutive windows of about split_target products each, which
     * persistent CTAs take from a device queue.  0 = the default (2^20);
     * negative = never split (each tile row's CTA runs its windows in
     * sequence).  Every setting gives bitwise the same C. */
    int split_target;
    /* Replay the numeric phase as a CUDA graph when nonzero (the default).
     * rtt_spgemm_numeric, rtt_spgemm_numeric_values and
     * rtt_spgemm_batched_numeric capture their launches on the second call
     * in a row with the same shapes, pointers, configuration and workspace,
     * and replay that graph while those stay the same.  Off with
     * stage_timing or fused_csr_output == 0. */
    int cuda_graphs;
    /* 64-bit products (rtt_spgemm_symbolic64): both phases run over chunks of
     * A's tile rows holding at most chunk_tiles C tiles (0 = 2^25, about
     * 2 GiB of C tile structure), and a chunk whose C holds more than
     * chunk_nnz entries (0 = INT32_MAX) is halved. */
    int chunk_tiles;
    int chunk_nnz;
    /* Numeric step from B's row segments when nonzero (default 0: the
     * entry-per-lane walk): where every tile row fits one window, B has no
     * repeated columns and no B row has more than 32 segments, a half-warp
     * walks a row's A entries and its lanes take the segments of each
     * entry's B row.  Both give bitwise the same C; on B200 the segment walk
     * measured slower on the 27-point stencil (numeric 4.18 against 2.29 ms
     * at 96^3: one A entry per half-warp in flight leaves the walk
     * latency-bound), so it is opt-in. */
    int segment_walk;
    /* Numeric step's tile-row CTAs as one resident wave taking tile rows
     * from a device queue (nonzero) instead of one CTA per tile row (0, the
     * default).  For a batch the queue spans every instance's tile rows.
     * Both give bitwise the same C. */
    int persistent_rows;
    /* Symbolic step 2 of C tile rows with more C tiles than 254 (R-MAT
     * rows): every window of C tiles walks the tile row's A entries again,
     * so such rows run in CTAs whose windows hold up to sym_window_slots C
     * tiles (0 = the default, 2045; 255..6000 to choose; -1 = off, every
     * row in windows of 254).  Every setting gives bitwise the same C. */
    int sym_window_slots;
    /* Numeric step on the FP64 tensor cores straight from hybrid leaf tiles
     * when nonzero (the reference's dmma_numeric_kernel path): A and B are
     * cut into 8x4 / 4x8 leaves (dense when they hold >= 24 of 32 entries),
     * each 8x8 quadrant of a C tile is a sum of mma.sync.m8n8k4.f64 over
     * the matching K blocks, and tile2csr writes the CSR.  Same structure;
     * values within the FP64 bound (other summation order).  Default 0: the
     * scalar kernel is faster on every workload measured. */
    int leaf_dmma;
    /* C tile rows that need several shared-memory windows (R-MAT rows) are
     * cut into tasks of about 8192 C entries that accumulate straight into
     * C's CSR values in device memory, so each A entry is walked once per
     * task instead of once per window: 0 = off (the default), 1 =
     * read-modify-write in each row's (K, k) order (bitwise the same C, but
     * slower than the windows: a warp per row leaves the others waiting on
     * hub rows), 2 = atomic adds for rows of at least 4 windows, the task's
     * tables in shared memory and its entries shared by all warps (rows of
     * fewer windows keep them; R-MAT 2^16 A*A^T numeric 21.0 -> 13.0 ms
     * on B200; values within the FP64 bound, their last bits depending on
     * the order of the adds).  Only with the fused CSR output and sorted B
     * rows without repeated columns (1: at most 2^20 tile columns);
     * otherwise the windows. */
    int global_rows;
} rtt_config;

RTT_API void rtt_config_default(rtt_config *config);

/* Per-context statistics of the last product. */
typedef struct
{
    long long nnz_a;
    long long nnz_b;
    long long nnz_c;
    long long nnz_cub; /* sum over (i,k) in A of nnz(B row k); flops = 2*nnz_cub */
    long long tiles_a;
    long long tiles_b;
    long long tiles_c;
    long long dmma_pairs;
    long long sparse_pairs;
    int kernel_launches; /* kernels launched by the last symbolic+numeric */
    int host_syncs;      /* stream synchronisations in the last symbolic */
    /* Stage times of the last product in ms (stage_timing != 0, else 0):
     * csr2tile of A and B + tile CSC index, symbolic steps 1-2 with their
     * scans, and the numeric kernel alone. */
    double csr2tile_ms;
    double symbolic_ms;
    double numeric_kernel_ms;
    /* Window tasks of the last numeric step: C tile rows that need several
     * windows of C tiles are cut into windows that persistent CTAs take from
     * a device queue (the early split of src/dmma_tile_early_split.h). */
    long long split_windows;
    /* 1 when the last numeric phase ran as a launch of a captured CUDA graph
     * (cuda_graphs), else 0. */
    int graph_launched;
    /* Window tasks of the last numeric step that hold two or more windows
     * (a worker keeps per-entry cursors from one window to the next). */
    long long split_multi_window_tasks;
} rtt_stats;

/* A context owns a CUDA stream handle (borrowed), workspace and the state
 * carried from rtt_spgemm_symbolic to rtt_spgemm_numeric.  One context must
 * not be used by two host threads at once. */
RTT_API int rtt_context_create(rtt_context *ctx, int device);
RTT_API void rtt_context_destroy(rtt_context ctx);
/* Releases every device buffer the context has grown (tiles, C structure,
 * workspace) and its captured graphs; the context stays usable (stream and
 * configuration kept) and the next product grows them again.  The state of
 * the last symbolic phase is dropped.  For long-running callers under memory
 * pressure (the serving loop calls it before a product that ran out of
 * memory is tried alone).  No counterpart in the reference. */
RTT_API int rtt_context_trim(rtt_context ctx);
/* stream is a cudaStream_t (NULL = legacy default stream). */
RTT_API int rtt_context_set_stream(rtt_context ctx, void *stream);
RTT_API int rtt_context_set_config(rtt_context ctx, const rtt_config *config);
RTT_API int rtt_context_get_stats(rtt_context ctx, rtt_stats *stats);

/* Phase 1: csr2tile of A (and B), the three-step symbolic, exact sizes.
 * A and B stay borrowed until rtt_spgemm_numeric returns.  Writes the exact
 * nnz(C) and tile count of C.  Returns RTT_ERR_UNREPRESENTABLE when nnz(C)
 * exceeds INT32_MAX. */
RTT_API int rtt_spgemm_symbolic(rtt_context ctx, const rtt_csr_view *A,
                        const rtt_csr_view *B, int op, long long *nnz_c,
                        long long *tiles_c);

/* Phase 2: numeric into caller-owned device buffers: c_row_ptr (rows + 1),
 * c_col_idx and c_values (nnz_c from phase 1).  Rows come out sorted by
 * column. */
RTT_API int rtt_spgemm_numeric(rtt_context ctx, int *c_row_ptr, int *c_col_idx,
                       double *c_values);

/* 64-bit output (the SMatrix64 case: C with more than INT32_MAX entries).
 * The reference stops there with WIDE_OUTPUT_UNREPRESENTABLE
 * (src/main.cu:2203-2219; candidates capped at INT_MAX, src/dmma_spgemm.h:171-176);
 * these two replace rtt_spgemm_symbolic / rtt_spgemm_numeric for such
 * products (any product works through them).  Phase 1 takes the same
 * operands and writes the exact nnz(C) as int64.  Phase 2 writes C into
 * caller-owned device buffers: c_row_ptr (rows + 1 int64), c_col_idx (int32)
 * and c_values (nnz_c entries each); rows sorted by column, results equal to
 * the 32-bit path's.  The C tile structure never exists for the whole
 * product: both phases run over chunks of A's tile rows (rtt_config
 * chunk_tiles, chunk_nnz), and phase 2 runs steps 1-2 of each chunk again
 * before its numeric step.  A and B stay borrowed until phase 2 returns. */
RTT_API int rtt_spgemm_symbolic64(rtt_context ctx, const rtt_csr_view *A,
                                  const rtt_csr_view *B, int op, long long *nnz_c);
RTT_API int rtt_spgemm_numeric64(rtt_context ctx, long long *c_row_ptr, int *c_col_idx,
                                 double *c_values);

/* Dynamic B (the reference's B update modes, src/main.cu:26-32 and
 * rebuild_b, :1406-1453): C = A*B for the A of the last rtt_spgemm_symbolic
 * on ctx (op RTT_OP_AB, B or A*A) and a new B.  A's tiles are kept (A stays
 * borrowed); B is tiled anew and the symbolic phase runs, writing nnz(C) and
 * its tile count; rtt_spgemm_numeric follows.
 *   - row_new_to_old == NULL: the structure mode (B_UPDATE_STRUCTURE): B is
 *     any new matrix with B->rows == A's columns;
 *   - otherwise the permutation mode (B_UPDATE_PERMUTATION): B's rows are
 *     taken in the order row_new_to_old (a device array of B->rows ints,
 *     checked to be a permutation: RTT_ERR_DEVICE_CHECK otherwise), the inner
 *     order of an A whose columns were permuted the same way.
 * The values mode (B_UPDATE_VALUES) is rtt_spgemm_numeric_values.
 * RTT_ERR_STATE without such a symbolic phase (or after A*A^T or a batch). */
RTT_API int rtt_spgemm_update_b(rtt_context ctx, const rtt_csr_view *B,
                                const int *row_new_to_old, long long *nnz_c,
                                long long *tiles_c);

/* Values-only update (the reference's dynamic-B "values-only" mode,
 * src/main.cu:26-32, :1406-1453, for A and B): the same product as the last
 * rtt_spgemm_symbolic, with new values for A (a_values, device, A's CSR order)
 * and B (b_values, B's CSR order; NULL keeps B's values; ignored for
 * C = A*A and C = A*A^T, whose B follows A).  The structure arrays given to
 * rtt_spgemm_symbolic stay borrowed while such updates are made.  Skips
 * csr2tile's counting and the symbolic phase: A's tiles (and B's) are refilled
 * in place and the numeric step runs into the caller's C buffers, whose
 * structure equals the first product's. */
RTT_API int rtt_spgemm_numeric_values(rtt_context ctx, const double *a_values,
                                      const double *b_values, int *c_row_ptr, int *c_col_idx,
                                      double *c_values);

/* Device pointers to C's 16x16 tiles from the last numeric (legacy SMatrix
 * layout, plain column bytes).  Valid until the next symbolic on ctx. */
RTT_API int rtt_spgemm_tiles_view(rtt_context ctx, SMatrix *c_tiles_device);

/* Host-buffer CSR product through the device path: copies A (and B) to the
 * device, runs both phases, copies C back into malloc'd rowpointer /
 * columnindex / value of C (m, n, nnz set).  A and B are CSR SMatrix (only
 * the CSR fields are read).  B == NULL means B = A for RTT_OP_AB. */
RTT_API int rtt_spgemm_csr_host(rtt_context ctx, const SMatrix *A, const SMatrix *B,
                        int op, SMatrix *C);

/* The same product into caller-owned host arrays, for callers that keep
 * their output buffers from one product to the next (a serving loop): C's
 * row pointer (A->m + 1 ints) always, its columns and values when nnz(C) <=
 * capacity.  Page-locked arrays receive the DMA directly; pageable ones go
 * through the context's staging buffers.  *nnz_c receives nnz(C); when it
 * exceeds capacity nothing else is written and the call returns
 * RTT_ERR_INVALID_ARGUMENT (grow the arrays to *nnz_c and call again). */
RTT_API int rtt_spgemm_csr_host_into(rtt_context ctx, const SMatrix *A, const SMatrix *B, int op,
                                     int *c_row_ptr, int *c_col_idx, double *c_values,
                                     long long capacity, long long *nnz_c);

/* Batched form (no single reference function: it batches the device path
 * above over independent products, many SpGEMMs of uneven sizes in one
 * pipeline run).  count products C_i = A_i * B_i (B == NULL: C_i =
 * A_i^2, A_i square), device CSR views in; all instances run through ONE
 * csr2tile, ONE symbolic and ONE numeric pass over their block diagonal
 * (every instance padded to a multiple of 16 rows and columns).
 * nnz_c[i] receives nnz(C_i); *nnz_total their sum.  A and B stay borrowed
 * until rtt_spgemm_batched_numeric returns.  Limits: the padded totals and
 * the total nnz must fit int32 (else RTT_ERR_UNREPRESENTABLE). */
RTT_API int rtt_spgemm_batched_symbolic(rtt_context ctx, int count, const rtt_csr_view *A,
                                        const rtt_csr_view *B, long long *nnz_c,
                                        long long *nnz_total);

/* Device CSR transpose (A^T of a device CSR view into caller-owned device
 * arrays of A->cols + 1 and A->nnz entries; rows sorted).  The serving loop
 * uses it to turn A*A^T requests into A*B instances of one batch. */
RTT_API int rtt_csr_transpose(rtt_context ctx, const rtt_csr_view *A, int *t_row_ptr,
                              int *t_col_idx, double *t_values);

/* Stages of a reorder plan: the reference's DmmaReorderVariant ablations
 * (src/dmma_reorder.h:63-71, resolved as at :123-137). */
enum
{
    RTT_REORDER_FULL = 0,         /* coarse traversal, then the row and inner fine passes */
    RTT_REORDER_COARSE = 1,       /* the coarse traversal only */
    RTT_REORDER_FINE = 2,         /* the fine passes only, from A's own order */
    RTT_REORDER_COARSE_ROW = 3,   /* coarse, then the row fine pass */
    RTT_REORDER_COARSE_INNER = 4, /* coarse, then the inner fine pass */
    RTT_REORDER_UNGUARDED = 5     /* every stage's proposal taken without the exact rule */
};

/* Replaces build_dmma_reorder_plan (src/dmma_reorder.h:2651) for a device CSR
 * A, in the stages of RTT_REORDER_FULL:
 *  1. coarse: a bipartite Cuthill-McKee traversal of A's rows and columns
 *     proposes a joint row / K order, committed only if it cuts A's distinct
 *     8x4 tiles (the exact commit rule, :1671-1727);
 *  2. row fine pass (:2865-2920): in each window of 32 consecutive rows,
 *     rows are packed into groups of 8 - an anchor (most entries, widest
 *     fingerprint of 4-column panels, leftmost panel...), then the rows
 *     adding the fewest new panel bits to the group's fingerprint - and a
 *     window's packing is committed only if it has fewer 8x4 tiles, or as
 *     many and a smaller fan-out (:1841-1887);
 *  3. inner fine pass (:2922-2990): the same over windows of 16 inner
 *     indices in groups of 4, against 8-row panels.
 * Every committed step keeps or cuts the tile count, so the plan never has
 * more 8x4 tiles than A.  The traversal's permutations are this build's
 * (not BGRF-v1's); the fine passes follow the reference's rules with this
 * build's fingerprint hash.  With A' = P A Q^T and B' = Q B, C' = A' B' =
 * P C.  Uses the context's tile buffers as scratch (a following product
 * starts with rtt_spgemm_symbolic). */
RTT_API int rtt_reorder_plan_build(rtt_context ctx, const rtt_csr_view *A, rtt_reorder_plan *plan);
/* The same with the stages of variant (RTT_REORDER_*). */
RTT_API int rtt_reorder_plan_build_variant(rtt_context ctx, const rtt_csr_view *A, int variant,
                                           rtt_reorder_plan *plan);
RTT_API void rtt_reorder_plan_destroy(rtt_reorder_plan *plan);

/* Replaces dump_dmma_reorder_plan (src/dmma_reorder.h:3087-3209): writes
 * <stem>_permutations.csv (axis,old_id,new_id,new_to_old_at_new_id for every
 * row and inner index), <stem>_unified_stats.csv (key,value: the plan's
 * counters) and, when dump_matrix != 0, <stem>_A_reordered.mtx (A's pattern
 * under the plan, from A's device row pointer and columns). */
RTT_API int rtt_reorder_plan_dump(const rtt_reorder_plan *plan, const char *stem,
                                  const int *d_row_ptr, const int *d_col_idx, int dump_matrix);

/* Tile-layout heatmap (the role of export_diagnostic_heatmaps,
 * src/super16_symbolic.cuh:2034, for this build's 16x16 tiles): the tiles of
 * A (which = 0), B (1) or C (2) of the last symbolic phase on ctx, counted on
 * a bins x bins grid over the tile grid (tile (I, J) -> bin (I * bins /
 * tilem, J * bins / tilen)); hist is a host array of bins * bins counts, row
 * major.  1 <= bins <= 4096.  After rtt_spgemm_symbolic64, C is the last
 * chunk's. */
RTT_API int rtt_tile_heatmap(rtt_context ctx, int which, int bins, unsigned long long *hist);

/* Device CSR permutation: out row i = A row row_new_to_old[i] (NULL: i), each
 * column c replaced by col_old_to_new[c] (NULL: c) and every row sorted by
 * its new columns (stable).  Maps are device arrays and must be
 * permutations (else RTT_ERR_DEVICE_CHECK); out_row_ptr has A->rows + 1
 * entries, out_col_idx / out_values A->nnz. */
RTT_API int rtt_csr_permute(rtt_context ctx, const rtt_csr_view *A, const int *row_new_to_old,
                            const int *col_old_to_new, int *out_row_ptr, int *out_col_idx,
                            double *out_values);

/* Writes the products of the last batched symbolic.  c_row_ptr: the
 * instances' row pointers one after another (instance i's A_i.rows + 1
 * entries, starting at 0, at offset sum_{j<i} (A_j.rows + 1)); c_col_idx /
 * c_values: nnz_total entries, instance i's at offset sum_{j<i} nnz_c[j], with
 * columns local to the instance.  Work is queued on the context's stream. */
RTT_API int rtt_spgemm_batched_numeric(rtt_context ctx, int *c_row_ptr, int *c_col_idx,
                                       double *c_values);

/* Values-only update of the last batch (Galerkin products, time steps: the
 * same instances' structures, new values): a_values[i] holds instance i's
 * new A values in its CSR order (b_values[i] its B values, or b_values ==
 * NULL to keep B's, which a batch of A_i^2 takes from A).  The values are
 * gathered into the block diagonal on the device, its tiles refilled and the
 * numeric step run as in rtt_spgemm_batched_numeric (same outputs); neither
 * csr2tile's counting nor the symbolic phase runs again, and a repeated call
 * replays a CUDA graph (rtt_config.cuda_graphs). */
RTT_API int rtt_spgemm_batched_numeric_values(rtt_context ctx, const double *const *a_values,
                                              const double *const *b_values, int *c_row_ptr,
                                              int *c_col_idx, double *c_values);

#ifdef __cplusplus
}
#endif

#endif /* RTT_SPGEMM_H_ */
