/*
 * ref_tiles.cpp - C entry points over the reference's own CPU code.
 *
 * TEST INFRASTRUCTURE ONLY.  This translation unit contains no algorithm: it
 * #includes the unmodified headers of for-the-juan/RTT-SpGEMM where they lie
 * (the Makefile passes -I <reference>/src) and exposes their functions with C
 * linkage for the oracle tests:
 *   csr2tile_row_major / csr2tile_col_major  src/csr2tile.h:196, :261
 *   spgemm_cpu                               src/spgemm-cpu.h:369
 *   tile2csr / tile2csr_restore_rows         src/tile2csr.h:232, :337
 *   spgemm_spa (structure, OpenMP)           src/spgemm_serialref_spa_new.h:7
 *   csr_to_hybrid_tiles                      src/dmma_tiles.h:243
 *   dmma_plan_tile_tail_queue                src/dmma_tile_tail_queue.h:190
 *   dmma_plan_tile_early_split               src/dmma_tile_early_split.h:152
 *   mmio_allinone (Matrix Market reader)     src/mmio_highlevel.h:593
 * The output is built into oracle/_ref/ and never shipped with the product.
 */
#include <unistd.h>
#include <fcntl.h>
#include <cstdio>

#include "common.h"
#include "csr2tile.h"
#include "spgemm-cpu.h"
#include "tile2csr.h"
#include "dmma_tile_tail_queue.h"
#include "dmma_tile_early_split.h"
#include "spgemm_serialref_spa_new.h"
#include "mmio_highlevel.h"

namespace
{
/* spgemm_cpu reports progress with printf; keep it off the test's stdout. */
struct QuietStdout
{
    int saved = -1;
    QuietStdout()
    {
        std::fflush(stdout);
        saved = dup(STDOUT_FILENO);
        int devnull = open("/dev/null", O_WRONLY);
        if (devnull >= 0)
        {
            dup2(devnull, STDOUT_FILENO);
            close(devnull);
        }
    }
    ~QuietStdout()
    {
        std::fflush(stdout);
        if (saved >= 0)
        {
            dup2(saved, STDOUT_FILENO);
            close(saved);
        }
    }
};
} // namespace

extern "C" {

void ref_csr2tile_row_major(SMatrix *m) { csr2tile_row_major(m); }

void ref_csr2tile_col_major(SMatrix *m) { csr2tile_col_major(m); }

/* spgemm_cpu with the in-tile column fix applied at the call site: A's packed
 * (row << 4) | col bytes are handed over as plain columns (byte & 0xF).  The
 * reference function itself runs unmodified. */
void ref_spgemm_cpu_fixed(SMatrix *A, SMatrix *B, SMatrix *C)
{
    unsigned char *packed = A->tile_csr_Col;
    unsigned char *plain = (unsigned char *)malloc(A->nnz > 0 ? A->nnz : 1);
    for (int i = 0; i < A->nnz; ++i)
        plain[i] = packed[i] & 0xF;
    A->tile_csr_Col = plain;
    {
        QuietStdout quiet;
        spgemm_cpu(A, B, C);
    }
    A->tile_csr_Col = packed;
    free(plain);
}

int ref_tile2csr(SMatrix *m, int canonical) { return tile2csr(m, canonical != 0) ? 1 : 0; }

int ref_tile2csr_restore_rows(SMatrix *m, const int *new_to_old, int size, int canonical)
{
    return tile2csr_restore_rows(m, new_to_old, size, canonical != 0) ? 1 : 0;
}

int ref_output_tile_rows(void) { return OUTPUT_TILE_ROWS; }

void ref_spgemm_spa_structure(const int *rpA, const int *ciA, int mA, int nA, int nnzA,
                              const int *rpB, const int *ciB, int mB, int nB, int nnzB,
                              int *rpC, int *ciC, int *nnzC, int count_only)
{
    spgemm_spa(rpA, ciA, nullptr, mA, nA, nnzA, rpB, ciB, nullptr, mB, nB, nnzB,
               rpC, ciC, nullptr, mA, nB, nnzC, count_only ? 1 : 0);
}

/* csr_to_hybrid_tiles flattened into caller-visible arrays (malloc'd). */
struct ref_hybrid
{
    int rows, cols, tile_rows, tile_cols, tile_row_count, tile_col_count;
    int num_tiles, payload_size, dense_tiles, sparse_tiles;
    int *tile_row_ptr;
    int *tile_col_idx;
    int *value_offsets;
    unsigned int *masks;
    double *values;
    int *tile_col_ptr;
    int *tile_row_idx;
    int *csc_tile_ids;
};

int ref_csr_to_hybrid_tiles(const SMatrix *csr, int tile_rows, int tile_cols, int col_major,
                            int dense_threshold, int build_csc, ref_hybrid *out)
{
    HybridTileMatrix h;
    if (!csr_to_hybrid_tiles(csr, tile_rows, tile_cols, col_major != 0, dense_threshold,
                             build_csc != 0, &h))
        return 0;
    out->rows = h.rows;
    out->cols = h.cols;
    out->tile_rows = h.tile_rows;
    out->tile_cols = h.tile_cols;
    out->tile_row_count = h.tile_row_count;
    out->tile_col_count = h.tile_col_count;
    out->num_tiles = h.num_tiles;
    out->payload_size = h.payload_size;
    out->dense_tiles = h.dense_tiles;
    out->sparse_tiles = h.sparse_tiles;
    out->tile_row_ptr = h.tile_row_ptr;
    out->tile_col_idx = h.tile_col_idx;
    out->value_offsets = h.value_offsets;
    out->masks = h.masks;
    out->values = h.values;
    out->tile_col_ptr = h.tile_col_ptr;
    out->tile_row_idx = h.tile_row_idx;
    out->csc_tile_ids = h.csc_tile_ids;
    return 1;
}

/* Tail-queue planner: tasks as flat arrays; returns the gate reason and
 * writes the admitted chunk count per task (0 = ordinary). */
int ref_plan_tile_tail_queue(int ntasks, const int *scans, const int *matches, const int *out_nnz,
                             double admission_threshold, double chunk_target, int max_chunks,
                             double max_heavy_fraction, int record_capacity,
                             long long workspace_limit_bytes, int workspace_reduction,
                             double m_intercept, double m_scan, double m_match, double m_output,
                             int *chunks_out, long long *summary)
{
    std::vector<DmmaTileTailQueueExactTask> tasks((size_t)ntasks);
    for (int i = 0; i < ntasks; ++i)
    {
        tasks[(size_t)i].task = i;
        tasks[(size_t)i].scans = scans[i];
        tasks[(size_t)i].matches = matches[i];
        tasks[(size_t)i].output_nnz = out_nnz[i];
    }
    DmmaTileTailQueuePolicy policy;
    policy.enabled = true;
    policy.admission_threshold = admission_threshold;
    policy.chunk_target = chunk_target;
    policy.max_chunks = max_chunks;
    policy.max_heavy_fraction = max_heavy_fraction;
    policy.record_capacity = record_capacity;
    policy.workspace_limit_bytes = (std::size_t)workspace_limit_bytes;
    policy.workspace_reduction = workspace_reduction != 0;
    DmmaTileTailQueueCostModel model;
    model.intercept = m_intercept;
    model.scan = m_scan;
    model.match = m_match;
    model.output = m_output;
    DmmaTileTailQueuePlan plan = dmma_plan_tile_tail_queue(tasks, policy, model);
    for (int i = 0; i < ntasks; ++i)
        chunks_out[i] = 0;
    for (const auto &h : plan.heavy)
        chunks_out[h.task] = h.chunks;
    summary[0] = (long long)plan.heavy_tasks;
    summary[1] = (long long)plan.chunks;
    summary[2] = (long long)plan.descriptor_bytes;
    summary[3] = (long long)plan.partial_workspace_bytes;
    summary[4] = (long long)plan.heavy_flag_bytes;
    return (int)plan.reason;
}

/* Early-split planner: same task arrays; returns the gate reason and writes
 * the admitted chunk count per task, summary = {base reason, ordinary,
 * heavy, chunks, cap, heavy workers, reduction workers, descriptor bytes,
 * heavy flag bytes, partial workspace bytes, exact parent partition}. */
int ref_plan_tile_early_split(int ntasks, const int *scans, const int *matches,
                              const int *out_nnz, int enabled, double admission_threshold,
                              double chunk_target, int max_chunks, double max_heavy_fraction,
                              int record_capacity, long long workspace_limit_bytes,
                              int workspace_reduction, double m_intercept, double m_scan,
                              double m_match, double m_output, int sm_count, int *chunks_out,
                              long long *summary)
{
    std::vector<DmmaTileTailQueueExactTask> tasks((size_t)ntasks);
    for (int i = 0; i < ntasks; ++i)
    {
        tasks[(size_t)i].task = i;
        tasks[(size_t)i].scans = scans[i];
        tasks[(size_t)i].matches = matches[i];
        tasks[(size_t)i].output_nnz = out_nnz[i];
    }
    DmmaTileEarlySplitPolicy policy;
    policy.enabled = enabled != 0;
    policy.admission_threshold = admission_threshold;
    policy.chunk_target = chunk_target;
    policy.max_chunks = max_chunks;
    policy.max_heavy_fraction = max_heavy_fraction;
    policy.record_capacity = record_capacity;
    policy.workspace_limit_bytes = (std::size_t)workspace_limit_bytes;
    policy.workspace_reduction = workspace_reduction != 0;
    DmmaTileTailQueueCostModel model;
    model.intercept = m_intercept;
    model.scan = m_scan;
    model.match = m_match;
    model.output = m_output;
    DmmaTileEarlySplitPlan plan = dmma_plan_tile_early_split(tasks, policy, model, sm_count);
    for (int i = 0; i < ntasks; ++i)
        chunks_out[i] = 0;
    for (const auto &h : plan.heavy)
        chunks_out[h.task] = h.chunks;
    summary[0] = (long long)plan.base_reason;
    summary[1] = (long long)plan.ordinary_tasks;
    summary[2] = (long long)plan.heavy_tasks;
    summary[3] = (long long)plan.chunks;
    summary[4] = (long long)plan.global_heavy_worker_block_cap;
    summary[5] = (long long)plan.heavy_worker_blocks;
    summary[6] = (long long)plan.reduction_worker_blocks;
    summary[7] = (long long)plan.descriptor_bytes;
    summary[8] = (long long)plan.heavy_flag_bytes;
    summary[9] = (long long)plan.partial_workspace_bytes;
    summary[10] = plan.exact_parent_partition ? 1 : 0;
    return (int)plan.reason;
}

/* mmio_allinone (src/mmio_highlevel.h:593-760): Matrix Market file -> CSR */
int ref_mmio_allinone(const char *path, int *m, int *n, int *nnz, int *is_sym, int **rowptr,
                      int **col, double **val)
{
    QuietStdout quiet;
    return mmio_allinone(m, n, nnz, is_sym, rowptr, col, val, const_cast<char *>(path));
}

void ref_free(void *p) { free(p); }

} /* extern "C" */
