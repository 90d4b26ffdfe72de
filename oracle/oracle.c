/*
 * oracle.c - CPU restatement of the reference's tiled SpGEMM path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library under
 * rtt-spgemm_b200/) links, loads or calls this file; only tests/, the smoke
 * check and bench.py's CPU-baseline leg do, as the checker.
 *
 * Each function restates one reference function of for-the-juan/RTT-SpGEMM
 * (file:line cited at the function) in plain C + OpenMP.  Semantics are kept
 * bit-for-bit, with two documented departures:
 *   - orc_spgemm_tile masks A's packed in-tile column byte with 0xF.  The
 *     reference spgemm_cpu uses the packed byte (row << 4) | col directly as
 *     a column (src/spgemm-cpu.h:231, :324); that is wrong for every A row
 *     but row 0 and reads other tiles' row pointers.
 *   - orc_spgemm_tile finds the C tiles of a tile row by a union over B's
 *     tile rows instead of testing every (A tile row, B tile column) pair
 *     (src/spgemm-cpu.h:3-96).  Both yield the same set in the same order:
 *     C(I,J) exists iff some K has A(I,K) and B(K,J).
 * The reference's step-3 row-length quirk (src/spgemm-cpu.h:206, :232: the
 * last B row of a tile is taken as C's column-tile width) is reproducible
 * with ref_step3_quirk = 1 so that the restatement can be pinned against the
 * reference on ragged shapes too; the default (0) is the intended semantics,
 * which is what step 4 of the reference computes.
 *
 * Floating point: products and sums are separate IEEE operations in the
 * reference's order; build with -ffp-contract=off so no FMA is formed.
 */
#include "rtt_spgemm.h"

#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <omp.h>

#define TD 16

static int ceil_div(int a, int b) { return a / b + (a % b != 0 ? 1 : 0); }

static void *xcalloc(size_t count, size_t size)
{
    /* calloc(0, ...) may return NULL; keep every array non-NULL. */
    return calloc(count ? count : 1, size ? size : 1);
}

/* Basic CSR validation, mirroring validate_csr (src/dmma_tiles.h:126-161). */
int orc_validate_csr(int m, int n, int nnz, const int *rowptr, const int *col)
{
    if (m < 0 || n < 0 || nnz < 0)
        return 0;
    if (m == 0)
        return nnz == 0;
    if (rowptr == NULL || rowptr[0] != 0 || rowptr[m] != nnz)
        return 0;
    for (int i = 0; i < m; ++i)
        if (rowptr[i + 1] < rowptr[i])
            return 0;
    for (int j = 0; j < nnz; ++j)
        if (col[j] < 0 || col[j] >= n)
            return 0;
    return 1;
}

/* ------------------------------------------------------------------------
 * csr2tile_row_major (src/csr2tile.h:196-259, steps at :6-194).
 * Per tile row: the distinct column tiles (ascending), per-tile per-row
 * counts, then entries placed row by row in CSR order.
 * ------------------------------------------------------------------------ */
int orc_csr2tile_row_major(SMatrix *mat)
{
    const int m = mat->m, n = mat->n, nnz = mat->nnz;
    if (!orc_validate_csr(m, n, nnz, mat->rowpointer, mat->columnindex))
        return RTT_ERR_INVALID_CSR;
    const int tilem = ceil_div(m, TD), tilen = ceil_div(n, TD);
    const int *rp = mat->rowpointer, *ci = mat->columnindex;
    const double *val = mat->value;

    int *tile_ptr = (int *)xcalloc((size_t)tilem + 1, sizeof(int));
    /* step 1: number of tiles per tile row (:6-39) */
#pragma omp parallel
    {
        char *flag = (char *)xcalloc((size_t)tilen, 1);
#pragma omp for schedule(dynamic, 64)
        for (int I = 0; I < tilem; ++I)
        {
            int r0 = I * TD, r1 = I == tilem - 1 ? m : (I + 1) * TD;
            int cnt = 0;
            for (int j = rp[r0]; j < rp[r1]; ++j)
            {
                int J = ci[j] / TD;
                if (!flag[J])
                {
                    flag[J] = 1;
                    ++cnt;
                }
            }
            for (int j = rp[r0]; j < rp[r1]; ++j)
                flag[ci[j] / TD] = 0;
            tile_ptr[I] = cnt;
        }
        free(flag);
    }
    /* exclusive scan (src/utils.h:33-48) */
    {
        int run = 0;
        for (int I = 0; I <= tilem; ++I)
        {
            int c = I < tilem ? tile_ptr[I] : 0;
            tile_ptr[I] = run;
            run += c;
        }
    }
    const int numtile = tile_ptr[tilem];
    int *tile_col = (int *)xcalloc((size_t)numtile, sizeof(int));
    int *tile_row = (int *)xcalloc((size_t)numtile, sizeof(int));
    int *tile_nnz = (int *)xcalloc((size_t)numtile + 1, sizeof(int));
    unsigned char *Ptr = (unsigned char *)xcalloc((size_t)numtile * TD, 1);
    unsigned char *Col = (unsigned char *)xcalloc((size_t)nnz, 1);
    double *Val = (double *)xcalloc((size_t)nnz, sizeof(double));
    unsigned short *mask = (unsigned short *)xcalloc((size_t)numtile * TD, sizeof(unsigned short));

    /* steps 2 + 3 per tile row (:43-110, :112-194) */
#pragma omp parallel
    {
        int *slot = (int *)xcalloc((size_t)tilen, sizeof(int)); /* J -> local index + 1 */
#pragma omp for schedule(dynamic, 64)
        for (int I = 0; I < tilem; ++I)
        {
            int r0 = I * TD, r1 = I == tilem - 1 ? m : (I + 1) * TD;
            int t0 = tile_ptr[I], nt = tile_ptr[I + 1] - t0;
            if (nt == 0)
                continue;
            /* ascending distinct J (step2 walks blkj = 0..tilen-1) */
            int k = 0;
            for (int j = rp[r0]; j < rp[r1]; ++j)
            {
                int J = ci[j] / TD;
                if (!slot[J])
                {
                    slot[J] = 1;
                    tile_col[t0 + k++] = J;
                }
            }
            /* insertion sort of the (small) tile list */
            for (int a = 1; a < nt; ++a)
            {
                int v = tile_col[t0 + a], b = a - 1;
                while (b >= 0 && tile_col[t0 + b] > v)
                {
                    tile_col[t0 + b + 1] = tile_col[t0 + b];
                    --b;
                }
                tile_col[t0 + b + 1] = v;
            }
            for (int a = 0; a < nt; ++a)
            {
                slot[tile_col[t0 + a]] = a + 1;
                tile_row[t0 + a] = I;
            }
            /* per-tile per-row counts */
            int *cnt = (int *)xcalloc((size_t)nt * TD, sizeof(int));
            for (int r = r0; r < r1; ++r)
                for (int j = rp[r]; j < rp[r + 1]; ++j)
                    cnt[(slot[ci[j] / TD] - 1) * TD + (r - r0)]++;
            int *tot = (int *)xcalloc((size_t)nt, sizeof(int));
            for (int a = 0; a < nt; ++a)
            {
                unsigned char run = 0; /* exclusive_scan_char keeps u8 arithmetic */
                int t = 0;
                for (int r = 0; r < TD; ++r)
                {
                    Ptr[(size_t)(t0 + a) * TD + r] = run;
                    run = (unsigned char)(run + (unsigned char)cnt[a * TD + r]);
                    t += cnt[a * TD + r];
                }
                tot[a] = t;
                tile_nnz[t0 + a] = t; /* scanned below */
            }
            free(cnt);
            free(tot);
            for (int a = 0; a < nt; ++a)
                slot[tile_col[t0 + a]] = 0;
        }
        free(slot);
    }
    {
        int run = 0;
        for (int t = 0; t <= numtile; ++t)
        {
            int c = t < numtile ? tile_nnz[t] : 0;
            tile_nnz[t] = run;
            run += c;
        }
    }
    /* place entries: tile base + row offset + rank within (tile,row) in CSR order */
#pragma omp parallel
    {
        int *slot = (int *)xcalloc((size_t)tilen, sizeof(int));
#pragma omp for schedule(dynamic, 64)
        for (int I = 0; I < tilem; ++I)
        {
            int r0 = I * TD, r1 = I == tilem - 1 ? m : (I + 1) * TD;
            int t0 = tile_ptr[I], nt = tile_ptr[I + 1] - t0;
            for (int a = 0; a < nt; ++a)
                slot[tile_col[t0 + a]] = a + 1;
            for (int r = r0; r < r1; ++r)
            {
                int ri = r - r0;
                int fill[64];
                int *cursor = nt <= 64 ? fill : (int *)xcalloc((size_t)nt, sizeof(int));
                for (int a = 0; a < nt; ++a)
                    cursor[a] = 0;
                /* the row offset is the exact count of earlier rows (int),
                   the reference stores it as u8 but indexes with the int
                   exclusive prefix of its own u8 array; for tiles of <= 255
                   entries per prefix the two agree. */
                for (int j = rp[r]; j < rp[r + 1]; ++j)
                {
                    int a = slot[ci[j] / TD] - 1;
                    int t = t0 + a;
                    int dst = tile_nnz[t] + Ptr[(size_t)t * TD + ri] + cursor[a]++;
                    int c = ci[j] - (ci[j] / TD) * TD;
                    Col[dst] = (unsigned char)((ri << 4) + c);
                    Val[dst] = val[j];
                    mask[(size_t)t * TD + ri] |= (unsigned short)(1u << (TD - c - 1));
                }
                if (cursor != fill)
                    free(cursor);
            }
            for (int a = 0; a < nt; ++a)
                slot[tile_col[t0 + a]] = 0;
        }
        free(slot);
    }
    mat->tilem = tilem;
    mat->tilen = tilen;
    mat->numtile = numtile;
    mat->tile_ptr = tile_ptr;
    mat->tile_columnidx = tile_col;
    mat->tile_rowidx = tile_row;
    mat->tile_nnz = tile_nnz;
    mat->tile_csr_Ptr = Ptr;
    mat->tile_csr_Col = Col;
    mat->tile_csr_Value = Val;
    mat->mask = mask;
    return RTT_OK;
}

/* ------------------------------------------------------------------------
 * csr2tile_col_major (src/csr2tile.h:261-478).
 * Tile structure of the matrix itself (tile_ptr, tile_columnidx), tile CSC
 * (csc_tile_ptr, csc_tile_rowidx) and, in tile-CSC order, per-tile CSR with
 * rows in order, columns ascending within a row (duplicates stay in CSR
 * order: both transpositions are stable), plain column bytes, rows past a
 * partial tile padded with the tile count.  tile_rowidx is allocated zeroed
 * and never written, as in the reference.
 * ------------------------------------------------------------------------ */
typedef struct
{
    int row, col, src;
} orc_entry;

static int entry_cmp_colmajor(const void *x, const void *y)
{
    const orc_entry *a = (const orc_entry *)x, *b = (const orc_entry *)y;
    int ta = a->col / TD, tb = b->col / TD;
    if (ta != tb)
        return ta < tb ? -1 : 1;
    int ra = a->row / TD, rb = b->row / TD;
    if (ra != rb)
        return ra < rb ? -1 : 1;
    if (a->row != b->row)
        return a->row < b->row ? -1 : 1;
    if (a->col != b->col)
        return a->col < b->col ? -1 : 1;
    return a->src < b->src ? -1 : (a->src > b->src);
}

int orc_csr2tile_col_major(SMatrix *mat)
{
    const int m = mat->m, n = mat->n, nnz = mat->nnz;
    if (!orc_validate_csr(m, n, nnz, mat->rowpointer, mat->columnindex))
        return RTT_ERR_INVALID_CSR;
    const int tilem = ceil_div(m, TD), tilen = ceil_div(n, TD);
    const int *rp = mat->rowpointer, *ci = mat->columnindex;

    /* row-major tile structure (:310-370) */
    SMatrix tmp;
    memset(&tmp, 0, sizeof(tmp));
    tmp.m = m;
    tmp.n = n;
    tmp.nnz = nnz;
    tmp.rowpointer = mat->rowpointer;
    tmp.columnindex = mat->columnindex;
    tmp.value = mat->value;
    int st = orc_csr2tile_row_major(&tmp);
    if (st != RTT_OK)
        return st;
    const int numtile = tmp.numtile;

    /* entries sorted by (tile col, tile row, row, col, CSR position) */
    orc_entry *e = (orc_entry *)xcalloc((size_t)nnz, sizeof(orc_entry));
    for (int r = 0; r < m; ++r)
        for (int j = rp[r]; j < rp[r + 1]; ++j)
        {
            e[j].row = r;
            e[j].col = ci[j];
            e[j].src = j;
        }
    qsort(e, (size_t)nnz, sizeof(orc_entry), entry_cmp_colmajor);

    int *csc_ptr = (int *)xcalloc((size_t)tilen + 1, sizeof(int));
    int *csc_row = (int *)xcalloc((size_t)numtile, sizeof(int));
    int *tile_nnz = (int *)xcalloc((size_t)numtile + 1, sizeof(int));
    unsigned char *Ptr = (unsigned char *)xcalloc((size_t)numtile * TD, 1);
    unsigned char *Col = (unsigned char *)xcalloc((size_t)nnz, 1);
    double *Val = (double *)xcalloc((size_t)nnz, sizeof(double));
    unsigned short *mask = (unsigned short *)xcalloc((size_t)numtile * TD, sizeof(unsigned short));

    int t = -1, curJ = -1, curR = -1;
    for (int p = 0; p < nnz; ++p)
    {
        int J = e[p].col / TD, R = e[p].row / TD;
        if (J != curJ || R != curR)
        {
            ++t;
            curJ = J;
            curR = R;
            csc_ptr[J + 1]++;
            csc_row[t] = R;
            tile_nnz[t] = p; /* exclusive offset of this tile */
        }
        int ri = e[p].row - R * TD, c = e[p].col - J * TD;
        Col[p] = (unsigned char)c;
        Val[p] = mat->value[e[p].src];
        mask[(size_t)t * TD + ri] |= (unsigned short)(1u << (TD - c - 1));
    }
    tile_nnz[numtile] = nnz;
    for (int J = 0; J < tilen; ++J)
        csc_ptr[J + 1] += csc_ptr[J];
    /* per-tile row offsets; rows past the tile's height get the tile count */
    for (int tt = 0; tt < numtile; ++tt)
    {
        int R = csc_row[tt];
        int height = R == tilem - 1 ? m - (tilem - 1) * TD : TD;
        int cnt[TD] = {0};
        for (int p = tile_nnz[tt]; p < tile_nnz[tt + 1]; ++p)
            cnt[e[p].row - R * TD]++;
        int run = 0;
        for (int r = 0; r < TD; ++r)
        {
            if (r < height)
            {
                Ptr[(size_t)tt * TD + r] = (unsigned char)run;
                run += cnt[r];
            }
            else
                Ptr[(size_t)tt * TD + r] = (unsigned char)run;
        }
    }
    free(e);
    free(tmp.tile_nnz);
    free(tmp.tile_csr_Ptr);
    free(tmp.tile_csr_Col);
    free(tmp.tile_csr_Value);
    free(tmp.mask);
    free(tmp.tile_rowidx);

    mat->tilem = tilem;
    mat->tilen = tilen;
    mat->numtile = numtile;
    mat->tile_ptr = tmp.tile_ptr;
    mat->tile_columnidx = tmp.tile_columnidx;
    mat->tile_rowidx = (int *)xcalloc((size_t)numtile, sizeof(int));
    mat->tile_nnz = tile_nnz;
    mat->csc_tile_ptr = csc_ptr;
    mat->csc_tile_rowidx = csc_row;
    mat->tile_csr_Ptr = Ptr;
    mat->tile_csr_Col = Col;
    mat->tile_csr_Value = Val;
    mat->mask = mask;
    return RTT_OK;
}

/* ------------------------------------------------------------------------
 * spgemm_cpu (src/spgemm-cpu.h:369-455): steps 1-2 (C tile structure),
 * step 3 (structural nnz per C tile, :185-281), step 4 (values, :284-367).
 * A: row-major tiles.  B: column-major tiles (csc_tile_ptr/csc_tile_rowidx
 * index its per-tile arrays).
 * ------------------------------------------------------------------------ */
int orc_spgemm_tile(const SMatrix *A, const SMatrix *B, SMatrix *C, int ref_step3_quirk)
{
    if (A == NULL || B == NULL || C == NULL)
        return RTT_ERR_INVALID_ARGUMENT;
    if (A->n != B->m)
        return RTT_ERR_SHAPE_MISMATCH;
    const int tilemA = A->tilem, tilenB = B->tilen, mA = A->m, nB = B->n;
    const int *aptr = A->tile_ptr, *acol = A->tile_columnidx, *annz = A->tile_nnz;
    const int *bcp = B->csc_tile_ptr, *brow = B->csc_tile_rowidx, *bnnz = B->tile_nnz;
    const unsigned char *aP = A->tile_csr_Ptr, *aC = A->tile_csr_Col;
    const unsigned char *bP = B->tile_csr_Ptr, *bC = B->tile_csr_Col;
    const double *aV = A->tile_csr_Value, *bV = B->tile_csr_Value;
    const int tilemB = B->tilem;

    /* B tile rows from its tile CSC (transpose of the tile structure) */
    int nb = bcp[tilenB];
    int *brp = (int *)xcalloc((size_t)tilemB + 1, sizeof(int));
    int *bcolJ = (int *)xcalloc((size_t)nb, sizeof(int));
    for (int p = 0; p < nb; ++p)
        brp[brow[p] + 1]++;
    for (int K = 0; K < tilemB; ++K)
        brp[K + 1] += brp[K];
    {
        int *cur = (int *)xcalloc((size_t)tilemB + 1, sizeof(int));
        memcpy(cur, brp, sizeof(int) * (size_t)tilemB);
        for (int J = 0; J < tilenB; ++J)
            for (int p = bcp[J]; p < bcp[J + 1]; ++p)
                bcolJ[cur[brow[p]]++] = J; /* ascending J within each row */
        free(cur);
    }

    /* steps 1 + 2: C tiles per tile row, ascending columns */
    int *cptr = (int *)xcalloc((size_t)tilemA + 1, sizeof(int));
#pragma omp parallel
    {
        char *flag = (char *)xcalloc((size_t)tilenB, 1);
#pragma omp for schedule(dynamic, 16)
        for (int I = 0; I < tilemA; ++I)
        {
            int cnt = 0;
            for (int a = aptr[I]; a < aptr[I + 1]; ++a)
            {
                int K = acol[a];
                for (int q = brp[K]; q < brp[K + 1]; ++q)
                    if (!flag[bcolJ[q]])
                    {
                        flag[bcolJ[q]] = 1;
                        ++cnt;
                    }
            }
            for (int a = aptr[I]; a < aptr[I + 1]; ++a)
            {
                int K = acol[a];
                for (int q = brp[K]; q < brp[K + 1]; ++q)
                    flag[bcolJ[q]] = 0;
            }
            cptr[I] = cnt;
        }
        free(flag);
    }
    {
        long long run = 0;
        for (int I = 0; I <= tilemA; ++I)
        {
            int c = I < tilemA ? cptr[I] : 0;
            cptr[I] = (int)run;
            run += c;
        }
        if (run > 0x7fffffffLL)
        {
            free(brp);
            free(bcolJ);
            free(cptr);
            return RTT_ERR_UNREPRESENTABLE;
        }
    }
    const int numtileC = cptr[tilemA];
    int *ccol = (int *)xcalloc((size_t)numtileC, sizeof(int));
    int *crow = (int *)xcalloc((size_t)numtileC, sizeof(int));
#pragma omp parallel
    {
        char *flag = (char *)xcalloc((size_t)tilenB, 1);
#pragma omp for schedule(dynamic, 16)
        for (int I = 0; I < tilemA; ++I)
        {
            int c0 = cptr[I], k = 0;
            for (int a = aptr[I]; a < aptr[I + 1]; ++a)
            {
                int K = acol[a];
                for (int q = brp[K]; q < brp[K + 1]; ++q)
                    if (!flag[bcolJ[q]])
                    {
                        flag[bcolJ[q]] = 1;
                        ccol[c0 + k++] = bcolJ[q];
                    }
            }
            for (int x = 0; x < k; ++x)
                flag[ccol[c0 + x]] = 0;
            for (int x = 1; x < k; ++x)
            {
                int v = ccol[c0 + x], y = x - 1;
                while (y >= 0 && ccol[c0 + y] > v)
                {
                    ccol[c0 + y + 1] = ccol[c0 + y];
                    --y;
                }
                ccol[c0 + y + 1] = v;
            }
            for (int x = 0; x < k; ++x)
                crow[c0 + x] = I;
        }
        free(flag);
    }
    free(brp);
    free(bcolJ);

    /* steps 3 + 4 per C tile */
    int *cnnz = (int *)xcalloc((size_t)numtileC + 1, sizeof(int));
    unsigned short *cmask = (unsigned short *)xcalloc((size_t)numtileC * TD, sizeof(unsigned short));
    /* structure first (step 3) */
#pragma omp parallel for schedule(dynamic, 256)
    for (int s = 0; s < numtileC; ++s)
    {
        int I = crow[s], J = ccol[s];
        int rowlen = I == tilemA - 1 ? mA - (tilemA - 1) * TD : TD;
        int collen = J == tilenB - 1 ? nB - (tilenB - 1) * TD : TD;
        unsigned short flags[TD] = {0};
        int pa = aptr[I], pb = bcp[J];
        while (pa < aptr[I + 1] && pb < bcp[J + 1])
        {
            int ka = acol[pa], kb = brow[pb];
            if (ka == kb)
            {
                int tna = annz[pa + 1] - annz[pa], tnb = bnnz[pb + 1] - bnnz[pb];
                for (int ri = 0; ri < rowlen; ++ri)
                {
                    int stopa = ri == rowlen - 1 ? tna : aP[(size_t)pa * TD + ri + 1];
                    for (int i = aP[(size_t)pa * TD + ri]; i < stopa; ++i)
                    {
                        int cola = aC[annz[pa] + i] & 0xF;
                        int stopb;
                        if (ref_step3_quirk)
                            stopb = cola == collen - 1 ? tnb : bP[(size_t)pb * TD + cola + 1];
                        else
                            stopb = cola == TD - 1 ? tnb : bP[(size_t)pb * TD + cola + 1];
                        for (int bi = bP[(size_t)pb * TD + cola]; bi < stopb; ++bi)
                            flags[ri] |= (unsigned short)(1u << (TD - 1 - bC[bnnz[pb] + bi]));
                    }
                }
                ++pa;
                ++pb;
            }
            else if (ka < kb)
                ++pa;
            else
                ++pb;
        }
        int cnt = 0;
        for (int r = 0; r < TD; ++r)
            cnt += __builtin_popcount(flags[r]);
        cnnz[s] = cnt;
    }
    {
        long long run = 0;
        for (int s = 0; s <= numtileC; ++s)
        {
            int c = s < numtileC ? cnnz[s] : 0;
            if (run > 0x7fffffffLL)
            {
                free(cptr);
                free(ccol);
                free(crow);
                free(cnnz);
                free(cmask);
                return RTT_ERR_UNREPRESENTABLE;
            }
            cnnz[s] = (int)run;
            run += c;
        }
    }
    const int nnzC = cnnz[numtileC];
    double *cval = (double *)xcalloc((size_t)nnzC, sizeof(double));
    unsigned char *ccolb = (unsigned char *)xcalloc((size_t)nnzC, 1);
    unsigned char *cP = (unsigned char *)xcalloc((size_t)numtileC * TD, 1);
    /* values (step 4): dense 16x16 accumulator, flags, row-major compaction */
#pragma omp parallel for schedule(dynamic, 256)
    for (int s = 0; s < numtileC; ++s)
    {
        int I = crow[s], J = ccol[s];
        int rowlen = I == tilemA - 1 ? mA - (tilemA - 1) * TD : TD;
        double acc[TD * TD];
        char flag[TD * TD];
        memset(acc, 0, sizeof(acc));
        memset(flag, 0, sizeof(flag));
        int pa = aptr[I], pb = bcp[J];
        while (pa < aptr[I + 1] && pb < bcp[J + 1])
        {
            int ka = acol[pa], kb = brow[pb];
            if (ka == kb)
            {
                int tna = annz[pa + 1] - annz[pa], tnb = bnnz[pb + 1] - bnnz[pb];
                for (int ri = 0; ri < TD; ++ri)
                {
                    if (ri == rowlen)
                        break;
                    int stopa = ri == TD - 1 ? tna : aP[(size_t)pa * TD + ri + 1];
                    for (int i = aP[(size_t)pa * TD + ri]; i < stopa; ++i)
                    {
                        int cola = aC[annz[pa] + i] & 0xF;
                        int stopb = cola == TD - 1 ? tnb : bP[(size_t)pb * TD + cola + 1];
                        for (int bi = bP[(size_t)pb * TD + cola]; bi < stopb; ++bi)
                        {
                            int colb = bC[bnnz[pb] + bi];
                            double prod = aV[annz[pa] + i] * bV[bnnz[pb] + bi];
                            acc[ri * TD + colb] = acc[ri * TD + colb] + prod;
                            flag[ri * TD + colb] = 1;
                        }
                    }
                }
                ++pa;
                ++pb;
            }
            else if (ka < kb)
                ++pa;
            else
                ++pb;
        }
        int count = 0;
        for (int ri = 0; ri < TD; ++ri)
        {
            for (int c = 0; c < TD; ++c)
                if (flag[ri * TD + c])
                {
                    cval[cnnz[s] + count] = acc[ri * TD + c];
                    ccolb[cnnz[s] + count] = (unsigned char)c;
                    cmask[(size_t)s * TD + ri] |= (unsigned short)(1u << (TD - 1 - c));
                    ++count;
                }
            if (ri < TD - 1)
                cP[(size_t)s * TD + ri + 1] = (unsigned char)count;
        }
    }
    C->m = A->m;
    C->n = B->n;
    C->tilem = tilemA;
    C->tilen = tilenB;
    C->numtile = numtileC;
    C->nnz = nnzC;
    C->tile_ptr = cptr;
    C->tile_columnidx = ccol;
    C->tile_rowidx = crow;
    C->tile_nnz = cnnz;
    C->tile_csr_Ptr = cP;
    C->tile_csr_Col = ccolb;
    C->tile_csr_Value = cval;
    C->mask = cmask;
    return RTT_OK;
}

/* ------------------------------------------------------------------------
 * tile2csr / tile2csr_restore_rows (src/tile2csr.h:232-329, :337-523) for a
 * square tile edge td (the reference fixes td = 8).
 * ------------------------------------------------------------------------ */
static int t2c_row_count(int tile_row, int m, int td)
{
    long long b = (long long)tile_row * td, rem = (long long)m - b;
    if (rem <= 0)
        return 0;
    return rem < td ? (int)rem : td;
}

static void t2c_bounds(const unsigned char *P, size_t off, int lr, int rc, int tnz, int *s, int *e)
{
    int a = P[off + lr];
    int b = lr + 1 == rc ? tnz : P[off + lr + 1];
    if (a < 0)
        a = 0;
    if (a > tnz)
        a = tnz;
    if (b < a)
        b = a;
    if (b > tnz)
        b = tnz;
    *s = a;
    *e = b;
}

static int t2c_col(int tile_col, unsigned char enc, int n, int td, int *g)
{
    int lc = enc;
    if (lc >= td || tile_col < 0)
        return 0;
    long long c = (long long)tile_col * td + lc;
    if (c < 0 || c >= n)
        return 0;
    *g = (int)c;
    return 1;
}

static void t2c_swap(int *ci, double *v, int x, int y)
{
    int c = ci[x];
    double t = v[x];
    ci[x] = ci[y];
    v[x] = v[y];
    ci[y] = c;
    v[y] = t;
}

/* heap sort of one row by column (tile2csr_sort_rows, :179-223) */
static void t2c_sift(int *ci, double *v, int b, int root, int count)
{
    for (;;)
    {
        int child = root * 2 + 1;
        if (child >= count)
            return;
        if (child + 1 < count && ci[b + child] < ci[b + child + 1])
            ++child;
        if (ci[b + root] >= ci[b + child])
            return;
        t2c_swap(ci, v, b + root, b + child);
        root = child;
    }
}

static void t2c_sort_rows(int m, const int *rp, int *ci, double *v)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int r = 0; r < m; ++r)
    {
        int b = rp[r], cnt = rp[r + 1] - rp[r];
        for (int root = cnt / 2; root > 0; --root)
            t2c_sift(ci, v, b, root - 1, cnt);
        for (int rem = cnt; rem > 1; --rem)
        {
            t2c_swap(ci, v, b, b + rem - 1);
            t2c_sift(ci, v, b, 0, rem - 1);
        }
    }
}

static int t2c_check(const SMatrix *M)
{
    return !(M == NULL || M->m < 0 || M->n < 0 || M->tilem < 0 || M->numtile < 0 ||
             M->tile_ptr == NULL || M->tile_nnz == NULL ||
             (M->numtile > 0 && (M->tile_columnidx == NULL || M->tile_csr_Ptr == NULL)) ||
             (M->nnz > 0 && (M->tile_csr_Col == NULL || M->tile_csr_Value == NULL)));
}

int orc_tile2csr_restore_rows(SMatrix *M, const int *new_to_old, int perm_size, int td, int canonical)
{
    if (!t2c_check(M) || td <= 0 || td > 16)
        return RTT_ERR_INVALID_ARGUMENT;
    const int identity = new_to_old == NULL && perm_size < 0;
    if (!identity)
    {
        if (perm_size < 0 || perm_size > M->m || (perm_size > 0 && new_to_old == NULL))
            return RTT_ERR_INVALID_ARGUMENT;
        char *seen = (char *)xcalloc((size_t)M->m, 1);
        for (int i = 0; i < perm_size; ++i)
        {
            int o = new_to_old[i];
            if (o < 0 || o >= M->m || seen[o])
            {
                free(seen);
                return RTT_ERR_INVALID_PERMUTATION;
            }
            seen[o] = 1;
        }
        free(seen);
    }
    const int m = M->m, n = M->n;
    int *rp = (int *)xcalloc((size_t)m + 1, sizeof(int));
    int tail = 0;
#pragma omp parallel for reduction(| : tail) schedule(dynamic, 64)
    for (int tr = 0; tr < M->tilem; ++tr)
    {
        int rc = t2c_row_count(tr, m, td);
        int cnt[16] = {0};
        for (int t = M->tile_ptr[tr]; t < M->tile_ptr[tr + 1]; ++t)
        {
            int tnz = M->tile_nnz[t + 1] - M->tile_nnz[t], off = M->tile_nnz[t];
            size_t poff = (size_t)t * td;
            for (int lr = 0; lr < rc; ++lr)
            {
                int s, e, g;
                t2c_bounds(M->tile_csr_Ptr, poff, lr, rc, tnz, &s, &e);
                for (int x = s; x < e; ++x)
                    if (t2c_col(M->tile_columnidx[t], M->tile_csr_Col[off + x], n, td, &g))
                        cnt[lr]++;
            }
        }
        for (int lr = 0; lr < rc; ++lr)
        {
            int row = tr * td + lr;
            if (identity)
                rp[row] = cnt[lr];
            else if (row >= perm_size)
            {
                if (cnt[lr])
                    tail = 1;
            }
            else
                rp[new_to_old[row]] = cnt[lr];
        }
    }
    if (tail)
    {
        free(rp);
        return RTT_ERR_TAIL_NONEMPTY;
    }
    long long run = 0;
    for (int r = 0; r <= m; ++r)
    {
        int c = r < m ? rp[r] : 0;
        rp[r] = (int)run;
        run += c;
    }
    if (run > 0x7fffffffLL)
    {
        free(rp);
        return RTT_ERR_UNREPRESENTABLE;
    }
    const int nnz = rp[m];
    int *ci = (int *)xcalloc((size_t)nnz, sizeof(int));
    double *v = (double *)xcalloc((size_t)nnz, sizeof(double));
#pragma omp parallel for schedule(dynamic, 64)
    for (int tr = 0; tr < M->tilem; ++tr)
    {
        int rc = t2c_row_count(tr, m, td);
        int cur[16] = {0};
        for (int t = M->tile_ptr[tr]; t < M->tile_ptr[tr + 1]; ++t)
        {
            int tnz = M->tile_nnz[t + 1] - M->tile_nnz[t], off = M->tile_nnz[t];
            size_t poff = (size_t)t * td;
            for (int lr = 0; lr < rc; ++lr)
            {
                int row = tr * td + lr;
                int dst_row;
                if (identity)
                    dst_row = row;
                else if (row >= perm_size)
                    continue;
                else
                    dst_row = new_to_old[row];
                int s, e, g;
                t2c_bounds(M->tile_csr_Ptr, poff, lr, rc, tnz, &s, &e);
                for (int x = s; x < e; ++x)
                    if (t2c_col(M->tile_columnidx[t], M->tile_csr_Col[off + x], n, td, &g))
                    {
                        int o = rp[dst_row] + cur[lr]++;
                        ci[o] = g;
                        v[o] = M->tile_csr_Value[off + x];
                    }
            }
        }
    }
    if (!canonical)
        t2c_sort_rows(m, rp, ci, v);
    M->rowpointer = rp;
    M->columnindex = ci;
    M->value = v;
    M->nnz = nnz;
    return RTT_OK;
}

int orc_tile2csr(SMatrix *M, int td, int canonical)
{
    return orc_tile2csr_restore_rows(M, NULL, -1, td, canonical);
}

/* ------------------------------------------------------------------------
 * 16x16 legacy C tiles -> native 8x8 output tiles: the SMatrix layout that
 * dmma_copy_output_to_host exports (src/dmma_spgemm.h:6399-6488) with the
 * per-tile row offsets of dmma_numeric_kernel (:4266-4283).  Empty 8x8
 * quadrants are not emitted.
 * ------------------------------------------------------------------------ */
int orc_tile16_to_tile8(const SMatrix *C, SMatrix *O)
{
    const int m = C->m, n = C->n;
    const int tm8 = ceil_div(m, 8), tn8 = ceil_div(n, 8);
    /* first pass: count tiles and entries per 8-row tile row */
    int *tp = (int *)xcalloc((size_t)tm8 + 1, sizeof(int));
    long long ntile = 0;
    for (int I = 0; I < C->tilem; ++I)
        for (int h = 0; h < 2; ++h)
        {
            int R8 = 2 * I + h;
            if (R8 >= tm8)
                continue;
            int cnt = 0;
            for (int t = C->tile_ptr[I]; t < C->tile_ptr[I + 1]; ++t)
                for (int q = 0; q < 2; ++q)
                {
                    int any = 0;
                    for (int r = 8 * h; r < 8 * h + 8; ++r)
                        if ((C->mask[(size_t)t * TD + r] >> (8 - 8 * q)) & 0xFF)
                            any = 1;
                    cnt += any;
                }
            tp[R8] = cnt;
            ntile += cnt;
        }
    long long run = 0;
    for (int R = 0; R <= tm8; ++R)
    {
        int c = R < tm8 ? tp[R] : 0;
        tp[R] = (int)run;
        run += c;
    }
    int nt = (int)ntile;
    int *tc = (int *)xcalloc((size_t)nt, sizeof(int));
    int *tr = (int *)xcalloc((size_t)nt, sizeof(int));
    int *tn = (int *)xcalloc((size_t)nt + 1, sizeof(int));
    unsigned char *P = (unsigned char *)xcalloc((size_t)nt * 8, 1);
    unsigned char *Cc = (unsigned char *)xcalloc((size_t)(C->nnz), 1);
    double *V = (double *)xcalloc((size_t)(C->nnz), sizeof(double));
    int k = 0, pos = 0;
    for (int I = 0; I < C->tilem; ++I)
        for (int h = 0; h < 2; ++h)
        {
            if (2 * I + h >= tm8)
                continue;
            for (int t = C->tile_ptr[I]; t < C->tile_ptr[I + 1]; ++t)
                for (int q = 0; q < 2; ++q)
                {
                    int any = 0;
                    for (int r = 8 * h; r < 8 * h + 8; ++r)
                        if ((C->mask[(size_t)t * TD + r] >> (8 - 8 * q)) & 0xFF)
                            any = 1;
                    if (!any)
                        continue;
                    tc[k] = 2 * C->tile_columnidx[t] + q;
                    tr[k] = 2 * I + h;
                    tn[k] = pos;
                    int cnt = 0;
                    for (int r = 8 * h; r < 8 * h + 8; ++r)
                    {
                        P[(size_t)k * 8 + (r - 8 * h)] = (unsigned char)cnt;
                        int rs = C->tile_nnz[t] + C->tile_csr_Ptr[(size_t)t * TD + r];
                        int re = r == TD - 1 ? C->tile_nnz[t + 1]
                                             : C->tile_nnz[t] + C->tile_csr_Ptr[(size_t)t * TD + r + 1];
                        for (int x = rs; x < re; ++x)
                        {
                            int c = C->tile_csr_Col[x];
                            if (c >= 8 * q && c < 8 * q + 8)
                            {
                                Cc[pos] = (unsigned char)(c - 8 * q);
                                V[pos] = C->tile_csr_Value[x];
                                ++pos;
                                ++cnt;
                            }
                        }
                    }
                    ++k;
                }
        }
    tn[nt] = pos;
    memset(O, 0, sizeof(*O));
    O->m = m;
    O->n = n;
    O->tilem = tm8;
    O->tilen = tn8;
    O->numtile = nt;
    O->nnz = pos;
    O->tile_ptr = tp;
    O->tile_columnidx = tc;
    O->tile_rowidx = tr;
    O->tile_nnz = tn;
    O->tile_csr_Ptr = P;
    O->tile_csr_Col = Cc;
    O->tile_csr_Value = V;
    return RTT_OK;
}

/* ------------------------------------------------------------------------
 * FP64 row SPA C = A*B on CSR with sorted output columns, plus the bound
 * (|A||B|)_ij.  Restates spgemm_serialref (dense row accumulator, values
 * summed in A-row CSR order; src/external/cusparse/spgemm_serialref_spa.h:7-121),
 * with OpenMP and a sparse reset of the accumulator.
 * Call with colC == NULL to get row counts in rpC (m + 1, exclusive scan).
 * ------------------------------------------------------------------------ */
long long orc_spgemm_csr(int m, int k, int n,
                         const int *rpA, const int *ciA, const double *vA,
                         const int *rpB, const int *ciB, const double *vB,
                         long long *rpC, int *colC, double *valC, double *absC)
{
    (void)k;
    const int fill = colC != NULL;
#pragma omp parallel
    {
        double *acc = (double *)xcalloc((size_t)n, sizeof(double));
        double *aab = (double *)xcalloc((size_t)n, sizeof(double));
        char *flag = (char *)xcalloc((size_t)n, 1);
        int *list = (int *)xcalloc((size_t)n, sizeof(int));
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < m; ++i)
        {
            int cnt = 0;
            for (int p = rpA[i]; p < rpA[i + 1]; ++p)
            {
                int kk = ciA[p];
                double a = vA ? vA[p] : 0.0;
                for (int q = rpB[kk]; q < rpB[kk + 1]; ++q)
                {
                    int j = ciB[q];
                    if (!flag[j])
                    {
                        flag[j] = 1;
                        list[cnt++] = j;
                    }
                    if (fill)
                    {
                        double prod = a * vB[q];
                        acc[j] = acc[j] + prod;
                        aab[j] = aab[j] + fabs(a) * fabs(vB[q]);
                    }
                }
            }
            if (!fill)
                rpC[i] = cnt;
            else
            {
                /* sorted columns: counting over the row's list */
                for (int x = 1; x < cnt; ++x)
                {
                    int v = list[x], y = x - 1;
                    while (y >= 0 && list[y] > v)
                    {
                        list[y + 1] = list[y];
                        --y;
                    }
                    list[y + 1] = v;
                }
                long long o = rpC[i];
                for (int x = 0; x < cnt; ++x)
                {
                    int j = list[x];
                    colC[o + x] = j;
                    valC[o + x] = acc[j];
                    if (absC)
                        absC[o + x] = aab[j];
                }
            }
            for (int x = 0; x < cnt; ++x)
            {
                flag[list[x]] = 0;
                acc[list[x]] = 0.0;
                aab[list[x]] = 0.0;
            }
        }
        free(acc);
        free(aab);
        free(flag);
        free(list);
    }
    if (!fill)
    {
        long long run = 0;
        for (int i = 0; i <= m; ++i)
        {
            long long c = i < m ? rpC[i] : 0;
            rpC[i] = run;
            run += c;
        }
        return run;
    }
    return rpC[m];
}

/* nnzCub = sum over (i,k) in A of nnz(B row k) (src/gpu_dmma_tiles.h:752-762). */
long long orc_nnzcub(int m, const int *rpA, const int *ciA, const int *rpB)
{
    long long s = 0;
#pragma omp parallel for reduction(+ : s)
    for (int i = 0; i < m; ++i)
        for (int p = rpA[i]; p < rpA[i + 1]; ++p)
            s += rpB[ciA[p] + 1] - rpB[ciA[p]];
    return s;
}

void orc_matrix_free(SMatrix *M)
{
    free(M->tile_ptr);
    free(M->tile_columnidx);
    free(M->tile_rowidx);
    free(M->tile_nnz);
    free(M->tile_csr_Ptr);
    free(M->tile_csr_Col);
    free(M->tile_csr_Value);
    free(M->mask);
    free(M->csc_tile_ptr);
    free(M->csc_tile_rowidx);
    M->tile_ptr = M->tile_columnidx = M->tile_rowidx = M->tile_nnz = NULL;
    M->csc_tile_ptr = M->csc_tile_rowidx = NULL;
    M->tile_csr_Ptr = M->tile_csr_Col = NULL;
    M->tile_csr_Value = NULL;
    M->mask = NULL;
}

/* free() for buffers handed out by this library (ctypes callers). */
void orc_free(void *p) { free(p); }

int orc_num_threads(void) { return omp_get_max_threads(); }
