/*
 * ref_layout.cpp - prints the layout of the reference's SMatrix.
 *
 * TEST INFRASTRUCTURE ONLY.  Includes the unmodified src/common.h of
 * for-the-juan/RTT-SpGEMM (SMatrix, :50-72) and prints sizeof and the
 * offsetof of every field, one "name offset" line each, for the C-ABI layout
 * test to compare against include/rtt_spgemm.h.
 */
#include <cstddef>
#include <cstdio>

#include "common.h"

#define F(name) std::printf(#name " %zu\n", offsetof(SMatrix, name))

int main()
{
    std::printf("sizeof %zu\n", sizeof(SMatrix));
    F(m); F(n); F(nnz); F(isSymmetric); F(value); F(columnindex); F(rowpointer);
    F(tilem); F(tilen); F(tile_ptr); F(tile_columnidx); F(tile_rowidx); F(tile_nnz);
    F(numtile); F(tile_csr_Value); F(tile_csr_Col); F(tile_csr_Ptr); F(mask);
    F(csc_tile_ptr); F(csc_tile_rowidx);
    return 0;
}
