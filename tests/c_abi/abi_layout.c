/*
 * abi_layout.c - a plain C caller of the library: includes
 * include/rtt_spgemm.h, links librtt_spgemm.so and prints the SMatrix layout
 * (sizeof and offsetof of every field, one "name offset" line each) plus the
 * library's version and one status string.  No GPU call is made.
 */
#include <stddef.h>
#include <stdio.h>

#include "rtt_spgemm.h"

#define F(name) printf(#name " %zu\n", offsetof(SMatrix, name))

int main(void)
{
    printf("sizeof %zu\n", sizeof(SMatrix));
    F(m); F(n); F(nnz); F(isSymmetric); F(value); F(columnindex); F(rowpointer);
    F(tilem); F(tilen); F(tile_ptr); F(tile_columnidx); F(tile_rowidx); F(tile_nnz);
    F(numtile); F(tile_csr_Value); F(tile_csr_Col); F(tile_csr_Ptr); F(mask);
    F(csc_tile_ptr); F(csc_tile_rowidx);
    printf("version %s\n", rtt_version());
    printf("status2 %s\n", rtt_status_string(RTT_ERR_INVALID_CSR));
    return 0;
}
