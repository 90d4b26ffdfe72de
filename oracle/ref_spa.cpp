/*
 * ref_spa.cpp - C entry point over the reference's serial FP64 row SPA.
 *
 * TEST INFRASTRUCTURE ONLY.  Includes the unmodified
 * src/external/cusparse/spgemm_serialref_spa.h of for-the-juan/RTT-SpGEMM
 * (dense-row accumulator, :7-121) and exposes spgemm_serialref with C
 * linkage.  Kept in its own library because that directory's common.h and
 * utils.h define functions that clash with src/utils.h.
 */
#include "spgemm_serialref_spa.h"

extern "C" int ref_spgemm_serialref(const int *rpA, const int *ciA, const double *vA, int mA,
                                    int nA, int nnzA, const int *rpB, const int *ciB,
                                    const double *vB, int mB, int nB, int nnzB, int *rpC,
                                    int *ciC, double *vC, int *nnzC, int count_only)
{
    return spgemm_serialref(rpA, ciA, vA, mA, nA, nnzA, rpB, ciB, vB, mB, nB, nnzB, rpC, ciC, vC,
                            mA, nB, nnzC, count_only != 0);
}
