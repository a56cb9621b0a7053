/*
 * oracle_common.h -- shared helpers of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a plain-C restatement of the
 * AMSS-NCKU Fortran kernels on the BSSN/Z4c evolution path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, and only
 * as the checker.  The product path (nr-amssncku_b200/) never links it.
 *
 * Parity status: UNPINNED.  The reference ships no golden vectors or tests
 * for this path and its Fortran cannot be compiled in this image (no Fortran
 * compiler).  The restatement keeps the Fortran's array layout (column-major,
 * i fastest), its statement order and the left-to-right association of every
 * expression, and it is built with -ffp-contract=off, so it evaluates the
 * same IEEE double operations the Fortran does when gfortran -O3 builds it
 * for baseline x86-64 (no FMA contraction).  It is checked by analytic
 * known answers and convergence tests instead (tests/test_oracle_*.py).
 */
#ifndef AMSS_ORACLE_COMMON_H
#define AMSS_ORACLE_COMMON_H

#include <stdlib.h>
#include <string.h>
#include <math.h>

/* Fortran-order index of a 1-based (i,j,k) point of an ex[0]*ex[1]*ex[2] array. */
#define OIDX(ex, i, j, k) \
    ((long)((i) - 1) + (long)(ex)[0] * ((long)((j) - 1) + (long)(ex)[1] * (long)((k) - 1)))

/* Array padded on the low side by `ord` cells, Fortran bounds (-ord+1:ex). */
typedef struct {
    double *a;
    int lo;          /* lowest index, -ord+1 */
    long n0, n1, n2; /* extents ex+ord */
} padded_t;

#define PH(P, i, j, k) \
    ((P).a[(long)((i) - (P).lo) + (P).n0 * ((long)((j) - (P).lo) + (P).n1 * (long)((k) - (P).lo))])

#define NO_SYMM 0
#define EQ_SYMM 1
#define OCTANT 2

static inline long npts3(const int *ex) { return (long)ex[0] * ex[1] * ex[2]; }

static inline double *oalloc(long n)
{
    double *p = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    if (!p) abort();
    return p;
}

/* fmisc.f90:877-901 symmetry_bd: copy f into an array padded by `ord` cells on
 * the low side of every direction, the pad mirrored cell-centred with parity. */
void oracle_symmetry_bd(int ord, const int *ex, const double *f, padded_t *fh, const double *SoA);
void oracle_padded_free(padded_t *fh);

#endif
