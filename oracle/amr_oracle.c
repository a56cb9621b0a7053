/*
 * amr_oracle.c -- CPU oracle of the AMR transfer operators and of one RK4
 * substep of one block.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle_common.h).  Parity unpinned.
 *
 * Restates, cell-centred (the active "#if 1" branches):
 *   prolong3   prolongrestrict_cell.f90:1915-2164 (5th-order, 6-point tensor
 *              Lagrange; the "#else" branch at :2129-2156 that picks the weight
 *              order per direction from the parity of the fine index)
 *   restrict3  prolongrestrict_cell.f90:2330-2468 (6-point symmetric average)
 * on boxes given in global level indices: a block array whose element 0 sits
 * at global index org[] of its level.  Fine cell g (0-based global) has the
 * coarse parent g >> 1; the reference's 1-based index arithmetic
 * (cxI = (i + lbf - 1)/2, cxI = 2*(i + lbc - 1) - 1) maps to
 *   prolong, g odd  (right child): coarse k-2..k+3, weights C1..C6
 *   prolong, g even (left child):  coarse k-3..k+2, weights C6..C1
 *   restrict: fine 2k-2..2k+3, weights C1 C2 C3 C3 C2 C1
 * and both apply the 1-D weights z first, then y, then x, as the Fortran's
 * tmp2/tmp1 passes do.
 */
#include "oracle_common.h"

static inline long aidx(const int *ex, int i, int j, int k)
{
    return (long)i + (long)ex[0] * ((long)j + (long)ex[1] * (long)k);
}

/* prolongrestrict_cell.f90:1937-1942 */
static const double PC1 = 7.7e1 / 8.192e3, PC2 = -6.93e2 / 8.192e3, PC3 = 3.465e3 / 4.096e3;
static const double PC6 = 6.3e1 / 8.192e3, PC5 = -4.95e2 / 8.192e3, PC4 = 1.155e3 / 4.096e3;

static void prolong_axis(int g, int *s0, double *w)
{
    int k = g >> 1;
    if (g & 1) {
        *s0 = k - 2;
        w[0] = PC1; w[1] = PC2; w[2] = PC3; w[3] = PC4; w[4] = PC5; w[5] = PC6;
    } else {
        *s0 = k - 3;
        w[0] = PC6; w[1] = PC5; w[2] = PC4; w[3] = PC3; w[4] = PC2; w[5] = PC1;
    }
}

/* Fine cells [flo, fhi) (global fine indices) of array funf from array func. */
void oracle_prolong3_box(const int *exc, const int *corg, const double *func, const int *exf, const int *forg,
                         double *funf, const int *flo, const int *fhi)
{
#pragma omp parallel for schedule(static)
    for (int gk = flo[2]; gk < fhi[2]; ++gk)
        for (int gj = flo[1]; gj < fhi[1]; ++gj)
            for (int gi = flo[0]; gi < fhi[0]; ++gi) {
                int sx, sy, sz;
                double wx[6], wy[6], wz[6];
                prolong_axis(gi, &sx, wx);
                prolong_axis(gj, &sy, wy);
                prolong_axis(gk, &sz, wz);
                double tmp2[6][6], tmp1[6];
                for (int a = 0; a < 6; ++a)
                    for (int b = 0; b < 6; ++b) {
                        int ci = sx + a - corg[0], cj = sy + b - corg[1], ck = sz - corg[2];
                        double v = wz[0] * func[aidx(exc, ci, cj, ck)];
                        for (int m = 1; m < 6; ++m) v = v + wz[m] * func[aidx(exc, ci, cj, ck + m)];
                        tmp2[a][b] = v;
                    }
                for (int a = 0; a < 6; ++a) {
                    double v = wy[0] * tmp2[a][0];
                    for (int b = 1; b < 6; ++b) v = v + wy[b] * tmp2[a][b];
                    tmp1[a] = v;
                }
                double v = wx[0] * tmp1[0];
                for (int a = 1; a < 6; ++a) v = v + wx[a] * tmp1[a];
                funf[aidx(exf, gi - forg[0], gj - forg[1], gk - forg[2])] = v;
            }
}

/* prolongrestrict_cell.f90:2350 */
static const double RC1 = 3.0 / 2.56e2, RC2 = -2.5e1 / 2.56e2, RC3 = 7.5e1 / 1.28e2;

/* Coarse cells [clo, chi) (global coarse indices) of array func from array funf. */
void oracle_restrict3_box(const int *exc, const int *corg, double *func, const int *exf, const int *forg,
                          const double *funf, const int *clo, const int *chi)
{
#pragma omp parallel for schedule(static)
    for (int ck = clo[2]; ck < chi[2]; ++ck)
        for (int cj = clo[1]; cj < chi[1]; ++cj)
            for (int ci = clo[0]; ci < chi[0]; ++ci) {
                int fi = 2 * ci - 2 - forg[0], fj = 2 * cj - 2 - forg[1], fk = 2 * ck - 2 - forg[2];
                double tmp2[6][6], tmp1[6];
                for (int a = 0; a < 6; ++a)
                    for (int b = 0; b < 6; ++b) {
#define FF(m) funf[aidx(exf, fi + a, fj + b, fk + (m))]
                        tmp2[a][b] = RC1 * (FF(0) + FF(5)) + RC2 * (FF(1) + FF(4)) + RC3 * (FF(2) + FF(3));
#undef FF
                    }
                for (int a = 0; a < 6; ++a)
                    tmp1[a] = RC1 * (tmp2[a][0] + tmp2[a][5]) + RC2 * (tmp2[a][1] + tmp2[a][4]) +
                              RC3 * (tmp2[a][2] + tmp2[a][3]);
                func[aidx(exc, ci - corg[0], cj - corg[1], ck - corg[2])] =
                    RC1 * (tmp1[0] + tmp1[5]) + RC2 * (tmp1[1] + tmp1[4]) + RC3 * (tmp1[2] + tmp1[3]);
            }
}
