/*
 * fd_oracle.c -- CPU oracle of the finite-difference building blocks.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle_common.h).  Parity unpinned.
 *
 * Restates, for ghost_width == 3 (4th-order code) and the Cell layout:
 *   symmetry_bd  fmisc.f90:877-901
 *   fderivs      diff_new.f90:946-1104   (the "for bam comparison" branch)
 *   fdderivs     diff_new.f90:1338-1528  (the "for bam comparison" branch)
 *   lopsided     lopsidediff.f90:186-488 (the "new code, 2012dec27" branch)
 *   kodis        kodiss.f90:120-216      (the combined-direction branch)
 * Loops, gates and expression association follow those lines.
 */
#include "oracle_common.h"

void oracle_symmetry_bd(int ord, const int *ex, const double *f, padded_t *fh, const double *SoA)
{
    fh->lo = -ord + 1;
    fh->n0 = ex[0] + ord;
    fh->n1 = ex[1] + ord;
    fh->n2 = ex[2] + ord;
    fh->a = oalloc(fh->n0 * fh->n1 * fh->n2);
    for (int k = 1; k <= ex[2]; ++k)
        for (int j = 1; j <= ex[1]; ++j)
            for (int i = 1; i <= ex[0]; ++i) PH(*fh, i, j, k) = f[OIDX(ex, i, j, k)];
    for (int i = 0; i <= ord - 1; ++i)
        for (int k = 1; k <= ex[2]; ++k)
            for (int j = 1; j <= ex[1]; ++j) PH(*fh, -i, j, k) = PH(*fh, i + 1, j, k) * SoA[0];
    for (int j = 0; j <= ord - 1; ++j)
        for (int k = 1; k <= ex[2]; ++k)
            for (int i = fh->lo; i <= ex[0]; ++i) PH(*fh, i, -j, k) = PH(*fh, i, j + 1, k) * SoA[1];
    for (int k = 0; k <= ord - 1; ++k)
        for (int j = fh->lo; j <= ex[1]; ++j)
            for (int i = fh->lo; i <= ex[0]; ++i) PH(*fh, i, j, -k) = PH(*fh, i, j, k + 1) * SoA[2];
}

void oracle_padded_free(padded_t *fh)
{
    free(fh->a);
    fh->a = NULL;
}

/* diff_new.f90:946-1104 */
void oracle_fderivs(const int *ex, const double *f, double *fx, double *fy, double *fz,
                    const double *X, const double *Y, const double *Z,
                    double SYM1, double SYM2, double SYM3, int Symmetry)
{
    const double ONE = 1.0, TWO = 2.0, EIT = 8.0, F12 = 12.0;
    double dX = X[1] - X[0], dY = Y[1] - Y[0], dZ = Z[1] - Z[0];
    int imax = ex[0], jmax = ex[1], kmax = ex[2];
    int imin = 1, jmin = 1, kmin = 1;
    if (Symmetry > NO_SYMM && fabs(Z[0]) < dZ) kmin = -1;
    if (Symmetry > EQ_SYMM && fabs(X[0]) < dX) imin = -1;
    if (Symmetry > EQ_SYMM && fabs(Y[0]) < dY) jmin = -1;
    double SoA[3] = {SYM1, SYM2, SYM3};
    padded_t fh;
    oracle_symmetry_bd(2, ex, f, &fh, SoA);
    double d12dx = ONE / F12 / dX, d12dy = ONE / F12 / dY, d12dz = ONE / F12 / dZ;
    double d2dx = ONE / TWO / dX, d2dy = ONE / TWO / dY, d2dz = ONE / TWO / dZ;
    long n = npts3(ex);
    memset(fx, 0, n * sizeof(double));
    memset(fy, 0, n * sizeof(double));
    memset(fz, 0, n * sizeof(double));
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= ex[2] - 1; ++k)
        for (int j = 1; j <= ex[1] - 1; ++j)
            for (int i = 1; i <= ex[0] - 1; ++i) {
                long p = OIDX(ex, i, j, k);
                if (i + 2 <= imax && i - 2 >= imin && j + 2 <= jmax && j - 2 >= jmin &&
                    k + 2 <= kmax && k - 2 >= kmin) {
                    fx[p] = d12dx * (PH(fh, i - 2, j, k) - EIT * PH(fh, i - 1, j, k) +
                                     EIT * PH(fh, i + 1, j, k) - PH(fh, i + 2, j, k));
                    fy[p] = d12dy * (PH(fh, i, j - 2, k) - EIT * PH(fh, i, j - 1, k) +
                                     EIT * PH(fh, i, j + 1, k) - PH(fh, i, j + 2, k));
                    fz[p] = d12dz * (PH(fh, i, j, k - 2) - EIT * PH(fh, i, j, k - 1) +
                                     EIT * PH(fh, i, j, k + 1) - PH(fh, i, j, k + 2));
                } else if (i + 1 <= imax && i - 1 >= imin && j + 1 <= jmax && j - 1 >= jmin &&
                           k + 1 <= kmax && k - 1 >= kmin) {
                    fx[p] = d2dx * (-PH(fh, i - 1, j, k) + PH(fh, i + 1, j, k));
                    fy[p] = d2dy * (-PH(fh, i, j - 1, k) + PH(fh, i, j + 1, k));
                    fz[p] = d2dz * (-PH(fh, i, j, k - 1) + PH(fh, i, j, k + 1));
                }
            }
    oracle_padded_free(&fh);
}

/* diff_new.f90:1338-1528 */
void oracle_fdderivs(const int *ex, const double *f, double *fxx, double *fxy, double *fxz,
                     double *fyy, double *fyz, double *fzz,
                     const double *X, const double *Y, const double *Z,
                     double SYM1, double SYM2, double SYM3, int Symmetry)
{
    const double ONE = 1.0, TWO = 2.0, F1o4 = 2.5e-1, F8 = 8.0, F16 = 16.0, F30 = 30.0;
    const double F1o12 = ONE / 12.0, F1o144 = ONE / 144.0;
    double dX = X[1] - X[0], dY = Y[1] - Y[0], dZ = Z[1] - Z[0];
    int imax = ex[0], jmax = ex[1], kmax = ex[2];
    int imin = 1, jmin = 1, kmin = 1;
    if (Symmetry > NO_SYMM && fabs(Z[0]) < dZ) kmin = -1;
    if (Symmetry > EQ_SYMM && fabs(X[0]) < dX) imin = -1;
    if (Symmetry > EQ_SYMM && fabs(Y[0]) < dY) jmin = -1;
    double SoA[3] = {SYM1, SYM2, SYM3};
    padded_t fh;
    oracle_symmetry_bd(2, ex, f, &fh, SoA);
    double Sdxdx = ONE / (dX * dX), Sdydy = ONE / (dY * dY), Sdzdz = ONE / (dZ * dZ);
    double Fdxdx = F1o12 / (dX * dX), Fdydy = F1o12 / (dY * dY), Fdzdz = F1o12 / (dZ * dZ);
    double Sdxdy = F1o4 / (dX * dY), Sdxdz = F1o4 / (dX * dZ), Sdydz = F1o4 / (dY * dZ);
    double Fdxdy = F1o144 / (dX * dY), Fdxdz = F1o144 / (dX * dZ), Fdydz = F1o144 / (dY * dZ);
    long n = npts3(ex);
    memset(fxx, 0, n * sizeof(double));
    memset(fyy, 0, n * sizeof(double));
    memset(fzz, 0, n * sizeof(double));
    memset(fxy, 0, n * sizeof(double));
    memset(fxz, 0, n * sizeof(double));
    memset(fyz, 0, n * sizeof(double));
#define H(a, b, c) PH(fh, a, b, c)
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= ex[2] - 1; ++k)
        for (int j = 1; j <= ex[1] - 1; ++j)
            for (int i = 1; i <= ex[0] - 1; ++i) {
                long p = OIDX(ex, i, j, k);
                if (i + 2 <= imax && i - 2 >= imin && j + 2 <= jmax && j - 2 >= jmin &&
                    k + 2 <= kmax && k - 2 >= kmin) {
                    fxx[p] = Fdxdx * (-H(i - 2, j, k) + F16 * H(i - 1, j, k) - F30 * H(i, j, k) -
                                      H(i + 2, j, k) + F16 * H(i + 1, j, k));
                    fyy[p] = Fdydy * (-H(i, j - 2, k) + F16 * H(i, j - 1, k) - F30 * H(i, j, k) -
                                      H(i, j + 2, k) + F16 * H(i, j + 1, k));
                    fzz[p] = Fdzdz * (-H(i, j, k - 2) + F16 * H(i, j, k - 1) - F30 * H(i, j, k) -
                                      H(i, j, k + 2) + F16 * H(i, j, k + 1));
                    fxy[p] = Fdxdy * ((H(i - 2, j - 2, k) - F8 * H(i - 1, j - 2, k) + F8 * H(i + 1, j - 2, k) - H(i + 2, j - 2, k)) -
                                      F8 * (H(i - 2, j - 1, k) - F8 * H(i - 1, j - 1, k) + F8 * H(i + 1, j - 1, k) - H(i + 2, j - 1, k)) +
                                      F8 * (H(i - 2, j + 1, k) - F8 * H(i - 1, j + 1, k) + F8 * H(i + 1, j + 1, k) - H(i + 2, j + 1, k)) -
                                      (H(i - 2, j + 2, k) - F8 * H(i - 1, j + 2, k) + F8 * H(i + 1, j + 2, k) - H(i + 2, j + 2, k)));
                    fxz[p] = Fdxdz * ((H(i - 2, j, k - 2) - F8 * H(i - 1, j, k - 2) + F8 * H(i + 1, j, k - 2) - H(i + 2, j, k - 2)) -
                                      F8 * (H(i - 2, j, k - 1) - F8 * H(i - 1, j, k - 1) + F8 * H(i + 1, j, k - 1) - H(i + 2, j, k - 1)) +
                                      F8 * (H(i - 2, j, k + 1) - F8 * H(i - 1, j, k + 1) + F8 * H(i + 1, j, k + 1) - H(i + 2, j, k + 1)) -
                                      (H(i - 2, j, k + 2) - F8 * H(i - 1, j, k + 2) + F8 * H(i + 1, j, k + 2) - H(i + 2, j, k + 2)));
                    fyz[p] = Fdydz * ((H(i, j - 2, k - 2) - F8 * H(i, j - 1, k - 2) + F8 * H(i, j + 1, k - 2) - H(i, j + 2, k - 2)) -
                                      F8 * (H(i, j - 2, k - 1) - F8 * H(i, j - 1, k - 1) + F8 * H(i, j + 1, k - 1) - H(i, j + 2, k - 1)) +
                                      F8 * (H(i, j - 2, k + 1) - F8 * H(i, j - 1, k + 1) + F8 * H(i, j + 1, k + 1) - H(i, j + 2, k + 1)) -
                                      (H(i, j - 2, k + 2) - F8 * H(i, j - 1, k + 2) + F8 * H(i, j + 1, k + 2) - H(i, j + 2, k + 2)));
                } else if (i + 1 <= imax && i - 1 >= imin && j + 1 <= jmax && j - 1 >= jmin &&
                           k + 1 <= kmax && k - 1 >= kmin) {
                    fxx[p] = Sdxdx * (H(i - 1, j, k) - TWO * H(i, j, k) + H(i + 1, j, k));
                    fyy[p] = Sdydy * (H(i, j - 1, k) - TWO * H(i, j, k) + H(i, j + 1, k));
                    fzz[p] = Sdzdz * (H(i, j, k - 1) - TWO * H(i, j, k) + H(i, j, k + 1));
                    fxy[p] = Sdxdy * (H(i - 1, j - 1, k) - H(i + 1, j - 1, k) - H(i - 1, j + 1, k) + H(i + 1, j + 1, k));
                    fxz[p] = Sdxdz * (H(i - 1, j, k - 1) - H(i + 1, j, k - 1) - H(i - 1, j, k + 1) + H(i + 1, j, k + 1));
                    fyz[p] = Sdydz * (H(i, j - 1, k - 1) - H(i, j + 1, k - 1) - H(i, j - 1, k + 1) + H(i, j + 1, k + 1));
                }
            }
#undef H
    oracle_padded_free(&fh);
}

/* lopsidediff.f90:186-488: f_rhs += beta^d * (upwinded D_d f). */
void oracle_lopsided(const int *ex, const double *X, const double *Y, const double *Z,
                     const double *f, double *f_rhs, const double *Sfx, const double *Sfy,
                     const double *Sfz, int Symmetry, const double *SoA)
{
    const double ZEO = 0.0, ONE = 1.0, F3 = 3.0, F6 = 6.0, F18 = 18.0, F12 = 12.0, F10 = 10.0, EIT = 8.0;
    double dX = X[1] - X[0], dY = Y[1] - Y[0], dZ = Z[1] - Z[0];
    double d12dx = ONE / F12 / dX, d12dy = ONE / F12 / dY, d12dz = ONE / F12 / dZ;
    int imax = ex[0], jmax = ex[1], kmax = ex[2];
    int imin = 1, jmin = 1, kmin = 1;
    if (Symmetry > NO_SYMM && fabs(Z[0]) < dZ) kmin = -2;
    if (Symmetry > EQ_SYMM && fabs(X[0]) < dX) imin = -2;
    if (Symmetry > EQ_SYMM && fabs(Y[0]) < dY) jmin = -2;
    padded_t fh;
    oracle_symmetry_bd(3, ex, f, &fh, SoA);
#define H(a, b, c) PH(fh, a, b, c)
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= ex[2] - 1; ++k)
        for (int j = 1; j <= ex[1] - 1; ++j)
            for (int i = 1; i <= ex[0] - 1; ++i) {
                long p = OIDX(ex, i, j, k);
                double r = f_rhs[p];
                /* x direction */
                if (Sfx[p] > ZEO) {
                    if (i + 3 <= imax)
                        r = r + Sfx[p] * d12dx * (-F3 * H(i - 1, j, k) - F10 * H(i, j, k) + F18 * H(i + 1, j, k) - F6 * H(i + 2, j, k) + H(i + 3, j, k));
                    else if (i + 2 <= imax)
                        r = r + Sfx[p] * d12dx * (H(i - 2, j, k) - EIT * H(i - 1, j, k) + EIT * H(i + 1, j, k) - H(i + 2, j, k));
                    else if (i + 1 <= imax)
                        r = r - Sfx[p] * d12dx * (-F3 * H(i + 1, j, k) - F10 * H(i, j, k) + F18 * H(i - 1, j, k) - F6 * H(i - 2, j, k) + H(i - 3, j, k));
                } else if (Sfx[p] < ZEO) {
                    if (i - 3 >= imin)
                        r = r - Sfx[p] * d12dx * (-F3 * H(i + 1, j, k) - F10 * H(i, j, k) + F18 * H(i - 1, j, k) - F6 * H(i - 2, j, k) + H(i - 3, j, k));
                    else if (i - 2 >= imin)
                        r = r + Sfx[p] * d12dx * (H(i - 2, j, k) - EIT * H(i - 1, j, k) + EIT * H(i + 1, j, k) - H(i + 2, j, k));
                    else if (i - 1 >= imin)
                        r = r + Sfx[p] * d12dx * (-F3 * H(i - 1, j, k) - F10 * H(i, j, k) + F18 * H(i + 1, j, k) - F6 * H(i + 2, j, k) + H(i + 3, j, k));
                }
                /* y direction */
                if (Sfy[p] > ZEO) {
                    if (j + 3 <= jmax)
                        r = r + Sfy[p] * d12dy * (-F3 * H(i, j - 1, k) - F10 * H(i, j, k) + F18 * H(i, j + 1, k) - F6 * H(i, j + 2, k) + H(i, j + 3, k));
                    else if (j + 2 <= jmax)
                        r = r + Sfy[p] * d12dy * (H(i, j - 2, k) - EIT * H(i, j - 1, k) + EIT * H(i, j + 1, k) - H(i, j + 2, k));
                    else if (j + 1 <= jmax)
                        r = r - Sfy[p] * d12dy * (-F3 * H(i, j + 1, k) - F10 * H(i, j, k) + F18 * H(i, j - 1, k) - F6 * H(i, j - 2, k) + H(i, j - 3, k));
                } else if (Sfy[p] < ZEO) {
                    if (j - 3 >= jmin)
                        r = r - Sfy[p] * d12dy * (-F3 * H(i, j + 1, k) - F10 * H(i, j, k) + F18 * H(i, j - 1, k) - F6 * H(i, j - 2, k) + H(i, j - 3, k));
                    else if (j - 2 >= jmin)
                        r = r + Sfy[p] * d12dy * (H(i, j - 2, k) - EIT * H(i, j - 1, k) + EIT * H(i, j + 1, k) - H(i, j + 2, k));
                    else if (j - 1 >= jmin)
                        r = r + Sfy[p] * d12dy * (-F3 * H(i, j - 1, k) - F10 * H(i, j, k) + F18 * H(i, j + 1, k) - F6 * H(i, j + 2, k) + H(i, j + 3, k));
                }
                /* z direction */
                if (Sfz[p] > ZEO) {
                    if (k + 3 <= kmax)
                        r = r + Sfz[p] * d12dz * (-F3 * H(i, j, k - 1) - F10 * H(i, j, k) + F18 * H(i, j, k + 1) - F6 * H(i, j, k + 2) + H(i, j, k + 3));
                    else if (k + 2 <= kmax)
                        r = r + Sfz[p] * d12dz * (H(i, j, k - 2) - EIT * H(i, j, k - 1) + EIT * H(i, j, k + 1) - H(i, j, k + 2));
                    else if (k + 1 <= kmax)
                        r = r - Sfz[p] * d12dz * (-F3 * H(i, j, k + 1) - F10 * H(i, j, k) + F18 * H(i, j, k - 1) - F6 * H(i, j, k - 2) + H(i, j, k - 3));
                } else if (Sfz[p] < ZEO) {
                    if (k - 3 >= kmin)
                        r = r - Sfz[p] * d12dz * (-F3 * H(i, j, k + 1) - F10 * H(i, j, k) + F18 * H(i, j, k - 1) - F6 * H(i, j, k - 2) + H(i, j, k - 3));
                    else if (k - 2 >= kmin)
                        r = r + Sfz[p] * d12dz * (H(i, j, k - 2) - EIT * H(i, j, k - 1) + EIT * H(i, j, k + 1) - H(i, j, k + 2));
                    else if (k - 1 >= kmin)
                        r = r + Sfz[p] * d12dz * (-F3 * H(i, j, k - 1) - F10 * H(i, j, k) + F18 * H(i, j, k + 1) - F6 * H(i, j, k + 2) + H(i, j, k + 3));
                }
                f_rhs[p] = r;
            }
#undef H
    oracle_padded_free(&fh);
}

/* kodiss.f90:120-216: f_rhs += eps/64 * sum_d (D+D-)^3 f * h_d^5, where all +-3 fit. */
void oracle_kodis(const int *ex, const double *X, const double *Y, const double *Z,
                  const double *f, double *f_rhs, const double *SoA, int Symmetry, double eps)
{
    const double SIX = 6.0, FIT = 15.0, TWT = 20.0, cof = 64.0;
    double dX = X[1] - X[0], dY = Y[1] - Y[0], dZ = Z[1] - Z[0];
    int imax = ex[0], jmax = ex[1], kmax = ex[2];
    int imin = 1, jmin = 1, kmin = 1;
    if (Symmetry > NO_SYMM && fabs(Z[0]) < dZ) kmin = -2;
    if (Symmetry == OCTANT && fabs(X[0]) < dX) imin = -2;
    if (Symmetry == OCTANT && fabs(Y[0]) < dY) jmin = -2;
    padded_t fh;
    oracle_symmetry_bd(3, ex, f, &fh, SoA);
#define H(a, b, c) PH(fh, a, b, c)
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= ex[2]; ++k)
        for (int j = 1; j <= ex[1]; ++j)
            for (int i = 1; i <= ex[0]; ++i) {
                if (i - 3 >= imin && i + 3 <= imax && j - 3 >= jmin && j + 3 <= jmax &&
                    k - 3 >= kmin && k + 3 <= kmax) {
                    long p = OIDX(ex, i, j, k);
                    f_rhs[p] = f_rhs[p] + eps / cof *
                        (((H(i - 3, j, k) + H(i + 3, j, k)) - SIX * (H(i - 2, j, k) + H(i + 2, j, k)) +
                          FIT * (H(i - 1, j, k) + H(i + 1, j, k)) - TWT * H(i, j, k)) / dX +
                         ((H(i, j - 3, k) + H(i, j + 3, k)) - SIX * (H(i, j - 2, k) + H(i, j + 2, k)) +
                          FIT * (H(i, j - 1, k) + H(i, j + 1, k)) - TWT * H(i, j, k)) / dY +
                         ((H(i, j, k - 3) + H(i, j, k + 3)) - SIX * (H(i, j, k - 2) + H(i, j, k + 2)) +
                          FIT * (H(i, j, k - 1) + H(i, j, k + 1)) - TWT * H(i, j, k)) / dZ);
                }
            }
#undef H
    oracle_padded_free(&fh);
}
