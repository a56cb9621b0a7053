/*
 * step_oracle.c -- CPU oracle of the per-block update pieces and of one
 * single-block RK4 step.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle_common.h).  Parity unpinned.
 *
 * Restates:
 *   enforce_ga          enforce_algebra.f90:72-133
 *   rungekutta4_rout    rungekutta4_rout.f90:94-139
 *   sommerfeld_routbam  sommerfeld_rout.f90:223-449 (the "new code, 2012dec26" branch)
 *   sommerfeld_rout     sommerfeld_rout.f90:9-221, precor == 1 (copy branch) only
 *   lowerboundset       fmisc.f90:1644-1657
 *   get_lousto_nbhs     initial_puncture.f90:1970-2202
 *   l2normhelper        fmisc.f90:1263-1309
 *   average2            fmisc.f90:1569-1592
 * and the order of calls inside one level-0 step of bssn_class::Step
 * (bssn_class.C:2981-3915) for a single block that is the whole patch:
 * enforce_ga -> compute_rhs_bssn -> sommerfeld_routbam -> rungekutta4_rout ->
 * lowerboundset, predictor then three correctors, lists swapped as there.
 */
#include "oracle_common.h"
#include <stdio.h>

int oracle_compute_rhs_bssn(const int *ex, double T, const double *X, const double *Y, const double *Z,
                            double *chi, double *trK, double *dxx, double *gxy, double *gxz, double *dyy,
                            double *gyz, double *dzz, double *Axx, double *Axy, double *Axz, double *Ayy,
                            double *Ayz, double *Azz, double *Gamx, double *Gamy, double *Gamz, double *Lap,
                            double *betax, double *betay, double *betaz, double *dtSfx, double *dtSfy,
                            double *dtSfz, double *chi_rhs, double *trK_rhs, double *gxx_rhs,
                            double *gxy_rhs, double *gxz_rhs, double *gyy_rhs, double *gyz_rhs,
                            double *gzz_rhs, double *Axx_rhs, double *Axy_rhs, double *Axz_rhs,
                            double *Ayy_rhs, double *Ayz_rhs, double *Azz_rhs, double *Gamx_rhs,
                            double *Gamy_rhs, double *Gamz_rhs, double *Lap_rhs, double *betax_rhs,
                            double *betay_rhs, double *betaz_rhs, double *dtSfx_rhs, double *dtSfy_rhs,
                            double *dtSfz_rhs, const double *rho, const double *Sx, const double *Sy,
                            const double *Sz, const double *Sxx, const double *Sxy, const double *Sxz,
                            const double *Syy, const double *Syz, const double *Szz, double *Gamxxx,
                            double *Gamxxy, double *Gamxxz, double *Gamxyy, double *Gamxyz, double *Gamxzz,
                            double *Gamyxx, double *Gamyxy, double *Gamyxz, double *Gamyyy, double *Gamyyz,
                            double *Gamyzz, double *Gamzxx, double *Gamzxy, double *Gamzxz, double *Gamzyy,
                            double *Gamzyz, double *Gamzzz, double *Rxx, double *Rxy, double *Rxz,
                            double *Ryy, double *Ryz, double *Rzz, double *ham_Res, double *movx_Res,
                            double *movy_Res, double *movz_Res, double *Gmx_Res, double *Gmy_Res,
                            double *Gmz_Res, int Symmetry, int Lev, double eps, int co);

/* enforce_algebra.f90:72-133 */
void oracle_enforce_ga(const int *ex, double *dxx, double *gxy, double *gxz, double *dyy, double *gyz,
                       double *dzz, double *Axx, double *Axy, double *Axz, double *Ayy, double *Ayz,
                       double *Azz)
{
    const double F1o3 = 1.0 / 3.0, ONE = 1.0, TWO = 2.0;
    long n = npts3(ex);
#pragma omp parallel for schedule(static)
    for (long p = 0; p < n; ++p) {
        double gxx = dxx[p] + ONE, gyy = dyy[p] + ONE, gzz = dzz[p] + ONE;
        double xy = gxy[p], xz = gxz[p], yz = gyz[p];
        double gupzz = gxx * gyy * gzz + xy * yz * xz + xz * xy * yz - xz * gyy * xz - xy * xy * gzz -
                       gxx * yz * yz;
        gupzz = ONE / pow(gupzz, F1o3);
        gxx = gxx * gupzz;
        xy = xy * gupzz;
        xz = xz * gupzz;
        gyy = gyy * gupzz;
        yz = yz * gupzz;
        gzz = gzz * gupzz;
        gxy[p] = xy;
        gxz[p] = xz;
        gyz[p] = yz;
        dxx[p] = gxx - ONE;
        dyy[p] = gyy - ONE;
        dzz[p] = gzz - ONE;
        double uxx = (gyy * gzz - yz * yz);
        double uxy = -(xy * gzz - yz * xz);
        double uxz = (xy * yz - gyy * xz);
        double uyy = (gxx * gzz - xz * xz);
        double uyz = -(gxx * yz - xy * xz);
        double uzz = (gxx * gyy - xy * xy);
        double trA = uxx * Axx[p] + uyy * Ayy[p] + uzz * Azz[p] +
                     TWO * (uxy * Axy[p] + uxz * Axz[p] + uyz * Ayz[p]);
        Axx[p] = Axx[p] - F1o3 * gxx * trA;
        Axy[p] = Axy[p] - F1o3 * xy * trA;
        Axz[p] = Axz[p] - F1o3 * xz * trA;
        Ayy[p] = Ayy[p] - F1o3 * gyy * trA;
        Ayz[p] = Ayz[p] - F1o3 * yz * trA;
        Azz[p] = Azz[p] - F1o3 * gzz * trA;
    }
}

/* rungekutta4_rout.f90:94-139; returns 1 on a bad RK4 counter (the Fortran stops). */
int oracle_rungekutta4_rout(const int *ex, double dT, const double *f0, double *f1, double *f_rhs, int RK4)
{
    const double F1o6 = 1.0 / 6.0, HLF = 0.5, TWO = 2.0;
    long n = npts3(ex);
    if (RK4 < 0 || RK4 > 3) return 1;
#pragma omp parallel for schedule(static)
    for (long p = 0; p < n; ++p) {
        if (RK4 == 0) {
            f1[p] = f0[p] + HLF * dT * f_rhs[p];
        } else if (RK4 == 1) {
            f_rhs[p] = f_rhs[p] + TWO * f1[p];
            f1[p] = f0[p] + HLF * dT * f1[p];
        } else if (RK4 == 2) {
            f_rhs[p] = f_rhs[p] + TWO * f1[p];
            f1[p] = f0[p] + dT * f1[p];
        } else {
            f1[p] = f0[p] + F1o6 * dT * (f1[p] + f_rhs[p]);
        }
    }
    return 0;
}

/* fmisc.f90:1644-1657 */
void oracle_lowerboundset(const int *ex, double *chi, double tinny)
{
    long n = npts3(ex);
    for (long p = 0; p < n; ++p)
        if (chi[p] < tinny) chi[p] = tinny;
}

/* The six face layers of sommerfeld_rout.f90:274-339 (also :56-121).  layer[gp]
 * holds imin,jmin,kmin,imax,jmax,kmax (1-based) of face gp, or all -1 when the
 * block does not touch that face of the patch. */
static void sommerfeld_layers(const int *ex, const double *X, const double *Y, const double *Z,
                              double xmin, double ymin, double zmin, double xmax, double ymax,
                              double zmax, int Symmetry, int layer[6][6])
{
    double dX = X[1] - X[0], dY = Y[1] - Y[0], dZ = Z[1] - Z[0];
    for (int gp = 0; gp < 6; ++gp) {
        for (int m = 0; m < 3; ++m) layer[gp][m] = 1;
        for (int m = 3; m < 6; ++m) layer[gp][m] = -1;
    }
    if (fabs(X[ex[0] - 1] - xmax) < dX) {
        int v[6] = {ex[0], 1, 1, ex[0], ex[1], ex[2]};
        memcpy(layer[0], v, sizeof v);
    }
    if (fabs(Y[ex[1] - 1] - ymax) < dY) {
        int v[6] = {1, ex[1], 1, ex[0], ex[1], ex[2]};
        memcpy(layer[1], v, sizeof v);
    }
    if (fabs(Z[ex[2] - 1] - zmax) < dZ) {
        int v[6] = {1, 1, ex[2], ex[0], ex[1], ex[2]};
        memcpy(layer[2], v, sizeof v);
    }
    if (fabs(X[0] - xmin) < dX && !(Symmetry == OCTANT && fabs(xmin) < dX / 2)) {
        int v[6] = {1, 1, 1, 1, ex[1], ex[2]};
        memcpy(layer[3], v, sizeof v);
    }
    if (fabs(Y[0] - ymin) < dY && !(Symmetry == OCTANT && fabs(ymin) < dY / 2)) {
        int v[6] = {1, 1, 1, ex[0], 1, ex[2]};
        memcpy(layer[4], v, sizeof v);
    }
    if (fabs(Z[0] - zmin) < dZ && !(Symmetry > NO_SYMM && fabs(zmin) < dZ / 2)) {
        int v[6] = {1, 1, 1, ex[0], ex[1], 1};
        memcpy(layer[5], v, sizeof v);
    }
}

/* sommerfeld_rout.f90:223-449 ("new code, 2012dec26"): on the outer faces of
 * the patch, f_rhs = -v (x.grad f0 + f0)/r with one-sided 2nd-order upwinding. */
void oracle_sommerfeld_routbam(const int *ex, const double *X, const double *Y, const double *Z,
                               double xmin, double ymin, double zmin, double xmax, double ymax,
                               double zmax, double *f_rhs, const double *f0, double velocity,
                               const double *SoA, int Symmetry)
{
    const double ONE = 1.0, TWO = 2.0;
    double dX = X[1] - X[0], dY = Y[1] - Y[0], dZ = Z[1] - Z[0];
    double d2dx = ONE / TWO / dX, d2dy = ONE / TWO / dY, d2dz = ONE / TWO / dZ;
    int imax = ex[0], jmax = ex[1], kmax = ex[2];
    int imin = 1, jmin = 1, kmin = 1;
    if (Symmetry > NO_SYMM && fabs(Z[0]) < dZ) kmin = 0;
    if (Symmetry > EQ_SYMM && fabs(X[0]) < dX) imin = 0;
    if (Symmetry > EQ_SYMM && fabs(Y[0]) < dY) jmin = 0;
    padded_t fh;
    oracle_symmetry_bd(1, ex, f0, &fh, SoA);
    int layer[6][6];
    sommerfeld_layers(ex, X, Y, Z, xmin, ymin, zmin, xmax, ymax, zmax, Symmetry, layer);
#define H(a, b, c) PH(fh, a, b, c)
    for (int gp = 0; gp < 6; ++gp) {
        int gont = 0;
        for (int m = 0; m < 6; ++m) gont |= (layer[gp][m] == -1);
        if (gont) continue;
        for (int k = layer[gp][2]; k <= layer[gp][5]; ++k)
            for (int j = layer[gp][1]; j <= layer[gp][4]; ++j)
                for (int i = layer[gp][0]; i <= layer[gp][3]; ++i) {
                    /* fx, fy, fz keep no stale value here: where w_d == 0 the
                     * coordinate is 0 and the term it multiplies is 0 as well. */
                    double fx = 0.0, fy = 0.0, fz = 0.0;
                    double x = X[i - 1], y = Y[j - 1], z = Z[k - 1];
                    double R = sqrt(x * x + y * y + z * z);
                    double wx = velocity * x / R, wy = velocity * y / R, wz = velocity * z / R;
                    if (wx > 0) {
                        if (i - 2 >= imin) fx = d2dx * (3 * H(i, j, k) - 4 * H(i - 1, j, k) + H(i - 2, j, k));
                        else if (i - 1 >= imin) fx = d2dx * (-H(i - 1, j, k) + H(i + 1, j, k));
                        else fx = d2dx * (-H(i + 2, j, k) + 4 * H(i + 1, j, k) - 3 * H(i, j, k));
                    } else if (wx < 0) {
                        if (i + 2 <= imax) fx = d2dx * (-H(i + 2, j, k) + 4 * H(i + 1, j, k) - 3 * H(i, j, k));
                        else if (i + 1 <= imax) fx = d2dx * (-H(i - 1, j, k) + H(i + 1, j, k));
                        else fx = d2dx * (3 * H(i, j, k) - 4 * H(i - 1, j, k) + H(i - 2, j, k));
                    }
                    if (wy > 0) {
                        if (j - 2 >= jmin) fy = d2dy * (3 * H(i, j, k) - 4 * H(i, j - 1, k) + H(i, j - 2, k));
                        else if (j - 1 >= jmin) fy = d2dy * (-H(i, j - 1, k) + H(i, j + 1, k));
                        else fy = d2dy * (-H(i, j + 2, k) + 4 * H(i, j + 1, k) - 3 * H(i, j, k));
                    } else if (wy < 0) {
                        if (j + 2 <= jmax) fy = d2dy * (-H(i, j + 2, k) + 4 * H(i, j + 1, k) - 3 * H(i, j, k));
                        else if (j + 1 <= jmax) fy = d2dy * (-H(i, j - 1, k) + H(i, j + 1, k));
                        else fy = d2dy * (3 * H(i, j, k) - 4 * H(i, j - 1, k) + H(i, j - 2, k));
                    }
                    if (wz > 0) {
                        if (k - 2 >= kmin) fz = d2dz * (3 * H(i, j, k) - 4 * H(i, j, k - 1) + H(i, j, k - 2));
                        else if (k - 1 >= kmin) fz = d2dz * (-H(i, j, k - 1) + H(i, j, k + 1));
                        else fz = d2dz * (-H(i, j, k + 2) + 4 * H(i, j, k + 1) - 3 * H(i, j, k));
                    } else if (wz < 0) {
                        if (k + 2 <= kmax) fz = d2dz * (-H(i, j, k + 2) + 4 * H(i, j, k + 1) - 3 * H(i, j, k));
                        else if (k + 1 <= kmax) fz = d2dz * (-H(i, j, k - 1) + H(i, j, k + 1));
                        else fz = d2dz * (3 * H(i, j, k) - 4 * H(i, j, k - 1) + H(i, j, k - 2));
                    }
                    f_rhs[OIDX(ex, i, j, k)] = -velocity * (fx * x + fy * y + fz * z + f0[OIDX(ex, i, j, k)]) / R;
                }
    }
#undef H
    oracle_padded_free(&fh);
}

/* sommerfeld_rout.f90:122-139 (precor == 1): freeze the outer faces at f0.
 * Returns 1 for precor != 1, whose interpolating branch is not restated. */
int oracle_sommerfeld_rout(const int *ex, const double *X, const double *Y, const double *Z,
                           double xmin, double ymin, double zmin, double xmax, double ymax, double zmax,
                           const double *f0, double *f, int Symmetry, int precor)
{
    if (precor != 1) return 1;
    int layer[6][6];
    sommerfeld_layers(ex, X, Y, Z, xmin, ymin, zmin, xmax, ymax, zmax, Symmetry, layer);
    for (int gp = 0; gp < 6; ++gp) {
        int gont = 0;
        for (int m = 0; m < 6; ++m) gont |= (layer[gp][m] == -1);
        if (gont) continue;
        for (int k = layer[gp][2]; k <= layer[gp][5]; ++k)
            for (int j = layer[gp][1]; j <= layer[gp][4]; ++j)
                for (int i = layer[gp][0]; i <= layer[gp][3]; ++i) f[OIDX(ex, i, j, k)] = f0[OIDX(ex, i, j, k)];
    }
    return 0;
}

/* initial_puncture.f90:1970-2202 with P = S = 0 terms kept as written. */
void oracle_get_lousto_nbhs(const int *ex, const double *X, const double *Y, const double *Z,
                            double **st /* 24 fields in state order */, const double *Mass,
                            const double *Porg, const double *Pmom, const double *Spin, int N)
{
    const double HLF = 0.5, ONE = 1.0, THR = 3.0, TINYRR = 1e-14;
    long n = npts3(ex);
    double *psi = oalloc(n);
    double *chi = st[0], *Axx = st[8], *Axy = st[9], *Axz = st[10], *Ayy = st[11], *Ayz = st[12], *Azz = st[13];
    double *Lap = st[17];
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= ex[2]; ++k)
        for (int j = 1; j <= ex[1]; ++j)
            for (int i = 1; i <= ex[0]; ++i) {
                long p = OIDX(ex, i, j, k);
                double ps = 0, axx = 0, ayy = 0, azz = 0, axy = 0, axz = 0, ayz = 0;
                for (int bhi = 0; bhi < N; ++bhi) {
                    double M = Mass[bhi];
                    double nx = X[i - 1] - Porg[3 * bhi], ny = Y[j - 1] - Porg[3 * bhi + 1], nz = Z[k - 1] - Porg[3 * bhi + 2];
                    double Px = Pmom[3 * bhi], Py = Pmom[3 * bhi + 1], Pz = Pmom[3 * bhi + 2];
                    double Sx = Spin[3 * bhi], Sy = Spin[3 * bhi + 1], Sz = Spin[3 * bhi + 2];
                    double rr = sqrt(nx * nx + ny * ny + nz * nz);
                    if (rr < TINYRR) rr = (X[1] - X[0]) / 2.0;
                    nx = nx / rr;
                    ny = ny / rr;
                    nz = nz / rr;
                    double PP = sqrt(Px * Px + Py * Py + Pz * Pz);
                    double mup = PP > 0.0 ? (Px * nx + Py * ny + Pz * nz) / PP : 0.0;
                    double SS = sqrt(Sx * Sx + Sy * Sy + Sz * Sz);
                    double mus = SS > 0.0 ? (Sx * nx + Sy * ny + Sz * nz) / SS : 0.0;
                    double b = 2.0 * rr / M;
                    double ell = 1.0 / (1.0 + b);
                    double l2 = ell * ell, l3 = l2 * ell, l4 = l2 * l2, l5 = l4 * ell;
                    double u1 = 5.0 / 8.0 * ell * (1.0 - 2.0 * ell + 2.0 * l2 - l3 + l4 / 5.0);
                    double u2 = (15.0 + 117.0 * ell - 79.0 * l2 + 43.0 * l3 - 14.0 * l4 + 2.0 * l5 +
                                 84.0 * log(ell) / b) / 40.0 / (b * b);
                    double u3 = ell + l2 + l3 - 4.0 * l4 + 2.0 * l5;
                    double u4 = -(b * b) * l5;
                    double u5 = b * (1.0 + 5.0 * b + 10.0 * (b * b)) * l5 / 80.0;
                    double tmp = (Py * Sz - Pz * Sy) * nx + (Pz * Sx - Px * Sz) * ny + (Px * Sy - Py * Sx) * nz;
                    double u = (PP * PP) / (M * M) * (u1 + u2 * (3.0 * (mup * mup) - ONE)) +
                               2.0 * (SS * SS) / 5.0 / ((M * M) * (M * M)) * (u3 + u4 * (3.0 * (mus * mus) - ONE)) +
                               u5 * tmp;
                    if (bhi == 0) ps = ONE + u + HLF * M / rr;
                    else ps = ps + u + HLF * M / rr;
                    tmp = Px * nx + Py * ny + Pz * nz;
                    double r2 = rr * rr;
                    axx = axx + (HLF * (Px * nx + nx * Px - (ONE - nx * nx) * tmp) +
                                 (nx * Sy * nz - nx * Sz * ny + nx * Sy * nz - nx * Sz * ny) / rr) * THR / r2;
                    ayy = ayy + (HLF * (Py * ny + ny * Py - (ONE - ny * ny) * tmp) +
                                 (ny * Sz * nx - ny * Sx * nz + ny * Sz * nx - ny * Sx * nz) / rr) * THR / r2;
                    azz = azz + (HLF * (Pz * nz + nz * Pz - (ONE - nz * nz) * tmp) +
                                 (nz * Sx * ny - nz * Sy * nx + nz * Sx * ny - nz * Sy * nx) / rr) * THR / r2;
                    axy = axy + (HLF * (Px * ny + nx * Py + nx * ny * tmp) +
                                 (nx * Sz * nx - nx * Sx * nz + ny * Sy * nz - ny * Sz * ny) / rr) * THR / r2;
                    axz = axz + (HLF * (Px * nz + nx * Pz + nx * nz * tmp) +
                                 (nx * Sx * ny - nx * Sy * nx + nz * Sy * nz - nz * Sz * ny) / rr) * THR / r2;
                    ayz = ayz + (HLF * (Py * nz + ny * Pz + ny * nz * tmp) +
                                 (ny * Sx * ny - ny * Sy * nx + nz * Sz * nx - nz * Sx * nz) / rr) * THR / r2;
                }
                psi[p] = ps;
                Axx[p] = axx;
                Ayy[p] = ayy;
                Azz[p] = azz;
                Axy[p] = axy;
                Axz[p] = axz;
                Ayz[p] = ayz;
            }
#pragma omp parallel for schedule(static)
    for (long p = 0; p < n; ++p) {
        double ps = psi[p];
        double p2 = ps * ps;
        chi[p] = ONE / (p2 * p2) - ONE;
        Lap[p] = ONE / (ps * ps) - ONE;
        double p6 = ps * ps * ps * ps * ps * ps;
        Axx[p] = Axx[p] / p6;
        Ayy[p] = Ayy[p] / p6;
        Azz[p] = Azz[p] / p6;
        Axy[p] = Axy[p] / p6;
        Axz[p] = Axz[p] / p6;
        Ayz[p] = Ayz[p] / p6;
        static const int zero_fields[] = {1, 2, 3, 4, 5, 6, 7, 14, 15, 16, 18, 19, 20, 21, 22, 23};
        for (size_t z = 0; z < sizeof(zero_fields) / sizeof(zero_fields[0]); ++z) st[zero_fields[z]][p] = 0.0;
    }
    free(psi);
}

/* fmisc.f90:1263-1309: sum f^2 dV over owned points (ghosts excluded, the
 * patch boundary included). */
double oracle_l2normhelper(const int *ex, const double *X, const double *Y, const double *Z,
                           double xmin, double ymin, double zmin, double xmax, double ymax, double zmax,
                           const double *f, int gw)
{
    double dX = X[1] - X[0], dY = Y[1] - Y[0], dZ = Z[1] - Z[0];
    int imin = gw + 1, jmin = gw + 1, kmin = gw + 1;
    int imax = ex[0] - gw, jmax = ex[1] - gw, kmax = ex[2] - gw;
    if (fabs(X[ex[0] - 1] - xmax) < dX) imax = ex[0];
    if (fabs(Y[ex[1] - 1] - ymax) < dY) jmax = ex[1];
    if (fabs(Z[ex[2] - 1] - zmax) < dZ) kmax = ex[2];
    if (fabs(X[0] - xmin) < dX) imin = 1;
    if (fabs(Y[0] - ymin) < dY) jmin = 1;
    if (fabs(Z[0] - zmin) < dZ) kmin = 1;
    double s = 0.0;
    for (int k = kmin; k <= kmax; ++k)
        for (int j = jmin; j <= jmax; ++j)
            for (int i = imin; i <= imax; ++i) {
                double v = f[OIDX(ex, i, j, k)];
                s = s + v * v;
            }
    return s * dX * dY * dZ;
}

/* fmisc.f90:1569-1592 */
void oracle_average2(long n, const double *f1, const double *f2, const double *f3, double *fout)
{
    const double C1 = 3.0 / 8.0, C2 = 3.0 / 4.0, C3 = -1.0 / 8.0;
    for (long p = 0; p < n; ++p) fout[p] = C1 * f1[p] + C2 * f2[p] + C3 * f3[p];
}

/* Parity (SoA) and Sommerfeld speed of the 24 BSSN state fields in state order,
 * bssn_class.C:177-330 (parities) and :390-410 (speed sqrt(2) for chi, trK,
 * Lap; var.C:30 default 1). */
static const double BSSN_SOA[25][3] = {
    {1, 1, 1}, {1, 1, 1}, {1, 1, 1}, {-1, -1, 1}, {-1, 1, -1}, {1, 1, 1}, {1, -1, -1}, {1, 1, 1},
    {1, 1, 1}, {-1, -1, 1}, {-1, 1, -1}, {1, 1, 1}, {1, -1, -1}, {1, 1, 1},
    {-1, 1, 1}, {1, -1, 1}, {1, 1, -1}, {1, 1, 1}, {-1, 1, 1}, {1, -1, 1}, {1, 1, -1},
    {-1, 1, 1}, {1, -1, 1}, {1, 1, -1},
    {1, 1, 1}};   /* Z4c Theta (Z4c_class.C var table: SSS, propspeed 1) */

const double *oracle_bssn_soa(int field) { return BSSN_SOA[field]; }
double oracle_bssn_propspeed(int field) { return (field == 0 || field == 1 || field == 17) ? sqrt(2.0) : 1.0; }

int oracle_compute_rhs_z4c(
    const int *ex, double T, const double *X, const double *Y, const double *Z,
    double *chi, double *trK, double *dxx, double *gxy, double *gxz, double *dyy, double *gyz, double *dzz,
    double *Axx, double *Axy, double *Axz, double *Ayy, double *Ayz, double *Azz,
    double *Gamx, double *Gamy, double *Gamz,
    double *Lap, double *betax, double *betay, double *betaz,
    double *dtSfx, double *dtSfy, double *dtSfz, double *TZ,
    double *chi_rhs, double *trK_rhs,
    double *gxx_rhs, double *gxy_rhs, double *gxz_rhs, double *gyy_rhs, double *gyz_rhs, double *gzz_rhs,
    double *Axx_rhs, double *Axy_rhs, double *Axz_rhs, double *Ayy_rhs, double *Ayz_rhs, double *Azz_rhs,
    double *Gamx_rhs, double *Gamy_rhs, double *Gamz_rhs,
    double *Lap_rhs, double *betax_rhs, double *betay_rhs, double *betaz_rhs,
    double *dtSfx_rhs, double *dtSfy_rhs, double *dtSfz_rhs, double *TZ_rhs,
    const double *rho, const double *Sx, const double *Sy, const double *Sz,
    const double *Sxx, const double *Sxy, const double *Sxz, const double *Syy, const double *Syz, const double *Szz,
    double *Gamxxx, double *Gamxxy, double *Gamxxz, double *Gamxyy, double *Gamxyz, double *Gamxzz,
    double *Gamyxx, double *Gamyxy, double *Gamyxz, double *Gamyyy, double *Gamyyz, double *Gamyzz,
    double *Gamzxx, double *Gamzxy, double *Gamzxz, double *Gamzyy, double *Gamzyz, double *Gamzzz,
    double *Rxx, double *Rxy, double *Rxz, double *Ryy, double *Ryz, double *Rzz,
    double *ham_Res, double *movx_Res, double *movy_Res, double *movz_Res,
    double *Gmx_Res, double *Gmy_Res, double *Gmz_Res,
    int Symmetry, int Lev, double eps, int co);

/* Z4c rhs call on 25-pointer lists (Z4c_class.C:207, :575) */
static int rhs_call_z4c(const int *ex, double T, const double *X, const double *Y, const double *Z, double **u,
                        double **r, double **s, const double *zero, int Symmetry, int lev, double eps, double **c)
{
    return oracle_compute_rhs_z4c(
        ex, T, X, Y, Z, u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7], u[8], u[9], u[10], u[11], u[12], u[13],
        u[14], u[15], u[16], u[17], u[18], u[19], u[20], u[21], u[22], u[23], u[24], r[0], r[1], r[2], r[3], r[4],
        r[5], r[6], r[7], r[8], r[9], r[10], r[11], r[12], r[13], r[14], r[15], r[16], r[17], r[18], r[19], r[20],
        r[21], r[22], r[23], r[24], zero, zero, zero, zero, zero, zero, zero, zero, zero, zero, s[0], s[1], s[2],
        s[3], s[4], s[5], s[6], s[7], s[8], s[9], s[10], s[11], s[12], s[13], s[14], s[15], s[16], s[17], s[18],
        s[19], s[20], s[21], s[22], s[23], c[0], c[1], c[2], c[3], c[4], c[5], c[6], Symmetry, lev, eps, 0);
}

/* rhs call on 24-pointer state / rhs lists with vacuum matter and scratch outputs */
static int rhs_call(const int *ex, double T, const double *X, const double *Y, const double *Z, double **u,
                    double **r, double **scratch31, const double *zero, int Symmetry, int lev, double eps, int co,
                    double **cons7)
{
    return oracle_compute_rhs_bssn(
        ex, T, X, Y, Z, u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7], u[8], u[9], u[10], u[11], u[12], u[13],
        u[14], u[15], u[16], u[17], u[18], u[19], u[20], u[21], u[22], u[23], r[0], r[1], r[2], r[3], r[4], r[5],
        r[6], r[7], r[8], r[9], r[10], r[11], r[12], r[13], r[14], r[15], r[16], r[17], r[18], r[19], r[20], r[21],
        r[22], r[23], zero, zero, zero, zero, zero, zero, zero, zero, zero, zero, scratch31[0], scratch31[1],
        scratch31[2], scratch31[3], scratch31[4], scratch31[5], scratch31[6], scratch31[7], scratch31[8],
        scratch31[9], scratch31[10], scratch31[11], scratch31[12], scratch31[13], scratch31[14], scratch31[15],
        scratch31[16], scratch31[17], scratch31[18], scratch31[19], scratch31[20], scratch31[21], scratch31[22],
        scratch31[23], cons7[0], cons7[1], cons7[2], cons7[3], cons7[4], cons7[5], cons7[6], Symmetry, lev, eps, co);
}

/*
 * One RK4 step of a single level-0 block that is the whole patch, in the order
 * of bssn_class::Step (bssn_class.C:3043-3158 predictor, :3401-3525
 * correctors, :3765-3795 and :3852-3853 list rotation).  u0 holds the state in
 * and out (24 fields).  chitiny is the already-shifted floor (chitiny - 1).
 * bbox = xmin,ymin,zmin,xmax,ymax,zmax of the patch.  Returns the NaN flag.
 */
int oracle_bssn_step_single(const int *ex, const double *X, const double *Y, const double *Z,
                            const double *bbox, double **u0, double dT, double eps, double chitiny,
                            int Symmetry, double T)
{
    long n = npts3(ex);
    double *buf = oalloc(n * (24 * 3 + 24 + 7 + 1));
    double *pre[24], *cor[24], *K[24], *scr[24], *cons[7];
    for (int f = 0; f < 24; ++f) {
        pre[f] = buf + n * f;
        cor[f] = buf + n * (24 + f);
        K[f] = buf + n * (48 + f);
        scr[f] = buf + n * (72 + f);
    }
    for (int c = 0; c < 7; ++c) cons[c] = buf + n * (96 + c);
    double *zero = buf + n * 103;
    int err = 0;
    /* predictor */
    oracle_enforce_ga(ex, u0[2], u0[3], u0[4], u0[5], u0[6], u0[7], u0[8], u0[9], u0[10], u0[11], u0[12], u0[13]);
    err |= rhs_call(ex, T, X, Y, Z, u0, K, scr, zero, Symmetry, 0, eps, 1, cons);
    for (int f = 0; f < 24; ++f) {
        oracle_sommerfeld_routbam(ex, X, Y, Z, bbox[0], bbox[1], bbox[2], bbox[3], bbox[4], bbox[5], K[f], u0[f],
                                  oracle_bssn_propspeed(f), oracle_bssn_soa(f), Symmetry);
        oracle_rungekutta4_rout(ex, dT, u0[f], pre[f], K[f], 0);
    }
    oracle_lowerboundset(ex, pre[0], chitiny);
    /* correctors */
    for (int it = 1; it < 4; ++it) {
        oracle_enforce_ga(ex, pre[2], pre[3], pre[4], pre[5], pre[6], pre[7], pre[8], pre[9], pre[10], pre[11],
                          pre[12], pre[13]);
        err |= rhs_call(ex, T, X, Y, Z, pre, cor, scr, zero, Symmetry, 0, eps, 1, cons);
        for (int f = 0; f < 24; ++f) {
            oracle_sommerfeld_routbam(ex, X, Y, Z, bbox[0], bbox[1], bbox[2], bbox[3], bbox[4], bbox[5], cor[f],
                                      pre[f], oracle_bssn_propspeed(f), oracle_bssn_soa(f), Symmetry);
            oracle_rungekutta4_rout(ex, dT, u0[f], cor[f], K[f], it);
        }
        oracle_lowerboundset(ex, cor[0], chitiny);
        if (it < 3)
            for (int f = 0; f < 24; ++f) {
                double *t = pre[f];
                pre[f] = cor[f];
                cor[f] = t;
            }
    }
    for (int f = 0; f < 24; ++f) memcpy(u0[f], cor[f], n * sizeof(double));
    free(buf);
    return err;
}

/*
 * One RK4 substep of one block, as bssn_class::Step runs it per block
 * (bssn_class.C:3043-3158 for sub == 0, :3401-3525 for sub = 1..3):
 * enforce_ga on the stage input (in place), compute_rhs_bssn, then per field
 * sommerfeld_routbam (lev == 0), rungekutta4_rout, sommerfeld_rout precor=1
 * (lev > 0), then lowerboundset on the stage output.
 *   sub == 0: input u0, rhs -> K, output -> out
 *   sub >= 1: input in,  rhs -> out (the reference's SynchList_cor), output -> out
 * pbbox is the patch bbox (with buffer) that decides the outer faces.
 * nf = 25 runs the Z4c right-hand side (Z4c_class::Step, Z4c_class.C:173-1045,
 * the same sequence with Theta as the 25th field).
 * Returns the NaN flag of the right-hand side.
 */
int oracle_evolve_substep(const int *ex, const double *X, const double *Y, const double *Z, const double *pbbox,
                          double **u0, double **in, double **out, double **K, int sub, double dT, double eps,
                          double chitiny, int Symmetry, int lev, int nf)
{
    long n = npts3(ex);
    double *buf = oalloc(n * (24 + 7 + 1));
    double *scr[24], *cons[7];
    for (int f = 0; f < 24; ++f) scr[f] = buf + n * f;
    for (int c = 0; c < 7; ++c) cons[c] = buf + n * (24 + c);
    double *zero = buf + n * 31;
    double **src = sub == 0 ? u0 : in;
    double **rtarget = sub == 0 ? K : out;
    oracle_enforce_ga(ex, src[2], src[3], src[4], src[5], src[6], src[7], src[8], src[9], src[10], src[11], src[12],
                      src[13]);
    int err = nf == 25 ? rhs_call_z4c(ex, 0.0, X, Y, Z, src, rtarget, scr, zero, Symmetry, lev, eps, cons)
                       : rhs_call(ex, 0.0, X, Y, Z, src, rtarget, scr, zero, Symmetry, lev, eps, 1, cons);
    for (int f = 0; f < nf; ++f) {
        if (lev == 0)
            oracle_sommerfeld_routbam(ex, X, Y, Z, pbbox[0], pbbox[1], pbbox[2], pbbox[3], pbbox[4], pbbox[5],
                                      rtarget[f], src[f], oracle_bssn_propspeed(f), oracle_bssn_soa(f), Symmetry);
        oracle_rungekutta4_rout(ex, dT, u0[f], out[f], K[f], sub);
        if (lev > 0)
            oracle_sommerfeld_rout(ex, X, Y, Z, pbbox[0], pbbox[1], pbbox[2], pbbox[3], pbbox[4], pbbox[5], u0[f],
                                   out[f], Symmetry, 1);
    }
    oracle_lowerboundset(ex, out[0], chitiny);
    free(buf);
    return err;
}

int oracle_bssn_substep(const int *ex, const double *X, const double *Y, const double *Z, const double *pbbox,
                        double **u0, double **in, double **out, double **K, int sub, double dT, double eps,
                        double chitiny, int Symmetry, int lev)
{
    return oracle_evolve_substep(ex, X, Y, Z, pbbox, u0, in, out, K, sub, dT, eps, chitiny, Symmetry, lev, 24);
}
