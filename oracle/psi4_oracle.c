/*
 * psi4_oracle.c -- the Newman-Penrose scalar Psi4 of a BSSN block
 * (getnp4.f90:12-452, the build's Psi4type 0 with tetradtype 2 and ABV 0,
 * macrodef.h:35, macrodef.fh:18, :71).
 *
 * TEST INFRASTRUCTURE ONLY (see oracle_common.h).  The physical Christoffel
 * symbols and Ricci tensor are inputs, as getnp4 takes them from
 * compute_rhs_bssn's outputs (bssn_class.C:6230-6262).  Statement order and
 * the left-to-right association of every expression are the Fortran's; the
 * whole-array statements are evaluated point by point, which changes nothing
 * since no statement reads a neighbour except the fderivs calls, made first.
 */
#include "oracle_common.h"

void oracle_fderivs(const int *ex, const double *f, double *fx, double *fy, double *fz,
                    const double *X, const double *Y, const double *Z,
                    double SYM1, double SYM2, double SYM3, int Symmetry);

/* getnp4.f90:12-452.  G: the 18 Christoffel arrays in the order Gamxxx ..
 * Gamzzz; R: Rxx Rxy Rxz Ryy Ryz Rzz. */
void oracle_getnp4(const int *ex, const double *X, const double *Y, const double *Z,
                   const double *chi, const double *trK,
                   const double *dxx, const double *gxy, const double *gxz,
                   const double *dyy, const double *gyz, const double *dzz,
                   const double *Axx, const double *Axy, const double *Axz,
                   const double *Ayy, const double *Ayz, const double *Azz,
                   const double *const *G, const double *const *R,
                   double *Rpsi4, double *Ipsi4, int symmetry)
{
    const double ONE = 1.0, TWO = 2.0, F1o3 = 1.0 / 3.0, SYM = 1.0, ANTI = -1.0;
    const double TINYRR = 1.0e-14;
    const long n = npts3(ex);
    /* derivatives first (:346-353) */
    double *d[8][3];
    for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 3; ++b) d[a][b] = oalloc(n);
    oracle_fderivs(ex, Axx, d[0][0], d[0][1], d[0][2], X, Y, Z, SYM, SYM, SYM, symmetry);
    oracle_fderivs(ex, Axy, d[1][0], d[1][1], d[1][2], X, Y, Z, ANTI, ANTI, SYM, symmetry);
    oracle_fderivs(ex, Axz, d[2][0], d[2][1], d[2][2], X, Y, Z, ANTI, SYM, ANTI, symmetry);
    oracle_fderivs(ex, Ayy, d[3][0], d[3][1], d[3][2], X, Y, Z, SYM, SYM, SYM, symmetry);
    oracle_fderivs(ex, Ayz, d[4][0], d[4][1], d[4][2], X, Y, Z, SYM, ANTI, ANTI, symmetry);
    oracle_fderivs(ex, Azz, d[5][0], d[5][1], d[5][2], X, Y, Z, SYM, SYM, SYM, symmetry);
    oracle_fderivs(ex, chi, d[6][0], d[6][1], d[6][2], X, Y, Z, SYM, SYM, SYM, symmetry);
    oracle_fderivs(ex, trK, d[7][0], d[7][1], d[7][2], X, Y, Z, SYM, SYM, SYM, symmetry);

    for (int k = 1; k <= ex[2]; ++k)
        for (int j = 1; j <= ex[1]; ++j)
            for (int i = 1; i <= ex[0]; ++i) {
                const long p = OIDX(ex, i, j, k);
                const double x = X[i - 1], y = Y[j - 1], z = Z[k - 1];
                const double gxx = dxx[p] + ONE, gyy = dyy[p] + ONE, gzz = dzz[p] + ONE;
                const double Gxy = gxy[p], Gxz = gxz[p], Gyz = gyz[p];
                const double chipn1 = chi[p] + ONE;
                /* :118-126 inverse conformal metric */
                double gupzz = gxx * gyy * gzz + Gxy * Gyz * Gxz + Gxz * Gxy * Gyz -
                               Gxz * gyy * Gxz - Gxy * Gxy * gzz - gxx * Gyz * Gyz;
                const double gupxx = (gyy * gzz - Gyz * Gyz) / gupzz;
                const double gupxy = -(Gxy * gzz - Gyz * Gxz) / gupzz;
                const double gupxz = (Gxy * Gyz - gyy * Gxz) / gupzz;
                const double gupyy = (gxx * gzz - Gxz * Gxz) / gupzz;
                const double gupyz = -(gxx * Gyz - Gxy * Gxz) / gupzz;
                gupzz = (gxx * gyy - Gxy * Gxy) / gupzz;
                /* :280-303 tetradtype 2: v radial, u azimuthal, w polar */
                double vx, vy, vz, ux, uy, uz, wx, wy, wz;
                if (fabs(x) < TINYRR && fabs(y) < TINYRR && fabs(z) < TINYRR) {
                    vx = TINYRR; vy = TINYRR; vz = TINYRR;
                } else {
                    vx = x; vy = y; vz = z;
                }
                if (fabs(x) < TINYRR && fabs(y) < TINYRR) {
                    ux = -TINYRR; uy = TINYRR; uz = 0.0;
                    wx = TINYRR * z; wy = TINYRR * z; wz = -2 * TINYRR * TINYRR;
                } else {
                    ux = -y; uy = x; uz = 0.0;
                    wx = x * z; wy = y * z; wz = -(x * x + y * y);
                }
                /* :305-310 raise v */
                {
                    const double fx = vx, fy = vy, fz = vz;
                    vx = gupxx * fx + gupxy * fy + gupxz * fz;
                    vy = gupxy * fx + gupyy * fy + gupyz * fz;
                    vz = gupxz * fx + gupyz * fy + gupzz * fz;
                }
                const double f = 1.0 / chipn1;
                /* :314-344 Gram-Schmidt in the physical metric gamma = g / chi */
                double fx = gxx * vx * vx + gyy * vy * vy + gzz * vz * vz +
                            (Gxy * vx * vy + Gxz * vx * vz + Gyz * vy * vz) * TWO;
                fx = sqrt(fx * f);
                vx = vx / fx; vy = vy / fx; vz = vz / fx;
                fx = gxx * vx * ux + Gxy * vx * uy + Gxz * vx * uz +
                     Gxy * vy * ux + gyy * vy * uy + Gyz * vy * uz +
                     Gxz * vz * ux + Gyz * vz * uy + gzz * vz * uz;
                fx = fx * f;
                ux = ux - fx * vx; uy = uy - fx * vy; uz = uz - fx * vz;
                fx = gxx * ux * ux + gyy * uy * uy + gzz * uz * uz +
                     (Gxy * ux * uy + Gxz * ux * uz + Gyz * uy * uz) * TWO;
                fx = sqrt(fx * f);
                ux = ux / fx; uy = uy / fx; uz = uz / fx;
                fx = gxx * vx * wx + Gxy * vx * wy + Gxz * vx * wz +
                     Gxy * vy * wx + gyy * vy * wy + Gyz * vy * wz +
                     Gxz * vz * wx + Gyz * vz * wy + gzz * vz * wz;
                fx = fx * f;
                wx = wx - fx * vx; wy = wy - fx * vy; wz = wz - fx * vz;
                fx = gxx * ux * wx + Gxy * ux * wy + Gxz * ux * wz +
                     Gxy * uy * wx + gyy * uy * wy + Gyz * uy * wz +
                     Gxz * uz * wx + Gyz * uz * wy + gzz * uz * wz;
                fx = fx * f;
                wx = wx - fx * ux; wy = wy - fx * uy; wz = wz - fx * uz;
                fx = gxx * wx * wx + gyy * wy * wy + gzz * wz * wz +
                     (Gxy * wx * wy + Gxz * wx * wz + Gyz * wy * wz) * TWO;
                fx = sqrt(fx * f);
                wx = wx / fx; wy = wy / fx; wz = wz / fx;

                const double axx = Axx[p], axy = Axy[p], axz = Axz[p], ayy = Ayy[p], ayz = Ayz[p], azz = Azz[p];
                const double K = trK[p];
                const double chix = d[6][0][p], chiy = d[6][1][p], chiz = d[6][2][p];
                const double tx = d[7][0][p], ty = d[7][1][p], tz = d[7][2][p];
                const double Gxxx = G[0][p], Gxxy = G[1][p], Gxxz = G[2][p], Gxyy = G[3][p], Gxyz = G[4][p], Gxzz = G[5][p];
                const double Gyxx = G[6][p], Gyxy = G[7][p], Gyxz = G[8][p], Gyyy = G[9][p], Gyyz = G[10][p], Gyzz = G[11][p];
                const double Gzxx = G[12][p], Gzxy = G[13][p], Gzxz = G[14][p], Gzyy = G[15][p], Gzyz = G[16][p], Gzzz = G[17][p];
                /* :355-390 D_k K_ij up to chi^-1 */
                double Axxx = d[0][0][p], Axxy = d[0][1][p], Axxz = d[0][2][p];
                double Axyx = d[1][0][p], Axyy = d[1][1][p], Axyz = d[1][2][p];
                double Axzx = d[2][0][p], Axzy = d[2][1][p], Axzz = d[2][2][p];
                double Ayyx = d[3][0][p], Ayyy = d[3][1][p], Ayyz = d[3][2][p];
                double Ayzx = d[4][0][p], Ayzy = d[4][1][p], Ayzz = d[4][2][p];
                double Azzx = d[5][0][p], Azzy = d[5][1][p], Azzz = d[5][2][p];
                Axxx = Axxx - (Gxxx * axx + Gyxx * axy + Gzxx * axz) * TWO - chix / chipn1 * axx + F1o3 * gxx * tx;
                Axxy = Axxy - (Gxxy * axx + Gyxy * axy + Gzxy * axz) * TWO - chiy / chipn1 * axx + F1o3 * gxx * ty;
                Axxz = Axxz - (Gxxz * axx + Gyxz * axy + Gzxz * axz) * TWO - chiz / chipn1 * axx + F1o3 * gxx * tz;
                Ayyx = Ayyx - (Gxxy * axy + Gyxy * ayy + Gzxy * ayz) * TWO - chix / chipn1 * ayy + F1o3 * gyy * tx;
                Ayyy = Ayyy - (Gxyy * axy + Gyyy * ayy + Gzyy * ayz) * TWO - chiy / chipn1 * ayy + F1o3 * gyy * ty;
                Ayyz = Ayyz - (Gxyz * axy + Gyyz * ayy + Gzyz * ayz) * TWO - chiz / chipn1 * ayy + F1o3 * gyy * tz;
                Azzx = Azzx - (Gxxz * axz + Gyxz * ayz + Gzxz * azz) * TWO - chix / chipn1 * azz + F1o3 * gzz * tx;
                Azzy = Azzy - (Gxyz * axz + Gyyz * ayz + Gzyz * azz) * TWO - chiy / chipn1 * azz + F1o3 * gzz * ty;
                Azzz = Azzz - (Gxzz * axz + Gyzz * ayz + Gzzz * azz) * TWO - chiz / chipn1 * azz + F1o3 * gzz * tz;
                Axyx = Axyx - (Gxxy * axx + Gyxy * axy + Gzxy * axz +
                               Gxxx * axy + Gyxx * ayy + Gzxx * ayz) - chix / chipn1 * axy + F1o3 * Gxy * tx;
                Axyy = Axyy - (Gxyy * axx + Gyyy * axy + Gzyy * axz +
                               Gxxy * axy + Gyxy * ayy + Gzxy * ayz) - chiy / chipn1 * axy + F1o3 * Gxy * ty;
                Axyz = Axyz - (Gxyz * axx + Gyyz * axy + Gzyz * axz +
                               Gxxz * axy + Gyxz * ayy + Gzxz * ayz) - chiz / chipn1 * axy + F1o3 * Gxy * tz;
                Axzx = Axzx - (Gxxz * axx + Gyxz * axy + Gzxz * axz +
                               Gxxx * axz + Gyxx * ayz + Gzxx * azz) - chix / chipn1 * axz + F1o3 * Gxz * tx;
                Axzy = Axzy - (Gxyz * axx + Gyyz * axy + Gzyz * axz +
                               Gxxy * axz + Gyxy * ayz + Gzxy * azz) - chiy / chipn1 * axz + F1o3 * Gxz * ty;
                Axzz = Axzz - (Gxzz * axx + Gyzz * axy + Gzzz * axz +
                               Gxxz * axz + Gyxz * ayz + Gzxz * azz) - chiz / chipn1 * axz + F1o3 * Gxz * tz;
                Ayzx = Ayzx - (Gxxz * axy + Gyxz * ayy + Gzxz * ayz +
                               Gxxy * axz + Gyxy * ayz + Gzxy * azz) - chix / chipn1 * ayz + F1o3 * Gyz * tx;
                Ayzy = Ayzy - (Gxyz * axy + Gyyz * ayy + Gzyz * ayz +
                               Gxyy * axz + Gyyy * ayz + Gzyy * azz) - chiy / chipn1 * ayz + F1o3 * Gyz * ty;
                Ayzz = Ayzz - (Gxzz * axy + Gyzz * ayy + Gzzz * ayz +
                               Gxyz * axz + Gyyz * ayz + Gzyz * azz) - chiz / chipn1 * ayz + F1o3 * Gyz * tz;
                /* :392-397 B_ij = v^k (D_k K_ij - D_j K_ik), symmetrised */
                const double Bxx = (vy * (Axxy - Axyx) + vz * (Axxz - Axzx)) * f;
                const double Byy = (vx * (Ayyx - Axyy) + vz * (Ayyz - Ayzy)) * f;
                const double Bzz = (vx * (Azzx - Axzz) + vy * (Azzy - Ayzz)) * f;
                const double Bxy = (vx * (Axyx - (Axxy + Axyx) / TWO) + vy * (Axyy - Ayyx) / TWO +
                                    vz * (Axyz - (Axzy + Ayzx) / TWO)) * f;
                const double Bxz = (vx * (Axzx - (Axxz + Axzx) / TWO) + vy * (Axzy - (Axyz + Ayzx) / TWO) +
                                    vz * (Axzz - Azzx) / TWO) * f;
                const double Byz = (vx * (Ayzx - (Axyz + Axzy) / TWO) + vy * (Ayzy - (Ayyz + Ayzy) / TWO) +
                                    vz * (Ayzz - Azzy) / TWO) * f;
                /* :401-407 K_ij up to chi^-1 */
                const double Kxx = axx + F1o3 * K * gxx, Kxy = axy + F1o3 * K * Gxy, Kxz = axz + F1o3 * K * Gxz;
                const double Kyy = ayy + F1o3 * K * gyy, Kyz = ayz + F1o3 * K * Gyz, Kzz = azz + F1o3 * K * gzz;
                /* :409-428 K_ik K^k_j */
                double Exx = gupxx * Kxx * Kxx + gupyy * Kxy * Kxy + gupzz * Kxz * Kxz +
                             TWO * (gupxy * Kxx * Kxy + gupxz * Kxx * Kxz + gupyz * Kxy * Kxz);
                double Eyy = gupxx * Kxy * Kxy + gupyy * Kyy * Kyy + gupzz * Kyz * Kyz +
                             TWO * (gupxy * Kxy * Kyy + gupxz * Kxy * Kyz + gupyz * Kyy * Kyz);
                double Ezz = gupxx * Kxz * Kxz + gupyy * Kyz * Kyz + gupzz * Kzz * Kzz +
                             TWO * (gupxy * Kxz * Kyz + gupxz * Kxz * Kzz + gupyz * Kyz * Kzz);
                double Exy = gupxx * Kxx * Kxy + gupyy * Kxy * Kyy + gupzz * Kxz * Kyz +
                             gupxy * (Kxx * Kyy + Kxy * Kxy) +
                             gupxz * (Kxx * Kyz + Kxz * Kxy) +
                             gupyz * (Kxy * Kyz + Kxz * Kyy);
                double Exz = gupxx * Kxx * Kxz + gupyy * Kxy * Kyz + gupzz * Kxz * Kzz +
                             gupxy * (Kxx * Kyz + Kxy * Kxz) +
                             gupxz * (Kxx * Kzz + Kxz * Kxz) +
                             gupyz * (Kxy * Kzz + Kxz * Kyz);
                double Eyz = gupxx * Kxy * Kxz + gupyy * Kyy * Kyz + gupzz * Kyz * Kzz +
                             gupxy * (Kxy * Kyz + Kyy * Kxz) +
                             gupxz * (Kxy * Kzz + Kyz * Kxz) +
                             gupyz * (Kyy * Kzz + Kyz * Kyz);
                /* :430-435 E_ij = R_ij - K_ik K^k_j + K K_ij - B_ij */
                Exx = R[0][p] - (Exx - Kxx * K) * f - Bxx;
                Exy = R[1][p] - (Exy - Kxy * K) * f - Bxy;
                Exz = R[2][p] - (Exz - Kxz * K) * f - Bxz;
                Eyy = R[3][p] - (Eyy - Kyy * K) * f - Byy;
                Eyz = R[4][p] - (Eyz - Kyz * K) * f - Byz;
                Ezz = R[5][p] - (Ezz - Kzz * K) * f - Bzz;
                /* :436-451 m = (u - i w)/sqrt(2): Psi4 = -(E_ij (u^i u^j - w^i w^j) + i E_ij (u^i w^j + w^i u^j))/2 */
                const double uuwwxx = ux * ux - wx * wx, uuwwxy = ux * uy - wx * wy, uuwwxz = ux * uz - wx * wz;
                const double uuwwyy = uy * uy - wy * wy, uuwwyz = uy * uz - wy * wz, uuwwzz = uz * uz - wz * wz;
                const double uwxx = ux * wx + wx * ux, uwxy = ux * wy + wx * uy, uwxz = ux * wz + wx * uz;
                const double uwyy = uy * wy + wy * uy, uwyz = uy * wz + wy * uz, uwzz = uz * wz + wz * uz;
                double rp = Exx * uuwwxx + Eyy * uuwwyy + Ezz * uuwwzz +
                            (Exy * uuwwxy + Exz * uuwwxz + Eyz * uuwwyz) * TWO;
                double ip = Exx * uwxx + Eyy * uwyy + Ezz * uwzz + (Exy * uwxy + Exz * uwxz + Eyz * uwyz) * TWO;
                Rpsi4[p] = -rp / TWO;
                Ipsi4[p] = -ip / TWO;
            }
    for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 3; ++b) free(d[a][b]);
}

/* fadmquantites_bssn.f90:5-65 admmass_bssn: the ADM-mass integrand
 * mass^i = (Gam^i / 8 + gup^ij chi_j / (4 (chi + 1)^1.25)) / (2 pi). */
void oracle_admmass_bssn(const int *ex, const double *X, const double *Y, const double *Z,
                         const double *chi, const double *dxx, const double *gxy, const double *gxz,
                         const double *dyy, const double *gyz, const double *dzz,
                         const double *Gamx, const double *Gamy, const double *Gamz,
                         double *massx, double *massy, double *massz, int symmetry)
{
    const double ONE = 1.0, F1o8 = 1.0 / 8.0, SYM = 1.0;
    const double PI = acos(-ONE);
    const double F1o2pi = ONE / (2.0 * PI);
    const long n = npts3(ex);
    double *chix = oalloc(n), *chiy = oalloc(n), *chiz = oalloc(n);
    oracle_fderivs(ex, chi, chix, chiy, chiz, X, Y, Z, SYM, SYM, SYM, symmetry);
    for (long p = 0; p < n; ++p) {
        const double gxx = dxx[p] + ONE, gyy = dyy[p] + ONE, gzz = dzz[p] + ONE;
        const double Gxy = gxy[p], Gxz = gxz[p], Gyz = gyz[p];
        double gupzz = gxx * gyy * gzz + Gxy * Gyz * Gxz + Gxz * Gxy * Gyz -
                       Gxz * gyy * Gxz - Gxy * Gxy * gzz - gxx * Gyz * Gyz;
        const double gupxx = (gyy * gzz - Gyz * Gyz) / gupzz;
        const double gupxy = -(Gxy * gzz - Gyz * Gxz) / gupzz;
        const double gupxz = (Gxy * Gyz - gyy * Gxz) / gupzz;
        const double gupyy = (gxx * gzz - Gxz * Gxz) / gupzz;
        const double gupyz = -(gxx * Gyz - Gxy * Gxz) / gupzz;
        gupzz = (gxx * gyy - Gxy * Gxy) / gupzz;
        const double f = 1 / 4.0 / pow(chi[p] + ONE, 1.25);
        massx[p] = (F1o8 * Gamx[p] + f * (gupxx * chix[p] + gupxy * chiy[p] + gupxz * chiz[p])) * F1o2pi;
        massy[p] = (F1o8 * Gamy[p] + f * (gupxy * chix[p] + gupyy * chiy[p] + gupyz * chiz[p])) * F1o2pi;
        massz[p] = (F1o8 * Gamz[p] + f * (gupxz * chix[p] + gupyz * chiy[p] + gupzz * chiz[p])) * F1o2pi;
    }
    free(chix);
    free(chiy);
    free(chiz);
}
