/*
 * z4c_oracle.c -- CPU oracle of compute_rhs_z4c (Z4c_rhs.f90:126-1295; GAUGE 0,
 * Cell, ghost_width 3; kappa1 = 0.02, kappa2 = 0, FF = 0.75, eta = 2 from
 * get_Z4cparameters, cpbc.f90:5-20).
 *
 * TEST INFRASTRUCTURE ONLY (see oracle_common.h).  Parity unpinned.
 *
 * Restates the Z4c right-hand side as whole-array loops in the Fortran's
 * order.  It shares its skeleton with bssn_oracle.c (comments citing
 * bssn_rhs.f90 mark that shared skeleton) and differs where
 * Z4c_rhs.f90 differs from bssn_rhs.f90: Theta (TZ) as the 25th field,
 * trKd = trK + 2 Theta in chi_rhs, A_ij_rhs and trK_rhs (:277, :1016-1050),
 * K_,i + Theta_,i / 2 in Gamma^i_rhs (:582-586), the trace of the A_ij
 * source taken from the Ricci scalar (:961-982), Theta_rhs = alpha H / 2
 * (:1077-1165), the constraint damping terms after advection (:1228-1233),
 * and KO on the full diagonal metric (:1240-1245).  Two blocks of the
 * Fortran are not restated because their results are overwritten before any
 * use: the polynomial and geometric Theta_rhs of :360-549 (overwritten at
 * :1165) and the inline momentum constraint of :1111-1161 (overwritten by
 * constraint_bssn at :1278).  The diagnostic outputs come from ricci_gamma
 * and constraint_bssn (:1266-1290), which evaluate the same formulas as the
 * inline Christoffel / Ricci / constraint blocks of bssn_rhs.f90 (ricci_gamma.f90:2-413,
 * bssn_constraint.f90:10-214); they are produced here by oracle_compute_rhs_bssn
 * with co = 0 on the first 24 fields.
 */
#include "oracle_common.h"
#include <stdio.h>

void oracle_fderivs(const int *ex, const double *f, double *fx, double *fy, double *fz,
                    const double *X, const double *Y, const double *Z,
                    double SYM1, double SYM2, double SYM3, int Symmetry);
void oracle_fdderivs(const int *ex, const double *f, double *fxx, double *fxy, double *fxz,
                     double *fyy, double *fyz, double *fzz,
                     const double *X, const double *Y, const double *Z,
                     double SYM1, double SYM2, double SYM3, int Symmetry);
void oracle_lopsided(const int *ex, const double *X, const double *Y, const double *Z,
                     const double *f, double *f_rhs, const double *Sfx, const double *Sfy,
                     const double *Sfz, int Symmetry, const double *SoA);
void oracle_kodis(const int *ex, const double *X, const double *Y, const double *Z,
                  const double *f, double *f_rhs, const double *SoA, int Symmetry, double eps);

int oracle_state_has_nan(long n, double *const *fields, int nfields);

#define PL _Pragma("omp parallel for schedule(static)") for (long p = 0; p < n; ++p)

int oracle_compute_rhs_bssn(
    const int *ex, double T, const double *X, const double *Y, const double *Z,
    double *chi, double *trK, double *dxx, double *gxy, double *gxz, double *dyy, double *gyz, double *dzz,
    double *Axx, double *Axy, double *Axz, double *Ayy, double *Ayz, double *Azz,
    double *Gamx, double *Gamy, double *Gamz,
    double *Lap, double *betax, double *betay, double *betaz,
    double *dtSfx, double *dtSfy, double *dtSfz,
    double *chi_rhs, double *trK_rhs,
    double *gxx_rhs, double *gxy_rhs, double *gxz_rhs, double *gyy_rhs, double *gyz_rhs, double *gzz_rhs,
    double *Axx_rhs, double *Axy_rhs, double *Axz_rhs, double *Ayy_rhs, double *Ayz_rhs, double *Azz_rhs,
    double *Gamx_rhs, double *Gamy_rhs, double *Gamz_rhs,
    double *Lap_rhs, double *betax_rhs, double *betay_rhs, double *betaz_rhs,
    double *dtSfx_rhs, double *dtSfy_rhs, double *dtSfz_rhs,
    const double *rho, const double *Sx, const double *Sy, const double *Sz,
    const double *Sxx, const double *Sxy, const double *Sxz, const double *Syy, const double *Syz, const double *Szz,
    double *Gamxxx, double *Gamxxy, double *Gamxxz, double *Gamxyy, double *Gamxyz, double *Gamxzz,
    double *Gamyxx, double *Gamyxy, double *Gamyxz, double *Gamyyy, double *Gamyyz, double *Gamyzz,
    double *Gamzxx, double *Gamzxy, double *Gamzxz, double *Gamzyy, double *Gamzyz, double *Gamzzz,
    double *Rxx, double *Rxy, double *Rxz, double *Ryy, double *Ryz, double *Rzz,
    double *ham_Res, double *movx_Res, double *movy_Res, double *movz_Res,
    double *Gmx_Res, double *Gmy_Res, double *Gmz_Res,
    int Symmetry, int Lev, double eps, int co);

int oracle_compute_rhs_z4c(
    const int *ex, double T, const double *X, const double *Y, const double *Z,
    double *chi, double *trK, double *dxx, double *gxy, double *gxz, double *dyy, double *gyz, double *dzz,
    double *Axx, double *Axy, double *Axz, double *Ayy, double *Ayz, double *Azz,
    double *Gamx, double *Gamy, double *Gamz,
    double *Lap, double *betax, double *betay, double *betaz,
    double *dtSfx, double *dtSfy, double *dtSfz,
    double *TZ,
    double *chi_rhs, double *trK_rhs,
    double *gxx_rhs, double *gxy_rhs, double *gxz_rhs, double *gyy_rhs, double *gyz_rhs, double *gzz_rhs,
    double *Axx_rhs, double *Axy_rhs, double *Axz_rhs, double *Ayy_rhs, double *Ayz_rhs, double *Azz_rhs,
    double *Gamx_rhs, double *Gamy_rhs, double *Gamz_rhs,
    double *Lap_rhs, double *betax_rhs, double *betay_rhs, double *betaz_rhs,
    double *dtSfx_rhs, double *dtSfy_rhs, double *dtSfz_rhs,
    double *TZ_rhs,
    const double *rho, const double *Sx, const double *Sy, const double *Sz,
    const double *Sxx, const double *Sxy, const double *Sxz, const double *Syy, const double *Syz, const double *Szz,
    double *Gamxxx, double *Gamxxy, double *Gamxxz, double *Gamxyy, double *Gamxyz, double *Gamxzz,
    double *Gamyxx, double *Gamyxy, double *Gamyxz, double *Gamyyy, double *Gamyyz, double *Gamyzz,
    double *Gamzxx, double *Gamzxy, double *Gamzxz, double *Gamzyy, double *Gamzyz, double *Gamzzz,
    double *Rxx, double *Rxy, double *Rxz, double *Ryy, double *Ryz, double *Rzz,
    double *ham_Res, double *movx_Res, double *movy_Res, double *movz_Res,
    double *Gmx_Res, double *Gmy_Res, double *Gmz_Res,
    int Symmetry, int Lev, double eps, int co)
{
    (void)co;   /* Z4c_rhs.f90:147: the constraints are always computed */
    const double kappa1 = 0.02, kappa2 = 0.0;   /* cpbc.f90:5-20 */
    (void)T;
    (void)Lev;
    const double ONE = 1.0, TWO = 2.0, FOUR = 4.0, EIGHT = 8.0, HALF = 0.5;
    const double SYM = 1.0, ANTI = -1.0;
    const double FF = 0.75, eta = 2.0;
    const double F1o3 = 1.0 / 3.0, F2o3 = 2.0 / 3.0, F3o2 = 1.5;
    const double F16 = 16.0, F8 = 8.0;
    long n = npts3(ex);

    {
        /* Z4c_rhs.f90:233-262: 25 fields summed */
        double *chk[25] = {chi, trK, dxx, gxy, gxz, dyy, gyz, dzz, Axx, Axy, Axz, Ayy, Ayz, Azz,
                           Gamx, Gamy, Gamz, Lap, betax, betay, betaz, dtSfx, dtSfy, dtSfz, TZ};
        if (oracle_state_has_nan(n, chk, 25)) return 1;
    }

    const double PI = acos(-ONE);
    /* temporaries, bssn_rhs.f90:68-84 */
    double *gxx = oalloc(n), *gyy = oalloc(n), *gzz = oalloc(n);
    double *chix = oalloc(n), *chiy = oalloc(n), *chiz = oalloc(n);
    double *gxxx = oalloc(n), *gxyx = oalloc(n), *gxzx = oalloc(n), *gyyx = oalloc(n), *gyzx = oalloc(n), *gzzx = oalloc(n);
    double *gxxy = oalloc(n), *gxyy = oalloc(n), *gxzy = oalloc(n), *gyyy = oalloc(n), *gyzy = oalloc(n), *gzzy = oalloc(n);
    double *gxxz = oalloc(n), *gxyz = oalloc(n), *gxzz = oalloc(n), *gyyz = oalloc(n), *gyzz = oalloc(n), *gzzz = oalloc(n);
    double *Lapx = oalloc(n), *Lapy = oalloc(n), *Lapz = oalloc(n);
    double *betaxx = oalloc(n), *betaxy = oalloc(n), *betaxz = oalloc(n);
    double *betayx = oalloc(n), *betayy = oalloc(n), *betayz = oalloc(n);
    double *betazx = oalloc(n), *betazy = oalloc(n), *betazz = oalloc(n);
    double *Gamxx = oalloc(n), *Gamxy = oalloc(n), *Gamxz = oalloc(n);
    double *Gamyx = oalloc(n), *Gamyy_ = oalloc(n), *Gamyz_ = oalloc(n);
    double *Gamzx = oalloc(n), *Gamzy = oalloc(n), *Gamzz_ = oalloc(n);
    double *Kx = oalloc(n), *Ky = oalloc(n), *Kz = oalloc(n), *div_beta = oalloc(n), *S = oalloc(n);
    double *f = oalloc(n), *fxx = oalloc(n), *fxy = oalloc(n), *fxz = oalloc(n), *fyy = oalloc(n), *fyz = oalloc(n), *fzz = oalloc(n);
    double *Gamxa = oalloc(n), *Gamya = oalloc(n), *Gamza = oalloc(n), *alpn1 = oalloc(n), *chin1 = oalloc(n);
    double *gupxx = oalloc(n), *gupxy = oalloc(n), *gupxz = oalloc(n), *gupyy = oalloc(n), *gupyz = oalloc(n), *gupzz = oalloc(n);
    double *trKd = oalloc(n), *Hc = oalloc(n);

    /* bssn_rhs.f90:146-150 */
    PL {
        alpn1[p] = Lap[p] + ONE;
        chin1[p] = chi[p] + ONE;
        gxx[p] = dxx[p] + ONE;
        gyy[p] = dyy[p] + ONE;
        gzz[p] = dzz[p] + ONE;
        trKd[p] = trK[p] + TWO * TZ[p];   /* Z4c_rhs.f90:277 */
    }
    /* bssn_rhs.f90:152-156 */
    oracle_fderivs(ex, betax, betaxx, betaxy, betaxz, X, Y, Z, ANTI, SYM, SYM, Symmetry);
    oracle_fderivs(ex, betay, betayx, betayy, betayz, X, Y, Z, SYM, ANTI, SYM, Symmetry);
    oracle_fderivs(ex, betaz, betazx, betazy, betazz, X, Y, Z, SYM, SYM, ANTI, Symmetry);
    PL div_beta[p] = betaxx[p] + betayy[p] + betazz[p];
    /* bssn_rhs.f90:158-160 */
    oracle_fderivs(ex, chi, chix, chiy, chiz, X, Y, Z, SYM, SYM, SYM, Symmetry);
    PL chi_rhs[p] = F2o3 * chin1[p] * (alpn1[p] * trKd[p] - div_beta[p]);   /* Z4c_rhs.f90:287 */
    /* bssn_rhs.f90:162-167 */
    oracle_fderivs(ex, dxx, gxxx, gxxy, gxxz, X, Y, Z, SYM, SYM, SYM, Symmetry);
    oracle_fderivs(ex, gxy, gxyx, gxyy, gxyz, X, Y, Z, ANTI, ANTI, SYM, Symmetry);
    oracle_fderivs(ex, gxz, gxzx, gxzy, gxzz, X, Y, Z, ANTI, SYM, ANTI, Symmetry);
    oracle_fderivs(ex, dyy, gyyx, gyyy, gyyz, X, Y, Z, SYM, SYM, SYM, Symmetry);
    oracle_fderivs(ex, gyz, gyzx, gyzy, gyzz, X, Y, Z, SYM, ANTI, ANTI, Symmetry);
    oracle_fderivs(ex, dzz, gzzx, gzzy, gzzz, X, Y, Z, SYM, SYM, SYM, Symmetry);

    PL {
        /* bssn_rhs.f90:169-191 */
        gxx_rhs[p] = -TWO * alpn1[p] * Axx[p] - F2o3 * gxx[p] * div_beta[p] +
                     TWO * (gxx[p] * betaxx[p] + gxy[p] * betayx[p] + gxz[p] * betazx[p]);
        gyy_rhs[p] = -TWO * alpn1[p] * Ayy[p] - F2o3 * gyy[p] * div_beta[p] +
                     TWO * (gxy[p] * betaxy[p] + gyy[p] * betayy[p] + gyz[p] * betazy[p]);
        gzz_rhs[p] = -TWO * alpn1[p] * Azz[p] - F2o3 * gzz[p] * div_beta[p] +
                     TWO * (gxz[p] * betaxz[p] + gyz[p] * betayz[p] + gzz[p] * betazz[p]);
        gxy_rhs[p] = -TWO * alpn1[p] * Axy[p] + F1o3 * gxy[p] * div_beta[p] +
                     gxx[p] * betaxy[p] + gxz[p] * betazy[p] + gyy[p] * betayx[p] + gyz[p] * betazx[p] -
                     gxy[p] * betazz[p];
        gyz_rhs[p] = -TWO * alpn1[p] * Ayz[p] + F1o3 * gyz[p] * div_beta[p] +
                     gxy[p] * betaxz[p] + gyy[p] * betayz[p] + gxz[p] * betaxy[p] + gzz[p] * betazy[p] -
                     gyz[p] * betaxx[p];
        gxz_rhs[p] = -TWO * alpn1[p] * Axz[p] + F1o3 * gxz[p] * div_beta[p] +
                     gxx[p] * betaxz[p] + gxy[p] * betayz[p] + gyz[p] * betayx[p] + gzz[p] * betazx[p] -
                     gxz[p] * betayy[p];
        /* bssn_rhs.f90:194-201 invert the conformal metric */
        gupzz[p] = gxx[p] * gyy[p] * gzz[p] + gxy[p] * gyz[p] * gxz[p] + gxz[p] * gxy[p] * gyz[p] -
                   gxz[p] * gyy[p] * gxz[p] - gxy[p] * gxy[p] * gzz[p] - gxx[p] * gyz[p] * gyz[p];
        gupxx[p] = (gyy[p] * gzz[p] - gyz[p] * gyz[p]) / gupzz[p];
        gupxy[p] = -(gxy[p] * gzz[p] - gyz[p] * gxz[p]) / gupzz[p];
        gupxz[p] = (gxy[p] * gyz[p] - gyy[p] * gxz[p]) / gupzz[p];
        gupyy[p] = (gxx[p] * gzz[p] - gxz[p] * gxz[p]) / gupzz[p];
        gupyz[p] = -(gxx[p] * gyz[p] - gxy[p] * gxz[p]) / gupzz[p];
        gupzz[p] = (gxx[p] * gyy[p] - gxy[p] * gxy[p]) / gupzz[p];
    }
    PL {
        double uxx = gupxx[p], uxy = gupxy[p], uxz = gupxz[p], uyy = gupyy[p], uyz = gupyz[p], uzz = gupzz[p];
        /* bssn_rhs.f90:235-257 second kind of connection (conformal) */
        Gamxxx[p] = HALF * (uxx * gxxx[p] + uxy * (TWO * gxyx[p] - gxxy[p]) + uxz * (TWO * gxzx[p] - gxxz[p]));
        Gamyxx[p] = HALF * (uxy * gxxx[p] + uyy * (TWO * gxyx[p] - gxxy[p]) + uyz * (TWO * gxzx[p] - gxxz[p]));
        Gamzxx[p] = HALF * (uxz * gxxx[p] + uyz * (TWO * gxyx[p] - gxxy[p]) + uzz * (TWO * gxzx[p] - gxxz[p]));
        Gamxyy[p] = HALF * (uxx * (TWO * gxyy[p] - gyyx[p]) + uxy * gyyy[p] + uxz * (TWO * gyzy[p] - gyyz[p]));
        Gamyyy[p] = HALF * (uxy * (TWO * gxyy[p] - gyyx[p]) + uyy * gyyy[p] + uyz * (TWO * gyzy[p] - gyyz[p]));
        Gamzyy[p] = HALF * (uxz * (TWO * gxyy[p] - gyyx[p]) + uyz * gyyy[p] + uzz * (TWO * gyzy[p] - gyyz[p]));
        Gamxzz[p] = HALF * (uxx * (TWO * gxzz[p] - gzzx[p]) + uxy * (TWO * gyzz[p] - gzzy[p]) + uxz * gzzz[p]);
        Gamyzz[p] = HALF * (uxy * (TWO * gxzz[p] - gzzx[p]) + uyy * (TWO * gyzz[p] - gzzy[p]) + uyz * gzzz[p]);
        Gamzzz[p] = HALF * (uxz * (TWO * gxzz[p] - gzzx[p]) + uyz * (TWO * gyzz[p] - gzzy[p]) + uzz * gzzz[p]);
        Gamxxy[p] = HALF * (uxx * gxxy[p] + uxy * gyyx[p] + uxz * (gxzy[p] + gyzx[p] - gxyz[p]));
        Gamyxy[p] = HALF * (uxy * gxxy[p] + uyy * gyyx[p] + uyz * (gxzy[p] + gyzx[p] - gxyz[p]));
        Gamzxy[p] = HALF * (uxz * gxxy[p] + uyz * gyyx[p] + uzz * (gxzy[p] + gyzx[p] - gxyz[p]));
        Gamxxz[p] = HALF * (uxx * gxxz[p] + uxy * (gxyz[p] + gyzx[p] - gxzy[p]) + uxz * gzzx[p]);
        Gamyxz[p] = HALF * (uxy * gxxz[p] + uyy * (gxyz[p] + gyzx[p] - gxzy[p]) + uyz * gzzx[p]);
        Gamzxz[p] = HALF * (uxz * gxxz[p] + uyz * (gxyz[p] + gyzx[p] - gxzy[p]) + uzz * gzzx[p]);
        Gamxyz[p] = HALF * (uxx * (gxyz[p] + gxzy[p] - gyzx[p]) + uxy * gyyz[p] + uxz * gzzy[p]);
        Gamyyz[p] = HALF * (uxy * (gxyz[p] + gxzy[p] - gyzx[p]) + uyy * gyyz[p] + uyz * gzzy[p]);
        Gamzyz[p] = HALF * (uxz * (gxyz[p] + gxzy[p] - gyzx[p]) + uyz * gyyz[p] + uzz * gzzy[p]);
        /* bssn_rhs.f90:260-282 raise the indices of A~_ij, stored in R_ij */
        double axx = Axx[p], axy = Axy[p], axz = Axz[p], ayy = Ayy[p], ayz = Ayz[p], azz = Azz[p];
        Rxx[p] = uxx * uxx * axx + uxy * uxy * ayy + uxz * uxz * azz +
                 TWO * (uxx * uxy * axy + uxx * uxz * axz + uxy * uxz * ayz);
        Ryy[p] = uxy * uxy * axx + uyy * uyy * ayy + uyz * uyz * azz +
                 TWO * (uxy * uyy * axy + uxy * uyz * axz + uyy * uyz * ayz);
        Rzz[p] = uxz * uxz * axx + uyz * uyz * ayy + uzz * uzz * azz +
                 TWO * (uxz * uyz * axy + uxz * uzz * axz + uyz * uzz * ayz);
        Rxy[p] = uxx * uxy * axx + uxy * uyy * ayy + uxz * uyz * azz +
                 (uxx * uyy + uxy * uxy) * axy + (uxx * uyz + uxz * uxy) * axz + (uxy * uyz + uxz * uyy) * ayz;
        Rxz[p] = uxx * uxz * axx + uxy * uyz * ayy + uxz * uzz * azz +
                 (uxx * uyz + uxy * uxz) * axy + (uxx * uzz + uxz * uxz) * axz + (uxy * uzz + uxz * uyz) * ayz;
        Ryz[p] = uxy * uxz * axx + uyy * uyz * ayy + uyz * uzz * azz +
                 (uxy * uyz + uyy * uxz) * axy + (uxy * uzz + uyz * uxz) * axz + (uyy * uzz + uyz * uyz) * ayz;
    }
    /* bssn_rhs.f90:285-313 */
    oracle_fderivs(ex, Lap, Lapx, Lapy, Lapz, X, Y, Z, SYM, SYM, SYM, Symmetry);
    oracle_fderivs(ex, trK, Kx, Ky, Kz, X, Y, Z, SYM, SYM, SYM, Symmetry);
    /* Z4c_rhs.f90:582-586 K_,i + Theta_,i / 2 */
    oracle_fderivs(ex, TZ, fxx, fxy, fxz, X, Y, Z, SYM, SYM, SYM, Symmetry);
    PL {
        Kx[p] = Kx[p] + fxx[p] / TWO;
        Ky[p] = Ky[p] + fxy[p] / TWO;
        Kz[p] = Kz[p] + fxz[p] / TWO;
    }
    PL {
        Gamx_rhs[p] = -TWO * (Lapx[p] * Rxx[p] + Lapy[p] * Rxy[p] + Lapz[p] * Rxz[p]) +
                      TWO * alpn1[p] * (-F3o2 / chin1[p] * (chix[p] * Rxx[p] + chiy[p] * Rxy[p] + chiz[p] * Rxz[p]) -
                                        gupxx[p] * (F2o3 * Kx[p] + EIGHT * PI * Sx[p]) -
                                        gupxy[p] * (F2o3 * Ky[p] + EIGHT * PI * Sy[p]) -
                                        gupxz[p] * (F2o3 * Kz[p] + EIGHT * PI * Sz[p]) +
                                        Gamxxx[p] * Rxx[p] + Gamxyy[p] * Ryy[p] + Gamxzz[p] * Rzz[p] +
                                        TWO * (Gamxxy[p] * Rxy[p] + Gamxxz[p] * Rxz[p] + Gamxyz[p] * Ryz[p]));
        Gamy_rhs[p] = -TWO * (Lapx[p] * Rxy[p] + Lapy[p] * Ryy[p] + Lapz[p] * Ryz[p]) +
                      TWO * alpn1[p] * (-F3o2 / chin1[p] * (chix[p] * Rxy[p] + chiy[p] * Ryy[p] + chiz[p] * Ryz[p]) -
                                        gupxy[p] * (F2o3 * Kx[p] + EIGHT * PI * Sx[p]) -
                                        gupyy[p] * (F2o3 * Ky[p] + EIGHT * PI * Sy[p]) -
                                        gupyz[p] * (F2o3 * Kz[p] + EIGHT * PI * Sz[p]) +
                                        Gamyxx[p] * Rxx[p] + Gamyyy[p] * Ryy[p] + Gamyzz[p] * Rzz[p] +
                                        TWO * (Gamyxy[p] * Rxy[p] + Gamyxz[p] * Rxz[p] + Gamyyz[p] * Ryz[p]));
        Gamz_rhs[p] = -TWO * (Lapx[p] * Rxz[p] + Lapy[p] * Ryz[p] + Lapz[p] * Rzz[p]) +
                      TWO * alpn1[p] * (-F3o2 / chin1[p] * (chix[p] * Rxz[p] + chiy[p] * Ryz[p] + chiz[p] * Rzz[p]) -
                                        gupxz[p] * (F2o3 * Kx[p] + EIGHT * PI * Sx[p]) -
                                        gupyz[p] * (F2o3 * Ky[p] + EIGHT * PI * Sy[p]) -
                                        gupzz[p] * (F2o3 * Kz[p] + EIGHT * PI * Sz[p]) +
                                        Gamzxx[p] * Rxx[p] + Gamzyy[p] * Ryy[p] + Gamzzz[p] * Rzz[p] +
                                        TWO * (Gamzxy[p] * Rxy[p] + Gamzxz[p] * Rxz[p] + Gamzyz[p] * Ryz[p]));
    }
    /* bssn_rhs.f90:315-331: second derivatives of the shift into the gij_k arrays */
    oracle_fdderivs(ex, betax, gxxx, gxyx, gxzx, gyyx, gyzx, gzzx, X, Y, Z, ANTI, SYM, SYM, Symmetry);
    oracle_fdderivs(ex, betay, gxxy, gxyy, gxzy, gyyy, gyzy, gzzy, X, Y, Z, SYM, ANTI, SYM, Symmetry);
    oracle_fdderivs(ex, betaz, gxxz, gxyz, gxzz, gyyz, gyzz, gzzz, X, Y, Z, SYM, SYM, ANTI, Symmetry);
    PL {
        fxx[p] = gxxx[p] + gxyy[p] + gxzz[p];
        fxy[p] = gxyx[p] + gyyy[p] + gyzz[p];
        fxz[p] = gxzx[p] + gyzy[p] + gzzz[p];
        Gamxa[p] = gupxx[p] * Gamxxx[p] + gupyy[p] * Gamxyy[p] + gupzz[p] * Gamxzz[p] +
                   TWO * (gupxy[p] * Gamxxy[p] + gupxz[p] * Gamxxz[p] + gupyz[p] * Gamxyz[p]);
        Gamya[p] = gupxx[p] * Gamyxx[p] + gupyy[p] * Gamyyy[p] + gupzz[p] * Gamyzz[p] +
                   TWO * (gupxy[p] * Gamyxy[p] + gupxz[p] * Gamyxz[p] + gupyz[p] * Gamyyz[p]);
        Gamza[p] = gupxx[p] * Gamzxx[p] + gupyy[p] * Gamzyy[p] + gupzz[p] * Gamzzz[p] +
                   TWO * (gupxy[p] * Gamzxy[p] + gupxz[p] * Gamzxz[p] + gupyz[p] * Gamzyz[p]);
    }
    /* bssn_rhs.f90:333-335 */
    oracle_fderivs(ex, Gamx, Gamxx, Gamxy, Gamxz, X, Y, Z, ANTI, SYM, SYM, Symmetry);
    oracle_fderivs(ex, Gamy, Gamyx, Gamyy_, Gamyz_, X, Y, Z, SYM, ANTI, SYM, Symmetry);
    oracle_fderivs(ex, Gamz, Gamzx, Gamzy, Gamzz_, X, Y, Z, SYM, SYM, ANTI, Symmetry);
    PL {
        /* bssn_rhs.f90:337-353 */
        Gamx_rhs[p] = Gamx_rhs[p] + F2o3 * Gamxa[p] * div_beta[p] -
                      Gamxa[p] * betaxx[p] - Gamya[p] * betaxy[p] - Gamza[p] * betaxz[p] +
                      F1o3 * (gupxx[p] * fxx[p] + gupxy[p] * fxy[p] + gupxz[p] * fxz[p]) +
                      gupxx[p] * gxxx[p] + gupyy[p] * gyyx[p] + gupzz[p] * gzzx[p] +
                      TWO * (gupxy[p] * gxyx[p] + gupxz[p] * gxzx[p] + gupyz[p] * gyzx[p]);
        Gamy_rhs[p] = Gamy_rhs[p] + F2o3 * Gamya[p] * div_beta[p] -
                      Gamxa[p] * betayx[p] - Gamya[p] * betayy[p] - Gamza[p] * betayz[p] +
                      F1o3 * (gupxy[p] * fxx[p] + gupyy[p] * fxy[p] + gupyz[p] * fxz[p]) +
                      gupxx[p] * gxxy[p] + gupyy[p] * gyyy[p] + gupzz[p] * gzzy[p] +
                      TWO * (gupxy[p] * gxyy[p] + gupxz[p] * gxzy[p] + gupyz[p] * gyzy[p]);
        Gamz_rhs[p] = Gamz_rhs[p] + F2o3 * Gamza[p] * div_beta[p] -
                      Gamxa[p] * betazx[p] - Gamya[p] * betazy[p] - Gamza[p] * betazz[p] +
                      F1o3 * (gupxz[p] * fxx[p] + gupyz[p] * fxy[p] + gupzz[p] * fxz[p]) +
                      gupxx[p] * gxxz[p] + gupyy[p] * gyyz[p] + gupzz[p] * gzzz[p] +
                      TWO * (gupxy[p] * gxyz[p] + gupxz[p] * gxzz[p] + gupyz[p] * gyzz[p]);
        /* bssn_rhs.f90:356-375 first kind of connection stored in gij_k */
        double g11 = gxx[p], g12 = gxy[p], g13 = gxz[p], g22 = gyy[p], g23 = gyz[p], g33 = gzz[p];
        gxxx[p] = g11 * Gamxxx[p] + g12 * Gamyxx[p] + g13 * Gamzxx[p];
        gxyx[p] = g11 * Gamxxy[p] + g12 * Gamyxy[p] + g13 * Gamzxy[p];
        gxzx[p] = g11 * Gamxxz[p] + g12 * Gamyxz[p] + g13 * Gamzxz[p];
        gyyx[p] = g11 * Gamxyy[p] + g12 * Gamyyy[p] + g13 * Gamzyy[p];
        gyzx[p] = g11 * Gamxyz[p] + g12 * Gamyyz[p] + g13 * Gamzyz[p];
        gzzx[p] = g11 * Gamxzz[p] + g12 * Gamyzz[p] + g13 * Gamzzz[p];
        gxxy[p] = g12 * Gamxxx[p] + g22 * Gamyxx[p] + g23 * Gamzxx[p];
        gxyy[p] = g12 * Gamxxy[p] + g22 * Gamyxy[p] + g23 * Gamzxy[p];
        gxzy[p] = g12 * Gamxxz[p] + g22 * Gamyxz[p] + g23 * Gamzxz[p];
        gyyy[p] = g12 * Gamxyy[p] + g22 * Gamyyy[p] + g23 * Gamzyy[p];
        gyzy[p] = g12 * Gamxyz[p] + g22 * Gamyyz[p] + g23 * Gamzyz[p];
        gzzy[p] = g12 * Gamxzz[p] + g22 * Gamyzz[p] + g23 * Gamzzz[p];
        gxxz[p] = g13 * Gamxxx[p] + g23 * Gamyxx[p] + g33 * Gamzxx[p];
        gxyz[p] = g13 * Gamxxy[p] + g23 * Gamyxy[p] + g33 * Gamzxy[p];
        gxzz[p] = g13 * Gamxxz[p] + g23 * Gamyxz[p] + g33 * Gamzxz[p];
        gyyz[p] = g13 * Gamxyy[p] + g23 * Gamyyy[p] + g33 * Gamzyy[p];
        gyzz[p] = g13 * Gamxyz[p] + g23 * Gamyyz[p] + g33 * Gamzyz[p];
        gzzz[p] = g13 * Gamxzz[p] + g23 * Gamyzz[p] + g33 * Gamzzz[p];
    }
    /* bssn_rhs.f90:378-400 Ricci tensor of the conformal metric: gup^kl d_k d_l g_ij */
#define RICCI_CONTRACT(R)                                                               \
    PL R[p] = gupxx[p] * fxx[p] + gupyy[p] * fyy[p] + gupzz[p] * fzz[p] +              \
              (gupxy[p] * fxy[p] + gupxz[p] * fxz[p] + gupyz[p] * fyz[p]) * TWO;
    oracle_fdderivs(ex, dxx, fxx, fxy, fxz, fyy, fyz, fzz, X, Y, Z, SYM, SYM, SYM, Symmetry);
    RICCI_CONTRACT(Rxx)
    oracle_fdderivs(ex, dyy, fxx, fxy, fxz, fyy, fyz, fzz, X, Y, Z, SYM, SYM, SYM, Symmetry);
    RICCI_CONTRACT(Ryy)
    oracle_fdderivs(ex, dzz, fxx, fxy, fxz, fyy, fyz, fzz, X, Y, Z, SYM, SYM, SYM, Symmetry);
    RICCI_CONTRACT(Rzz)
    oracle_fdderivs(ex, gxy, fxx, fxy, fxz, fyy, fyz, fzz, X, Y, Z, ANTI, ANTI, SYM, Symmetry);
    RICCI_CONTRACT(Rxy)
    oracle_fdderivs(ex, gxz, fxx, fxy, fxz, fyy, fyz, fzz, X, Y, Z, ANTI, SYM, ANTI, Symmetry);
    RICCI_CONTRACT(Rxz)
    oracle_fdderivs(ex, gyz, fxx, fxy, fxz, fyy, fyz, fzz, X, Y, Z, SYM, ANTI, ANTI, Symmetry);
    RICCI_CONTRACT(Ryz)
#undef RICCI_CONTRACT
    PL {
        /* bssn_rhs.f90:402-601 */
#define G(a) a[p]
        Rxx[p] = -HALF * G(Rxx) +
                 G(gxx) * G(Gamxx) + G(gxy) * G(Gamyx) + G(gxz) * G(Gamzx) +
                 G(Gamxa) * G(gxxx) + G(Gamya) * G(gxyx) + G(Gamza) * G(gxzx) +
                 G(gupxx) * (TWO * (G(Gamxxx) * G(gxxx) + G(Gamyxx) * G(gxyx) + G(Gamzxx) * G(gxzx)) +
                             G(Gamxxx) * G(gxxx) + G(Gamyxx) * G(gxxy) + G(Gamzxx) * G(gxxz)) +
                 G(gupxy) * (TWO * (G(Gamxxx) * G(gxyx) + G(Gamyxx) * G(gyyx) + G(Gamzxx) * G(gyzx) +
                                    G(Gamxxy) * G(gxxx) + G(Gamyxy) * G(gxyx) + G(Gamzxy) * G(gxzx)) +
                             G(Gamxxy) * G(gxxx) + G(Gamyxy) * G(gxxy) + G(Gamzxy) * G(gxxz) +
                             G(Gamxxx) * G(gxyx) + G(Gamyxx) * G(gxyy) + G(Gamzxx) * G(gxyz)) +
                 G(gupxz) * (TWO * (G(Gamxxx) * G(gxzx) + G(Gamyxx) * G(gyzx) + G(Gamzxx) * G(gzzx) +
                                    G(Gamxxz) * G(gxxx) + G(Gamyxz) * G(gxyx) + G(Gamzxz) * G(gxzx)) +
                             G(Gamxxz) * G(gxxx) + G(Gamyxz) * G(gxxy) + G(Gamzxz) * G(gxxz) +
                             G(Gamxxx) * G(gxzx) + G(Gamyxx) * G(gxzy) + G(Gamzxx) * G(gxzz)) +
                 G(gupyy) * (TWO * (G(Gamxxy) * G(gxyx) + G(Gamyxy) * G(gyyx) + G(Gamzxy) * G(gyzx)) +
                             G(Gamxxy) * G(gxyx) + G(Gamyxy) * G(gxyy) + G(Gamzxy) * G(gxyz)) +
                 G(gupyz) * (TWO * (G(Gamxxy) * G(gxzx) + G(Gamyxy) * G(gyzx) + G(Gamzxy) * G(gzzx) +
                                    G(Gamxxz) * G(gxyx) + G(Gamyxz) * G(gyyx) + G(Gamzxz) * G(gyzx)) +
                             G(Gamxxz) * G(gxyx) + G(Gamyxz) * G(gxyy) + G(Gamzxz) * G(gxyz) +
                             G(Gamxxy) * G(gxzx) + G(Gamyxy) * G(gxzy) + G(Gamzxy) * G(gxzz)) +
                 G(gupzz) * (TWO * (G(Gamxxz) * G(gxzx) + G(Gamyxz) * G(gyzx) + G(Gamzxz) * G(gzzx)) +
                             G(Gamxxz) * G(gxzx) + G(Gamyxz) * G(gxzy) + G(Gamzxz) * G(gxzz));

        Ryy[p] = -HALF * G(Ryy) +
                 G(gxy) * G(Gamxy) + G(gyy) * G(Gamyy_) + G(gyz) * G(Gamzy) +
                 G(Gamxa) * G(gxyy) + G(Gamya) * G(gyyy) + G(Gamza) * G(gyzy) +
                 G(gupxx) * (TWO * (G(Gamxxy) * G(gxxy) + G(Gamyxy) * G(gxyy) + G(Gamzxy) * G(gxzy)) +
                             G(Gamxxy) * G(gxyx) + G(Gamyxy) * G(gxyy) + G(Gamzxy) * G(gxyz)) +
                 G(gupxy) * (TWO * (G(Gamxxy) * G(gxyy) + G(Gamyxy) * G(gyyy) + G(Gamzxy) * G(gyzy) +
                                    G(Gamxyy) * G(gxxy) + G(Gamyyy) * G(gxyy) + G(Gamzyy) * G(gxzy)) +
                             G(Gamxyy) * G(gxyx) + G(Gamyyy) * G(gxyy) + G(Gamzyy) * G(gxyz) +
                             G(Gamxxy) * G(gyyx) + G(Gamyxy) * G(gyyy) + G(Gamzxy) * G(gyyz)) +
                 G(gupxz) * (TWO * (G(Gamxxy) * G(gxzy) + G(Gamyxy) * G(gyzy) + G(Gamzxy) * G(gzzy) +
                                    G(Gamxyz) * G(gxxy) + G(Gamyyz) * G(gxyy) + G(Gamzyz) * G(gxzy)) +
                             G(Gamxyz) * G(gxyx) + G(Gamyyz) * G(gxyy) + G(Gamzyz) * G(gxyz) +
                             G(Gamxxy) * G(gyzx) + G(Gamyxy) * G(gyzy) + G(Gamzxy) * G(gyzz)) +
                 G(gupyy) * (TWO * (G(Gamxyy) * G(gxyy) + G(Gamyyy) * G(gyyy) + G(Gamzyy) * G(gyzy)) +
                             G(Gamxyy) * G(gyyx) + G(Gamyyy) * G(gyyy) + G(Gamzyy) * G(gyyz)) +
                 G(gupyz) * (TWO * (G(Gamxyy) * G(gxzy) + G(Gamyyy) * G(gyzy) + G(Gamzyy) * G(gzzy) +
                                    G(Gamxyz) * G(gxyy) + G(Gamyyz) * G(gyyy) + G(Gamzyz) * G(gyzy)) +
                             G(Gamxyz) * G(gyyx) + G(Gamyyz) * G(gyyy) + G(Gamzyz) * G(gyyz) +
                             G(Gamxyy) * G(gyzx) + G(Gamyyy) * G(gyzy) + G(Gamzyy) * G(gyzz)) +
                 G(gupzz) * (TWO * (G(Gamxyz) * G(gxzy) + G(Gamyyz) * G(gyzy) + G(Gamzyz) * G(gzzy)) +
                             G(Gamxyz) * G(gyzx) + G(Gamyyz) * G(gyzy) + G(Gamzyz) * G(gyzz));

        Rzz[p] = -HALF * G(Rzz) +
                 G(gxz) * G(Gamxz) + G(gyz) * G(Gamyz_) + G(gzz) * G(Gamzz_) +
                 G(Gamxa) * G(gxzz) + G(Gamya) * G(gyzz) + G(Gamza) * G(gzzz) +
                 G(gupxx) * (TWO * (G(Gamxxz) * G(gxxz) + G(Gamyxz) * G(gxyz) + G(Gamzxz) * G(gxzz)) +
                             G(Gamxxz) * G(gxzx) + G(Gamyxz) * G(gxzy) + G(Gamzxz) * G(gxzz)) +
                 G(gupxy) * (TWO * (G(Gamxxz) * G(gxyz) + G(Gamyxz) * G(gyyz) + G(Gamzxz) * G(gyzz) +
                                    G(Gamxyz) * G(gxxz) + G(Gamyyz) * G(gxyz) + G(Gamzyz) * G(gxzz)) +
                             G(Gamxyz) * G(gxzx) + G(Gamyyz) * G(gxzy) + G(Gamzyz) * G(gxzz) +
                             G(Gamxxz) * G(gyzx) + G(Gamyxz) * G(gyzy) + G(Gamzxz) * G(gyzz)) +
                 G(gupxz) * (TWO * (G(Gamxxz) * G(gxzz) + G(Gamyxz) * G(gyzz) + G(Gamzxz) * G(gzzz) +
                                    G(Gamxzz) * G(gxxz) + G(Gamyzz) * G(gxyz) + G(Gamzzz) * G(gxzz)) +
                             G(Gamxzz) * G(gxzx) + G(Gamyzz) * G(gxzy) + G(Gamzzz) * G(gxzz) +
                             G(Gamxxz) * G(gzzx) + G(Gamyxz) * G(gzzy) + G(Gamzxz) * G(gzzz)) +
                 G(gupyy) * (TWO * (G(Gamxyz) * G(gxyz) + G(Gamyyz) * G(gyyz) + G(Gamzyz) * G(gyzz)) +
                             G(Gamxyz) * G(gyzx) + G(Gamyyz) * G(gyzy) + G(Gamzyz) * G(gyzz)) +
                 G(gupyz) * (TWO * (G(Gamxyz) * G(gxzz) + G(Gamyyz) * G(gyzz) + G(Gamzyz) * G(gzzz) +
                                    G(Gamxzz) * G(gxyz) + G(Gamyzz) * G(gyyz) + G(Gamzzz) * G(gyzz)) +
                             G(Gamxzz) * G(gyzx) + G(Gamyzz) * G(gyzy) + G(Gamzzz) * G(gyzz) +
                             G(Gamxyz) * G(gzzx) + G(Gamyyz) * G(gzzy) + G(Gamzyz) * G(gzzz)) +
                 G(gupzz) * (TWO * (G(Gamxzz) * G(gxzz) + G(Gamyzz) * G(gyzz) + G(Gamzzz) * G(gzzz)) +
                             G(Gamxzz) * G(gzzx) + G(Gamyzz) * G(gzzy) + G(Gamzzz) * G(gzzz));

        Rxy[p] = HALF * (-G(Rxy) +
                         G(gxx) * G(Gamxy) + G(gxy) * G(Gamyy_) + G(gxz) * G(Gamzy) +
                         G(gxy) * G(Gamxx) + G(gyy) * G(Gamyx) + G(gyz) * G(Gamzx) +
                         G(Gamxa) * G(gxyx) + G(Gamya) * G(gyyx) + G(Gamza) * G(gyzx) +
                         G(Gamxa) * G(gxxy) + G(Gamya) * G(gxyy) + G(Gamza) * G(gxzy)) +
                 G(gupxx) * (G(Gamxxx) * G(gxxy) + G(Gamyxx) * G(gxyy) + G(Gamzxx) * G(gxzy) +
                             G(Gamxxy) * G(gxxx) + G(Gamyxy) * G(gxyx) + G(Gamzxy) * G(gxzx) +
                             G(Gamxxx) * G(gxyx) + G(Gamyxx) * G(gxyy) + G(Gamzxx) * G(gxyz)) +
                 G(gupxy) * (G(Gamxxx) * G(gxyy) + G(Gamyxx) * G(gyyy) + G(Gamzxx) * G(gyzy) +
                             G(Gamxxy) * G(gxyx) + G(Gamyxy) * G(gyyx) + G(Gamzxy) * G(gyzx) +
                             G(Gamxxy) * G(gxyx) + G(Gamyxy) * G(gxyy) + G(Gamzxy) * G(gxyz) +
                             G(Gamxxy) * G(gxxy) + G(Gamyxy) * G(gxyy) + G(Gamzxy) * G(gxzy) +
                             G(Gamxyy) * G(gxxx) + G(Gamyyy) * G(gxyx) + G(Gamzyy) * G(gxzx) +
                             G(Gamxxx) * G(gyyx) + G(Gamyxx) * G(gyyy) + G(Gamzxx) * G(gyyz)) +
                 G(gupxz) * (G(Gamxxx) * G(gxzy) + G(Gamyxx) * G(gyzy) + G(Gamzxx) * G(gzzy) +
                             G(Gamxxy) * G(gxzx) + G(Gamyxy) * G(gyzx) + G(Gamzxy) * G(gzzx) +
                             G(Gamxxz) * G(gxyx) + G(Gamyxz) * G(gxyy) + G(Gamzxz) * G(gxyz) +
                             G(Gamxxz) * G(gxxy) + G(Gamyxz) * G(gxyy) + G(Gamzxz) * G(gxzy) +
                             G(Gamxyz) * G(gxxx) + G(Gamyyz) * G(gxyx) + G(Gamzyz) * G(gxzx) +
                             G(Gamxxx) * G(gyzx) + G(Gamyxx) * G(gyzy) + G(Gamzxx) * G(gyzz)) +
                 G(gupyy) * (G(Gamxxy) * G(gxyy) + G(Gamyxy) * G(gyyy) + G(Gamzxy) * G(gyzy) +
                             G(Gamxyy) * G(gxyx) + G(Gamyyy) * G(gyyx) + G(Gamzyy) * G(gyzx) +
                             G(Gamxxy) * G(gyyx) + G(Gamyxy) * G(gyyy) + G(Gamzxy) * G(gyyz)) +
                 G(gupyz) * (G(Gamxxy) * G(gxzy) + G(Gamyxy) * G(gyzy) + G(Gamzxy) * G(gzzy) +
                             G(Gamxyy) * G(gxzx) + G(Gamyyy) * G(gyzx) + G(Gamzyy) * G(gzzx) +
                             G(Gamxxz) * G(gyyx) + G(Gamyxz) * G(gyyy) + G(Gamzxz) * G(gyyz) +
                             G(Gamxxz) * G(gxyy) + G(Gamyxz) * G(gyyy) + G(Gamzxz) * G(gyzy) +
                             G(Gamxyz) * G(gxyx) + G(Gamyyz) * G(gyyx) + G(Gamzyz) * G(gyzx) +
                             G(Gamxxy) * G(gyzx) + G(Gamyxy) * G(gyzy) + G(Gamzxy) * G(gyzz)) +
                 G(gupzz) * (G(Gamxxz) * G(gxzy) + G(Gamyxz) * G(gyzy) + G(Gamzxz) * G(gzzy) +
                             G(Gamxyz) * G(gxzx) + G(Gamyyz) * G(gyzx) + G(Gamzyz) * G(gzzx) +
                             G(Gamxxz) * G(gyzx) + G(Gamyxz) * G(gyzy) + G(Gamzxz) * G(gyzz));

        Rxz[p] = HALF * (-G(Rxz) +
                         G(gxx) * G(Gamxz) + G(gxy) * G(Gamyz_) + G(gxz) * G(Gamzz_) +
                         G(gxz) * G(Gamxx) + G(gyz) * G(Gamyx) + G(gzz) * G(Gamzx) +
                         G(Gamxa) * G(gxzx) + G(Gamya) * G(gyzx) + G(Gamza) * G(gzzx) +
                         G(Gamxa) * G(gxxz) + G(Gamya) * G(gxyz) + G(Gamza) * G(gxzz)) +
                 G(gupxx) * (G(Gamxxx) * G(gxxz) + G(Gamyxx) * G(gxyz) + G(Gamzxx) * G(gxzz) +
                             G(Gamxxz) * G(gxxx) + G(Gamyxz) * G(gxyx) + G(Gamzxz) * G(gxzx) +
                             G(Gamxxx) * G(gxzx) + G(Gamyxx) * G(gxzy) + G(Gamzxx) * G(gxzz)) +
                 G(gupxy) * (G(Gamxxx) * G(gxyz) + G(Gamyxx) * G(gyyz) + G(Gamzxx) * G(gyzz) +
                             G(Gamxxz) * G(gxyx) + G(Gamyxz) * G(gyyx) + G(Gamzxz) * G(gyzx) +
                             G(Gamxxy) * G(gxzx) + G(Gamyxy) * G(gxzy) + G(Gamzxy) * G(gxzz) +
                             G(Gamxxy) * G(gxxz) + G(Gamyxy) * G(gxyz) + G(Gamzxy) * G(gxzz) +
                             G(Gamxyz) * G(gxxx) + G(Gamyyz) * G(gxyx) + G(Gamzyz) * G(gxzx) +
                             G(Gamxxx) * G(gyzx) + G(Gamyxx) * G(gyzy) + G(Gamzxx) * G(gyzz)) +
                 G(gupxz) * (G(Gamxxx) * G(gxzz) + G(Gamyxx) * G(gyzz) + G(Gamzxx) * G(gzzz) +
                             G(Gamxxz) * G(gxzx) + G(Gamyxz) * G(gyzx) + G(Gamzxz) * G(gzzx) +
                             G(Gamxxz) * G(gxzx) + G(Gamyxz) * G(gxzy) + G(Gamzxz) * G(gxzz) +
                             G(Gamxxz) * G(gxxz) + G(Gamyxz) * G(gxyz) + G(Gamzxz) * G(gxzz) +
                             G(Gamxzz) * G(gxxx) + G(Gamyzz) * G(gxyx) + G(Gamzzz) * G(gxzx) +
                             G(Gamxxx) * G(gzzx) + G(Gamyxx) * G(gzzy) + G(Gamzxx) * G(gzzz)) +
                 G(gupyy) * (G(Gamxxy) * G(gxyz) + G(Gamyxy) * G(gyyz) + G(Gamzxy) * G(gyzz) +
                             G(Gamxyz) * G(gxyx) + G(Gamyyz) * G(gyyx) + G(Gamzyz) * G(gyzx) +
                             G(Gamxxy) * G(gyzx) + G(Gamyxy) * G(gyzy) + G(Gamzxy) * G(gyzz)) +
                 G(gupyz) * (G(Gamxxy) * G(gxzz) + G(Gamyxy) * G(gyzz) + G(Gamzxy) * G(gzzz) +
                             G(Gamxyz) * G(gxzx) + G(Gamyyz) * G(gyzx) + G(Gamzyz) * G(gzzx) +
                             G(Gamxxz) * G(gyzx) + G(Gamyxz) * G(gyzy) + G(Gamzxz) * G(gyzz) +
                             G(Gamxxz) * G(gxyz) + G(Gamyxz) * G(gyyz) + G(Gamzxz) * G(gyzz) +
                             G(Gamxzz) * G(gxyx) + G(Gamyzz) * G(gyyx) + G(Gamzzz) * G(gyzx) +
                             G(Gamxxy) * G(gzzx) + G(Gamyxy) * G(gzzy) + G(Gamzxy) * G(gzzz)) +
                 G(gupzz) * (G(Gamxxz) * G(gxzz) + G(Gamyxz) * G(gyzz) + G(Gamzxz) * G(gzzz) +
                             G(Gamxzz) * G(gxzx) + G(Gamyzz) * G(gyzx) + G(Gamzzz) * G(gzzx) +
                             G(Gamxxz) * G(gzzx) + G(Gamyxz) * G(gzzy) + G(Gamzxz) * G(gzzz));

        Ryz[p] = HALF * (-G(Ryz) +
                         G(gxy) * G(Gamxz) + G(gyy) * G(Gamyz_) + G(gyz) * G(Gamzz_) +
                         G(gxz) * G(Gamxy) + G(gyz) * G(Gamyy_) + G(gzz) * G(Gamzy) +
                         G(Gamxa) * G(gxzy) + G(Gamya) * G(gyzy) + G(Gamza) * G(gzzy) +
                         G(Gamxa) * G(gxyz) + G(Gamya) * G(gyyz) + G(Gamza) * G(gyzz)) +
                 G(gupxx) * (G(Gamxxy) * G(gxxz) + G(Gamyxy) * G(gxyz) + G(Gamzxy) * G(gxzz) +
                             G(Gamxxz) * G(gxxy) + G(Gamyxz) * G(gxyy) + G(Gamzxz) * G(gxzy) +
                             G(Gamxxy) * G(gxzx) + G(Gamyxy) * G(gxzy) + G(Gamzxy) * G(gxzz)) +
                 G(gupxy) * (G(Gamxxy) * G(gxyz) + G(Gamyxy) * G(gyyz) + G(Gamzxy) * G(gyzz) +
                             G(Gamxxz) * G(gxyy) + G(Gamyxz) * G(gyyy) + G(Gamzxz) * G(gyzy) +
                             G(Gamxyy) * G(gxzx) + G(Gamyyy) * G(gxzy) + G(Gamzyy) * G(gxzz) +
                             G(Gamxyy) * G(gxxz) + G(Gamyyy) * G(gxyz) + G(Gamzyy) * G(gxzz) +
                             G(Gamxyz) * G(gxxy) + G(Gamyyz) * G(gxyy) + G(Gamzyz) * G(gxzy) +
                             G(Gamxxy) * G(gyzx) + G(Gamyxy) * G(gyzy) + G(Gamzxy) * G(gyzz)) +
                 G(gupxz) * (G(Gamxxy) * G(gxzz) + G(Gamyxy) * G(gyzz) + G(Gamzxy) * G(gzzz) +
                             G(Gamxxz) * G(gxzy) + G(Gamyxz) * G(gyzy) + G(Gamzxz) * G(gzzy) +
                             G(Gamxyz) * G(gxzx) + G(Gamyyz) * G(gxzy) + G(Gamzyz) * G(gxzz) +
                             G(Gamxyz) * G(gxxz) + G(Gamyyz) * G(gxyz) + G(Gamzyz) * G(gxzz) +
                             G(Gamxzz) * G(gxxy) + G(Gamyzz) * G(gxyy) + G(Gamzzz) * G(gxzy) +
                             G(Gamxxy) * G(gzzx) + G(Gamyxy) * G(gzzy) + G(Gamzxy) * G(gzzz)) +
                 G(gupyy) * (G(Gamxyy) * G(gxyz) + G(Gamyyy) * G(gyyz) + G(Gamzyy) * G(gyzz) +
                             G(Gamxyz) * G(gxyy) + G(Gamyyz) * G(gyyy) + G(Gamzyz) * G(gyzy) +
                             G(Gamxyy) * G(gyzx) + G(Gamyyy) * G(gyzy) + G(Gamzyy) * G(gyzz)) +
                 G(gupyz) * (G(Gamxyy) * G(gxzz) + G(Gamyyy) * G(gyzz) + G(Gamzyy) * G(gzzz) +
                             G(Gamxyz) * G(gxzy) + G(Gamyyz) * G(gyzy) + G(Gamzyz) * G(gzzy) +
                             G(Gamxyz) * G(gyzx) + G(Gamyyz) * G(gyzy) + G(Gamzyz) * G(gyzz) +
                             G(Gamxyz) * G(gxyz) + G(Gamyyz) * G(gyyz) + G(Gamzyz) * G(gyzz) +
                             G(Gamxzz) * G(gxyy) + G(Gamyzz) * G(gyyy) + G(Gamzzz) * G(gyzy) +
                             G(Gamxyy) * G(gzzx) + G(Gamyyy) * G(gzzy) + G(Gamzyy) * G(gzzz)) +
                 G(gupzz) * (G(Gamxyz) * G(gxzz) + G(Gamyyz) * G(gyzz) + G(Gamzyz) * G(gzzz) +
                             G(Gamxzz) * G(gxzy) + G(Gamyzz) * G(gyzy) + G(Gamzzz) * G(gzzy) +
                             G(Gamxyz) * G(gzzx) + G(Gamyyz) * G(gzzy) + G(Gamzyz) * G(gzzz));
    }
    /* bssn_rhs.f90:603-626 covariant second derivative of chi w.r.t. the conformal metric */
    oracle_fdderivs(ex, chi, fxx, fxy, fxz, fyy, fyz, fzz, X, Y, Z, SYM, SYM, SYM, Symmetry);
    PL {
        fxx[p] = fxx[p] - G(Gamxxx) * G(chix) - G(Gamyxx) * G(chiy) - G(Gamzxx) * G(chiz);
        fxy[p] = fxy[p] - G(Gamxxy) * G(chix) - G(Gamyxy) * G(chiy) - G(Gamzxy) * G(chiz);
        fxz[p] = fxz[p] - G(Gamxxz) * G(chix) - G(Gamyxz) * G(chiy) - G(Gamzxz) * G(chiz);
        fyy[p] = fyy[p] - G(Gamxyy) * G(chix) - G(Gamyyy) * G(chiy) - G(Gamzyy) * G(chiz);
        fyz[p] = fyz[p] - G(Gamxyz) * G(chix) - G(Gamyyz) * G(chiy) - G(Gamzyz) * G(chiz);
        fzz[p] = fzz[p] - G(Gamxzz) * G(chix) - G(Gamyzz) * G(chiy) - G(Gamzzz) * G(chiz);
        double c = chin1[p];
        f[p] = G(gupxx) * (G(fxx) - F3o2 / c * G(chix) * G(chix)) +
               G(gupyy) * (G(fyy) - F3o2 / c * G(chiy) * G(chiy)) +
               G(gupzz) * (G(fzz) - F3o2 / c * G(chiz) * G(chiz)) +
               TWO * G(gupxy) * (G(fxy) - F3o2 / c * G(chix) * G(chiy)) +
               TWO * G(gupxz) * (G(fxz) - F3o2 / c * G(chix) * G(chiz)) +
               TWO * G(gupyz) * (G(fyz) - F3o2 / c * G(chiy) * G(chiz));
        Rxx[p] = Rxx[p] + (G(fxx) - G(chix) * G(chix) / c / TWO + G(gxx) * G(f)) / c / TWO;
        Ryy[p] = Ryy[p] + (G(fyy) - G(chiy) * G(chiy) / c / TWO + G(gyy) * G(f)) / c / TWO;
        Rzz[p] = Rzz[p] + (G(fzz) - G(chiz) * G(chiz) / c / TWO + G(gzz) * G(f)) / c / TWO;
        Rxy[p] = Rxy[p] + (G(fxy) - G(chix) * G(chiy) / c / TWO + G(gxy) * G(f)) / c / TWO;
        Rxz[p] = Rxz[p] + (G(fxz) - G(chix) * G(chiz) / c / TWO + G(gxz) * G(f)) / c / TWO;
        Ryz[p] = Ryz[p] + (G(fyz) - G(chiy) * G(chiz) / c / TWO + G(gyz) * G(f)) / c / TWO;
        /* Z4c_rhs.f90:913-915 R / chi */
        Hc[p] = G(gupxx) * G(Rxx) + G(gupyy) * G(Ryy) + G(gupzz) * G(Rzz) +
                TWO * (G(gupxy) * G(Rxy) + G(gupxz) * G(Rxz) + G(gupyz) * G(Ryz));
    }
    /* bssn_rhs.f90:629-799 */
    oracle_fdderivs(ex, Lap, fxx, fxy, fxz, fyy, fyz, fzz, X, Y, Z, SYM, SYM, SYM, Symmetry);
    PL {
        double c = chin1[p];
        gxxx[p] = (G(gupxx) * G(chix) + G(gupxy) * G(chiy) + G(gupxz) * G(chiz)) / c;
        gxxy[p] = (G(gupxy) * G(chix) + G(gupyy) * G(chiy) + G(gupyz) * G(chiz)) / c;
        gxxz[p] = (G(gupxz) * G(chix) + G(gupyz) * G(chiy) + G(gupzz) * G(chiz)) / c;
        /* physical second kind of connection */
        Gamxxx[p] = Gamxxx[p] - ((G(chix) + G(chix)) / c - G(gxx) * G(gxxx)) * HALF;
        Gamyxx[p] = Gamyxx[p] - (-G(gxx) * G(gxxy)) * HALF;
        Gamzxx[p] = Gamzxx[p] - (-G(gxx) * G(gxxz)) * HALF;
        Gamxyy[p] = Gamxyy[p] - (-G(gyy) * G(gxxx)) * HALF;
        Gamyyy[p] = Gamyyy[p] - ((G(chiy) + G(chiy)) / c - G(gyy) * G(gxxy)) * HALF;
        Gamzyy[p] = Gamzyy[p] - (-G(gyy) * G(gxxz)) * HALF;
        Gamxzz[p] = Gamxzz[p] - (-G(gzz) * G(gxxx)) * HALF;
        Gamyzz[p] = Gamyzz[p] - (-G(gzz) * G(gxxy)) * HALF;
        Gamzzz[p] = Gamzzz[p] - ((G(chiz) + G(chiz)) / c - G(gzz) * G(gxxz)) * HALF;
        Gamxxy[p] = Gamxxy[p] - (G(chiy) / c - G(gxy) * G(gxxx)) * HALF;
        Gamyxy[p] = Gamyxy[p] - (G(chix) / c - G(gxy) * G(gxxy)) * HALF;
        Gamzxy[p] = Gamzxy[p] - (-G(gxy) * G(gxxz)) * HALF;
        Gamxxz[p] = Gamxxz[p] - (G(chiz) / c - G(gxz) * G(gxxx)) * HALF;
        Gamyxz[p] = Gamyxz[p] - (-G(gxz) * G(gxxy)) * HALF;
        Gamzxz[p] = Gamzxz[p] - (G(chix) / c - G(gxz) * G(gxxz)) * HALF;
        Gamxyz[p] = Gamxyz[p] - (-G(gyz) * G(gxxx)) * HALF;
        Gamyyz[p] = Gamyyz[p] - (G(chiz) / c - G(gyz) * G(gxxy)) * HALF;
        Gamzyz[p] = Gamzyz[p] - (G(chiy) / c - G(gyz) * G(gxxz)) * HALF;

        fxx[p] = fxx[p] - G(Gamxxx) * G(Lapx) - G(Gamyxx) * G(Lapy) - G(Gamzxx) * G(Lapz);
        fyy[p] = fyy[p] - G(Gamxyy) * G(Lapx) - G(Gamyyy) * G(Lapy) - G(Gamzyy) * G(Lapz);
        fzz[p] = fzz[p] - G(Gamxzz) * G(Lapx) - G(Gamyzz) * G(Lapy) - G(Gamzzz) * G(Lapz);
        fxy[p] = fxy[p] - G(Gamxxy) * G(Lapx) - G(Gamyxy) * G(Lapy) - G(Gamzxy) * G(Lapz);
        fxz[p] = fxz[p] - G(Gamxxz) * G(Lapx) - G(Gamyxz) * G(Lapy) - G(Gamzxz) * G(Lapz);
        fyz[p] = fyz[p] - G(Gamxyz) * G(Lapx) - G(Gamyyz) * G(Lapy) - G(Gamzyz) * G(Lapz);

        /* store D^i D_i Lap in trK_rhs up to chi */
        trK_rhs[p] = G(gupxx) * G(fxx) + G(gupyy) * G(fyy) + G(gupzz) * G(fzz) +
                     TWO * (G(gupxy) * G(fxy) + G(gupxz) * G(fxz) + G(gupyz) * G(fyz));
        /* Z4c_rhs.f90:961-982: trace of the source from the Ricci scalar */
        double uxx = gupxx[p], uxy = gupxy[p], uxz = gupxz[p], uyy = gupyy[p], uyz = gupyz[p], uzz = gupzz[p];
        double axx = Axx[p], axy = Axy[p], axz = Axz[p], ayy = Ayy[p], ayz = Ayz[p], azz = Azz[p];
        double al = alpn1[p];
        fxx[p] = EIGHT * PI * al * Sxx[p] + fxx[p];
        fxy[p] = EIGHT * PI * al * Sxy[p] + fxy[p];
        fxz[p] = EIGHT * PI * al * Sxz[p] + fxz[p];
        fyy[p] = EIGHT * PI * al * Syy[p] + fyy[p];
        fyz[p] = EIGHT * PI * al * Syz[p] + fyz[p];
        fzz[p] = EIGHT * PI * al * Szz[p] + fzz[p];
        double ff = uxx * fxx[p] + uyy * fyy[p] + uzz * fzz[p] +
                    TWO * (uxy * fxy[p] + uxz * fxz[p] + uyz * fyz[p]);
        ff = F1o3 * (Hc[p] * al - ff);
        fxx[p] = al * Rxx[p] - fxx[p];
        fxy[p] = al * Rxy[p] - fxy[p];
        fxz[p] = al * Rxz[p] - fxz[p];
        fyy[p] = al * Ryy[p] - fyy[p];
        fyz[p] = al * Ryz[p] - fyz[p];
        fzz[p] = al * Rzz[p] - fzz[p];
        /* Z4c_rhs.f90:984-989 */
        Axx_rhs[p] = fxx[p] - gxx[p] * ff;
        Ayy_rhs[p] = fyy[p] - gyy[p] * ff;
        Azz_rhs[p] = fzz[p] - gzz[p] * ff;
        Axy_rhs[p] = fxy[p] - gxy[p] * ff;
        Axz_rhs[p] = fxz[p] - gxz[p] * ff;
        Ayz_rhs[p] = fyz[p] - gyz[p] * ff;
        /* bssn_rhs.f90:729-746 A_il A^l_j */
        fxx[p] = uxx * axx * axx + uyy * axy * axy + uzz * axz * axz +
                 TWO * (uxy * axx * axy + uxz * axx * axz + uyz * axy * axz);
        fyy[p] = uxx * axy * axy + uyy * ayy * ayy + uzz * ayz * ayz +
                 TWO * (uxy * axy * ayy + uxz * axy * ayz + uyz * ayy * ayz);
        fzz[p] = uxx * axz * axz + uyy * ayz * ayz + uzz * azz * azz +
                 TWO * (uxy * axz * ayz + uxz * axz * azz + uyz * ayz * azz);
        fxy[p] = uxx * axx * axy + uyy * axy * ayy + uzz * axz * ayz +
                 uxy * (axx * ayy + axy * axy) + uxz * (axx * ayz + axz * axy) + uyz * (axy * ayz + axz * ayy);
        fxz[p] = uxx * axx * axz + uyy * axy * ayz + uzz * axz * azz +
                 uxy * (axx * ayz + axy * axz) + uxz * (axx * azz + axz * axz) + uyz * (axy * azz + axz * ayz);
        fyz[p] = uxx * axy * axz + uyy * ayy * ayz + uzz * ayz * azz +
                 uxy * (axy * ayz + ayy * axz) + uxz * (axy * azz + ayz * axz) + uyz * (ayy * azz + ayz * ayz);
        /* bssn_rhs.f90:748-777 */
        f[p] = c;
        double fc = c;
        trK_rhs[p] = fc * trK_rhs[p];
        double K = trK[p], Kd = trKd[p];
        double bxx = betaxx[p], bxy = betaxy[p], bxz = betaxz[p];
        double byx = betayx[p], byy = betayy[p], byz = betayz[p];
        double bzx = betazx[p], bzy = betazy[p], bzz = betazz[p], db = div_beta[p];
        Axx_rhs[p] = fc * Axx_rhs[p] + al * (Kd * axx - TWO * fxx[p]) +
                     TWO * (axx * bxx + axy * byx + axz * bzx) - F2o3 * axx * db;
        Ayy_rhs[p] = fc * Ayy_rhs[p] + al * (Kd * ayy - TWO * fyy[p]) +
                     TWO * (axy * bxy + ayy * byy + ayz * bzy) - F2o3 * ayy * db;
        Azz_rhs[p] = fc * Azz_rhs[p] + al * (Kd * azz - TWO * fzz[p]) +
                     TWO * (axz * bxz + ayz * byz + azz * bzz) - F2o3 * azz * db;
        Axy_rhs[p] = fc * Axy_rhs[p] + al * (Kd * axy - TWO * fxy[p]) +
                     axx * bxy + axz * bzy + ayy * byx + ayz * bzx + F1o3 * axy * db - axy * bzz;
        Ayz_rhs[p] = fc * Ayz_rhs[p] + al * (Kd * ayz - TWO * fyz[p]) +
                     axy * bxz + ayy * byz + axz * bxy + azz * bzy + F1o3 * ayz * db - ayz * bxx;
        Axz_rhs[p] = fc * Axz_rhs[p] + al * (Kd * axz - TWO * fxz[p]) +
                     axx * bxz + axy * byz + ayz * byx + azz * bzx + F1o3 * axz * db - axz * byy;
        /* bssn_rhs.f90:781-787 */
        S[p] = fc * (uxx * Sxx[p] + uyy * Syy[p] + uzz * Szz[p] +
                     TWO * (uxy * Sxy[p] + uxz * Sxz[p] + uyz * Syz[p]));
        trK_rhs[p] = -trK_rhs[p] + al * (F1o3 * Kd * Kd + uxx * fxx[p] + uyy * fyy[p] + uzz * fzz[p] +
                                         TWO * (uxy * fxy[p] + uxz * fxz[p] + uyz * fyz[p]) +
                                         FOUR * PI * (rho[p] + S[p]));
        /* bssn_rhs.f90:791-799 gauge, GAUGE == 0 */
        Lap_rhs[p] = -TWO * al * K;
        betax_rhs[p] = FF * dtSfx[p];
        betay_rhs[p] = FF * dtSfy[p];
        betaz_rhs[p] = FF * dtSfz[p];
        dtSfx_rhs[p] = Gamx_rhs[p] - eta * dtSfx[p];
        dtSfy_rhs[p] = Gamy_rhs[p] - eta * dtSfy[p];
        dtSfz_rhs[p] = Gamz_rhs[p] - eta * dtSfz[p];
        /* Z4c_rhs.f90:1077-1110 Hamiltonian constraint with trKd; :1165 Theta_rhs */
        double hh = c * Hc[p] + F2o3 * Kd * Kd -
                    (uxx * (uxx * axx * axx + uyy * axy * axy + uzz * axz * axz +
                            TWO * (uxy * axx * axy + uxz * axx * axz + uyz * axy * axz)) +
                     uyy * (uxx * axy * axy + uyy * ayy * ayy + uzz * ayz * ayz +
                            TWO * (uxy * axy * ayy + uxz * axy * ayz + uyz * ayy * ayz)) +
                     uzz * (uxx * axz * axz + uyy * ayz * ayz + uzz * azz * azz +
                            TWO * (uxy * axz * ayz + uxz * axz * azz + uyz * ayz * azz)) +
                     TWO * (uxy * (uxx * axx * axy + uyy * axy * ayy + uzz * axz * ayz +
                                   uxy * (axx * ayy + axy * axy) +
                                   uxz * (axx * ayz + axz * axy) +
                                   uyz * (axy * ayz + axz * ayy)) +
                            uxz * (uxx * axx * axz + uyy * axy * ayz + uzz * axz * azz +
                                   uxy * (axx * ayz + axy * axz) +
                                   uxz * (axx * azz + axz * axz) +
                                   uyz * (axy * azz + axz * ayz)) +
                            uyz * (uxx * axy * axz + uyy * ayy * ayz + uzz * ayz * azz +
                                   uxy * (axy * ayz + ayy * axz) +
                                   uxz * (axy * azz + ayz * axz) +
                                   uyz * (ayy * azz + ayz * ayz)))) -
                    F16 * PI * rho[p];
        TZ_rhs[p] = al * hh / TWO;
    }
#undef G
    /* bssn_rhs.f90:918-981 advection */
    const double SSS[3] = {SYM, SYM, SYM}, AAS[3] = {ANTI, ANTI, SYM}, ASA[3] = {ANTI, SYM, ANTI};
    const double SAA[3] = {SYM, ANTI, ANTI}, ASS[3] = {ANTI, SYM, SYM}, SAS[3] = {SYM, ANTI, SYM};
    const double SSA[3] = {SYM, SYM, ANTI};
#define LOP(F, R, P) oracle_lopsided(ex, X, Y, Z, F, R, betax, betay, betaz, Symmetry, P)
    LOP(gxx, gxx_rhs, SSS);
    LOP(gxy, gxy_rhs, AAS);
    LOP(gxz, gxz_rhs, ASA);
    LOP(gyy, gyy_rhs, SSS);
    LOP(gyz, gyz_rhs, SAA);
    LOP(gzz, gzz_rhs, SSS);
    LOP(Axx, Axx_rhs, SSS);
    LOP(Axy, Axy_rhs, AAS);
    LOP(Axz, Axz_rhs, ASA);
    LOP(Ayy, Ayy_rhs, SSS);
    LOP(Ayz, Ayz_rhs, SAA);
    LOP(Azz, Azz_rhs, SSS);
    LOP(chi, chi_rhs, SSS);
    LOP(trK, trK_rhs, SSS);
    LOP(Gamx, Gamx_rhs, ASS);
    LOP(Gamy, Gamy_rhs, SAS);
    LOP(Gamz, Gamz_rhs, SSA);
    LOP(Lap, Lap_rhs, SSS);
    LOP(betax, betax_rhs, ASS);
    LOP(betay, betay_rhs, SAS);
    LOP(betaz, betaz_rhs, SSA);
    LOP(dtSfx, dtSfx_rhs, ASS);
    LOP(dtSfy, dtSfy_rhs, SAS);
    LOP(dtSfz, dtSfz_rhs, SSA);
    LOP(TZ, TZ_rhs, SSS);
#undef LOP
    /* Z4c_rhs.f90:1228-1233 constraint damping */
    PL {
        double al = alpn1[p];
        TZ_rhs[p] = TZ_rhs[p] - al * (TWO + kappa2) * kappa1 * TZ[p];
        trK_rhs[p] = trK_rhs[p] + al * kappa1 * (ONE - kappa2) * TZ[p];
        Gamx_rhs[p] = Gamx_rhs[p] - TWO * al * kappa1 * (Gamx[p] - Gamxa[p]);
        Gamy_rhs[p] = Gamy_rhs[p] - TWO * al * kappa1 * (Gamy[p] - Gamya[p]);
        Gamz_rhs[p] = Gamz_rhs[p] - TWO * al * kappa1 * (Gamz[p] - Gamza[p]);
    }
    /* bssn_rhs.f90:983-1042 Kreiss-Oliger dissipation */
    if (eps > 0) {
#define KO(F, R, P) oracle_kodis(ex, X, Y, Z, F, R, P, Symmetry, eps)
        KO(chi, chi_rhs, SSS);
        KO(trK, trK_rhs, SSS);
        KO(gxx, gxx_rhs, SSS);   /* Z4c_rhs.f90:1240-1245: the full metric */
        KO(gxy, gxy_rhs, AAS);
        KO(gxz, gxz_rhs, ASA);
        KO(gyy, gyy_rhs, SSS);
        KO(gyz, gyz_rhs, SAA);
        KO(gzz, gzz_rhs, SSS);
        KO(Axx, Axx_rhs, SSS);
        KO(Axy, Axy_rhs, AAS);
        KO(Axz, Axz_rhs, ASA);
        KO(Ayy, Ayy_rhs, SSS);
        KO(Ayz, Ayz_rhs, SAA);
        KO(Azz, Azz_rhs, SSS);
        KO(Gamx, Gamx_rhs, ASS);
        KO(Gamy, Gamy_rhs, SAS);
        KO(Gamz, Gamz_rhs, SSA);
        KO(Lap, Lap_rhs, SSS);
        KO(betax, betax_rhs, ASS);
        KO(betay, betay_rhs, SAS);
        KO(betaz, betaz_rhs, SSA);
        KO(dtSfx, dtSfx_rhs, ASS);
        KO(dtSfy, dtSfy_rhs, SAS);
        KO(dtSfz, dtSfz_rhs, SSA);
        KO(TZ, TZ_rhs, SSS);
#undef KO
    }
    /* Z4c_rhs.f90:1266-1290 ricci_gamma + constraint_bssn: diagnostic outputs from the
     * first 24 fields (the RHS written there is scratch) */
    {
        double *scratch = oalloc(24 * n);
        double *r[24];
        for (int f = 0; f < 24; ++f) r[f] = scratch + (long)f * n;
        oracle_compute_rhs_bssn(ex, T, X, Y, Z, chi, trK, dxx, gxy, gxz, dyy, gyz, dzz, Axx, Axy, Axz, Ayy, Ayz,
                                Azz, Gamx, Gamy, Gamz, Lap, betax, betay, betaz, dtSfx, dtSfy, dtSfz, r[0], r[1],
                                r[2], r[3], r[4], r[5], r[6], r[7], r[8], r[9], r[10], r[11], r[12], r[13], r[14],
                                r[15], r[16], r[17], r[18], r[19], r[20], r[21], r[22], r[23], rho, Sx, Sy, Sz, Sxx,
                                Sxy, Sxz, Syy, Syz, Szz, Gamxxx, Gamxxy, Gamxxz, Gamxyy, Gamxyz, Gamxzz, Gamyxx,
                                Gamyxy, Gamyxz, Gamyyy, Gamyyz, Gamyzz, Gamzxx, Gamzxy, Gamzxz, Gamzyy, Gamzyz,
                                Gamzzz, Rxx, Rxy, Rxz, Ryy, Ryz, Rzz, ham_Res, movx_Res, movy_Res, movz_Res, Gmx_Res,
                                Gmy_Res, Gmz_Res, Symmetry, Lev, eps, 0);
        free(scratch);
    }

    double *tmp[] = {gxx, gyy, gzz, chix, chiy, chiz, gxxx, gxyx, gxzx, gyyx, gyzx, gzzx,
                     gxxy, gxyy, gxzy, gyyy, gyzy, gzzy, gxxz, gxyz, gxzz, gyyz, gyzz, gzzz,
                     Lapx, Lapy, Lapz, betaxx, betaxy, betaxz, betayx, betayy, betayz,
                     betazx, betazy, betazz, Gamxx, Gamxy, Gamxz, Gamyx, Gamyy_, Gamyz_,
                     Gamzx, Gamzy, Gamzz_, Kx, Ky, Kz, div_beta, S, f, fxx, fxy, fxz, fyy, fyz, fzz,
                     Gamxa, Gamya, Gamza, alpn1, chin1, gupxx, gupxy, gupxz, gupyy, gupyz, gupzz, trKd, Hc};
    for (size_t t = 0; t < sizeof(tmp) / sizeof(tmp[0]); ++t) free(tmp[t]);
    return 0;
}
